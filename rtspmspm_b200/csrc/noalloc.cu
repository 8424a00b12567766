// Allocation-free entry point: the plain two-pass product with every piece
// of scratch (widened row pointers, per-row products and counts, row bins,
// scan partials, the error word) in one file-scope device array, and the
// output written into buffers the caller owns.
//
// Who needs it: callers that cannot let a library call cudaMalloc -- e.g. a
// serving process whose device memory is owned by its own arena or held to
// a fixed budget, where a library growing the CUDA memory pool would break
// the accounting, and hot paths where an allocation's latency or a possible
// out-of-memory failure mid-call is not acceptable.
//
// Limits: A and B have at most kNoAllocMaxRows rows each, and every output
// row must fit the warp hash tables (intermediate products per row, capped
// at the column count, no more than 2048 with the default tables); larger
// inputs are rejected with SPG_ERR_UNSUPPORTED/SPG_ERR_INVALID_ARG and a
// message.  The scratch array (about 9.3 MB) stays resident on every GPU
// that loads the library until the process exits.  Its device address is
// looked up once per device and kept, so the entry point must not be used
// across a cudaDeviceReset of that device.  On any error return the
// contents of C's buffers are unspecified.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "context.hpp"

using namespace spg;

namespace {

constexpr int64_t kNoAllocMaxRows = int64_t(1) << 18;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

constexpr size_t kRpBytes = align256((size_t)(kNoAllocMaxRows + 1) * 8);
constexpr size_t kOffArp = 0;                                                // A row pointers (int64)
constexpr size_t kOffBrp = kOffArp + kRpBytes;                               // B row pointers (int64)
constexpr size_t kOffProd = kOffBrp + kRpBytes;                              // products per row
constexpr size_t kOffNnz = kOffProd + kRpBytes;                              // nnz per row -> row pointers
constexpr size_t kOffBins = kOffNnz + kRpBytes;                              // bin of each row (uint8)
constexpr size_t kOffLists = kOffBins + align256((size_t)kNoAllocMaxRows);   // rows grouped by bin
constexpr size_t kOffMeta = kOffLists + align256((size_t)kNoAllocMaxRows * 4);  // bin counts/offsets/cursors
constexpr size_t kOffScan = kOffMeta + 512;                                  // scan partials
constexpr size_t kScanBytes = 4096;
constexpr size_t kOffFlags = kOffScan + kScanBytes;                          // device error word
constexpr size_t kScratchBytes = kOffFlags + 256;

}  // namespace

// The scratch.  In host code this name is only a stand-in for the symbol:
// device addresses come from cudaGetSymbolAddress (scratch_address below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

std::mutex g_setup_mu;
constexpr int kMaxDevices = 64;
unsigned char* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch on the current device, looked up once per
// device (with that device current) on the first call.
spg_status scratch_address(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices) return SPG_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      (void)cudaGetLastError();
      return SPG_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_addr[dev];
  return SPG_OK;
}

spg_status err(char* buf, int32_t len, spg_status st, const char* fmt, ...) {
  if (buf && len > 0) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, (size_t)len, fmt, ap);
    va_end(ap);
  }
  return st;
}

#define NA_CUDA(call)                                                                          \
  do {                                                                                         \
    const cudaError_t _e = (call);                                                             \
    if (_e != cudaSuccess) {                                                                   \
      (void)cudaGetLastError();                                                                \
      return err(errbuf, errlen, _e == cudaErrorMemoryAllocation ? SPG_ERR_OUT_OF_MEMORY : SPG_ERR_CUDA, \
                 "%s: %s", #call, cudaGetErrorString(_e));                                     \
    }                                                                                          \
  } while (0)

spg_status check_input(const spg_csr* m, const char* name, char* errbuf, int32_t errlen) {
  if (!m) return err(errbuf, errlen, SPG_ERR_INVALID_ARG, "%s is null", name);
  if (m->location != SPG_DEVICE) return err(errbuf, errlen, SPG_ERR_INVALID_ARG, "%s must be on the device", name);
  if (m->index_bits != 32 && m->index_bits != 64)
    return err(errbuf, errlen, SPG_ERR_INVALID_ARG, "%s.index_bits must be 32 or 64", name);
  if (m->rows < 0 || m->cols < 0 || m->nnz < 0) return err(errbuf, errlen, SPG_ERR_INVALID_ARG, "%s has a negative size", name);
  if (m->rows > kNoAllocMaxRows)
    return err(errbuf, errlen, SPG_ERR_INVALID_ARG,
               "%s has %lld rows; the allocation-free entry point takes at most %lld (use spg_multiply)", name,
               (long long)m->rows, (long long)kNoAllocMaxRows);
  if (m->cols > INT32_MAX) return err(errbuf, errlen, SPG_ERR_UNSUPPORTED, "%s has more than 2^31-1 columns", name);
  if (!m->row_ptr || (m->nnz > 0 && (!m->col_idx || !m->val)))
    return err(errbuf, errlen, SPG_ERR_INVALID_ARG, "%s has a null array", name);
  return SPG_OK;
}

}  // namespace

extern "C" spg_status spg_multiply_noalloc(void* stream, const spg_csr* A, const spg_csr* B, spg_csr* C,
                                           char* errbuf, int32_t errlen) {
  if (errbuf && errlen > 0) errbuf[0] = 0;
  // an error left pending by the caller's earlier work is not this call's:
  // report it without clearing it, before any device work
  const cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess)
    return err(errbuf, errlen, SPG_ERR_CUDA, "a CUDA error was already pending when the call began: %s",
               cudaGetErrorString(pending));
  spg_status st;
  if ((st = check_input(A, "A", errbuf, errlen)) != SPG_OK) return st;
  if ((st = check_input(B, "B", errbuf, errlen)) != SPG_OK) return st;
  if (A->cols != B->rows) return err(errbuf, errlen, SPG_ERR_INVALID_ARG, "inner dimensions differ");
  if (!C || C->location != SPG_DEVICE || (C->index_bits != 32 && C->index_bits != 64) || !C->row_ptr ||
      C->capacity < 0 || (C->capacity > 0 && (!C->col_idx || !C->val)))
    return err(errbuf, errlen, SPG_ERR_INVALID_ARG,
               "C must carry caller-owned device buffers: row_ptr (rows+1 entries), col_idx and val (capacity)");
  int dev = 0;
  NA_CUDA(cudaGetDevice(&dev));
  unsigned char* base = nullptr;
  if ((st = scratch_address(dev, &base)) != SPG_OK)
    return err(errbuf, errlen, st, "cudaGetSymbolAddress of the scratch array failed");
  int sms = 0;
  NA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const LaunchCtx lc{static_cast<cudaStream_t>(stream), sms};
  const cudaStream_t s = lc.stream;
  const int64_t rows = A->rows;
  int64_t* arp = reinterpret_cast<int64_t*>(base + kOffArp);
  int64_t* brp = reinterpret_cast<int64_t*>(base + kOffBrp);
  int64_t* prod = reinterpret_cast<int64_t*>(base + kOffProd);
  int64_t* nnz = reinterpret_cast<int64_t*>(base + kOffNnz);
  uint8_t* bins = base + kOffBins;
  int32_t* lists = reinterpret_cast<int32_t*>(base + kOffLists);
  int64_t* meta = reinterpret_cast<int64_t*>(base + kOffMeta);
  int64_t* scan_tmp = reinterpret_cast<int64_t*>(base + kOffScan);
  int* flags = reinterpret_cast<int*>(base + kOffFlags);
  int64_t* counts = meta;
  int64_t* offsets = meta + kNumBins;
  int64_t* cursors = meta + 2 * kNumBins + 1;

  // the array keeps the previous call's contents: reset what must start at 0
  NA_CUDA(cudaMemsetAsync(flags, 0, sizeof(int), s));
  NA_CUDA(cudaMemsetAsync(nnz, 0, (size_t)(rows + 1) * 8, s));
  const spg_csr* src[2] = {A, B};
  int64_t* dst[2] = {arp, brp};
  for (int q = 0; q < 2; ++q) {
    if (src[q]->index_bits == 32) launch_widen_rp(static_cast<const int32_t*>(src[q]->row_ptr), src[q]->rows + 1, dst[q], lc);
    else NA_CUDA(cudaMemcpyAsync(dst[q], src[q]->row_ptr, (size_t)(src[q]->rows + 1) * 8, cudaMemcpyDeviceToDevice, s));
  }
  const DCsr dA{A->rows, A->cols, arp, A->col_idx, A->val,
                A->index_bits == 32 ? static_cast<const int32_t*>(A->row_ptr) : nullptr};
  const DCsr dB{B->rows, B->cols, brp, B->col_idx, B->val,
                B->index_bits == 32 ? static_cast<const int32_t*>(B->row_ptr) : nullptr};
  launch_validate(dA, A->nnz, flags, lc);
  launch_validate(dB, B->nnz, flags, lc);
  int hflags = 0;
  NA_CUDA(cudaMemcpyAsync(&hflags, flags, sizeof(int), cudaMemcpyDeviceToHost, s));
  NA_CUDA(cudaStreamSynchronize(s));
  if (hflags & kFlagBadIndex)
    return err(errbuf, errlen, SPG_ERR_INVALID_ARG,
               "input failed validation (index out of range, unsorted or duplicate columns, bad row pointers)");

  // the warp bins only (rows above them are rejected)
  const BinParams bp = without_block_bins(bin_params(default_tuning()));
  const int wpb = default_tuning().warps_per_block;
  launch_row_products(dA, dB, prod, lc);
  launch_binning(prod, rows, B->cols, kBinSymbolic, bp, bins, counts, offsets, cursors, lists, lc);
  int64_t off[kNumBins + 1];
  NA_CUDA(cudaMemcpyAsync(off, offsets, sizeof off, cudaMemcpyDeviceToHost, s));
  NA_CUDA(cudaStreamSynchronize(s));
  const int64_t big = (off[kBinBlock + 1] - off[kBinBlock]) + (off[kBinDense + 1] - off[kBinDense]);
  if (big > 0)
    return err(errbuf, errlen, SPG_ERR_UNSUPPORTED,
               "%lld rows have more than %lld intermediate products; the allocation-free entry point only takes "
               "rows that fit the warp hash tables (use spg_multiply)",
               (long long)big, (long long)bp.warp_cap);
  for (int b = 0; b < kNumWarpBins; ++b)
    launch_sym_warp(kMinLogT + b, dA, dB, lists + off[b], off[b + 1] - off[b], nnz, flags, lc, wpb);
  NA_CUDA(cudaGetLastError());  // a failed symbolic launch: the counts below would be wrong
  launch_binning(nnz, rows, B->cols, kBinNumeric, bp, bins, counts, offsets, cursors, lists, lc);
  launch_excl_scan(nnz, rows, nnz, scan_tmp, lc);
  int64_t total = 0;
  NA_CUDA(cudaMemcpyAsync(off, offsets, sizeof off, cudaMemcpyDeviceToHost, s));
  NA_CUDA(cudaMemcpyAsync(&total, nnz + rows, sizeof total, cudaMemcpyDeviceToHost, s));
  NA_CUDA(cudaStreamSynchronize(s));
  // only the warp bins are launched below: a non-empty row binned anywhere
  // else would leave its part of C unwritten
  int64_t outside = 0;
  for (int b = kNumWarpBins; b < kNumBins; ++b)
    if (b != kBinEmpty) outside += off[b + 1] - off[b];
  if (outside > 0)
    return err(errbuf, errlen, SPG_ERR_INTERNAL,
               "%lld output rows exceed the warp hash tables after the exact count (internal binning mismatch)",
               (long long)outside);
  C->rows = rows;
  C->cols = B->cols;
  if (total > C->capacity) {
    C->nnz = total;
    return err(errbuf, errlen, SPG_ERR_INVALID_ARG,
               "C needs room for %lld entries but its capacity is %lld (C->nnz holds the size needed)",
               (long long)total, (long long)C->capacity);
  }
  if (C->index_bits == 32 && total >= INT32_MAX)
    return err(errbuf, errlen, SPG_ERR_INVALID_ARG, "nnz(C) does not fit int32 row pointers");
  for (int b = 0; b < kNumWarpBins; ++b)
    launch_num_warp(kMinLogT + b, dA, dB, lists + off[b], off[b + 1] - off[b], nnz, C->col_idx, C->val, flags, lc,
                    wpb);
  NA_CUDA(cudaGetLastError());
  if (C->index_bits == 64)
    NA_CUDA(cudaMemcpyAsync(C->row_ptr, nnz, (size_t)(rows + 1) * 8, cudaMemcpyDeviceToDevice, s));
  else
    launch_narrow_rp(nnz, rows + 1, static_cast<int32_t*>(C->row_ptr), lc);
  NA_CUDA(cudaMemcpyAsync(&hflags, flags, sizeof(int), cudaMemcpyDeviceToHost, s));
  NA_CUDA(cudaStreamSynchronize(s));
  NA_CUDA(cudaGetLastError());
  if (hflags & (kFlagHashFull | kFlagCountDiff))
    return err(errbuf, errlen, SPG_ERR_INTERNAL, "device consistency check failed (flags %d)", hflags);
  C->nnz = total;
  return SPG_OK;
}
