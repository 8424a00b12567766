// Matrix Market reader / writer of the C ABI (host code).
//
// Reader: replaces the reference's three line-by-line istringstream parsers
// (cooFromFile cuSparse/src/util.cpp:9-44, mat1ToGPU
// optixSpMSpM/src/optixSpMSpM/optixSpMSpM.cpp:73-131, Sphere::Sphere
// optixSpMSpM/src/optixSpMSpM/Sphere.cpp:26-78).  The whole file is read
// at once and its body parsed with std::from_chars in newline-aligned slices
// on all host threads; entries may come in any order (the shipped fixtures
// are column-major), are converted to 0-based CSR with sorted columns (row
// blocks in parallel), and duplicate (i, j) pairs are summed in FP32 in file
// order.  `symmetric` files are expanded; `pattern` files get value 1; lines
// after the header's nnz entries are ignored.
//
// Writer: the reference's two writers -- printCooToFile
// (cuSparse/src/util.cpp:49-69, every structural entry) and printResult
// (optixSpMSpM.cpp:452-494, row-major, skips exact zeros).  Lines are
// `i j v`, 1-based, row-major with ascending columns; values use the
// shortest decimal form that reads back to the same FP32.
#include <algorithm>
#include <charconv>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/rtspmspm.h"

namespace {

struct Cursor {
  const char* p;
  const char* end;
  bool at_end() const { return p >= end; }
  void skip_blank() {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
  }
  void next_line() {
    while (p < end && *p != '\n') ++p;
    if (p < end) ++p;
  }
  template <typename T>
  bool read_int(T& v) {
    skip_blank();
    auto r = std::from_chars(p, end, v);
    if (r.ec != std::errc()) return false;
    p = r.ptr;
    return true;
  }
  bool read_float(float& v) {
    skip_blank();
    // accept a leading '+' which from_chars rejects
    if (p < end && *p == '+') ++p;
    auto r = std::from_chars(p, end, v);
    if (r.ec == std::errc::result_out_of_range) {
      // denormal / overflow literals: fall back to strtof semantics
      char buf[64];
      size_t n = std::min<size_t>(63, (size_t)(r.ptr - p));
      std::memcpy(buf, p, n);
      buf[n] = 0;
      v = std::strtof(buf, nullptr);
      p = r.ptr;
      return true;
    }
    if (r.ec != std::errc()) return false;
    p = r.ptr;
    return true;
  }
};

bool read_file(const char* path, std::vector<char>& buf) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  long n = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (n < 0) {
    std::fclose(f);
    return false;
  }
  buf.resize((size_t)n);
  size_t got = n ? std::fread(buf.data(), 1, (size_t)n, f) : 0;
  std::fclose(f);
  return got == (size_t)n;
}

std::string lower(std::string s) {
  for (auto& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

// Entries of one newline-aligned slice of the body, in file order.
struct Slice {
  std::vector<int32_t> ri, ci;
  std::vector<float> vv;
  int64_t entries = 0;  // file entries (before symmetric expansion)
  bool bad = false;
};

void parse_slice(const char* b, const char* e, bool pattern, bool symmetric, bool skew, int64_t rows, int64_t cols,
                 Slice& out) {
  Cursor c{b, e};
  while (!c.at_end()) {
    c.skip_blank();
    if (c.at_end()) break;
    if (*c.p == '\n' || *c.p == '%') {
      c.next_line();
      continue;
    }
    int64_t i = 0, j = 0;
    float v = 1.0f;
    if (!c.read_int(i) || !c.read_int(j) || (!pattern && !c.read_float(v)) || i < 1 || i > rows || j < 1 ||
        j > cols) {
      out.bad = true;
      return;
    }
    out.ri.push_back((int32_t)(i - 1));
    out.ci.push_back((int32_t)(j - 1));
    out.vv.push_back(v);
    if (symmetric && i != j) {
      out.ri.push_back((int32_t)(j - 1));
      out.ci.push_back((int32_t)(i - 1));
      out.vv.push_back(skew ? -v : v);
    }
    ++out.entries;
    c.next_line();
  }
}

int worker_count(size_t work, size_t per_worker) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t want = std::max<size_t>(1, work / std::max<size_t>(per_worker, 1));
  return (int)std::min<size_t>({(size_t)hw, want, (size_t)64});
}

template <typename F>
void run_workers(int n, F&& f) {
  if (n <= 1) {
    f(0);
    return;
  }
  std::vector<std::thread> th;
  th.reserve((size_t)n - 1);
  for (int t = 1; t < n; ++t) th.emplace_back(f, t);
  f(0);
  for (auto& x : th) x.join();
}

}  // namespace

// The parsed entries of a Matrix Market file: the header's shape and the
// slices holding its first nnz entries (slices [0, last]), m of them after
// the symmetric expansion.
struct Parsed {
  int64_t rows = 0, cols = 0, m = 0;
  int last = -1;
  std::vector<Slice> sl;
};

// Reads and parses `path` in newline-aligned slices on all host threads.
spg_status parse_mtx(const char* path, Parsed& P) {
  std::vector<char> buf;
  if (!read_file(path, buf)) return SPG_ERR_IO;
  Cursor c{buf.data(), buf.data() + buf.size()};
  bool pattern = false, symmetric = false, skew = false;
  // banner (optional) and comments
  if (buf.size() >= 2 && buf[0] == '%' && buf[1] == '%') {
    const char* e = c.p;
    while (e < c.end && *e != '\n') ++e;
    std::string banner = lower(std::string(c.p, e));
    if (banner.find("coordinate") == std::string::npos) return SPG_ERR_FORMAT;
    if (banner.find("complex") != std::string::npos) return SPG_ERR_UNSUPPORTED;
    pattern = banner.find("pattern") != std::string::npos;
    symmetric = banner.find("symmetric") != std::string::npos || banner.find("hermitian") != std::string::npos;
    skew = banner.find("skew-symmetric") != std::string::npos;
    c.next_line();
  }
  while (!c.at_end()) {
    c.skip_blank();
    if (c.at_end()) break;
    if (*c.p == '%' || *c.p == '\n') {
      c.next_line();
      continue;
    }
    break;
  }
  int64_t rows = 0, cols = 0, nnz = 0;
  if (!c.read_int(rows) || !c.read_int(cols) || !c.read_int(nnz)) return SPG_ERR_FORMAT;
  if (rows < 0 || cols < 0 || nnz < 0 || cols > INT32_MAX || rows > INT32_MAX) return SPG_ERR_FORMAT;
  c.next_line();
  // ---- parse: slices cut at line starts ----
  const char* body = c.p;
  const size_t blen = (size_t)(c.end - body);
  const int ns = worker_count(blen, (size_t)4 << 20);
  std::vector<const char*> cut((size_t)ns + 1);
  cut[0] = body;
  cut[(size_t)ns] = c.end;
  for (int t = 1; t < ns; ++t) {
    const char* q = body + blen * (size_t)t / (size_t)ns;
    if (q < cut[(size_t)t - 1]) q = cut[(size_t)t - 1];
    while (q < c.end && q[-1] != '\n') ++q;
    cut[(size_t)t] = q;
  }
  std::vector<Slice>& sl = P.sl;
  sl.assign((size_t)ns, Slice());
  run_workers(ns, [&](int t) {
    parse_slice(cut[(size_t)t], cut[(size_t)t + 1], pattern, symmetric, skew, rows, cols, sl[(size_t)t]);
  });
  // the first nnz entries count (later lines are ignored); a malformed line
  // before them is an error
  int64_t seen = 0, m = 0;
  int last = -1;
  for (int t = 0; t < ns && seen < nnz; ++t) {
    if (sl[(size_t)t].bad && seen + sl[(size_t)t].entries < nnz) return SPG_ERR_FORMAT;
    last = t;
    if (seen + sl[(size_t)t].entries > nnz) {
      // trim this slice to the entries still wanted (expanded pairs stay together)
      Slice& z = sl[(size_t)t];
      const int64_t keep = nnz - seen;
      size_t k = 0;
      for (int64_t x = 0; x < keep; ++x) k += (symmetric && z.ri[k] != z.ci[k]) ? 2 : 1;
      z.ri.resize(k);
      z.ci.resize(k);
      z.vv.resize(k);
      z.entries = keep;
    }
    seen += sl[(size_t)t].entries;
    m += (int64_t)sl[(size_t)t].ri.size();
  }
  if (seen < nnz) return SPG_ERR_FORMAT;
  P.rows = rows;
  P.cols = cols;
  P.m = m;
  P.last = last;
  return SPG_OK;
}

// Parses the body in newline-aligned slices on all host threads, then builds
// CSR: a counting sort by row keeps file order inside a row, and row blocks
// (balanced by entries) are sorted by column and their duplicates summed in
// file order in parallel.
extern "C" spg_status spg_mtx_read(const char* path, spg_csr* out) {
  if (!path || !out) return SPG_ERR_INVALID_ARG;
  std::memset(out, 0, sizeof *out);
  Parsed P;
  const spg_status st = parse_mtx(path, P);
  if (st != SPG_OK) return st;
  const int64_t rows = P.rows, cols = P.cols, m = P.m;
  const int last = P.last;
  std::vector<Slice>& sl = P.sl;
  // ---- counting sort by row (stable: file order inside a row) ----
  std::vector<int64_t> rp((size_t)rows + 1, 0);
  for (int t = 0; t <= last; ++t)
    for (int32_t r : sl[(size_t)t].ri) ++rp[(size_t)r + 1];
  for (int64_t r = 0; r < rows; ++r) rp[(size_t)r + 1] += rp[(size_t)r];
  std::vector<int32_t> col((size_t)m);
  std::vector<float> val((size_t)m);
  {
    std::vector<int64_t> pos(rp.begin(), rp.end() - 1);
    for (int t = 0; t <= last; ++t) {
      Slice& z = sl[(size_t)t];
      for (size_t k = 0; k < z.ri.size(); ++k) {
        const int64_t d = pos[(size_t)z.ri[k]]++;
        col[(size_t)d] = z.ci[k];
        val[(size_t)d] = z.vv[k];
      }
      z = Slice();
    }
  }
  // ---- per-row column sort + duplicate merge, row blocks in parallel ----
  const int nb = worker_count((size_t)m, (size_t)1 << 20);
  std::vector<int64_t> r0((size_t)nb + 1, rows);
  r0[0] = 0;
  for (int t = 1; t < nb; ++t) {
    const int64_t target = m * t / nb;
    r0[(size_t)t] = std::upper_bound(rp.begin(), rp.end(), target) - rp.begin() - 1;
    if (r0[(size_t)t] < r0[(size_t)t - 1]) r0[(size_t)t] = r0[(size_t)t - 1];
  }
  std::vector<int64_t> rowlen((size_t)rows, 0);
  run_workers(nb, [&](int t) {
    std::vector<std::pair<int32_t, float>> tmp;
    for (int64_t r = r0[(size_t)t]; r < r0[(size_t)t + 1]; ++r) {
      const int64_t s = rp[(size_t)r], e = rp[(size_t)r + 1];
      bool sorted = true;
      for (int64_t q = s + 1; q < e && sorted; ++q) sorted = col[(size_t)q - 1] < col[(size_t)q];
      if (sorted) {
        rowlen[(size_t)r] = e - s;
        continue;
      }
      tmp.assign((size_t)(e - s), {});
      for (int64_t q = s; q < e; ++q) tmp[(size_t)(q - s)] = {col[(size_t)q], val[(size_t)q]};
      std::stable_sort(tmp.begin(), tmp.end(),
                       [](const std::pair<int32_t, float>& x, const std::pair<int32_t, float>& y) {
                         return x.first < y.first;
                       });
      int64_t w = s;
      for (size_t q = 0; q < tmp.size(); ++q) {
        if (q > 0 && tmp[q].first == tmp[q - 1].first) {
          val[(size_t)w - 1] = val[(size_t)w - 1] + tmp[q].second;
        } else {
          col[(size_t)w] = tmp[q].first;
          val[(size_t)w] = tmp[q].second;
          ++w;
        }
      }
      rowlen[(size_t)r] = w - s;
    }
  });
  std::vector<int64_t> orp((size_t)rows + 1, 0);
  for (int64_t r = 0; r < rows; ++r) orp[(size_t)r + 1] = orp[(size_t)r] + rowlen[(size_t)r];
  const int64_t w = orp[(size_t)rows];
  const size_t rpb = ((size_t)rows + 1) * sizeof(int64_t);
  int64_t* hrp = (int64_t*)std::malloc(rpb);
  int32_t* hcol = (int32_t*)std::malloc(std::max<size_t>((size_t)w * 4, 4));
  float* hval = (float*)std::malloc(std::max<size_t>((size_t)w * 4, 4));
  if (!hrp || !hcol || !hval) {
    std::free(hrp);
    std::free(hcol);
    std::free(hval);
    return SPG_ERR_OUT_OF_MEMORY;
  }
  std::memcpy(hrp, orp.data(), rpb);
  run_workers(nb, [&](int t) {
    for (int64_t r = r0[(size_t)t]; r < r0[(size_t)t + 1]; ++r) {
      const int64_t n = rowlen[(size_t)r];
      if (!n) continue;
      std::memcpy(hcol + orp[(size_t)r], col.data() + rp[(size_t)r], (size_t)n * 4);
      std::memcpy(hval + orp[(size_t)r], val.data() + rp[(size_t)r], (size_t)n * 4);
    }
  });
  out->rows = rows;
  out->cols = cols;
  out->nnz = w;
  out->capacity = w;
  out->index_bits = 64;
  out->location = SPG_HOST;
  out->row_ptr = hrp;
  out->col_idx = hcol;
  out->val = hval;
  out->owner = 2;
  return SPG_OK;
}

// Parses on all host threads as spg_mtx_read does, then gathers the
// slices' entries (file order, symmetric mirrors after their entry) into one
// COO and builds the CSR on the GPU (spg_coo_to_csr): no host sort.
extern "C" spg_status spg_mtx_read_device(spg_ctx* ctx, const char* path, spg_csr* out) {
  if (!ctx || !path || !out) return SPG_ERR_INVALID_ARG;
  std::memset(out, 0, sizeof *out);
  Parsed P;
  const spg_status st = parse_mtx(path, P);
  if (st != SPG_OK) return st;
  std::vector<int64_t> at((size_t)P.last + 2, 0);
  for (int t = 0; t <= P.last; ++t) at[(size_t)t + 1] = at[(size_t)t] + (int64_t)P.sl[(size_t)t].ri.size();
  std::vector<int32_t> ri((size_t)P.m), ci((size_t)P.m);
  std::vector<float> vv((size_t)P.m);
  if (P.last >= 0) run_workers(P.last + 1, [&](int t) {
    const Slice& z = P.sl[(size_t)t];
    const size_t o = (size_t)at[(size_t)t], k = z.ri.size();
    if (!k) return;
    std::memcpy(ri.data() + o, z.ri.data(), k * 4);
    std::memcpy(ci.data() + o, z.ci.data(), k * 4);
    std::memcpy(vv.data() + o, z.vv.data(), k * 4);
  });
  P.sl.clear();
  return spg_coo_to_csr(ctx, P.rows, P.cols, P.m, ri.data(), ci.data(), vv.data(), SPG_HOST, out);
}

extern "C" spg_status spg_csr_transpose(const spg_csr* src, spg_csr* dst) {
  if (!src || !dst || src == dst) return SPG_ERR_INVALID_ARG;
  if (src->location != SPG_HOST) return SPG_ERR_INVALID_ARG;
  if (src->index_bits != 32 && src->index_bits != 64) return SPG_ERR_INVALID_ARG;
  if (src->rows > INT32_MAX || src->cols > INT32_MAX || src->nnz < 0) return SPG_ERR_UNSUPPORTED;
  auto rp_at = [&](int64_t r) -> int64_t {
    return src->index_bits == 64 ? static_cast<const int64_t*>(src->row_ptr)[r]
                                 : (int64_t) static_cast<const int32_t*>(src->row_ptr)[r];
  };
  const int64_t rows = src->rows, cols = src->cols, nnz = src->nnz;
  int64_t* trp = (int64_t*)std::calloc((size_t)cols + 1, sizeof(int64_t));
  int32_t* tcol = (int32_t*)std::malloc(std::max<size_t>((size_t)nnz * 4, 4));
  float* tval = (float*)std::malloc(std::max<size_t>((size_t)nnz * 4, 4));
  if (!trp || !tcol || !tval) {
    std::free(trp);
    std::free(tcol);
    std::free(tval);
    return SPG_ERR_OUT_OF_MEMORY;
  }
  for (int64_t t = 0; t < nnz; ++t) {
    const int32_t j = src->col_idx[t];
    if (j < 0 || j >= cols) {
      std::free(trp);
      std::free(tcol);
      std::free(tval);
      return SPG_ERR_INVALID_ARG;
    }
    ++trp[(size_t)j + 1];
  }
  for (int64_t j = 0; j < cols; ++j) trp[j + 1] += trp[j];
  std::vector<int64_t> pos(trp, trp + cols);
  for (int64_t r = 0; r < rows; ++r) {
    for (int64_t t = rp_at(r), e = rp_at(r + 1); t < e; ++t) {
      const int64_t d = pos[(size_t)src->col_idx[t]]++;
      tcol[d] = (int32_t)r;
      tval[d] = src->val[t];
    }
  }
  std::memset(dst, 0, sizeof *dst);
  dst->rows = cols;
  dst->cols = rows;
  dst->nnz = nnz;
  dst->capacity = nnz;
  dst->index_bits = 64;
  dst->location = SPG_HOST;
  dst->row_ptr = trp;
  dst->col_idx = tcol;
  dst->val = tval;
  dst->owner = 2;
  return SPG_OK;
}

extern "C" spg_status spg_mtx_write(spg_ctx* ctx, const char* path, const spg_csr* m, int32_t drop_zeros) {
  if (!path || !m) return SPG_ERR_INVALID_ARG;
  spg_csr host{};
  const spg_csr* src = m;
  if (m->location == SPG_DEVICE) {
    if (!ctx) return SPG_ERR_INVALID_ARG;
    spg_status st = spg_csr_copy(ctx, m, SPG_HOST, &host);
    if (st != SPG_OK) return st;
    src = &host;
  }
  auto rp_at = [&](int64_t r) -> int64_t {
    return src->index_bits == 64 ? static_cast<const int64_t*>(src->row_ptr)[r]
                                 : (int64_t) static_cast<const int32_t*>(src->row_ptr)[r];
  };
  int64_t count = 0;
  if (drop_zeros) {
    for (int64_t t = 0; t < src->nnz; ++t) count += src->val[t] != 0.0f;
  } else {
    count = src->nnz;
  }
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    spg_csr_free(ctx, &host);
    return SPG_ERR_IO;
  }
  std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%lld %lld %lld\n", (long long)src->rows,
               (long long)src->cols, (long long)count);
  std::vector<char> out;
  out.reserve(1 << 22);
  char tmp[64];
  bool ok = true;
  for (int64_t r = 0; r < src->rows && ok; ++r) {
    const int64_t s = rp_at(r), e = rp_at(r + 1);
    for (int64_t t = s; t < e; ++t) {
      const float v = src->val[t];
      if (drop_zeros && v == 0.0f) continue;
      char* p = tmp;
      p = std::to_chars(p, tmp + sizeof tmp, r + 1).ptr;
      *p++ = ' ';
      p = std::to_chars(p, tmp + sizeof tmp, (int64_t)src->col_idx[t] + 1).ptr;
      *p++ = ' ';
      p = std::to_chars(p, tmp + sizeof tmp, v).ptr;
      *p++ = '\n';
      out.insert(out.end(), tmp, p);
      if (out.size() > (1 << 22) - 64) {
        ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
        out.clear();
      }
    }
  }
  if (ok && !out.empty()) ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
  ok = (std::fclose(f) == 0) && ok;
  spg_csr_free(ctx, &host);
  return ok ? SPG_OK : SPG_ERR_IO;
}
