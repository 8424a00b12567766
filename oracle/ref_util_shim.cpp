// C-callable shim over the reference's Matrix Market helpers
// (cuSparse/src/util.cpp:9-69), compiled from the reference sources in place
// so tests can check the engine's .mtx reader and writer against the
// reference's own.  Test infrastructure only; builds into oracle/_ref/.
#include <cstdint>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <algorithm>
#include "util.cpp"

extern "C" {

// Reads a .mtx with the reference's cooFromFile; returns nnz, or -1 if the
// file could not be opened.  Arrays are released with ref_free.
int64_t ref_read_coo(const char* path, int** rows, int** cols, float** vals,
                     int* nrows, int* ncols) {
    {
        std::ifstream probe(path);
        if (!probe.is_open()) return -1;
    }
    uint64_t nnz = 0;
    cooFromFile(std::string(path), rows, cols, vals, nrows, ncols, &nnz);
    return (int64_t)nnz;
}

void ref_free(int* rows, int* cols, float* vals) {
    delete[] rows;
    delete[] cols;
    delete[] vals;
}

// Writes 1-based COO with the reference's printCooToFile.
void ref_write_coo(const char* path, const int* rows, const int* cols, const float* vals,
                   int nrows, int ncols, int64_t nnz) {
    printCooToFile(std::string(path), rows, cols, vals, nrows, ncols, (uint64_t)nnz);
}

}
