// sell.cuh -- sliced-ELL copies of CSR matrices, shared by the AMS fine-level
// passes and the Krylov SpMV of large system matrices.
//
// Layout: rows sorted by length (longest first, ties in row order) inside
// windows of kSellWindow rows, cut into slices of 32 consecutive sorted rows,
// each slice padded to its longest row; entry k of slice row t sits at
// off[slice] + 32 k + t, so step k of a slice is one coalesced load of 32
// values and one of 32 column indices. Padding carries column -1 and source
// -1. rows[32 slice + t] is the CSR row of slice row t (-1 past the end).
// (Storing the slices widest first, so that the last partial wave of a launch
// holds the shortest ones, measured no faster at 40^3 and 8% slower at 64^3:
// neighbouring slices then no longer run side by side and share fewer x rows
// in L1.)
#pragma once

#include <cstdint>

#include "ssv_common.cuh"

namespace ssv {

constexpr int kSellWindow = 256;

struct SellPattern {
    int slices = 0;
    int64_t entries = 0;
    int pat_n = -1;
    int64_t pat_nnz = -1;  // the pattern the layout was built for
    DevBuf<int> off, rows, ci;
    DevBuf<int> src;  // slot -> CSR entry index (-1 = padding), for value gathers
    // the layout of the device CSR pattern (rp, ci) of n rows; false (and no
    // copy: slices = 0) when the padded size exceeds the int range
    bool build_pattern(int n, int64_t nnz, const int* rp, const int* ci, cudaStream_t s);
    bool same_pattern(int n, int64_t nnz) const { return slices > 0 && pat_n == n && pat_nnz == nnz; }
    // no usable layout (set before a build, so that one that fails part way,
    // on an allocation, is never taken for a finished one)
    void invalidate() {
        slices = 0;
        entries = 0;
        pat_n = -1;
        pat_nnz = -1;
    }
};

// v[e] = csr_v[src[e]] for `words` doubles per entry (2 for complex), 0 on padding
void sell_gather(const SellPattern& P, const double* csr_v, int words, double* v, cudaStream_t s);

// exclusive scan of the slice widths into off (slices + 1 entries); the
// total, or -1 when it exceeds the int range (amg_device.cu)
int sell_offsets(int slices, const int* width, int* off, cudaStream_t s);

}  // namespace ssv
