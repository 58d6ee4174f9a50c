// amg_device.hpp -- the Compact AMS / AMG set-up of Update() on the device
// (compact_amg.hpp:66-156,252-632; compact_ams.hpp:300-421,605-659): the
// BC-modified matrix, the Galerkin products, strength, PMIS coarsening,
// direct interpolation, transposes, l1 norms and the fused level products
// that amg_setup.cpp computes on the host, with the same results bit for bit:
// every floating-point sum runs in the host's order (one thread per output
// row) with each product and sum rounded on its own (no FMA contraction), and
// PMIS reproduces the host's in-order sweep semantics exactly.
#pragma once

#include <cstdint>
#include <vector>

#include "amg_setup.hpp"
#include "host_threads.hpp"
#include "ssv_common.cuh"

namespace ssv {

// SSV_AMS_SETUP_LOG=1: the wall time of every set-up stage on stderr (the
// stream is synchronised at each mark; off, a mark costs nothing)
struct SetupLog {
    bool on = false;
    cudaStream_t s = nullptr;
    double t = 0;
    explicit SetupLog(cudaStream_t st);
    void mark(const char* fmt, ...);
};

// FP64 CSR in device memory (columns sorted per row where the producer says so)
struct DCsr {
    int n = 0, m = 0;
    int64_t nnz = 0;
    DevBuf<int> rp, ci;
    DevBuf<double> v;
    void from_host(const HostCsr& H, cudaStream_t s);
    HostCsr to_host(cudaStream_t s) const;
    void copy_from(const DCsr& o, cudaStream_t s);
};

struct DAmgLevel {
    DCsr A, P, Pt;
    DevBuf<double> l1;
    bool direct = false;
    std::vector<double> linv, linvt, piv;  // coarsest LDL^T pseudo-inverse factors (host, FP64)
    double piv_min = 1.0;                  // smallest kept |pivot| / |diagonal|
};

// A_bc (CreateBCModifiedMatrix, compact_amg.hpp:252-287): identity rows on
// constrained DOFs, zero columns; vals may be a device pointer to A's values.
void d_bc_matrix(int n, int m, int64_t nnz, const int* rp, const int* ci, const double* vals, const uint8_t* d_fd,
                 DCsr& out, cudaStream_t s);
// C = P^T A P with the structural product pattern (csr_rap's order); false if
// a row of C is too long for the device symbolic step
bool d_rap(const DCsr& A, const DCsr& P, const DCsr& Pt, DCsr& C, cudaStream_t s);
// T = A^T, each row in increasing source row (csr_transpose's order)
void d_transpose(const DCsr& A, DCsr& T, cudaStream_t s);
// FixZeroRows (compact_ams.hpp:638-659)
void d_fix_zero_rows(DCsr& A, cudaStream_t s);
// truncated l1 of the fine smoother (compact_ams.hpp:395-413)
void d_fine_l1(const DCsr& A, DevBuf<double>& out, cudaStream_t s);
// CompactAMG::Setup for freedofs = nullptr on the device; false when a row is
// too long for the device symbolic products (the caller then uses the host).
// The coarsest LDL^T factorisation runs on the host: inline, or, when
// `coarse` is given, on a host thread stored there (the caller joins it
// before the factors are read), so it overlaps the device work that follows.
bool d_amg_setup(const DCsr& A0, double theta, int max_levels, int min_coarse, std::vector<DAmgLevel>& out,
                 cudaStream_t s, WorkerThread* coarse = nullptr);
// fused_level (amg_setup.hpp) on the device: R = P^T (I - A D^{-1}),
// U = [D^{-1}(2I - A D^{-1}) | (I - D^{-1} A) P]
bool d_fused_level(const DCsr& A, const DCsr& P, const DCsr& Pt, const double* d, DCsr& R, DCsr& U,
                   cudaStream_t s);
// out.v[k] = A.v[k] * (rmul[row] * cmul[col]) (either may be null = 1), pattern copied
void d_scaled(const DCsr& A, const double* rmul, const double* cmul, DCsr& out, cudaStream_t s);
// sc[i] = sqrt|a_ii| (1 for a zero or missing diagonal); isc = 1 / sc
void d_diag_scale(const DCsr& A, DevBuf<double>& sc, DevBuf<double>& isc, cudaStream_t s);
// out[i] = in[i] * a[i] * b[i] (b may be null), out = 1 / in
void d_scale_vec(int n, const double* in, const double* a, const double* b, double* out, cudaStream_t s);
void d_reciprocal(int n, const double* in, double* out, cudaStream_t s);
void d_to_float(int64_t n, const double* in, float* out, cudaStream_t s);

}  // namespace ssv
