// amg_setup.hpp -- host set-up of the Compact AMS / AMG hierarchy
// (include/sparsesolv/preconditioners/compact_amg.hpp:66-156,292-632 and
// compact_ams.hpp:243-504,605-659). Produces the matrices the device cycle
// applies; runs once per Update().
#pragma once

#include <cstdint>
#include <vector>

namespace ssv {

struct HostCsr {
    int n = 0, m = 0;
    std::vector<int> rp, ci;
    std::vector<double> v;
    int nnz() const { return rp.empty() ? 0 : rp[n]; }
};

HostCsr csr_transpose(const HostCsr& A);
// P^T A P with the structural product pattern (explicit zeros kept, columns
// sorted) -- the semantics of NGSolve's SparseMatrix::Restrict.
HostCsr csr_rap(const HostCsr& A, const HostCsr& P);

// C = A B (columns of each row sorted)
HostCsr csr_mul(const HostCsr& A, const HostCsr& B);
// C = a A + b B on the union pattern (columns sorted)
HostCsr csr_add(const HostCsr& A, double a, const HostCsr& B, double b);

// One level's V-cycle steps (num_smooth = 1, l1-Jacobi with l1 = d) folded
// into two matrices, from the level's A, P, P^T and d:
//   down: b_next = R b,  R = P^T (I - A D^{-1})        (first sweep x = D^{-1} b,
//         residual b - A x and restriction in one product)
//   up:   x = U [b; e],  U = [D^{-1}(2I - A D^{-1}) | (I - D^{-1} A) P]
//         (prolongation x + P e and the post sweep in one product; columns
//         n.. of U address the coarse correction e)
struct FusedLevel {
    HostCsr R, U;
};
FusedLevel fused_level(const HostCsr& A, const HostCsr& P, const HostCsr& Pt, const std::vector<double>& d);

// Pseudo-inverse of the small coarsest matrix through LDL^T (pivots at or
// below tau of their row's diagonal dropped; the reference's tau is 1e-13):
// linv = L^{-1} row-major, linvt its transpose, piv the pivots (0 where
// dropped). Returns the smallest |pivot| / |diagonal| among the kept pivots
// (1 when none is kept).
double dense_ldlt_pseudo(const HostCsr& A, std::vector<double>& linv, std::vector<double>& linvt,
                         std::vector<double>& piv, double tau = 1e-13);

struct AmgHostLevel {
    HostCsr A, P, Pt;
    std::vector<double> l1;
    bool direct = false;          // coarsest: solved through the dense LDL^T pseudo-inverse
    std::vector<double> linv;     // n x n row-major L^{-1} (unit lower; direct only)
    std::vector<double> linvt;    // its transpose
    std::vector<double> piv;      // D, dropped pivots as 0
    double piv_min = 1.0;         // smallest kept |pivot| / |diagonal| (direct only)
};

struct AmgHost {
    double theta = 0.25;
    int max_levels = 25, min_coarse = 500, num_smooth = 1;
    std::vector<AmgHostLevel> levels;
    void setup(const HostCsr& A0);
};

struct AmsHost {
    int nhc = 0, nh1 = 0;
    HostCsr A_bc, G, Gt, Pi[3], Pit[3];
    std::vector<double> fine_l1;
    AmgHost amg[4];  // 0 = gradient space, 1..3 = Nedelec interpolation x, y, z
    double theta = 0.25;
    // Geometry (Pi from G and the vertex coordinates), once.
    void setup_geometry(const HostCsr& grad, const double* cx, const double* cy, const double* cz);
    // Matrix part: A_bc, Galerkin products, AMG hierarchies, fine l1 norms.
    void rebuild(const HostCsr& A, const uint8_t* freedofs);
};

}  // namespace ssv
