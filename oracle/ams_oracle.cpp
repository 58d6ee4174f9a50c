// ams_oracle.cpp -- TEST INFRASTRUCTURE: CPU restatement of the reference's
// Compact AMG / Compact AMS / ComplexCompactAMS preconditioners
// (include/sparsesolv/preconditioners/compact_amg.hpp, compact_ams.hpp,
// complex_compact_ams.hpp), which need NGSolve and cannot be compiled here.
// The NGSolve primitives they call are re-derived: SparseMatrix::Restrict
// (P^T A P with the structural product pattern, explicit zeros kept, columns
// sorted), CreateTranspose, Mult/MultAdd (row loops), SPARSECHOLESKY (an exact
// dense Cholesky solve of the small coarsest matrix). Agreement with NGSolve
// itself cannot be checked in this image ("parity unpinned" for the AMS part).
// Serial test infrastructure: used only by tests/ and bench.py's CPU-baseline leg, to check results.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif
#include <random>
#include <string>
#include <vector>

#include "../include/sparsesolv_b200.h"

namespace {

struct Csr {
    int n = 0, m = 0;
    std::vector<int> rp, ci;
    std::vector<double> v;
    int nnz() const { return rp.empty() ? 0 : rp[n]; }
};

Csr make_csr(int n, int m, const int* rp, const int* ci, const double* v) {
    Csr A;
    A.n = n; A.m = m;
    A.rp.assign(rp, rp + n + 1);
    A.ci.assign(ci, ci + rp[n]);
    A.v.assign(v, v + rp[n]);
    return A;
}

// CreateTranspose: entries of row i appended to rows col in ascending i
Csr transpose(const Csr& A) {
    Csr T;
    T.n = A.m; T.m = A.n;
    T.rp.assign(A.m + 1, 0);
    for (int k = 0; k < A.nnz(); ++k) T.rp[A.ci[k] + 1]++;
    for (int i = 0; i < A.m; ++i) T.rp[i + 1] += T.rp[i];
    T.ci.resize(A.nnz());
    T.v.resize(A.nnz());
    std::vector<int> pos(T.rp.begin(), T.rp.end() - 1);
    for (int i = 0; i < A.n; ++i)
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
            const int p = pos[A.ci[k]]++;
            T.ci[p] = i;
            T.v[p] = A.v[k];
        }
    return T;
}

// Restrict(P) = P^T A P: pattern = all (k,l) with k in P row i, l in P row j
// for an entry (i,j) of A; value sum over those products.
Csr restrict_rap(const Csr& A, const Csr& P) {
    const int nc = P.m;
    Csr Pt = transpose(P);
    // (P^T A) row k = sum over i in Pt row k of Pt(k,i) * A row i; then * P
    std::vector<double> acc(nc, 0.0);
    std::vector<int> mark(nc, -1), cols;
    Csr C;
    C.n = nc; C.m = nc;
    C.rp.assign(nc + 1, 0);
    for (int k = 0; k < nc; ++k) {
        cols.clear();
        for (int q = Pt.rp[k]; q < Pt.rp[k + 1]; ++q) {
            const int i = Pt.ci[q];
            const double pki = Pt.v[q];
            for (int a = A.rp[i]; a < A.rp[i + 1]; ++a) {
                const int j = A.ci[a];
                const double pa = pki * A.v[a];
                for (int b = P.rp[j]; b < P.rp[j + 1]; ++b) {
                    const int l = P.ci[b];
                    if (mark[l] != k) { mark[l] = k; acc[l] = 0.0; cols.push_back(l); }
                    acc[l] += pa * P.v[b];
                }
            }
        }
        std::sort(cols.begin(), cols.end());
        for (int l : cols) { C.ci.push_back(l); C.v.push_back(acc[l]); }
        C.rp[k + 1] = (int)C.ci.size();
    }
    return C;
}

// y = A x
void mult(const Csr& A, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < A.n; ++i) {
        double s = 0.0;
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) s += A.v[k] * x[A.ci[k]];
        y[i] = s;
    }
}

// y += s * A x (NGSolve MultAdd)
void mult_add(const Csr& A, double s, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < A.n; ++i) {
        double t = 0.0;
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) t += A.v[k] * x[A.ci[k]];
        y[i] += s * t;
    }
}

// CreateBCModifiedMatrix (compact_amg.hpp:252-287, compact_ams.hpp:605-633)
Csr bc_modified(const Csr& A, const unsigned char* fd) {
    Csr B = A;
    for (int i = 0; i < A.n; ++i)
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
            const int j = A.ci[k];
            if (!fd[i]) B.v[k] = (j == i) ? 1.0 : 0.0;
            else if (!fd[j]) B.v[k] = 0.0;
        }
    return B;
}

// Solve with the small coarsest matrix (stands in for SPARSECHOLESKY).
// Dense LDL^T; a pivot below 1e-13 of its row's diagonal is treated as zero
// and its component set to zero. The gradient-space Galerkin matrix
// G^T A_bc G is singular (constants are in the kernel of G), so its coarsest
// level meets a rounding-sized pivot; the dropped component is one that G
// (and constant-preserving interpolation) maps to nothing.
struct DenseChol {
    int n = 0;
    std::vector<double> L, d;
    void factor(const Csr& A) {
        n = A.n;
        L.assign((size_t)n * n, 0.0);
        d.assign(n, 0.0);
        for (int i = 0; i < n; ++i)
            for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) L[(size_t)i * n + A.ci[k]] += A.v[k];
        std::vector<double> diag0(n);
        for (int i = 0; i < n; ++i) diag0[i] = std::abs(L[(size_t)i * n + i]);
        std::vector<double> w(n);
        for (int j = 0; j < n; ++j) {
            for (int k = 0; k < j; ++k) w[k] = L[(size_t)j * n + k] * d[k];
            double dj = L[(size_t)j * n + j];
            for (int k = 0; k < j; ++k) dj -= L[(size_t)j * n + k] * w[k];
            const bool zero = !(std::abs(dj) > 1e-13 * diag0[j]);
            d[j] = zero ? 0.0 : dj;
            L[(size_t)j * n + j] = 1.0;
            for (int i = j + 1; i < n; ++i) {
                double s = L[(size_t)i * n + j];
                for (int k = 0; k < j; ++k) s -= L[(size_t)i * n + k] * w[k];
                L[(size_t)i * n + j] = zero ? 0.0 : s / dj;
            }
        }
    }
    void solve(const double* b, double* x) const {
        std::vector<double> y(n);
        for (int i = 0; i < n; ++i) {
            double s = b[i];
            for (int k = 0; k < i; ++k) s -= L[(size_t)i * n + k] * y[k];
            y[i] = s;
        }
        for (int i = 0; i < n; ++i) y[i] = d[i] != 0.0 ? y[i] / d[i] : 0.0;
        for (int i = n - 1; i >= 0; --i) {
            double s = y[i];
            for (int k = i + 1; k < n; ++k) s -= L[(size_t)k * n + i] * x[k];
            x[i] = s;
        }
    }
};

// ---------------------------------------------------------------------------
// CompactAMG (compact_amg.hpp)
// ---------------------------------------------------------------------------
struct Graph {
    int n = 0;
    std::vector<int> rp, ci;
};

struct AmgLevel {
    Csr A, P, Pt;
    std::vector<double> l1;
    bool has_inv = false;
    DenseChol inv;
};

struct Amg {
    double theta = 0.25;
    int max_levels = 25, min_coarse = 50, num_smooth = 1;
    std::vector<AmgLevel> lv;

    // ComputeStrength (:292-372)
    static Graph strength(const Csr& A, double theta) {
        Graph S;
        S.n = A.n;
        S.rp.assign(A.n + 1, 0);
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1) S.ci.resize(S.rp[A.n]);
            for (int i = 0; i < A.n; ++i) {
                double max_neg = 0, max_abs = 0;
                for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
                    if (A.ci[k] != i) {
                        const double v = A.v[k];
                        if (-v > max_neg) max_neg = -v;
                        const double av = std::abs(v);
                        if (av > max_abs) max_abs = av;
                    }
                const double ref = (max_neg > 0) ? max_neg : max_abs;
                const double thr = theta * ref;
                int cnt = 0, pos = pass ? S.rp[i] : 0;
                for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
                    if (A.ci[k] != i) {
                        const bool strong = (max_neg > 0) ? (-A.v[k] >= thr) : (std::abs(A.v[k]) >= thr);
                        if (strong) {
                            if (pass) S.ci[pos++] = A.ci[k];
                            else cnt++;
                        }
                    }
                if (!pass) S.rp[i + 1] = cnt;
            }
            if (pass == 0)
                for (int i = 0; i < A.n; ++i) S.rp[i + 1] += S.rp[i];
        }
        return S;
    }

    // TransposeGraph (:457-483)
    static Graph transpose_graph(const Graph& G) {
        Graph T;
        T.n = G.n;
        T.rp.assign(G.n + 1, 0);
        for (int i = 0; i < G.n; ++i)
            for (int k = G.rp[i]; k < G.rp[i + 1]; ++k) T.rp[G.ci[k] + 1]++;
        for (int i = 0; i < G.n; ++i) T.rp[i + 1] += T.rp[i];
        T.ci.resize(T.rp[G.n]);
        std::vector<int> pos(G.n, 0);
        for (int i = 0; i < G.n; ++i)
            for (int k = G.rp[i]; k < G.rp[i + 1]; ++k) {
                const int j = G.ci[k];
                T.ci[T.rp[j] + pos[j]++] = i;
            }
        return T;
    }

    // CoarsenPMIS (:378-454)
    static std::vector<int> pmis(const Graph& S) {
        const int n = S.n;
        std::vector<int> cf(n, -1);
        Graph St = transpose_graph(S);
        std::vector<double> measure(n);
        std::mt19937 rng(42);
        std::uniform_real_distribution<double> dist(0.0, 1.0);
        for (int i = 0; i < n; ++i) measure[i] = (double)(St.rp[i + 1] - St.rp[i]) + dist(rng);
        for (int iter = 0; iter < 100; ++iter) {
            bool changed = false;
            std::vector<int> new_c;
            for (int i = 0; i < n; ++i) {
                if (cf[i] != -1) continue;
                bool is_max = true;
                for (int k = S.rp[i]; k < S.rp[i + 1]; ++k) {
                    const int j = S.ci[k];
                    if (cf[j] == -1 && measure[j] > measure[i]) { is_max = false; break; }
                }
                if (is_max)
                    for (int k = St.rp[i]; k < St.rp[i + 1]; ++k) {
                        const int j = St.ci[k];
                        if (cf[j] == -1 && measure[j] > measure[i]) { is_max = false; break; }
                    }
                if (is_max) { cf[i] = 1; new_c.push_back(i); changed = true; }
            }
            for (int i : new_c) {
                for (int k = S.rp[i]; k < S.rp[i + 1]; ++k)
                    if (cf[S.ci[k]] == -1) { cf[S.ci[k]] = 0; changed = true; }
                for (int k = St.rp[i]; k < St.rp[i + 1]; ++k)
                    if (cf[St.ci[k]] == -1) { cf[St.ci[k]] = 0; changed = true; }
            }
            if (!changed) break;
        }
        for (int i = 0; i < n; ++i)
            if (cf[i] == -1) cf[i] = 1;
        return cf;
    }

    // BuildClassicalInterp (:488-612)
    static Csr interp(const Csr& A, const Graph& S, const std::vector<int>& cf, int nc) {
        const int nf = A.n;
        std::vector<int> cidx(nf, -1);
        int c = 0;
        for (int i = 0; i < nf; ++i)
            if (cf[i] == 1) cidx[i] = c++;
        std::vector<char> strong(A.nnz(), 0);
        for (int i = 0; i < nf; ++i)
            for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
                for (int q = S.rp[i]; q < S.rp[i + 1]; ++q)
                    if (S.ci[q] == A.ci[k]) { strong[k] = 1; break; }
        Csr P;
        P.n = nf; P.m = nc;
        P.rp.assign(nf + 1, 0);
        for (int i = 0; i < nf; ++i) {
            int cnt = 0;
            if (cf[i] == 1) cnt = 1;
            else {
                for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
                    if (strong[k] && cf[A.ci[k]] == 1) cnt++;
                if (cnt == 0) cnt = 1;
            }
            P.rp[i + 1] = P.rp[i] + cnt;
        }
        P.ci.assign(P.rp[nf], 0);
        P.v.assign(P.rp[nf], 0.0);
        for (int i = 0; i < nf; ++i) {
            const int p0 = P.rp[i];
            if (cf[i] == 1) { P.ci[p0] = cidx[i]; P.v[p0] = 1.0; continue; }
            double aii = 0;
            for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
                if (A.ci[k] == i) { aii = A.v[k]; break; }
            double sum_non = 0;
            for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
                if (A.ci[k] == i) continue;
                if (strong[k] && cf[A.ci[k]] == 1) continue;
                sum_non += A.v[k];
            }
            double denom = aii + sum_non;
            if (std::abs(denom) < 1e-30) denom = 1.0;
            int pos = 0;
            for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
                if (strong[k] && cf[A.ci[k]] == 1) {
                    P.ci[p0 + pos] = cidx[A.ci[k]];
                    P.v[p0 + pos] = -A.v[k] / denom;
                    pos++;
                }
            if (pos == 0) {
                int best_c = -1;
                double best_val = 0;
                for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
                    if (cf[A.ci[k]] == 1 && std::abs(A.v[k]) > best_val) {
                        best_val = std::abs(A.v[k]);
                        best_c = cidx[A.ci[k]];
                    }
                if (best_c >= 0) { P.ci[p0] = best_c; P.v[p0] = 1.0; }
                else { P.ci[p0] = 0; P.v[p0] = 0.0; }
            }
        }
        return P;
    }

    // ComputeL1Norms (:621-632): plain l1 row sums
    static void l1norms(const Csr& A, std::vector<double>& out) {
        out.resize(A.n);
        for (int i = 0; i < A.n; ++i) {
            double s = 0;
            for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) s += std::abs(A.v[k]);
            out[i] = (s > 0) ? s : 1.0;
        }
    }

    // Setup (:66-156), freedofs = nullptr (the AMS subspace use)
    void setup(const Csr& A0) {
        lv.clear();
        lv.emplace_back();
        lv[0].A = A0;
        l1norms(lv[0].A, lv[0].l1);
        for (int l = 0; l < max_levels - 1; ++l) {
            if (lv[l].A.n <= min_coarse) break;
            Graph S = strength(lv[l].A, theta);
            std::vector<int> cf = pmis(S);
            int nc = 0;
            for (int i = 0; i < lv[l].A.n; ++i) nc += (cf[i] == 1);
            if (nc == 0 || nc >= lv[l].A.n) break;
            Csr P = interp(lv[l].A, S, cf, nc);
            Csr Pt = transpose(P);
            Csr Ac = restrict_rap(lv[l].A, P);
            lv[l].P = std::move(P);
            lv[l].Pt = std::move(Pt);
            lv.emplace_back();
            lv.back().A = std::move(Ac);
            l1norms(lv.back().A, lv.back().l1);
        }
        AmgLevel& co = lv.back();
        if (co.A.n <= min_coarse * 10) {
            co.inv.factor(co.A);
            co.has_inv = true;
        }
    }

    // L1JacobiSmooth (:642-657): x_i += r_i / l1_i
    void smooth(int l, const double* b, double* x) const {
        const AmgLevel& L = lv[l];
        std::vector<double> r(b, b + L.A.n);
        mult_add(L.A, -1.0, x, r.data());
#pragma omp parallel for schedule(static)
        for (int i = 0; i < L.A.n; ++i) x[i] += r[i] / L.l1[i];
    }

    // VCycle (:801-841)
    void vcycle(int l, const double* b, double* x) const {
        const AmgLevel& L = lv[l];
        if (l == (int)lv.size() - 1) {
            if (L.has_inv) L.inv.solve(b, x);
            else for (int s = 0; s < 10; ++s) smooth(l, b, x);
            return;
        }
        for (int s = 0; s < num_smooth; ++s) smooth(l, b, x);
        std::vector<double> res(b, b + L.A.n);
        mult_add(L.A, -1.0, x, res.data());
        const int nc = lv[l + 1].A.n;
        std::vector<double> rc(nc), ec(nc, 0.0);
        mult(L.Pt, res.data(), rc.data());
        vcycle(l + 1, rc.data(), ec.data());
        mult_add(L.P, 1.0, ec.data(), x);
        for (int s = 0; s < num_smooth; ++s) smooth(l, b, x);
    }

    void apply(const double* b, double* x) const {
        std::fill(x, x + lv[0].A.n, 0.0);
        vcycle(0, b, x);
    }

    // DualL1JacobiSmooth (:709-729): x_i += r_i * (1 / l1_i)
    void dual_smooth(int l, const double* b1, double* x1, const double* b2, double* x2) const {
        const AmgLevel& L = lv[l];
        std::vector<double> r1(L.A.n), r2(L.A.n);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < L.A.n; ++i) {
            double d1 = 0, d2 = 0;
            for (int k = L.A.rp[i]; k < L.A.rp[i + 1]; ++k) {
                d1 += L.A.v[k] * x1[L.A.ci[k]];
                d2 += L.A.v[k] * x2[L.A.ci[k]];
            }
            r1[i] = b1[i] - d1;
            r2[i] = b2[i] - d2;
        }
#pragma omp parallel for schedule(static)
        for (int i = 0; i < L.A.n; ++i) {
            const double inv = 1.0 / L.l1[i];
            x1[i] += r1[i] * inv;
            x2[i] += r2[i] * inv;
        }
    }

    // DualVCycle (:662-706)
    void dual_vcycle(int l, const double* b1, double* x1, const double* b2, double* x2) const {
        const AmgLevel& L = lv[l];
        if (l == (int)lv.size() - 1) {
            if (L.has_inv) { L.inv.solve(b1, x1); L.inv.solve(b2, x2); }
            else for (int s = 0; s < 10; ++s) dual_smooth(l, b1, x1, b2, x2);
            return;
        }
        for (int s = 0; s < num_smooth; ++s) dual_smooth(l, b1, x1, b2, x2);
        const int n = L.A.n, nc = lv[l + 1].A.n;
        std::vector<double> r1(n), r2(n);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            double d1 = 0, d2 = 0;
            for (int k = L.A.rp[i]; k < L.A.rp[i + 1]; ++k) {
                d1 += L.A.v[k] * x1[L.A.ci[k]];
                d2 += L.A.v[k] * x2[L.A.ci[k]];
            }
            r1[i] = b1[i] - d1;
            r2[i] = b2[i] - d2;
        }
        std::vector<double> c1(nc), c2(nc), e1(nc, 0.0), e2(nc, 0.0);
        mult(L.Pt, r1.data(), c1.data());
        mult(L.Pt, r2.data(), c2.data());
        dual_vcycle(l + 1, c1.data(), e1.data(), c2.data(), e2.data());
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
            double s1 = 0, s2 = 0;
            for (int k = L.P.rp[i]; k < L.P.rp[i + 1]; ++k) {
                s1 += L.P.v[k] * e1[L.P.ci[k]];
                s2 += L.P.v[k] * e2[L.P.ci[k]];
            }
            x1[i] += s1;
            x2[i] += s2;
        }
        for (int s = 0; s < num_smooth; ++s) dual_smooth(l, b1, x1, b2, x2);
    }

    void dual_apply(const double* b1, double* x1, const double* b2, double* x2) const {
        std::fill(x1, x1 + lv[0].A.n, 0.0);
        std::fill(x2, x2 + lv[0].A.n, 0.0);
        dual_vcycle(0, b1, x1, b2, x2);
    }
};

// ---------------------------------------------------------------------------
// CompactAMS (compact_ams.hpp)
// ---------------------------------------------------------------------------
struct Ams {
    Csr mat, A_bc, G, Gt, Pi[3], Pit[3];
    std::vector<unsigned char> fd;
    bool has_fd = false;
    int nhc = 0, nh1 = 0, cycle_type = 1, num_smooth = 1;
    double theta = 0.25, w = 1.0;
    Amg B_G, B_Pi[3];
    std::vector<double> l1;

    // BuildPiComponents (:454-504) + transposes (:276-294)
    void setup_geometry(const double* cx, const double* cy, const double* cz) {
        const double* cs[3] = {cx, cy, cz};
        for (int d = 0; d < 3; ++d) {
            Pi[d] = G;
            for (int e = 0; e < G.n; ++e) {
                double gd = 0;
                for (int k = G.rp[e]; k < G.rp[e + 1]; ++k) gd += G.v[k] * cs[d][G.ci[k]];
                for (int k = G.rp[e]; k < G.rp[e + 1]; ++k) Pi[d].v[k] = std::abs(G.v[k]) * 0.5 * gd;
            }
        }
        Gt = transpose(G);
        for (int d = 0; d < 3; ++d) Pit[d] = transpose(Pi[d]);
    }

    // FixZeroRows (:638-659)
    static void fix_zero_rows(Csr& A) {
        for (int i = 0; i < A.n; ++i) {
            double l1n = 0;
            int dp = -1;
            for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
                l1n += std::abs(A.v[k]);
                if (A.ci[k] == i) dp = k;
            }
            if (l1n == 0.0 && dp >= 0) A.v[dp] = 1.0;
        }
    }

    // RebuildMatrix (:300-421)
    void rebuild() {
        A_bc = has_fd ? bc_modified(mat, fd.data()) : mat;
        Csr AG = restrict_rap(A_bc, G);
        Csr AP[3];
        for (int d = 0; d < 3; ++d) AP[d] = restrict_rap(A_bc, Pi[d]);
        fix_zero_rows(AG);
        for (int d = 0; d < 3; ++d) fix_zero_rows(AP[d]);
        B_G = Amg();
        B_G.theta = theta; B_G.max_levels = 25; B_G.min_coarse = 500; B_G.num_smooth = 1;
        B_G.setup(AG);
        for (int d = 0; d < 3; ++d) {
            B_Pi[d] = Amg();
            B_Pi[d].theta = theta; B_Pi[d].max_levels = 25; B_Pi[d].min_coarse = 500; B_Pi[d].num_smooth = 1;
            B_Pi[d].setup(AP[d]);
        }
        l1.resize(nhc);
        for (int i = 0; i < nhc; ++i) {
            double diag = 0, off = 0;
            for (int k = A_bc.rp[i]; k < A_bc.rp[i + 1]; ++k) {
                if (A_bc.ci[k] == i) diag = std::abs(A_bc.v[k]);
                else off += std::abs(A_bc.v[k]);
            }
            const double t = diag + 0.5 * off;
            if (t <= (4.0 / 3.0) * diag) l1[i] = (diag > 0) ? diag : 1.0;
            else l1[i] = (t > 0) ? t : 1.0;
        }
    }

    void residual(const double* b, const double* x, double* r) const {
        std::copy(b, b + nhc, r);
        mult_add(A_bc, -1.0, x, r);
    }

    void fine_smooth(const double* b, double* x) const {  // :525-542
        std::vector<double> r(nhc);
        for (int s = 0; s < num_smooth; ++s) {
            residual(b, x, r.data());
#pragma omp parallel for schedule(static)
            for (int i = 0; i < nhc; ++i) x[i] += r[i] / l1[i];
        }
    }

    void gradient_correct(const double* b, double* x) const {  // :547-574
        std::vector<double> r(nhc), rg(nh1), gg(nh1, 0.0);
        residual(b, x, r.data());
        mult(Gt, r.data(), rg.data());
        B_G.apply(rg.data(), gg.data());
        mult_add(G, w, gg.data(), x);
    }

    void nodal_correct(const double* b, double* x) const {  // :576-599
        std::vector<double> r(nhc), rp[3], gp[3];
        residual(b, x, r.data());
        for (int d = 0; d < 3; ++d) { rp[d].resize(nh1); gp[d].assign(nh1, 0.0); mult(Pit[d], r.data(), rp[d].data()); }
        for (int d = 0; d < 3; ++d) B_Pi[d].apply(rp[d].data(), gp[d].data());
        for (int d = 0; d < 3; ++d) mult_add(Pi[d], w, gp[d].data(), x);
    }

    // Mult (:136-195)
    void apply(const double* b, double* x) const {
        std::vector<double> b0(b, b + nhc);
        if (has_fd) for (int i = 0; i < nhc; ++i) if (!fd[i]) b0[i] = 0;
        std::fill(x, x + nhc, 0.0);
        if (cycle_type == 7) {
            fine_smooth(b0.data(), x); gradient_correct(b0.data(), x); fine_smooth(b0.data(), x);
            nodal_correct(b0.data(), x); fine_smooth(b0.data(), x); gradient_correct(b0.data(), x);
            fine_smooth(b0.data(), x);
        } else {
            fine_smooth(b0.data(), x); gradient_correct(b0.data(), x); nodal_correct(b0.data(), x);
            gradient_correct(b0.data(), x); fine_smooth(b0.data(), x);
        }
        if (has_fd) for (int i = 0; i < nhc; ++i) if (!fd[i]) x[i] = 0;
    }

    // ComplexCompactAMS (complex_compact_ams.hpp:112-341): fused Re/Im passes
    void fused_residual(const double* br, const double* xr, double* rr, const double* bi, const double* xi,
                        double* ri) const {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < nhc; ++i) {
            double d1 = 0, d2 = 0;
            for (int k = A_bc.rp[i]; k < A_bc.rp[i + 1]; ++k) {
                d1 += A_bc.v[k] * xr[A_bc.ci[k]];
                d2 += A_bc.v[k] * xi[A_bc.ci[k]];
            }
            rr[i] = br[i] - d1;
            ri[i] = bi[i] - d2;
        }
    }
    void fused_smooth(const double* br, double* xr, const double* bi, double* xi) const {
        std::vector<double> rr(nhc), ri(nhc);
        for (int s = 0; s < num_smooth; ++s) {
            fused_residual(br, xr, rr.data(), bi, xi, ri.data());
#pragma omp parallel for schedule(static)
            for (int i = 0; i < nhc; ++i) {
                const double inv = 1.0 / l1[i];
                xr[i] += rr[i] * inv;
                xi[i] += ri[i] * inv;
            }
        }
    }
    static void fused_prolong(const Csr& P, double w, const double* gr, double* xr, const double* gi, double* xi) {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < P.n; ++i) {
            double s1 = 0, s2 = 0;
            for (int k = P.rp[i]; k < P.rp[i + 1]; ++k) {
                s1 += P.v[k] * gr[P.ci[k]];
                s2 += P.v[k] * gi[P.ci[k]];
            }
            xr[i] += w * s1;
            xi[i] += w * s2;
        }
    }
    void fused_gradient(const double* br, double* xr, const double* bi, double* xi) const {
        std::vector<double> rr(nhc), ri(nhc), cr(nh1), ci(nh1), gr(nh1), gi(nh1);
        fused_residual(br, xr, rr.data(), bi, xi, ri.data());
        mult(Gt, rr.data(), cr.data());
        mult(Gt, ri.data(), ci.data());
        B_G.dual_apply(cr.data(), gr.data(), ci.data(), gi.data());
        fused_prolong(G, w, gr.data(), xr, gi.data(), xi);
    }
    void fused_nodal(const double* br, double* xr, const double* bi, double* xi) const {
        std::vector<double> rr(nhc), ri(nhc);
        fused_residual(br, xr, rr.data(), bi, xi, ri.data());
        std::vector<double> cr[3], ci[3], gr[3], gi[3];
        for (int d = 0; d < 3; ++d) {
            cr[d].resize(nh1); ci[d].resize(nh1); gr[d].resize(nh1); gi[d].resize(nh1);
            mult(Pit[d], rr.data(), cr[d].data());
            mult(Pit[d], ri.data(), ci[d].data());
        }
        for (int d = 0; d < 3; ++d) B_Pi[d].dual_apply(cr[d].data(), gr[d].data(), ci[d].data(), gi[d].data());
        for (int d = 0; d < 3; ++d) fused_prolong(Pi[d], w, gr[d].data(), xr, gi[d].data(), xi);
    }
    void apply_complex(const std::complex<double>* f, std::complex<double>* u) const {
        std::vector<double> br(nhc), bi(nhc), xr(nhc, 0.0), xi(nhc, 0.0);
        for (int i = 0; i < nhc; ++i) {
            const bool free = !has_fd || fd[i];
            br[i] = free ? f[i].real() : 0.0;
            bi[i] = free ? f[i].imag() : 0.0;
        }
        if (cycle_type == 7) {
            fused_smooth(br.data(), xr.data(), bi.data(), xi.data());
            fused_gradient(br.data(), xr.data(), bi.data(), xi.data());
            fused_smooth(br.data(), xr.data(), bi.data(), xi.data());
            fused_nodal(br.data(), xr.data(), bi.data(), xi.data());
            fused_smooth(br.data(), xr.data(), bi.data(), xi.data());
            fused_gradient(br.data(), xr.data(), bi.data(), xi.data());
            fused_smooth(br.data(), xr.data(), bi.data(), xi.data());
        } else {
            fused_smooth(br.data(), xr.data(), bi.data(), xi.data());
            fused_gradient(br.data(), xr.data(), bi.data(), xi.data());
            fused_nodal(br.data(), xr.data(), bi.data(), xi.data());
            fused_gradient(br.data(), xr.data(), bi.data(), xi.data());
            fused_smooth(br.data(), xr.data(), bi.data(), xi.data());
        }
        for (int i = 0; i < nhc; ++i) {
            const bool free = !has_fd || fd[i];
            u[i] = free ? std::complex<double>(xr[i], xi[i]) : std::complex<double>(0.0, 0.0);
        }
    }
};

thread_local std::string g_err;

}  // namespace

extern "C" {

const char* ams_oracle_last_error(void) { return g_err.c_str(); }

// Host threads of the row-parallel loops (SpMV, smoothers, transfers); the
// dot products stay sequential, so results do not depend on the count.
void ams_oracle_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : 1);
#else
    (void)n;
#endif
}

// CompactAMS / ComplexCompactAMS constructor: A (n_hc x n_hc), G (n_hc x
// n_h1), freedofs (NULL = all free), vertex coordinates (n_h1 each).
void* ams_oracle_create(int nhc, const int* arp, const int* aci, const double* av, int nh1, const int* grp,
                        const int* gci, const double* gv, const unsigned char* fd, const double* cx,
                        const double* cy, const double* cz, int cycle_type, int num_smooth, double theta,
                        double correction_weight) {
    Ams* a = new Ams();
    a->nhc = nhc;
    a->nh1 = nh1;
    a->mat = make_csr(nhc, nhc, arp, aci, av);
    a->G = make_csr(nhc, nh1, grp, gci, gv);
    a->has_fd = fd != nullptr;
    if (fd) a->fd.assign(fd, fd + nhc);
    a->cycle_type = cycle_type;
    a->num_smooth = num_smooth;
    a->theta = theta;
    a->w = correction_weight;
    a->setup_geometry(cx, cy, cz);
    a->rebuild();
    if (a->w <= 0.0) a->w = 1.0;
    return a;
}

// Update(new values, same pattern)
void ams_oracle_update(void* h, const double* av) {
    Ams* a = static_cast<Ams*>(h);
    std::copy(av, av + a->mat.nnz(), a->mat.v.begin());
    a->rebuild();
}

void ams_oracle_destroy(void* h) { delete static_cast<Ams*>(h); }

void ams_oracle_apply(void* h, const double* b, double* x) { static_cast<Ams*>(h)->apply(b, x); }

void ams_oracle_apply_complex(void* h, const double* f, double* u) {
    static_cast<Ams*>(h)->apply_complex(reinterpret_cast<const std::complex<double>*>(f),
                                        reinterpret_cast<std::complex<double>*>(u));
}

// CompactAMGPreconditioner (compact_amg.hpp:49-183): Setup on the FreeDofs
// view (CreateBCModifiedMatrix, :72-79) and Mult = x = 0, VCycle, constrained
// outputs zeroed (:166-183).
struct AmgOnly {
    Amg amg;
    std::vector<unsigned char> fd;
};

void* ams_oracle_amg_create(int n, const int* rp, const int* ci, const double* v, const unsigned char* fd,
                            double theta, int max_levels, int min_coarse, int num_smooth) {
    AmgOnly* g = new AmgOnly();
    Csr A = make_csr(n, n, rp, ci, v);
    if (fd) {
        g->fd.assign(fd, fd + n);
        A = bc_modified(A, fd);
    }
    g->amg.theta = theta;
    g->amg.max_levels = max_levels;
    g->amg.min_coarse = min_coarse;
    g->amg.num_smooth = num_smooth;
    g->amg.setup(A);
    return g;
}

void ams_oracle_amg_apply(void* h, const double* b, double* x) {
    AmgOnly* g = static_cast<AmgOnly*>(h);
    g->amg.apply(b, x);
    if (!g->fd.empty())
        for (size_t i = 0; i < g->fd.size(); ++i)
            if (!g->fd[i]) x[i] = 0.0;
}

int ams_oracle_amg_levels(void* h, int* sizes, int cap) {
    const Amg& m = static_cast<AmgOnly*>(h)->amg;
    const int nl = (int)m.lv.size();
    for (int l = 0; l < nl && 2 * l + 1 < cap; ++l) {
        sizes[2 * l] = m.lv[l].A.n;
        sizes[2 * l + 1] = m.lv[l].A.nnz();
    }
    return nl;
}

void ams_oracle_amg_destroy(void* h) { delete static_cast<AmgOnly*>(h); }

// Hierarchy shape: for subspace s (0 = G, 1..3 = Pi x,y,z) the number of
// levels, and per level (rows, nnz) into sizes[2*l], sizes[2*l+1].
int ams_oracle_levels(void* h, int s, int* sizes, int cap) {
    Ams* a = static_cast<Ams*>(h);
    const Amg& m = (s == 0) ? a->B_G : a->B_Pi[s - 1];
    const int nl = (int)m.lv.size();
    for (int l = 0; l < nl && 2 * l + 1 < cap; ++l) {
        sizes[2 * l] = m.lv[l].A.n;
        sizes[2 * l + 1] = m.lv[l].A.nnz();
    }
    return nl;
}

// Level matrices and interpolation of one subspace AMG (for parity checks):
// what = 0 A, 1 P; copies row_ptr / col_idx / values when the buffers fit.
int ams_oracle_level_matrix(void* h, int s, int l, int what, int* rp, int* ci, double* v, int cap) {
    Ams* a = static_cast<Ams*>(h);
    const Amg& m = (s == 0) ? a->B_G : a->B_Pi[s - 1];
    const Csr& M = what == 0 ? m.lv[l].A : m.lv[l].P;
    if (M.nnz() > cap) return M.nnz();
    std::copy(M.rp.begin(), M.rp.end(), rp);
    std::copy(M.ci.begin(), M.ci.end(), ci);
    std::copy(M.v.begin(), M.v.end(), v);
    return M.nnz();
}

// sparsesolv::CGSolver (solvers/cg_solver.hpp:64-146 + iterative_solver.hpp)
// with this AMS as the preconditioner, on A with the FreeDofs rule
// (identity rows) -- the CG-with-external-preconditioner entry of the AMS
// configurations. x is the initial guess (constrained entries kept).
int ams_oracle_pcg(void* h, const double* b, double* x, const ssv_config* cfg, ssv_result* res, double* hist,
                   int hist_cap) {
    Ams* a = static_cast<Ams*>(h);
    const int n = a->nhc;
    const Csr& A = a->A_bc;
    std::vector<double> bm(b, b + n), xm(x, x + n);
    if (a->has_fd)
        for (int i = 0; i < n; ++i)
            if (!a->fd[i]) { bm[i] = 0; xm[i] = 0; }
    std::vector<double> r(n), z(n), p(n), Ap(n), best;
    double best_res = 1.7976931348623157e308;
    if (cfg->save_best_result) best.assign(n, 0.0);
    mult(A, xm.data(), r.data());
    for (int i = 0; i < n; ++i) r[i] = bm[i] - r[i];
    auto nrm = [&](const std::vector<double>& v) { double s = 0; for (double t : v) s += t * t; return std::sqrt(s); };
    const double nb = nrm(bm), nr0 = nrm(r);
    double normalizer = cfg->norm_type == SSV_NORM_RHS ? nb : cfg->norm_type == SSV_NORM_INITIAL_RESIDUAL ? nr0 : cfg->custom_norm;
    if (normalizer < 1e-15) normalizer = 1.0;
    int hl = 0;
    auto push = [&](double v) { if (hist && hl < hist_cap) hist[hl] = v; hl++; };
    if (cfg->save_residual_history) push(nr0 / normalizer);
    int bad = 0;
    auto check = [&](double nr_) {
        const double rel = nr_ / normalizer;
        if (cfg->save_residual_history) push(rel);
        if (cfg->save_best_result && rel < best_res) { best_res = rel; best = xm; }
        if (rel < cfg->tolerance || nr_ < cfg->abs_tolerance) return true;
        if (cfg->divergence_check) {
            if (rel >= best_res * cfg->divergence_threshold) bad++; else bad = 0;
        }
        return false;
    };
    auto finish = [&](bool conv, int it, double fn) {
        std::memset(res, 0, sizeof(*res));
        res->converged = conv;
        res->iterations = it;
        res->final_residual = fn / normalizer;
        if (!conv && cfg->save_best_result) { xm = best; res->final_residual = best_res; }
        res->history_total = cfg->save_residual_history ? hl : 0;
        res->history_len = std::min(res->history_total, hist_cap);
        for (int i = 0; i < n; ++i) if (!a->has_fd || a->fd[i]) x[i] = xm[i];
        return 0;
    };
    a->apply(r.data(), z.data());
    double rz = 0;
    for (int i = 0; i < n; ++i) rz += r[i] * z[i];
    p = z;
    for (int it = 0; it < cfg->max_iterations; ++it) {
        double pAp = 0;
        for (int i = 0; i < n; ++i) {
            double s = 0;
            for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) s += A.v[k] * p[A.ci[k]];
            Ap[i] = s;
            pAp += p[i] * s;
        }
        if (std::abs(pAp) < 1e-30) {
            const double nr_ = nrm(r);
            if (check(nr_)) return finish(true, it + 1, nr_);
            return finish(false, it, nr_);
        }
        const double alpha = rz / pAp;
        double s2 = 0;
        for (int i = 0; i < n; ++i) { xm[i] += alpha * p[i]; r[i] -= alpha * Ap[i]; s2 += r[i] * r[i]; }
        const double nr_ = std::sqrt(s2);
        if (check(nr_)) return finish(true, it + 1, nr_);
        if (cfg->divergence_check && bad >= cfg->divergence_count) return finish(false, it + 1, nr_);
        a->apply(r.data(), z.data());
        double rzn = 0;
        for (int i = 0; i < n; ++i) rzn += r[i] * z[i];
        const double beta = rzn / rz;
        rz = rzn;
        for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    return finish(false, cfg->max_iterations, nrm(r));
}

// COCRSolverNGS::Mult (ngsolve/sparsesolv_solvers.hpp:273-369) on a complex
// A (interleaved CSR values) with ComplexCompactAMS as the preconditioner.
int ams_oracle_cocr(void* h, int n, const int* rp, const int* ci, const double* av, const unsigned char* fd,
                    int maxiter, double tol, const double* rhs, double* sol, int* iterations, double* hist,
                    int hist_cap, int* hist_len) {
    using Z = std::complex<double>;
    Ams* a = static_cast<Ams*>(h);
    const Z* v = reinterpret_cast<const Z*>(av);
    const Z* f = reinterpret_cast<const Z*>(rhs);
    Z* x = reinterpret_cast<Z*>(sol);
    std::vector<Z> r(n), rt(n), p(n), q(n), qt(n), t(n);
    auto spmv = [&](const std::vector<Z>& in, std::vector<Z>& out) {
        for (int i = 0; i < n; ++i) {
            Z s = 0;
            for (int k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * in[ci[k]];
            out[i] = s;
        }
        if (fd) for (int i = 0; i < n; ++i) if (!fd[i]) out[i] = 0;
    };
    auto udot = [&](const std::vector<Z>& x1, const std::vector<Z>& y1) { Z s = 0; for (int i = 0; i < n; ++i) s += x1[i] * y1[i]; return s; };
    for (int i = 0; i < n; ++i) { x[i] = 0; r[i] = (fd && !fd[i]) ? Z(0) : f[i]; }
    double rhs_norm = 0;
    for (int i = 0; i < n; ++i) rhs_norm += std::norm(r[i]);
    rhs_norm = std::sqrt(std::abs(rhs_norm));
    int hl = 0;
    if (rhs_norm < 1e-30) { *iterations = 0; if (hist_len) *hist_len = 0; return 0; }
    a->apply_complex(r.data(), rt.data());
    p = rt;
    spmv(p, q);
    Z rho = udot(rt, q);
    int j = 0;
    for (j = 0; j < maxiter; ++j) {
        a->apply_complex(q.data(), qt.data());
        const Z mu = udot(qt, q);
        if (std::abs(mu) < 1e-30) break;
        const Z alpha = rho / mu;
        for (int i = 0; i < n; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; rt[i] -= alpha * qt[i]; }
        double rr = 0;
        for (int i = 0; i < n; ++i) rr += std::norm(r[i]);
        const double res = std::sqrt(std::abs(rr));
        if (hist && hl < hist_cap) hist[hl] = res / rhs_norm;
        hl++;
        if (res / rhs_norm <= tol) { *iterations = j + 1; if (hist_len) *hist_len = hl; return 0; }
        spmv(rt, t);
        const Z rho_new = udot(rt, t);
        if (std::abs(rho) < 1e-30) break;
        const Z beta = rho_new / rho;
        rho = rho_new;
        for (int i = 0; i < n; ++i) { p[i] = rt[i] + beta * p[i]; q[i] = t[i] + beta * q[i]; }
    }
    *iterations = j;
    if (hist_len) *hist_len = hl;
    return 0;
}

}  // extern "C"
