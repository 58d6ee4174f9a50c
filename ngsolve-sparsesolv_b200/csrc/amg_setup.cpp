// amg_setup.cpp -- see amg_setup.hpp. The coarsening must follow the
// reference step for step (the hierarchy decides the iteration count):
// strength with the max-negative / max-absolute rule, PMIS with the measure
// |S^T_i| + U(0,1) drawn from std::mt19937(42), at most 100 rounds, classical
// direct interpolation with lumping of the non-interpolatory connections and
// the injection fall-back, Galerkin P^T A P, plain l1 row norms.
#include "amg_setup.hpp"
#include "host_threads.hpp"

#include <algorithm>
#include <cmath>
#include <random>
#include <thread>
#include <utility>

namespace ssv {

HostCsr csr_transpose(const HostCsr& A) {
    HostCsr T;
    T.n = A.m;
    T.m = A.n;
    T.rp.assign(A.m + 1, 0);
    const int nnz = A.nnz();
    for (int k = 0; k < nnz; ++k) T.rp[A.ci[k] + 1]++;
    for (int i = 0; i < A.m; ++i) T.rp[i + 1] += T.rp[i];
    T.ci.resize(nnz);
    T.v.resize(nnz);
    std::vector<int> pos(T.rp.begin(), T.rp.end() - 1);
    for (int i = 0; i < A.n; ++i)
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
            const int p = pos[A.ci[k]]++;
            T.ci[p] = i;
            T.v[p] = A.v[k];
        }
    return T;
}

HostCsr csr_mul(const HostCsr& A, const HostCsr& B) {
    HostCsr C;
    C.n = A.n;
    C.m = B.m;
    C.rp.assign(A.n + 1, 0);
    std::vector<double> acc(B.m, 0.0);
    std::vector<int> mark(B.m, -1), cols;
    for (int i = 0; i < A.n; ++i) {
        cols.clear();
        for (int a = A.rp[i]; a < A.rp[i + 1]; ++a) {
            const int j = A.ci[a];
            const double av = A.v[a];
            for (int b = B.rp[j]; b < B.rp[j + 1]; ++b) {
                const int l = B.ci[b];
                if (mark[l] != i) {
                    mark[l] = i;
                    acc[l] = 0.0;
                    cols.push_back(l);
                }
                acc[l] += av * B.v[b];
            }
        }
        std::sort(cols.begin(), cols.end());
        for (int l : cols) {
            C.ci.push_back(l);
            C.v.push_back(acc[l]);
        }
        C.rp[i + 1] = (int)C.ci.size();
    }
    return C;
}

HostCsr csr_add(const HostCsr& A, double a, const HostCsr& B, double b) {
    HostCsr C;
    C.n = A.n;
    C.m = std::max(A.m, B.m);
    C.rp.assign(A.n + 1, 0);
    std::vector<std::pair<int, double>> row;
    for (int i = 0; i < A.n; ++i) {
        row.clear();
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) row.push_back({A.ci[k], a * A.v[k]});
        for (int k = B.rp[i]; k < B.rp[i + 1]; ++k) row.push_back({B.ci[k], b * B.v[k]});
        std::stable_sort(row.begin(), row.end(),
                         [](const std::pair<int, double>& p, const std::pair<int, double>& q) { return p.first < q.first; });
        for (size_t k = 0; k < row.size();) {
            size_t e = k;
            double sum = 0.0;
            while (e < row.size() && row[e].first == row[k].first) sum += row[e++].second;
            C.ci.push_back(row[k].first);
            C.v.push_back(sum);
            k = e;
        }
        C.rp[i + 1] = (int)C.ci.size();
    }
    return C;
}

FusedLevel fused_level(const HostCsr& A, const HostCsr& P, const HostCsr& Pt, const std::vector<double>& d) {
    const int n = A.n;
    HostCsr AD = A;  // A D^{-1}
    for (int i = 0; i < n; ++i)
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) AD.v[k] = A.v[k] / d[A.ci[k]];
    FusedLevel F;
    F.R = csr_add(Pt, 1.0, csr_mul(Pt, AD), -1.0);
    HostCsr I2;  // 2 I
    I2.n = I2.m = n;
    I2.rp.resize(n + 1);
    I2.ci.resize(n);
    I2.v.assign(n, 2.0);
    for (int i = 0; i <= n; ++i) I2.rp[i] = i;
    for (int i = 0; i < n; ++i) I2.ci[i] = i;
    HostCsr S = csr_add(I2, 1.0, AD, -1.0);  // then rows by D^{-1}
    for (int i = 0; i < n; ++i)
        for (int k = S.rp[i]; k < S.rp[i + 1]; ++k) S.v[k] /= d[i];
    HostCsr DAP = csr_mul(A, P);  // then rows by D^{-1}
    for (int i = 0; i < n; ++i)
        for (int k = DAP.rp[i]; k < DAP.rp[i + 1]; ++k) DAP.v[k] /= d[i];
    const HostCsr Q = csr_add(P, 1.0, DAP, -1.0);
    HostCsr& U = F.U;
    U.n = n;
    U.m = n + P.m;
    U.rp.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        for (int k = S.rp[i]; k < S.rp[i + 1]; ++k) {
            U.ci.push_back(S.ci[k]);
            U.v.push_back(S.v[k]);
        }
        for (int k = Q.rp[i]; k < Q.rp[i + 1]; ++k) {
            U.ci.push_back(n + Q.ci[k]);
            U.v.push_back(Q.v[k]);
        }
        U.rp[i + 1] = (int)U.ci.size();
    }
    return F;
}

HostCsr csr_rap(const HostCsr& A, const HostCsr& P) {
    const int nc = P.m;
    const HostCsr Pt = csr_transpose(P);
    HostCsr C;
    C.n = nc;
    C.m = nc;
    C.rp.assign(nc + 1, 0);
    std::vector<double> acc(nc, 0.0);
    std::vector<int> mark(nc, -1), cols;
    C.ci.reserve((size_t)A.nnz() / std::max(1, A.n) * nc * 2);
    for (int k = 0; k < nc; ++k) {
        cols.clear();
        for (int q = Pt.rp[k]; q < Pt.rp[k + 1]; ++q) {
            const int i = Pt.ci[q];
            const double pki = Pt.v[q];
            for (int a = A.rp[i]; a < A.rp[i + 1]; ++a) {
                const double pa = pki * A.v[a];
                const int j = A.ci[a];
                for (int b = P.rp[j]; b < P.rp[j + 1]; ++b) {
                    const int l = P.ci[b];
                    if (mark[l] != k) {
                        mark[l] = k;
                        acc[l] = 0.0;
                        cols.push_back(l);
                    }
                    acc[l] += pa * P.v[b];
                }
            }
        }
        std::sort(cols.begin(), cols.end());
        for (int l : cols) {
            C.ci.push_back(l);
            C.v.push_back(acc[l]);
        }
        C.rp[k + 1] = (int)C.ci.size();
    }
    return C;
}

namespace {

struct Graph {
    int n = 0;
    std::vector<int> rp, ci;
};

// ComputeStrength (compact_amg.hpp:292-372)
Graph strength(const HostCsr& A, double theta) {
    Graph S;
    S.n = A.n;
    S.rp.assign(A.n + 1, 0);
    std::vector<double> thr(A.n);
    std::vector<char> neg(A.n);
    for (int i = 0; i < A.n; ++i) {
        double max_neg = 0, max_abs = 0;
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
            if (A.ci[k] != i) {
                const double v = A.v[k];
                if (-v > max_neg) max_neg = -v;
                const double av = std::abs(v);
                if (av > max_abs) max_abs = av;
            }
        neg[i] = max_neg > 0;
        thr[i] = theta * (neg[i] ? max_neg : max_abs);
        int c = 0;
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
            if (A.ci[k] != i && (neg[i] ? (-A.v[k] >= thr[i]) : (std::abs(A.v[k]) >= thr[i]))) ++c;
        S.rp[i + 1] = S.rp[i] + c;
    }
    S.ci.resize(S.rp[A.n]);
    for (int i = 0; i < A.n; ++i) {
        int p = S.rp[i];
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
            if (A.ci[k] != i && (neg[i] ? (-A.v[k] >= thr[i]) : (std::abs(A.v[k]) >= thr[i]))) S.ci[p++] = A.ci[k];
    }
    return S;
}

// TransposeGraph (:457-483)
Graph transpose_graph(const Graph& G) {
    Graph T;
    T.n = G.n;
    T.rp.assign(G.n + 1, 0);
    for (int k = 0; k < (int)G.ci.size(); ++k) T.rp[G.ci[k] + 1]++;
    for (int i = 0; i < G.n; ++i) T.rp[i + 1] += T.rp[i];
    T.ci.resize(G.ci.size());
    std::vector<int> pos(T.rp.begin(), T.rp.end() - 1);
    for (int i = 0; i < G.n; ++i)
        for (int k = G.rp[i]; k < G.rp[i + 1]; ++k) T.ci[pos[G.ci[k]]++] = i;
    return T;
}

// CoarsenPMIS (:378-454): 1 = C, 0 = F
std::vector<int> pmis(const Graph& S) {
    const int n = S.n;
    std::vector<int> cf(n, -1);
    const Graph St = transpose_graph(S);
    std::vector<double> measure(n);
    std::mt19937 rng(42);
    std::uniform_real_distribution<double> dist(0.0, 1.0);
    for (int i = 0; i < n; ++i) measure[i] = (double)(St.rp[i + 1] - St.rp[i]) + dist(rng);
    std::vector<int> fresh;
    for (int round = 0; round < 100; ++round) {
        bool changed = false;
        fresh.clear();
        for (int i = 0; i < n; ++i) {
            if (cf[i] != -1) continue;
            const double mi = measure[i];
            bool top = true;
            for (int k = S.rp[i]; k < S.rp[i + 1] && top; ++k)
                if (cf[S.ci[k]] == -1 && measure[S.ci[k]] > mi) top = false;
            for (int k = St.rp[i]; k < St.rp[i + 1] && top; ++k)
                if (cf[St.ci[k]] == -1 && measure[St.ci[k]] > mi) top = false;
            if (top) {
                cf[i] = 1;  // C immediately (later rows see it)
                fresh.push_back(i);
                changed = true;
            }
        }
        for (int i : fresh) {
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
HostCsr interpolation(const HostCsr& A, const Graph& S, const std::vector<int>& cf, int nc) {
    const int nf = A.n;
    std::vector<int> cidx(nf, -1);
    for (int i = 0, c = 0; i < nf; ++i)
        if (cf[i] == 1) cidx[i] = c++;
    // strong flag per matrix entry (S rows are a subsequence of A rows)
    std::vector<char> strong(A.nnz(), 0);
    for (int i = 0; i < nf; ++i) {
        int q = S.rp[i];
        for (int k = A.rp[i]; k < A.rp[i + 1] && q < S.rp[i + 1]; ++k)
            if (A.ci[k] == S.ci[q]) { strong[k] = 1; ++q; }
    }
    HostCsr P;
    P.n = nf;
    P.m = nc;
    P.rp.assign(nf + 1, 0);
    for (int i = 0; i < nf; ++i) {
        int c = 0;
        if (cf[i] == 1) c = 1;
        else {
            for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) c += (strong[k] && cf[A.ci[k]] == 1);
            if (c == 0) c = 1;
        }
        P.rp[i + 1] = P.rp[i] + c;
    }
    P.ci.assign(P.rp[nf], 0);
    P.v.assign(P.rp[nf], 0.0);
    for (int i = 0; i < nf; ++i) {
        const int p0 = P.rp[i];
        if (cf[i] == 1) { P.ci[p0] = cidx[i]; P.v[p0] = 1.0; continue; }
        double aii = 0;
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
            if (A.ci[k] == i) { aii = A.v[k]; break; }
        double lump = 0;
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
            if (A.ci[k] != i && !(strong[k] && cf[A.ci[k]] == 1)) lump += A.v[k];
        double denom = aii + lump;
        if (std::abs(denom) < 1e-30) denom = 1.0;
        int pos = 0;
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
            if (strong[k] && cf[A.ci[k]] == 1) {
                P.ci[p0 + pos] = cidx[A.ci[k]];
                P.v[p0 + pos] = -A.v[k] / denom;
                ++pos;
            }
        if (pos == 0) {  // inject to the largest C neighbour, else a zero row
            int best = -1;
            double bv = 0;
            for (int k = A.rp[i]; k < A.rp[i + 1]; ++k)
                if (cf[A.ci[k]] == 1 && std::abs(A.v[k]) > bv) { bv = std::abs(A.v[k]); best = cidx[A.ci[k]]; }
            P.ci[p0] = best >= 0 ? best : 0;
            P.v[p0] = best >= 0 ? 1.0 : 0.0;
        }
    }
    return P;
}

void l1_norms(const HostCsr& A, std::vector<double>& out) {
    out.resize(A.n);
    for (int i = 0; i < A.n; ++i) {
        double s = 0;
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) s += std::abs(A.v[k]);
        out[i] = (s > 0) ? s : 1.0;
    }
}

}  // namespace

// Pseudo-inverse of the small coarsest matrix through LDL^T: pivots below
// 1e-13 of the row's diagonal count as zero and drop their component (the
// gradient-space matrix is singular, constants being in the kernel of G).
// The factors stay separate: the device applies x = L^{-T} (D^+ (L^{-1} b))
// as two triangular products with the pivot division between them, which is
// the substitution's arithmetic regrouped. A single explicit X = L^{-T} D^+
// L^{-1} is not used: when the pivots span many decades (a conducting region
// next to the 1e-6 mass weight of air gives ~1e13) X's entries are dominated
// by the smallest pivots and X b loses the other components, enough to stall
// COCR on the eddy-current systems.
double dense_ldlt_pseudo(const HostCsr& A, std::vector<double>& linv, std::vector<double>& linvt,
                         std::vector<double>& piv, double tau) {
    const int n = A.n;
    std::vector<double> L((size_t)n * n, 0.0), w(n), diag0(n);
    piv.assign(n, 0.0);
    std::vector<double>& d = piv;
    for (int i = 0; i < n; ++i)
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) L[(size_t)i * n + A.ci[k]] += A.v[k];
    for (int i = 0; i < n; ++i) diag0[i] = std::abs(L[(size_t)i * n + i]);
    double kept_min = 1.0;
    for (int j = 0; j < n; ++j) {
        for (int k = 0; k < j; ++k) w[k] = L[(size_t)j * n + k] * d[k];
        double dj = L[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) dj -= L[(size_t)j * n + k] * w[k];
        const bool zero = !(std::abs(dj) > tau * diag0[j]);
        d[j] = zero ? 0.0 : dj;
        if (!zero) kept_min = std::min(kept_min, std::abs(dj) / diag0[j]);
        L[(size_t)j * n + j] = 1.0;
        for (int i = j + 1; i < n; ++i) {
            double s = L[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) s -= L[(size_t)i * n + k] * w[k];
            L[(size_t)i * n + j] = zero ? 0.0 : s / dj;
        }
        for (int k = j + 1; k < n; ++k) L[(size_t)j * n + k] = 0.0;
    }
    // L^{-1} (unit lower) by forward substitution, columns in parallel;
    // linv row-major, linvt = its transpose (row i holds column i of L^{-1})
    linv.assign((size_t)n * n, 0.0);
    linvt.assign((size_t)n * n, 0.0);
    auto columns = [&](int c0, int c1) {
        std::vector<double> y(n);
        for (int c = c0; c < c1; ++c) {
            for (int i = 0; i < n; ++i) {
                double s = (i == c) ? 1.0 : 0.0;
                for (int k = 0; k < i; ++k) s -= L[(size_t)i * n + k] * y[k];
                y[i] = s;
            }
            for (int i = 0; i < n; ++i) {
                linv[(size_t)i * n + c] = y[i];
                linvt[(size_t)c * n + i] = y[i];
            }
        }
    };
    const int nt = std::max(1, std::min(16, (int)std::thread::hardware_concurrency()));
    if (n < 256 || nt == 1) {
        columns(0, n);
    } else {
        run_threads(nt, [&](int t) { columns(n * t / nt, n * (t + 1) / nt); });
    }
    return kept_min;
}

// CompactAMG::Setup (:66-156) for freedofs = nullptr (the AMS subspaces)
void AmgHost::setup(const HostCsr& A0) {
    levels.clear();
    levels.emplace_back();
    levels[0].A = A0;
    l1_norms(levels[0].A, levels[0].l1);
    for (int l = 0; l < max_levels - 1; ++l) {
        const HostCsr& A = levels[l].A;
        if (A.n <= min_coarse) break;
        const Graph S = strength(A, theta);
        const std::vector<int> cf = pmis(S);
        int nc = 0;
        for (int i = 0; i < A.n; ++i) nc += (cf[i] == 1);
        if (nc == 0 || nc >= A.n) break;
        HostCsr P = interpolation(A, S, cf, nc);
        HostCsr Pt = csr_transpose(P);
        HostCsr Ac = csr_rap(A, P);
        levels[l].P = std::move(P);
        levels[l].Pt = std::move(Pt);
        levels.emplace_back();
        levels.back().A = std::move(Ac);
        l1_norms(levels.back().A, levels.back().l1);
    }
    AmgHostLevel& co = levels.back();
    if (co.A.n <= min_coarse * 10) {
        co.direct = true;
        co.piv_min = dense_ldlt_pseudo(co.A, co.linv, co.linvt, co.piv);
    }
}

// BuildPiComponents (compact_ams.hpp:454-504) and the transposes (:276-294)
void AmsHost::setup_geometry(const HostCsr& grad, const double* cx, const double* cy, const double* cz) {
    G = grad;
    nhc = G.n;
    nh1 = G.m;
    const double* cs[3] = {cx, cy, cz};
    for (int d = 0; d < 3; ++d) {
        Pi[d] = G;
        for (int e = 0; e < G.n; ++e) {
            double gd = 0;
            for (int k = G.rp[e]; k < G.rp[e + 1]; ++k) gd += G.v[k] * cs[d][G.ci[k]];
            for (int k = G.rp[e]; k < G.rp[e + 1]; ++k) Pi[d].v[k] = std::abs(G.v[k]) * 0.5 * gd;
        }
    }
    Gt = csr_transpose(G);
    for (int d = 0; d < 3; ++d) Pit[d] = csr_transpose(Pi[d]);
}

// RebuildMatrix (compact_ams.hpp:300-421)
void AmsHost::rebuild(const HostCsr& A, const uint8_t* fd) {
    A_bc = A;
    if (fd)  // CreateBCModifiedMatrix (:605-633)
        for (int i = 0; i < A.n; ++i)
            for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
                const int j = A.ci[k];
                if (!fd[i]) A_bc.v[k] = (j == i) ? 1.0 : 0.0;
                else if (!fd[j]) A_bc.v[k] = 0.0;
            }
    HostCsr sub[4];
    auto galerkin = [&](int s) {
        sub[s] = csr_rap(A_bc, s == 0 ? G : Pi[s - 1]);
        HostCsr& M = sub[s];  // FixZeroRows (:638-659)
        for (int i = 0; i < M.n; ++i) {
            double l1 = 0;
            int dp = -1;
            for (int k = M.rp[i]; k < M.rp[i + 1]; ++k) {
                l1 += std::abs(M.v[k]);
                if (M.ci[k] == i) dp = k;
            }
            if (l1 == 0.0 && dp >= 0) M.v[dp] = 1.0;
        }
        amg[s] = AmgHost();
        amg[s].theta = theta;
        amg[s].max_levels = 25;
        amg[s].min_coarse = 500;
        amg[s].num_smooth = 1;
        amg[s].setup(M);
    };
    run_threads(4, galerkin);
    // truncated l1 of the fine smoother (:395-413)
    fine_l1.resize(nhc);
    for (int i = 0; i < nhc; ++i) {
        double diag = 0, off = 0;
        for (int k = A_bc.rp[i]; k < A_bc.rp[i + 1]; ++k) {
            if (A_bc.ci[k] == i) diag = std::abs(A_bc.v[k]);
            else off += std::abs(A_bc.v[k]);
        }
        const double t = diag + 0.5 * off;
        fine_l1[i] = (t <= (4.0 / 3.0) * diag) ? ((diag > 0) ? diag : 1.0) : ((t > 0) ? t : 1.0);
    }
}

}  // namespace ssv
