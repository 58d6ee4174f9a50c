// Host check of the fused V-cycle level products (amg_setup.cpp:fused_level):
// on random sparse levels, R b must equal the restriction of the residual
// after the first l1-Jacobi sweep, and U [b; e] the prolongation followed by
// the post sweep, both computed step by step in FP64. Prints the relative
// errors; exits 0 when both are below 1e-13 on every case.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <utility>
#include <vector>

#include "amg_setup.hpp"

using ssv::HostCsr;

static std::vector<double> spmv(const HostCsr& M, const std::vector<double>& x) {
    std::vector<double> y(M.n, 0.0);
    for (int i = 0; i < M.n; ++i)
        for (int k = M.rp[i]; k < M.rp[i + 1]; ++k) y[i] += M.v[k] * x[M.ci[k]];
    return y;
}

static double rel(const std::vector<double>& a, const std::vector<double>& b) {
    double e = 0.0, m = 0.0;
    for (size_t i = 0; i < a.size(); ++i) {
        e = std::max(e, std::fabs(a[i] - b[i]));
        m = std::max(m, std::fabs(b[i]));
    }
    return m > 0.0 ? e / m : e;
}

int main() {
    bool ok = true;
    for (int seed = 1; seed <= 6; ++seed) {
        std::mt19937 g(seed);
        std::uniform_real_distribution<double> U(-1.0, 1.0);
        const int n = 40 + 17 * seed, nc = n / 3 + seed;
        HostCsr A;  // symmetric pattern and values, dominant diagonal
        A.n = A.m = n;
        std::vector<std::vector<std::pair<int, double>>> rows(n);
        for (int i = 0; i < n; ++i) rows[i].push_back({i, 6.0 + U(g)});
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j)
                if ((j - i <= 2) || ((i * 31 + j * 17 + seed) % 37 == 0)) {
                    const double v = U(g);
                    rows[i].push_back({j, v});
                    rows[j].push_back({i, v});
                }
        A.rp.assign(n + 1, 0);
        for (int i = 0; i < n; ++i) {
            std::sort(rows[i].begin(), rows[i].end());
            for (auto& p : rows[i]) {
                A.ci.push_back(p.first);
                A.v.push_back(p.second);
            }
            A.rp[i + 1] = (int)A.ci.size();
        }
        HostCsr P;  // one or two coarse columns per fine row
        P.n = n;
        P.m = nc;
        P.rp.assign(n + 1, 0);
        for (int i = 0; i < n; ++i) {
            const int c = std::min(nc - 1, i * nc / n);
            P.ci.push_back(c);
            P.v.push_back(0.5 + 0.5 * U(g));
            if (c + 1 < nc && (i + seed) % 3 == 0) {
                P.ci.push_back(c + 1);
                P.v.push_back(U(g));
            }
            P.rp[i + 1] = (int)P.ci.size();
        }
        const HostCsr Pt = ssv::csr_transpose(P);
        std::vector<double> d(n, 0.0);
        for (int i = 0; i < n; ++i)
            for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) d[i] += std::fabs(A.v[k]);
        const ssv::FusedLevel F = ssv::fused_level(A, P, Pt, d);
        std::vector<double> b(n), e(nc);
        for (auto& v : b) v = U(g);
        for (auto& v : e) v = U(g);
        // step by step: x = D^-1 b; r = b - A x; b' = P^T r
        std::vector<double> x(n);
        for (int i = 0; i < n; ++i) x[i] = b[i] / d[i];
        std::vector<double> Ax = spmv(A, x), r(n);
        for (int i = 0; i < n; ++i) r[i] = b[i] - Ax[i];
        const double e_down = rel(spmv(F.R, b), spmv(Pt, r));
        // x += P e; x' = x + D^-1 (b - A x)
        const std::vector<double> Pe = spmv(P, e);
        for (int i = 0; i < n; ++i) x[i] += Pe[i];
        const std::vector<double> Ax2 = spmv(A, x);
        std::vector<double> xp(n);
        for (int i = 0; i < n; ++i) xp[i] = x[i] + (b[i] - Ax2[i]) / d[i];
        std::vector<double> be(b);
        be.insert(be.end(), e.begin(), e.end());
        const double e_up = rel(spmv(F.U, be), xp);
        const bool shapes = F.R.n == nc && F.R.m == n && F.U.n == n && F.U.m == n + nc;
        std::printf("seed %d n %d nc %d: down %.2e up %.2e shapes %s\n", seed, n, nc, e_down, e_up,
                    shapes ? "ok" : "WRONG");
        ok = ok && shapes && e_down < 1e-13 && e_up < 1e-13;
    }
    return ok ? 0 : 1;
}
