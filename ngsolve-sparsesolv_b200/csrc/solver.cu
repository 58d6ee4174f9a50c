// solver.cu -- host orchestration of the device solve path: IC(0) set-up and
// factorisation, the CG / COCR iteration loops captured in CUDA graphs, the
// NGSolve-style COCR loop with an external preconditioner.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "objects.cuh"
#include "solver_api.hpp"

namespace ssv {

// ---------------------------------------------------------------------------
// Runtime plumbing
// ---------------------------------------------------------------------------
cudaStream_t stream() {
    static cudaStream_t s = nullptr;
    if (!s) SSV_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    return s;
}

int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        SSV_CUDA(cudaGetDevice(&dev));
        SSV_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
        if (n <= 0) n = 148;
    }
    return n;
}

double wall_seconds() {
    using clk = std::chrono::steady_clock;
    return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

int pick_lanes(double nnz_per_row) {
    if (nnz_per_row <= 3.0) return 2;
    if (nnz_per_row <= 6.0) return 4;
    if (nnz_per_row <= 12.0) return 8;
    if (nnz_per_row <= 24.0) return 16;
    return 32;
}

bool graph_while_mode() {
    const char* m = std::getenv("SSV_GRAPH_MODE");
    return !(m && std::strcmp(m, "chunk") == 0);
}

void GraphLoop::reset() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    key.clear();
}

__global__ void k_loop_ctl(KState* st, cudaGraphConditionalHandle h, int use_cond) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (!st->done) {
        st->it++;
        if (st->it >= st->maxiter) {
            st->done = 1;
            st->converged = 0;
            st->iters = st->maxiter;
            st->final_norm = st->norm_r;
        }
    }
    st->loops++;
    if (!st->done && st->loops >= st->max_loops) {
        st->done = 1;
        st->status = SSV_ERR_TIMEOUT;
    }
    if (use_cond) cudaGraphSetConditional(h, st->done ? 0u : 1u);
}

// Cap on the executed loop bodies of every device-looped solve: maxiter + 4
// (a loop that outruns its own iteration count means a stuck state), or the
// process-wide override of ssv_set_loop_guard (> 0). A solve that reaches it
// stops on the device and fails with SSV_ERR_TIMEOUT.
static int g_loop_guard = 0;
void set_loop_guard(int loops) { g_loop_guard = loops > 0 ? loops : 0; }
int loop_guard(int maxiter) { return g_loop_guard > 0 ? g_loop_guard : std::max(maxiter, 0) + 4; }

void run_graph_loop(GraphLoop& g, KState* d_st, int max_iters) {
    cudaStream_t s = stream();
    if (g.cond) {
        SSV_CUDA(cudaGraphLaunch(g.exec, s));
        SSV_CUDA(cudaStreamSynchronize(s));
        return;
    }
    // chunked: relaunch until done; bounded by the iteration cap
    int launches = 0;
    const int max_launches = max_iters / std::max(g.chunk, 1) + 2;
    int done = 0;
    while (!done && launches < max_launches) {
        SSV_CUDA(cudaGraphLaunch(g.exec, s));
        SSV_CUDA(cudaMemcpyAsync(&done, &d_st->done, sizeof(int), cudaMemcpyDeviceToHost, s));
        SSV_CUDA(cudaStreamSynchronize(s));
        ++launches;
    }
}

// `shape` = lanes per row | (rows per row group and pass) << 8
template <typename S, typename SV, int MODE>
void launch_spmv(int shape, int n, const int* rp, const int* ci, const SV* v, const S* x, S* y,
                 const S* b, const uint8_t* mask, KState* st, int op, RedBuf red, double2* out,
                 cudaStream_t s) {
    const int lanes = shape & 0xff;
    const int u = std::max(1, shape >> 8);
    const int rows_per_block = kBlock / lanes * u;
    int grid = (n + rows_per_block - 1) / rows_per_block;
    grid = std::max(1, std::min(grid, sm_count() * 8));
#define SSV_SPMV_CASE(L, UU)                                                                          \
    if (lanes == L && u == UU) {                                                                      \
        launch_k(k_spmv<S, SV, L, MODE, UU>, grid, kBlock, s, n, rp, ci, v, x, y, b, mask, st, op, red, out); \
        SSV_LAUNCH_CHECK();                                                                           \
        return;                                                                                       \
    }
    SSV_SPMV_CASE(2, 1)
    SSV_SPMV_CASE(4, 1)
    SSV_SPMV_CASE(8, 1)
    SSV_SPMV_CASE(16, 1)
    SSV_SPMV_CASE(4, 2)
    SSV_SPMV_CASE(8, 2)
#undef SSV_SPMV_CASE
    launch_k(k_spmv<S, SV, 32, MODE, 1>, grid, kBlock, s, n, rp, ci, v, x, y, b, mask, st, op, red, out);
    SSV_LAUNCH_CHECK();
}

// lanes and rows per group for a matrix of n rows and nnz_per_row: a large
// matrix takes two rows per group and half the lanes of the one-row shape
// (SSV_SPMV_ROWS_PER_GROUP=1 keeps one row per group everywhere)
int pick_shape(int n, double nnz_per_row) {
    static int rows = -1;
    if (rows < 0) {
        const char* e = std::getenv("SSV_SPMV_ROWS_PER_GROUP");
        rows = (e && e[0] == '1') ? 1 : 2;
    }
    const int lanes = pick_lanes(nnz_per_row);
    if (rows == 2 && n >= 65536 && (lanes == 8 || lanes == 16)) return (lanes / 2) | (2 << 8);
    return lanes;
}

template <typename S>
void KrylovWork<S>::ensure(int n_, int hist_cap) {
    if (n_ != n) {
        for (auto& b : xb) b.alloc(n_);
        r.alloc(n_); z.alloc(n_); p.alloc(n_); Ap.alloc(n_); t.alloc(n_); qt.alloc(n_); bw.alloc(n_);
        n = n_;
    }
    if (!st.get()) st.alloc(1);
    const size_t np = (size_t)sm_count() * 8 + 64;
    if (partials.size() < np) partials.alloc(np);
    if (!ticket.get()) {
        ticket.alloc(4);
        ticket.zero(stream());
    }
    if (scal.size() < 8) scal.alloc(8);
    if ((int)hist.size() < hist_cap) hist.alloc(hist_cap);
}

// ---------------------------------------------------------------------------
// IC(0)
// ---------------------------------------------------------------------------

template <typename S>
void ICDevice<S>::build_pattern(int n_, const std::vector<int>& rp, const std::vector<int>& ci,
                                const ssv_config& cfg) {
    cudaStream_t s = stream();
    n = n_;
    ++gen;
    abmc = cfg.use_abmc != 0;
    rcm = abmc && cfg.abmc_use_rcm != 0;
    bs = cfg.abmc_block_size;
    nct = cfg.abmc_num_colors;
    fwd_launch.clear();
    bwd_launch.clear();
    std::vector<int> lrp, lci, lsrc, urp, uci, usrc;
    if (abmc) {
        // abmc_use_rcm (ic_preconditioner.hpp:97-104): the ABMC schedule is
        // built on the RCM-reordered pattern, and the working numbering is the
        // composite old -> RCM -> ABMC (build_composite_permutations, :584-596)
        std::vector<int> rord, rrev, crp, cci, csrc;
        const int* brp = rp.data();
        const int* bci = ci.data();
        if (rcm) {
            rcm_order(n, rp.data(), ci.data(), rord, rrev);
            permute_pattern(n, rp.data(), ci.data(), rord.data(), crp, cci, csrc);
            brp = crp.data();
            bci = cci.data();
        }
        AbmcSchedule sched;
        build_abmc(n, brp, bci, cfg.abmc_block_size, cfg.abmc_num_colors, sched);
        num_colors = sched.num_colors;
        num_blocks = sched.num_blocks;
        h_perm = sched.ordering;
        if (rcm)
            for (int i = 0; i < n; ++i) h_perm[i] = sched.ordering[rord[i]];
        std::vector<int> prp, pci, psrc;
        permute_pattern(n, rp.data(), ci.data(), h_perm.data(), prp, pci, psrc);
        lower_pattern(n, prp.data(), pci.data(), lrp, lci, lsrc);
        // L value sources as positions in the ORIGINAL value array
        for (auto& k : lsrc) k = psrc[k];
        h_Arp = prp;
        Arp.upload(prp.data(), prp.size(), s);
        Aci.upload(pci.data(), pci.size(), s);
        Asrc.upload(psrc.data(), psrc.size(), s);
        Av.alloc(pci.size());
        lanes = pick_shape(n, n > 0 ? (double)pci.size() / n : 1.0);
        perm.upload(h_perm.data(), h_perm.size(), s);
        uoff.upload(sched.block_offsets.data(), sched.block_offsets.size(), s);
        h_boff = sched.block_offsets;
        sched_color_offsets = sched.color_offsets;
        rows_f.release();
        rows_b.release();
        for (int c = 0; c < num_colors; ++c)
            fwd_launch.push_back({sched.color_offsets[c], sched.color_offsets[c + 1]});
        for (int c = num_colors - 1; c >= 0; --c)
            bwd_launch.push_back({sched.color_offsets[c], sched.color_offsets[c + 1]});
    } else {
        lower_pattern(n, rp.data(), ci.data(), lrp, lci, lsrc);
        h_perm.clear();
        perm.release();
        Arp.release(); Aci.release(); Asrc.release(); Av.release();
        uoff.release();
    }
    transpose_pattern(n, lrp, lci, urp, uci, usrc);
    if (!abmc) {
        std::vector<int> lev, rws, off;
        num_levels_f = build_levels(n, lrp.data(), lci.data(), false, lev);
        group_by_level(lev, num_levels_f, rws, off);
        rows_f.upload(rws.data(), rws.size(), s);
        for (int l = 0; l < num_levels_f; ++l) fwd_launch.push_back({off[l], off[l + 1]});
        num_levels_b = build_levels(n, urp.data(), uci.data(), true, lev);
        group_by_level(lev, num_levels_b, rws, off);
        rows_b.upload(rws.data(), rws.size(), s);
        for (int l = 0; l < num_levels_b; ++l) bwd_launch.push_back({off[l], off[l + 1]});
    }
    // missing diagonal (ic_preconditioner.hpp:1221-1226 / :1358-1363): first
    // row in processing order whose last lower entry is not the diagonal
    missing_row = -1;
    for (int i = 0; i < n && missing_row < 0; ++i) {
        const int d = lrp[i + 1] - 1;
        if (d < lrp[i] || lci[d] != i) missing_row = i;
    }
    h_Lrp = lrp;
    h_Lci = lci;
    Lrp.upload(lrp.data(), lrp.size(), s);
    Lci.upload(lci.data(), lci.size(), s);
    Lsrc.upload(lsrc.data(), lsrc.size(), s);
    Urp.upload(urp.data(), urp.size(), s);
    Uci.upload(uci.data(), uci.size(), s);
    Usrc.upload(usrc.data(), usrc.size(), s);
    Lv.alloc(lci.size());
    Uv.alloc(uci.size());
    inv.alloc(n);
    tw.alloc(n);
    if (!flag.get()) flag.alloc(1);
    blk = false;
    fwd_blk.clear();
    bwd_blk.clear();
    fwd_cta.clear();
    bwd_cta.clear();
    if (abmc && missing_row < 0 && cfg.abmc_block_size <= 32) {
        // Ordinary blocks hold <= block_size rows; the aggregation appends any
        // rows it could not place to the last block
        // (abmc_ordering.hpp:217-226), which can be far larger. Such a block
        // is swept row-parallel by its own intra-block level sets.
        const std::vector<int>& bo = h_boff;
        const int cap = std::max(1, cfg.abmc_block_size);
        int bsmax = 1;
        for (int b = 0; b < num_blocks; ++b) {
            const int sz = bo[b + 1] - bo[b];
            if (sz <= cap) bsmax = std::max(bsmax, sz);
        }
        blk = true;
        blk_lanes = 1;
        while (blk_lanes < bsmax) blk_lanes <<= 1;
        tri = std::max(1, bsmax * (bsmax - 1) / 2);
        std::vector<int> h_erp(n + 1, 0), h_eci, h_esrc, h_urp(n + 1, 0), h_uci, h_usrc, h_dsrc(n);
        std::vector<int> h_isrc((size_t)num_blocks * tri, -1);
        std::vector<int> h_rows_f, h_rows_b, h_lev_f, h_lev_b;
        std::vector<int> h_sf_rp(1, 0), h_sf_src, h_sf_col, h_sf_loc, h_sb_rp(1, 0), h_sb_src, h_sb_col, h_sb_loc;
        std::vector<int> pos;
        int smem_optin = 0, staged_max = 0;
        SSV_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, 0));
        h_eci.reserve(lci.size());
        h_esrc.reserve(lci.size());
        h_uci.reserve(uci.size());
        h_usrc.reserve(uci.size());
        std::vector<int> lev;
        for (int b = 0; b < num_blocks; ++b) {
            const int r0 = bo[b], r1 = bo[b + 1];
            const bool big = (r1 - r0) > cap;
            for (int i = r0; i < r1; ++i) {
                for (int k = lrp[i]; k < lrp[i + 1] - 1; ++k) {
                    const int c = lci[k];
                    if (c < r0 || big) { h_eci.push_back(c); h_esrc.push_back(k); }
                    else {
                        const int j = i - r0, t = c - r0;
                        h_isrc[(size_t)b * tri + j * (j - 1) / 2 + t] = k;
                    }
                }
                h_erp[i + 1] = (int)h_eci.size();
                h_dsrc[i] = lrp[i + 1] - 1;
                for (int k = urp[i] + 1; k < urp[i + 1]; ++k)
                    if (uci[k] >= r1 || big) { h_uci.push_back(uci[k]); h_usrc.push_back(usrc[k]); }
                h_urp[i + 1] = (int)h_uci.size();
            }
        }
        // launch lists: colour by colour; runs of ordinary blocks, and the
        // level sets of oversized blocks (forward: dependencies on earlier
        // rows of the block, backward: on later rows)
        auto add_big = [&](int r0, int r1, bool fwd) {
            const int m = r1 - r0;
            lev.assign(m, 0);
            int nl = 0;
            if (fwd) {
                for (int i = r0; i < r1; ++i) {
                    int d = -1;
                    for (int k = lrp[i]; k < lrp[i + 1] - 1; ++k)
                        if (lci[k] >= r0) d = std::max(d, lev[lci[k] - r0]);
                    lev[i - r0] = d + 1;
                    nl = std::max(nl, d + 2);
                }
            } else {
                for (int i = r1 - 1; i >= r0; --i) {
                    int d = -1;
                    for (int k = urp[i] + 1; k < urp[i + 1]; ++k)
                        if (uci[k] < r1) d = std::max(d, lev[uci[k] - r0]);
                    lev[i - r0] = d + 1;
                    nl = std::max(nl, d + 2);
                }
            }
            std::vector<int>& rows = fwd ? h_rows_f : h_rows_b;
            std::vector<int>& lv = fwd ? h_lev_f : h_lev_b;
            const int p0 = (int)lv.size();
            lv.push_back((int)rows.size());
            const int qa = (int)rows.size();
            for (int l = 0; l < nl; ++l) {
                const int a = (int)rows.size();
                for (int i = r0; i < r1; ++i)
                    if (lev[i - r0] == l) rows.push_back(i);
                (fwd ? fwd_blk : bwd_blk).push_back({1, a, (int)rows.size()});
                lv.push_back((int)rows.size());
            }
            // staged copy: each row's entries in sweep order, couplings inside
            // the block by position, the others by column
            const int qb = (int)rows.size();
            pos.assign(m, -1);
            for (int q = qa; q < qb; ++q) pos[rows[q] - r0] = q - qa;
            std::vector<int>& srp = fwd ? h_sf_rp : h_sb_rp;
            std::vector<int>& ssrc = fwd ? h_sf_src : h_sb_src;
            std::vector<int>& scol = fwd ? h_sf_col : h_sb_col;
            std::vector<int>& sloc = fwd ? h_sf_loc : h_sb_loc;
            const int e0 = (int)ssrc.size();
            for (int q = qa; q < qb; ++q) {
                const int i = rows[q];
                const int ka = fwd ? lrp[i] : urp[i] + 1, kb = fwd ? lrp[i + 1] - 1 : urp[i + 1];
                for (int k = ka; k < kb; ++k) {
                    const int c = fwd ? lci[k] : uci[k];
                    ssrc.push_back(k);
                    scol.push_back(c);
                    sloc.push_back(c >= r0 && c < r1 ? pos[c - r0] : -1);
                }
                srp.push_back((int)ssrc.size());
            }
            // headroom for the launching kernel's static shared memory
            const size_t bytes = staged_bytes<S, S>(qb - qa, (int)ssrc.size() - e0, nl);
            const int smem = bytes + 1024 <= (size_t)smem_optin ? (int)bytes : 0;
            staged_max = std::max(staged_max, smem);
            (fwd ? fwd_cta : bwd_cta).push_back({2, p0, p0 + nl, smem});
        };
        auto add_colour = [&](int c, bool fwd) {
            const int b0 = sched_color_offsets[c], b1 = sched_color_offsets[c + 1];
            std::vector<Launch>& cta = fwd ? fwd_cta : bwd_cta;
            int run = b0;
            for (int b = b0; b < b1; ++b) {
                if (bo[b + 1] - bo[b] > cap) {
                    if (b > run) {
                        (fwd ? fwd_blk : bwd_blk).push_back({0, run, b});
                        cta.push_back({0, run, b, 0, c});
                    }
                    add_big(bo[b], bo[b + 1], fwd);
                    cta.back().color = c;
                    run = b + 1;
                }
            }
            if (b1 > run) {
                (fwd ? fwd_blk : bwd_blk).push_back({0, run, b1});
                cta.push_back({0, run, b1, 0, c});
            }
        };
        for (int c = 0; c < num_colors; ++c) add_colour(c, true);
        for (int c = num_colors - 1; c >= 0; --c) add_colour(c, false);
        erp.upload(h_erp.data(), h_erp.size(), s);
        eci.upload(h_eci.data(), h_eci.size(), s);
        esrc.upload(h_esrc.data(), h_esrc.size(), s);
        urpe.upload(h_urp.data(), h_urp.size(), s);
        ucie.upload(h_uci.data(), h_uci.size(), s);
        usrce.upload(h_usrc.data(), h_usrc.size(), s);
        isrc.upload(h_isrc.data(), h_isrc.size(), s);
        dsrc.upload(h_dsrc.data(), h_dsrc.size(), s);
        if (!h_rows_f.empty()) rows_f.upload(h_rows_f.data(), h_rows_f.size(), s);
        if (!h_rows_b.empty()) rows_b.upload(h_rows_b.data(), h_rows_b.size(), s);
        if (!h_lev_f.empty()) lev_f.upload(h_lev_f.data(), h_lev_f.size(), s);
        if (!h_lev_b.empty()) lev_b.upload(h_lev_b.data(), h_lev_b.size(), s);
        auto up = [&](DevBuf<int>& d, const std::vector<int>& h) {
            if (!h.empty()) d.upload(h.data(), h.size(), s);
        };
        up(sf_rp, h_sf_rp); up(sf_src, h_sf_src); up(sf_col, h_sf_col); up(sf_loc, h_sf_loc);
        up(sb_rp, h_sb_rp); up(sb_src, h_sb_src); up(sb_col, h_sb_col); up(sb_loc, h_sb_loc);
        if (staged_max > 0) {  // dynamic shared memory of the staged sweeps (<= optin - 1 KB)
            using SLo = typename ST<S>::lo;
            const int sm = staged_max;
            SSV_CUDA(cudaFuncSetAttribute(k_ic_sweep_staged<S, S, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            SSV_CUDA(cudaFuncSetAttribute(k_ic_sweep_staged<S, S, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            SSV_CUDA(cudaFuncSetAttribute(k_ic_sweep_staged<S, SLo, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
            SSV_CUDA(cudaFuncSetAttribute(k_ic_sweep_staged<S, SLo, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        }
        ev.alloc(h_eci.size()); uev.alloc(h_uci.size()); iv.alloc(h_isrc.size()); dv.alloc(n);
    }
    built = true;
    SSV_CUDA(cudaStreamSynchronize(s));
}

// scaling_i = 1/sqrt(|L_ii|) (ic_preconditioner.hpp:1120-1134) then
// L_ij *= scaling_i * scaling_j (:1139-1149), on the gathered originals.
template <typename S>
__global__ void k_ic_scaling(int n, const int* __restrict__ Lrp, const int* __restrict__ Lci,
                             const S* __restrict__ Lv, double* __restrict__ sc) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int d = Lrp[i + 1] - 1;
        double v = 1.0;
        if (d >= Lrp[i] && Lci[d] == i) {
            const double a = ST<S>::abs(Lv[d]);
            v = (a > 0.0) ? 1.0 / sqrt(a) : 1.0;
        }
        sc[i] = v;
    }
}

template <typename S>
__global__ void k_ic_apply_scaling(int n, const int* __restrict__ Lrp, const int* __restrict__ Lci,
                                   S* __restrict__ Lv, const double* __restrict__ sc) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = Lrp[i]; k < Lrp[i + 1]; ++k)
            Lv[k] = Lv[k] * ST<S>::from(sc[i]) * ST<S>::from(sc[Lci[k]]);
}

template <typename S>
int ICDevice<S>::factorize(const S* vals, const ssv_config& cfg) {
    cudaStream_t s = stream();
    int nk = 0;
    if (missing_row >= 0)
        fail(SSV_ERR_RUNTIME, std::string(abmc ? "IC decomposition failed: missing diagonal at row "
                                               : "IC decomposition failed: missing diagonal element at row ") +
                                  std::to_string(missing_row));
    const int64_t nl = (int64_t)h_Lci.size();
    if (abmc) {
        k_gather_values<S><<<grid_for(Asrc.size(), kBlock), kBlock, 0, s>>>((int64_t)Asrc.size(), Asrc.get(),
                                                                           vals, Av.get());
        SSV_LAUNCH_CHECK();
        ++nk;
    }
    const bool scale = cfg.diagonal_scaling != 0;
    if (scale) scaling.alloc(n);
    double shift = cfg.shift_parameter;
    double increment = cfg.shift_increment;
    int trials = 0;
    for (;;) {
        // (re)load the original values, then scale (restart path :1300-1307)
        k_gather_values<S><<<grid_for(nl, kBlock), kBlock, 0, s>>>(nl, Lsrc.get(), vals, Lv.get());
        SSV_LAUNCH_CHECK();
        nk += 1 + (scale ? 2 : 0) + (int)fwd_launch.size();
        if (scale) {
            k_ic_scaling<S><<<grid_for(n, kBlock), kBlock, 0, s>>>(n, Lrp.get(), Lci.get(), Lv.get(),
                                                                  scaling.get());
            k_ic_apply_scaling<S><<<grid_for(n, kBlock), kBlock, 0, s>>>(n, Lrp.get(), Lci.get(), Lv.get(),
                                                                        scaling.get());
            SSV_LAUNCH_CHECK();
        }
        flag.zero(s);
        if (blk) {
            for (const auto& g : fwd_blk) {
                const int units = g.b - g.a;
                if (units <= 0) continue;
                k_ic_factor<S><<<(units + 127) / 128, 128, 0, s>>>(
                    g.a, g.b, g.kind == 0 ? uoff.get() : nullptr, g.kind == 0 ? nullptr : rows_f.get(), Lrp.get(),
                    Lci.get(), Lv.get(), inv.get(), shift, cfg.min_diagonal_threshold, cfg.zero_diagonal_replacement,
                    cfg.auto_shift, flag.get());
            }
            nk += (int)fwd_blk.size() - (int)fwd_launch.size();
        } else {
            for (const auto& g : fwd_launch) {
                const int units = g.second - g.first;
                if (units <= 0) continue;
                k_ic_factor<S><<<(units + 127) / 128, 128, 0, s>>>(
                    g.first, g.second, abmc ? uoff.get() : nullptr, abmc ? nullptr : rows_f.get(), Lrp.get(),
                    Lci.get(), Lv.get(), inv.get(), shift, cfg.min_diagonal_threshold,
                    cfg.zero_diagonal_replacement, cfg.auto_shift, flag.get());
            }
        }
        SSV_LAUNCH_CHECK();
        int need = 0;
        SSV_CUDA(cudaMemcpyAsync(&need, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        SSV_CUDA(cudaStreamSynchronize(s));
        if (cfg.auto_shift && need && shift < cfg.max_shift_value && trials < cfg.max_shift_trials) {
            shift += increment;
            increment *= 2;  // exponential back-off (:1404-1406)
            ++trials;
            continue;
        }
        break;
    }
    actual_shift = shift;
    // the ABMC apply of the default path never scales (the scaling enters the
    // factor only); the reordered-space applies of paths 1 and 2 do
    // (ic_preconditioner.hpp:327-345)
    scaled_apply = scale && (!abmc || cfg.abmc_reorder_spmv || cfg.abmc_use_rcm);
    const int64_t nu = (int64_t)Usrc.size();
    k_gather_values<S><<<grid_for(nu, kBlock), kBlock, 0, s>>>(nu, Usrc.get(), Lv.get(), Uv.get());
    SSV_LAUNCH_CHECK();
    ++nk;
    lo = cfg.precision == SSV_PREC_FP32;
    if (blk) {
        auto gz = [&](const DevBuf<int>& src, auto& out) {
            const int64_t m = (int64_t)src.size();
            if (m > 0) k_gather_or_zero<S><<<grid_for(m, kBlock), kBlock, 0, s>>>(m, src.get(), Lv.get(), out.get());
            ++nk;
        };
        if (lo) {
            ev_lo.alloc(ev.size()); uev_lo.alloc(uev.size()); iv_lo.alloc(iv.size()); dv_lo.alloc(n);
            gz(esrc, ev_lo); gz(usrce, uev_lo); gz(isrc, iv_lo); gz(dsrc, dv_lo);
        } else {
            gz(esrc, ev); gz(usrce, uev); gz(isrc, iv); gz(dsrc, dv);
        }
        SSV_LAUNCH_CHECK();
    }
    if (lo) {
        nk += 3;
        Lv_lo.alloc(nl); Uv_lo.alloc(nu); inv_lo.alloc(n);
        k_to_lo<S, SL><<<grid_for(nl, kBlock), kBlock, 0, s>>>(nl, Lv.get(), Lv_lo.get());
        k_to_lo<S, SL><<<grid_for(nu, kBlock), kBlock, 0, s>>>(nu, Uv.get(), Uv_lo.get());
        k_to_lo<S, SL><<<grid_for(n, kBlock), kBlock, 0, s>>>(n, inv.get(), inv_lo.get());
        SSV_LAUNCH_CHECK();
    }
    return nk;
}

// one CTA of 256 threads with `smem` bytes of dynamic shared memory, PDL allowed
template <typename... KArgs, typename... Args>
static void launch_staged(void (*k)(KArgs...), int smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(1);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    SSV_CUDA(cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...));
}

template <typename S, typename SL, int L>
static void launch_fwd_blk(const ICDevice<S>& ic, const SL* ev, const SL* iv, const SL* dv, const S* x,
                           const double* sc, const KState* st, cudaStream_t s) {
    constexpr int per_cta = 128 / L;
    const SL* Lfull = ic.lo ? reinterpret_cast<const SL*>(ic.Lv_lo.get()) : reinterpret_cast<const SL*>(ic.Lv.get());
    for (const auto& g : ic.fwd_cta) {
        const int units = g.b - g.a;
        if (units <= 0) continue;
        if (g.kind == 0)
            launch_k(k_ic_fwd_blk<S, SL, L>, (units + per_cta - 1) / per_cta, 128, s, 
                g.a, g.b, ic.uoff.get(), ic.erp.get(), ic.eci.get(), ev, iv, ic.tri, dv, x, sc, ic.tw.get(), st);
        else if (g.smem > 0)
            launch_staged(k_ic_sweep_staged<S, SL, true>, g.smem, s, units, ic.lev_f.get() + g.a, ic.rows_f.get(),
                          ic.sf_rp.get(), ic.sf_src.get(), ic.sf_col.get(), ic.sf_loc.get(), ic.Lrp.get(), Lfull,
                          (const SL*)nullptr, x, sc, ic.tw.get(), st);
        else
            launch_k(k_ic_fwd_cta<S, SL>, 1, 256, s, units, ic.lev_f.get() + g.a, ic.rows_f.get(), ic.Lrp.get(),
                                                  ic.Lci.get(), Lfull, x, sc, ic.tw.get(), st);
    }
}

template <typename S, typename SL, int L>
static void launch_bwd_blk(const ICDevice<S>& ic, const SL* uev, const SL* iv, const SL* inv, S* y,
                           const KState* st, cudaStream_t s) {
    constexpr int per_cta = 128 / L;
    const SL* Ufull = ic.lo ? reinterpret_cast<const SL*>(ic.Uv_lo.get()) : reinterpret_cast<const SL*>(ic.Uv.get());
    for (const auto& g : ic.bwd_cta) {
        const int units = g.b - g.a;
        if (units <= 0) continue;
        if (g.kind == 0)
            launch_k(k_ic_bwd_blk<S, SL, L>, (units + per_cta - 1) / per_cta, 128, s, 
                g.a, g.b, ic.uoff.get(), ic.urpe.get(), ic.ucie.get(), uev, iv, ic.tri, inv, ic.tw.get(), y, st);
        else if (g.smem > 0)
            launch_staged(k_ic_sweep_staged<S, SL, false>, g.smem, s, units, ic.lev_b.get() + g.a, ic.rows_b.get(),
                          ic.sb_rp.get(), ic.sb_src.get(), ic.sb_col.get(), ic.sb_loc.get(), (const int*)nullptr,
                          Ufull, inv, (const S*)ic.tw.get(), (const double*)nullptr, y, st);
        else
            launch_k(k_ic_bwd_cta<S, SL>, 1, 256, s, units, ic.lev_b.get() + g.a, ic.rows_b.get(), ic.Urp.get(),
                                                  ic.Uci.get(), Ufull, inv, ic.tw.get(), y, st);
    }
}

#define SSV_BLK_DISPATCH(FN, SLT, ...)                         \
    switch (blk_lanes) {                                      \
        case 1: FN<S, SLT, 1>(__VA_ARGS__); break;            \
        case 2: FN<S, SLT, 2>(__VA_ARGS__); break;            \
        case 4: FN<S, SLT, 4>(__VA_ARGS__); break;            \
        case 8: FN<S, SLT, 8>(__VA_ARGS__); break;            \
        case 16: FN<S, SLT, 16>(__VA_ARGS__); break;          \
        default: FN<S, SLT, 32>(__VA_ARGS__); break;          \
    }

template <typename S>
void ICDevice<S>::apply_fwd(const S* x, const KState* st, cudaStream_t s) const {
    const int* uo = abmc ? uoff.get() : nullptr;
    const double* sc = scaled_apply ? scaling.get() : nullptr;
    if (blk) {
        if (lo) {
            SSV_BLK_DISPATCH(launch_fwd_blk, SL, *this, ev_lo.get(), iv_lo.get(), dv_lo.get(), x, sc, st, s)
        } else {
            SSV_BLK_DISPATCH(launch_fwd_blk, S, *this, ev.get(), iv.get(), dv.get(), x, sc, st, s)
        }
        SSV_LAUNCH_CHECK();
        return;
    }
    for (const auto& g : fwd_launch) {
        const int units = g.second - g.first;
        if (units <= 0) continue;
        if (lo)
            launch_k(k_ic_fwd<S, SL>, (units + 127) / 128, 128, s, g.first, g.second, uo, rows_f.get(), Lrp.get(),
                                                                Lci.get(), Lv_lo.get(), x, sc, tw.get(), st);
        else
            launch_k(k_ic_fwd<S, S>, (units + 127) / 128, 128, s, g.first, g.second, uo, rows_f.get(), Lrp.get(),
                                                               Lci.get(), Lv.get(), x, sc, tw.get(), st);
    }
    SSV_LAUNCH_CHECK();
}

template <typename S>
void ICDevice<S>::apply_bwd(S* y, const KState* st, cudaStream_t s) const {
    const int* uo = abmc ? uoff.get() : nullptr;
    const double* sc = scaled_apply ? scaling.get() : nullptr;
    if (blk) {
        if (lo) {
            SSV_BLK_DISPATCH(launch_bwd_blk, SL, *this, uev_lo.get(), iv_lo.get(), inv_lo.get(), y, st, s)
        } else {
            SSV_BLK_DISPATCH(launch_bwd_blk, S, *this, uev.get(), iv.get(), inv.get(), y, st, s)
        }
        if (sc) launch_k(k_scale_real<S>, grid_for(n, kBlock), kBlock, s, n, y, sc);
        SSV_LAUNCH_CHECK();
        return;
    }
    for (const auto& g : bwd_launch) {
        const int units = g.second - g.first;
        if (units <= 0) continue;
        if (lo)
            launch_k(k_ic_bwd<S, SL>, (units + 127) / 128, 128, s, g.first, g.second, uo, rows_b.get(), Urp.get(),
                                                                Uci.get(), Uv_lo.get(), inv_lo.get(), tw.get(), y, st);
        else
            launch_k(k_ic_bwd<S, S>, (units + 127) / 128, 128, s, g.first, g.second, uo, rows_b.get(), Urp.get(),
                                                               Uci.get(), Uv.get(), inv.get(), tw.get(), y, st);
    }
    if (sc) launch_k(k_scale_real<S>, grid_for(n, kBlock), kBlock, s, n, y, sc);
    SSV_LAUNCH_CHECK();
}

template struct ICDevice<double>;
template struct ICDevice<zdouble>;

// ---------------------------------------------------------------------------
// Krylov drivers (SparseSolvSolver::Solve)
// ---------------------------------------------------------------------------
template <typename S> ICDevice<S>& ic_of(ssv_solver* s);
template <> ICDevice<double>& ic_of<double>(ssv_solver* s) { return s->ic_d; }
template <> ICDevice<zdouble>& ic_of<zdouble>(ssv_solver* s) { return s->ic_z; }
template <typename S> KrylovWork<S>& work_of(ssv_solver* s);
template <> KrylovWork<double>& work_of<double>(ssv_solver* s) { return s->w_d; }
template <> KrylovWork<zdouble>& work_of<zdouble>(ssv_solver* s) { return s->w_z; }

static std::string ptr_key(const void* p) {
    char b[32];
    std::snprintf(b, sizeof(b), "%p;", p);
    return b;
}

int parse_method(const char* m) {
    if (!m) return -1;
    const std::string s(m);
    if (s == "ICCG" || s == "iccg") return SSV_METHOD_ICCG;
    if (s == "SGSMRTR" || s == "sgsmrtr") return SSV_METHOD_SGSMRTR;
    if (s == "CG" || s == "cg") return SSV_METHOD_CG;
    if (s == "COCR" || s == "cocr") return SSV_METHOD_COCR;
    return -1;
}

// SGS-MRTR lives in mrtr.cu
template <typename S>
void run_mrtr(ssv_solver* sv, const ssv_config& cfg, const S* d_b, S* d_x, ssv_result* res,
              double* hist, int hist_cap);

template <typename S>
static void run_krylov(ssv_solver* sv, int method, const ssv_config& cfg, const S* d_b, S* d_x,
                       ssv_result* res, double* hist, int hist_cap) {
    cudaStream_t s = stream();
    ssv_matrix* A = sv->A;
    const int n = A->rows;
    const double t0 = wall_seconds();
    const uint8_t* fd = sv->has_fd ? sv->fd.get() : nullptr;
    int64_t nk = 0;  // kernels launched outside the iteration graph

    // FreeDofs rule on the matrix values (BuildSparseMatrixView)
    const S* vals = reinterpret_cast<const S*>(A->val.get());
    if (fd) {
        sv->vals_bc.alloc(A->val.size());
        k_bc_values<S><<<grid_for(n, kBlock), kBlock, 0, s>>>(n, A->rp.get(), A->ci.get(), vals, fd,
                                                             reinterpret_cast<S*>(sv->vals_bc.get()));
        SSV_LAUNCH_CHECK();
        vals = reinterpret_cast<const S*>(sv->vals_bc.get());
        ++nk;
    }

    // preconditioner and working numbering
    const int* wrp = A->rp.get();
    const int* wci = A->ci.get();
    const S* wv = vals;
    int lanes = A->lanes;
    const int* perm = nullptr;
    ICDevice<S>* ic = nullptr;
    if (method == SSV_METHOD_ICCG) {
        ic = &ic_of<S>(sv);
        const bool same = ic->built && ic->abmc == (cfg.use_abmc != 0) &&
                          (!ic->abmc || (ic->bs == cfg.abmc_block_size && ic->nct == cfg.abmc_num_colors &&
                                         ic->rcm == (cfg.abmc_use_rcm != 0)));
        if (!same) ic->build_pattern(n, A->h_rp, A->h_ci, cfg);
        nk += ic->factorize(vals, cfg);
        res->actual_shift = ic->actual_shift;
        if (ic->abmc) {
            wrp = ic->Arp.get();
            wci = ic->Aci.get();
            wv = ic->Av.get();
            lanes = ic->lanes;
            perm = ic->perm.get();
        }
    }
    SSV_CUDA(cudaStreamSynchronize(s));
    const double t1 = wall_seconds();

    KrylovWork<S>& w = work_of<S>(sv);
    const int dev_hist = cfg.save_residual_history ? std::max(cfg.max_iterations, 0) + 2 : 1;
    w.ensure(n, dev_hist);
    const RedBuf red = w.red();
    const int g = grid_for(n, kBlock);

    // b and x into the working numbering, constrained entries zeroed
    if (perm) {
        launch_k(k_scatter_perm<S>, g, kBlock, s, n, perm, d_b, w.bw.get(), fd);
        launch_k(k_scatter_perm<S>, g, kBlock, s, n, perm, d_x, w.xb[0].get(), fd);
    } else {
        launch_k(k_gather_perm<S>, g, kBlock, s, n, nullptr, d_b, w.bw.get(), fd, 1);
        launch_k(k_gather_perm<S>, g, kBlock, s, n, nullptr, d_x, w.xb[0].get(), fd, 1);
    }
    SSV_LAUNCH_CHECK();
    // prepare_iteration (iterative_solver.hpp:135-180)
    launch_spmv<S, S, 2>(lanes, n, wrp, wci, wv, w.xb[0].get(), w.r.get(), w.bw.get(), nullptr, nullptr,
                         RED_STORE, red, nullptr, s);
    launch_k(k_norm2<S>, g, kBlock, s, n, w.bw.get(), red, w.scal.get());
    launch_k(k_norm2<S>, g, kBlock, s, n, w.r.get(), red, w.scal.get() + 1);
    SSV_LAUNCH_CHECK();
    nk += 5;
    double2 nrm[2];
    SSV_CUDA(cudaMemcpyAsync(nrm, w.scal.get(), sizeof(nrm), cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
    const double norm_b = std::sqrt(nrm[0].x), init_norm_r = std::sqrt(nrm[1].x);
    double normalizer = cfg.norm_type == SSV_NORM_RHS ? norm_b
                      : cfg.norm_type == SSV_NORM_INITIAL_RESIDUAL ? init_norm_r : cfg.custom_norm;
    if (normalizer < 1e-15) normalizer = 1.0;

    KState h;
    std::memset(&h, 0, sizeof(h));
    h.cur = 0;
    h.best = -1;
    h.normalizer = normalizer;
    h.best_residual = DBL_MAX;
    h.norm_r = init_norm_r;
    h.final_norm = init_norm_r;
    h.tol = cfg.tolerance;
    h.abs_tol = cfg.abs_tolerance;
    h.div_threshold = cfg.divergence_threshold;
    h.maxiter = cfg.max_iterations;
    h.div_check = cfg.divergence_check;
    h.div_count = cfg.divergence_count;
    h.save_best = cfg.save_best_result;
    h.save_hist = cfg.save_residual_history;
    h.conj = cfg.conjugate;
    h.hist_cap = dev_hist;
    h.hist = w.hist.get();
    h.max_loops = loop_guard(cfg.max_iterations);
    if (cfg.save_residual_history) {
        const double h0 = init_norm_r / normalizer;
        SSV_CUDA(cudaMemcpyAsync(w.hist.get(), &h0, sizeof(double), cudaMemcpyHostToDevice, s));
        h.hist_len = 1;
    }
    if (cfg.max_iterations <= 0) {
        h.done = 1;
        h.iters = std::max(cfg.max_iterations, 0);
    }
    KState* dst = w.st.get();
    SSV_CUDA(cudaMemcpyAsync(dst, &h, sizeof(h), cudaMemcpyHostToDevice, s));

    S* z = (method == SSV_METHOD_ICCG) ? w.z.get() : w.r.get();
    std::string key;
    if (method == SSV_METHOD_CG || method == SSV_METHOD_ICCG) {
        // z = M^{-1} r, rho = (r, z), p = z (cg_solver.hpp:428-432)
        if (ic) ic->apply(w.r.get(), w.z.get(), nullptr, s);
        launch_k(k_dot<S>, g, kBlock, s, n, w.r.get(), z, cfg.conjugate, nullptr, RED_STORE, red, &dst->rho);
        launch_k(k_copy<S>, g, kBlock, s, n, z, w.p.get());
        SSV_LAUNCH_CHECK();
        nk += 2 + (ic ? ic->kernels_per_apply() : 0);
        key = "cg" + std::to_string(method) + ";" + std::to_string(n) + ";" + std::to_string(lanes) + ";" +
              ptr_key(wrp) + ptr_key(wv) + ptr_key(w.r.get()) + ptr_key(dst) +
              ptr_key(red.partials) + std::to_string(fd != nullptr) +
              (ic ? ptr_key(ic) + std::to_string(ic->gen) + ";" + ptr_key(ic->Lv.get()) + ptr_key(ic->Lv_lo.get()) + std::to_string(ic->lo) +
                        std::to_string(ic->scaled_apply) + std::to_string(ic->fwd_launch.size())
                  : std::string());
        build_graph_loop(sv->loop, key, [&](cudaGraphConditionalHandle hc, int use_cond) {
            launch_spmv<S, S, 1>(lanes, n, wrp, wci, wv, w.p.get(), w.Ap.get(), nullptr, nullptr, dst,
                                 RED_CG_ALPHA, red, nullptr, s);
            launch_k(k_cg_update<S>, g, kBlock, s, n, w.xb[0].get(), w.xb[1].get(), w.xb[2].get(), w.p.get(),
                                               w.Ap.get(), w.r.get(), dst, red);
            if (ic) ic->apply(w.r.get(), w.z.get(), dst, s);
            launch_k(k_dot<S>, g, kBlock, s, n, w.r.get(), z, cfg.conjugate, dst, RED_CG_BETA, red, nullptr);
            launch_k(k_pupdate<S>, g, kBlock, s, n, z, w.p.get(), dst);
            k_loop_ctl<<<1, 32, 0, s>>>(dst, hc, use_cond);
            SSV_LAUNCH_CHECK();
        });
    } else {  // COCR without preconditioner (sparsesolv_solvers.hpp:120-123)
        S* rt = w.z.get();
        S* q = w.Ap.get();
        launch_k(k_copy<S>, g, kBlock, s, n, w.r.get(), rt);
        launch_k(k_copy<S>, g, kBlock, s, n, rt, w.p.get());
        launch_spmv<S, S, 0>(lanes, n, wrp, wci, wv, w.p.get(), q, nullptr, nullptr, nullptr, RED_STORE, red,
                             nullptr, s);
 launch_k(k_dot<S>, g, kBlock, s, n, rt, q, 0, nullptr, RED_STORE, red, &dst->rho);
        SSV_LAUNCH_CHECK();
        nk += 4;
        key = "cocr;" + std::to_string(n) + ";" + std::to_string(lanes) + ";" + ptr_key(wrp) + ptr_key(wv) +
              ptr_key(w.r.get()) + ptr_key(dst) + ptr_key(red.partials);
        build_graph_loop(sv->loop, key, [&](cudaGraphConditionalHandle hc, int use_cond) {
            // qt = q (identity preconditioner); mu = qt^T q
            launch_k(k_dot<S>, g, kBlock, s, n, q, q, 0, dst, RED_COCR_ALPHA, red, nullptr);
            launch_k(k_cocr_update<S>, g, kBlock, s, n, w.xb[0].get(), w.xb[1].get(), w.xb[2].get(), w.p.get(), q,
                                                 q, w.r.get(), rt, dst, red);
            launch_spmv<S, S, 3>(lanes, n, wrp, wci, wv, rt, w.t.get(), nullptr, nullptr, dst, RED_COCR_BETA,
                                 red, nullptr, s);
            launch_k(k_cocr_pq<S>, g, kBlock, s, n, rt, w.t.get(), w.p.get(), q, dst);
            k_loop_ctl<<<1, 32, 0, s>>>(dst, hc, use_cond);
            SSV_LAUNCH_CHECK();
        });
    }
    if (cfg.max_iterations > 0) run_graph_loop(sv->loop, dst, cfg.max_iterations);
    SSV_CUDA(cudaMemcpyAsync(&h, dst, sizeof(h), cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
    if (h.status == SSV_ERR_TIMEOUT) fail(SSV_ERR_TIMEOUT, "Krylov loop guard fired (iteration state never finished)");
    if (!h.done) fail(SSV_ERR_RUNTIME, "Krylov loop ended without a result");

    res->converged = h.converged;
    res->iterations = h.iters;
    res->final_residual = h.final_norm / h.normalizer;
    int xbuf = h.cur;
    if (!h.converged && cfg.save_best_result) {  // build_result (iterative_solver.hpp:272-276)
        res->final_residual = h.best_residual;
        xbuf = h.best;
    }
    const S* xsrc;
    if (xbuf < 0) {  // best_x never written: the reference's zero-initialised best_x_
        w.t.zero(s);
        xsrc = w.t.get();
    } else {
        xsrc = w.xb[xbuf].get();
    }
    launch_k(k_gather_perm<S>, g, kBlock, s, n, perm, xsrc, d_x, fd, 0);
    SSV_LAUNCH_CHECK();
    nk += 1;
    res->kernel_launches = nk + (int64_t)sv->loop.body_nodes * h.loops;
    res->history_total = cfg.save_residual_history ? h.hist_len : 0;
    res->history_len = std::min(std::min(res->history_total, dev_hist), std::max(hist_cap, 0));
    if (hist && res->history_len > 0)
        SSV_CUDA(cudaMemcpyAsync(hist, w.hist.get(), sizeof(double) * res->history_len,
                                 cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
    const double t2 = wall_seconds();
    res->setup_seconds = t1 - t0;
    res->solve_seconds = t2 - t1;
}

void solver_solve_dev(ssv_solver* sv, const char* method, const ssv_config& cfg, const void* d_b, void* d_x,
                      ssv_result* res, double* hist, int hist_cap) {
    const int m = parse_method(method);
    if (m < 0)
        fail(SSV_ERR_RUNTIME, std::string("SparseSolvSolver: Unknown method '") + (method ? method : "") +
                                  "'. Available: ICCG, SGSMRTR, CG, COCR");
    std::memset(res, 0, sizeof(*res));
    ssv_config c = cfg;
    if (sv->A->dtype == SSV_F64) {
        if (m == SSV_METHOD_SGSMRTR)
            run_mrtr<double>(sv, c, static_cast<const double*>(d_b), static_cast<double*>(d_x), res, hist, hist_cap);
        else
            run_krylov<double>(sv, m, c, static_cast<const double*>(d_b), static_cast<double*>(d_x), res, hist,
                               hist_cap);
    } else {
        if (m == SSV_METHOD_SGSMRTR)
            run_mrtr<zdouble>(sv, c, static_cast<const zdouble*>(d_b), static_cast<zdouble*>(d_x), res, hist,
                              hist_cap);
        else
            run_krylov<zdouble>(sv, m, c, static_cast<const zdouble*>(d_b), static_cast<zdouble*>(d_x), res,
                                hist, hist_cap);
    }
}

// ---------------------------------------------------------------------------
// Per-phase timing of one iteration (measurement hook)
// ---------------------------------------------------------------------------
template <typename S>
static void profile_krylov(ssv_solver* sv, int method, const ssv_config& cfg, int reps, ssv_phase_profile* out) {
    cudaStream_t s = stream();
    ssv_matrix* A = sv->A;
    const int n = A->rows;
    KrylovWork<S>& w = work_of<S>(sv);
    if (w.n != n || !w.st.get()) fail(SSV_ERR_RUNTIME, "ssv_solver_profile: run a solve on this handle first");
    const S* vals = sv->has_fd ? reinterpret_cast<const S*>(sv->vals_bc.get()) : reinterpret_cast<const S*>(A->val.get());
    const int* wrp = A->rp.get();
    const int* wci = A->ci.get();
    const S* wv = vals;
    int lanes = A->lanes;
    int64_t wnnz = A->nnz;
    ICDevice<S>* ic = nullptr;
    if (method == SSV_METHOD_ICCG) {
        ic = &ic_of<S>(sv);
        if (!ic->built) fail(SSV_ERR_RUNTIME, "ssv_solver_profile: run an ICCG solve on this handle first");
        if (ic->abmc) { wrp = ic->Arp.get(); wci = ic->Aci.get(); wv = ic->Av.get(); lanes = ic->lanes; }
    }
    KState h;
    std::memset(&h, 0, sizeof(h));
    h.normalizer = 1.0;
    h.best_residual = DBL_MAX;
    h.maxiter = 1 << 30;
    h.max_loops = 1 << 30;
    h.conj = cfg.conjugate;
    h.rho = make_double2(1.0, 0.0);
    h.beta = make_double2(0.5, 0.0);
    h.alpha = make_double2(1e-3, 0.0);
    h.hist = w.hist.get();
    h.hist_cap = 0;
    DevBuf<KState> pst(1);
    SSV_CUDA(cudaMemcpyAsync(pst.get(), &h, sizeof(h), cudaMemcpyHostToDevice, s));
    KState* dst = pst.get();
    const RedBuf red = w.red();
    const int g = grid_for(n, kBlock);
    cudaEvent_t e0, e1;
    SSV_CUDA(cudaEventCreate(&e0));
    SSV_CUDA(cudaEventCreate(&e1));
    std::memset(out, 0, sizeof(*out));
    auto timed = [&](const char* name, double bytes, int kernels, auto&& launch) {
        for (int k = 0; k < 2; ++k) launch();
        SSV_CUDA(cudaEventRecord(e0, s));
        for (int k = 0; k < reps; ++k) launch();
        SSV_CUDA(cudaEventRecord(e1, s));
        SSV_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        SSV_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        const int i = out->num_phases++;
        std::snprintf(out->names[i], sizeof(out->names[i]), "%s", name);
        out->ms[i] = (double)ms / reps;
        out->bytes[i] = bytes;
        out->kernels[i] = kernels;
    };
    const double N = n, Z = (double)wnnz, sb = sizeof(S);
    if (method == SSV_METHOD_CG || method == SSV_METHOD_ICCG) {
        S* z = ic ? w.z.get() : w.r.get();
        timed("spmv_dot", Z * (4 + sb) + (N + 1) * 4 + 2 * N * sb, 1, [&] {
            launch_spmv<S, S, 1>(lanes, n, wrp, wci, wv, w.p.get(), w.Ap.get(), nullptr, nullptr, dst, RED_CG_ALPHA,
                                 red, nullptr, s);
        });
        timed("axpy_norm", 6 * N * sb, 1, [&] {
            launch_k(k_cg_update<S>, g, kBlock, s, n, w.xb[0].get(), w.xb[1].get(), w.xb[2].get(), w.p.get(), w.Ap.get(),
                                               w.r.get(), dst, red);
        });
        if (ic) {
            const double ZL = (double)ic->h_Lci.size();
            const double lb = ic->lo ? sizeof(typename ST<S>::lo) : sb;
            const int kf = ic->blk ? (int)ic->fwd_cta.size() : (int)ic->fwd_launch.size();
            const int kb = ic->blk ? (int)ic->bwd_cta.size() : (int)ic->bwd_launch.size();
            timed("ic_forward", ZL * (4 + lb) + (N + 1) * 4 + 2 * N * sb, kf,
                  [&] { ic->apply_fwd(w.r.get(), dst, s); });
            timed("ic_backward", ZL * (4 + lb) + (N + 1) * 4 + N * lb + 2 * N * sb,
                  kb + (ic->scaled_apply ? 1 : 0), [&] { ic->apply_bwd(w.z.get(), dst, s); });
        }
        timed("dot_beta", 2 * N * sb, 1, [&] {
            launch_k(k_dot<S>, g, kBlock, s, n, w.r.get(), z, cfg.conjugate, dst, RED_CG_BETA, red, nullptr);
        });
        timed("p_update", 3 * N * sb, 1, [&] { launch_k(k_pupdate<S>, g, kBlock, s, n, z, w.p.get(), dst); });
    } else if (method == SSV_METHOD_COCR) {
        S* rt = w.z.get();
        S* q = w.Ap.get();
        timed("dot_mu", 2 * N * sb, 1, [&] {
            launch_k(k_dot<S>, g, kBlock, s, n, q, q, 0, dst, RED_COCR_ALPHA, red, nullptr);
        });
        timed("update3_norm", 8 * N * sb, 1, [&] {
            launch_k(k_cocr_update<S>, g, kBlock, s, n, w.xb[0].get(), w.xb[1].get(), w.xb[2].get(), w.p.get(), q, q,
                                                 w.r.get(), rt, dst, red);
        });
        timed("spmv_dot", Z * (4 + sb) + (N + 1) * 4 + 2 * N * sb, 1, [&] {
            launch_spmv<S, S, 3>(lanes, n, wrp, wci, wv, rt, w.t.get(), nullptr, nullptr, dst, RED_COCR_BETA, red,
                                 nullptr, s);
        });
        timed("pq_update", 6 * N * sb, 1, [&] { launch_k(k_cocr_pq<S>, g, kBlock, s, n, rt, w.t.get(), w.p.get(), q, dst); });
    } else {
        fail(SSV_ERR_INVALID_ARG, "ssv_solver_profile: method not profiled");
    }
    SSV_CUDA(cudaEventDestroy(e0));
    SSV_CUDA(cudaEventDestroy(e1));
    SSV_CUDA(cudaStreamSynchronize(s));
}

void solver_profile(ssv_solver* sv, const char* method, const ssv_config& cfg, int reps, ssv_phase_profile* out) {
    const int m = parse_method(method);
    if (m < 0) fail(SSV_ERR_RUNTIME, "ssv_solver_profile: unknown method");
    if (reps < 1) reps = 1;
    if (sv->A->dtype == SSV_F64) profile_krylov<double>(sv, m, cfg, reps, out);
    else profile_krylov<zdouble>(sv, m, cfg, reps, out);
}

// ---------------------------------------------------------------------------
// ICPreconditioner handle (SparseSolvICPreconditioner)
// ---------------------------------------------------------------------------
template <typename S> ICDevice<S>& pic_of(ssv_precond* p);
template <> ICDevice<double>& pic_of<double>(ssv_precond* p) { return p->ic_d; }
template <> ICDevice<zdouble>& pic_of<zdouble>(ssv_precond* p) { return p->ic_z; }

template <typename S>
static void ic_update(ssv_precond* p) {
    cudaStream_t s = stream();
    ssv_matrix* A = p->A;
    const int n = A->rows;
    const S* vals = reinterpret_cast<const S*>(A->val.get());
    if (p->has_fd) {
        p->vals_bc.alloc(A->val.size());
        k_bc_values<S><<<grid_for(n, kBlock), kBlock, 0, s>>>(n, A->rp.get(), A->ci.get(), vals, p->fd.get(),
                                                             reinterpret_cast<S*>(p->vals_bc.get()));
        SSV_LAUNCH_CHECK();
        vals = reinterpret_cast<const S*>(p->vals_bc.get());
    }
    ICDevice<S>& ic = pic_of<S>(p);
    const ssv_config& cfg = p->cfg;
    // the pattern cache of ICPreconditioner::setup (ic_preconditioner.hpp:78-81)
    const bool same = ic.built && ic.abmc == (cfg.use_abmc != 0) &&
                      (!ic.abmc || (ic.bs == cfg.abmc_block_size && ic.nct == cfg.abmc_num_colors &&
                                    ic.rcm == (cfg.abmc_use_rcm != 0)));
    if (!same) ic.build_pattern(n, A->h_rp, A->h_ci, cfg);
    ic.factorize(vals, cfg);
    // Mult goes through ICPreconditioner::apply -> apply_abmc (:215-225,
    // :655-700) in original numbering for every ABMC variant, which (single
    // threaded) does not scale
    if (ic.abmc) ic.scaled_apply = false;
    const size_t words = (size_t)n * (sizeof(S) / sizeof(double));
    p->xw.alloc(words);
    p->yw.alloc(words);
    SSV_CUDA(cudaStreamSynchronize(s));
    p->ready = true;
}

// Mult (sparsesolv_precond.hpp:123-136): y = M^{-1} x, constrained y = 0.
template <typename S>
void ic_apply_dev(ssv_precond* p, const S* x, S* y, const KState* st, cudaStream_t s) {
    ICDevice<S>& ic = pic_of<S>(p);
    const int n = p->A->rows;
    const uint8_t* fd = p->has_fd ? p->fd.get() : nullptr;
    const int g = grid_for(n, kBlock);
    S* xw = reinterpret_cast<S*>(p->xw.get());
    S* yw = reinterpret_cast<S*>(p->yw.get());
    if (ic.abmc) {
        launch_k(k_scatter_perm<S>, g, kBlock, s, n, ic.perm.get(), x, xw, nullptr);
        ic.apply(xw, yw, st, s);
        launch_k(k_gather_perm<S>, g, kBlock, s, n, ic.perm.get(), yw, y, fd, 1);
    } else {
        ic.apply(x, y, st, s);
        if (fd) launch_k(k_mask_zero<S>, g, kBlock, s, n, y, fd);
    }
    SSV_LAUNCH_CHECK();
}

void precond_update(ssv_precond* p) {
    if (p->kind == 5) amg_update(p->amg.get(), p->A);
    else if (p->kind == 4) sgs_update(p);
    else if (p->A->dtype == SSV_F64) ic_update<double>(p);
    else ic_update<zdouble>(p);
}

void precond_apply_dev(ssv_precond* p, const void* d_x, void* d_y) {
    if (!p->ready)
        fail(SSV_ERR_RUNTIME, p->kind == 4   ? "SGSPreconditioner::apply called before setup"
                              : p->kind == 5 ? "CompactAMG::Mult called before Setup"
                                             : "ICPreconditioner::apply called before setup");
    if (p->vdtype == SSV_F64)
        precond_apply_any<double>(p, static_cast<const double*>(d_x), static_cast<double*>(d_y), nullptr, stream());
    else
        precond_apply_any<zdouble>(p, static_cast<const zdouble*>(d_x), static_cast<zdouble*>(d_y), nullptr,
                                   stream());
    SSV_CUDA(cudaStreamSynchronize(stream()));
}

double precond_actual_shift(const ssv_precond* p) {
    return p->A->dtype == SSV_F64 ? p->ic_d.actual_shift : p->ic_z.actual_shift;
}

// ---------------------------------------------------------------------------
// y = A x
// ---------------------------------------------------------------------------
void matrix_spmv_dev(ssv_matrix* A, const void* d_x, void* d_y) {
    cudaStream_t s = stream();
    RedBuf red{nullptr, nullptr};
    if (A->dtype == SSV_F64)
        launch_spmv<double, double, 0>(A->lanes, A->rows, A->rp.get(), A->ci.get(), A->val.get(),
                                       static_cast<const double*>(d_x), static_cast<double*>(d_y), nullptr,
                                       nullptr, nullptr, RED_STORE, red, nullptr, s);
    else
        launch_spmv<zdouble, zdouble, 0>(A->lanes, A->rows, A->rp.get(), A->ci.get(),
                                         reinterpret_cast<const zdouble*>(A->val.get()),
                                         static_cast<const zdouble*>(d_x), static_cast<zdouble*>(d_y), nullptr,
                                         nullptr, nullptr, RED_STORE, red, nullptr, s);
    SSV_CUDA(cudaStreamSynchronize(s));
}

// explicit instantiations used by other translation units
template void launch_spmv<double, double, 0>(int, int, const int*, const int*, const double*, const double*,
                                             double*, const double*, const uint8_t*, KState*, int, RedBuf,
                                             double2*, cudaStream_t);
template void launch_spmv<zdouble, zdouble, 0>(int, int, const int*, const int*, const zdouble*,
                                               const zdouble*, zdouble*, const zdouble*, const uint8_t*,
                                               KState*, int, RedBuf, double2*, cudaStream_t);
template void launch_spmv<double, double, 2>(int, int, const int*, const int*, const double*, const double*,
                                             double*, const double*, const uint8_t*, KState*, int, RedBuf,
                                             double2*, cudaStream_t);
template void launch_spmv<zdouble, zdouble, 2>(int, int, const int*, const int*, const zdouble*,
                                               const zdouble*, zdouble*, const zdouble*, const uint8_t*,
                                               KState*, int, RedBuf, double2*, cudaStream_t);
template void launch_spmv<double, double, 3>(int, int, const int*, const int*, const double*, const double*,
                                             double*, const double*, const uint8_t*, KState*, int, RedBuf,
                                             double2*, cudaStream_t);
template void launch_spmv<zdouble, zdouble, 3>(int, int, const int*, const int*, const zdouble*,
                                               const zdouble*, zdouble*, const zdouble*, const uint8_t*,
                                               KState*, int, RedBuf, double2*, cudaStream_t);
template void ic_apply_dev<double>(ssv_precond*, const double*, double*, const KState*, cudaStream_t);
template void ic_apply_dev<zdouble>(ssv_precond*, const zdouble*, zdouble*, const KState*, cudaStream_t);
template struct KrylovWork<double>;
template struct KrylovWork<zdouble>;

}  // namespace ssv
