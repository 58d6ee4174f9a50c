// objects.cuh -- the device objects behind the C ABI handles.
#pragma once

#include <algorithm>
#include <cstdlib>
#include <memory>
#include <string>

#include "host_order.hpp"
#include "kernels.cuh"
#include "sell.cuh"

namespace ssv {

cudaStream_t stream();

// Kernel launch with programmatic dependent launch allowed (the kernel must
// start with pdl_gate()); SSV_PDL=0 launches without it.
inline bool pdl_enabled() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("SSV_PDL");
        v = (e && e[0] == '0') ? 0 : 1;
    }
    return v != 0;
}

template <typename... KArgs, typename... Args>
inline void launch_k(void (*k)(KArgs...), dim3 grid, dim3 block, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    SSV_CUDA(cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...));
}

// Host -> device copy of a large pageable array through threaded pinned staging
// (small copies: one cudaMemcpyAsync); ordered after the work queued on s.
void h2d_staged(void* dst, const void* src, size_t bytes, cudaStream_t s);

// Sub-warp width of the CSR kernels from the mean row length.
int pick_lanes(double nnz_per_row);
// SpMV launch shape: lanes | (rows per row group and pass) << 8
int pick_shape(int n, double nnz_per_row);

// Side streams for independent pieces of one stream's work: fork() makes k
// side streams wait for the work queued so far on s, join() makes s wait for
// them. Under stream capture the side work becomes parallel branches of the
// graph; outside capture it runs concurrently.
struct ForkSet {
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> ev;  // ev[0] fork point, ev[1 + i] side i done
    ForkSet() = default;
    ForkSet(const ForkSet&) = delete;
    ForkSet& operator=(const ForkSet&) = delete;
    ~ForkSet() {
        for (auto e : ev) cudaEventDestroy(e);
        for (auto t : side) cudaStreamDestroy(t);
    }
    void ensure(int k) {
        while ((int)side.size() < k) {
            cudaStream_t t;
            SSV_CUDA(cudaStreamCreateWithFlags(&t, cudaStreamNonBlocking));
            side.push_back(t);
        }
        while ((int)ev.size() < k + 1) {
            cudaEvent_t e;
            SSV_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            ev.push_back(e);
        }
    }
    void fork(cudaStream_t s, int k) {
        SSV_CUDA(cudaEventRecord(ev[0], s));
        for (int i = 0; i < k; ++i) SSV_CUDA(cudaStreamWaitEvent(side[i], ev[0], 0));
    }
    void join(cudaStream_t s, int k) {
        for (int i = 0; i < k; ++i) {
            SSV_CUDA(cudaEventRecord(ev[1 + i], side[i]));
            SSV_CUDA(cudaStreamWaitEvent(s, ev[1 + i], 0));
        }
    }
};

// Launch y = A x style SpMV for any lanes/mode (mask zeroes masked rows).
template <typename S, typename SV, int MODE>
void launch_spmv(int lanes, int n, const int* rp, const int* ci, const SV* v, const S* x, S* y,
                 const S* b, const uint8_t* mask, KState* st, int op, RedBuf red, double2* out,
                 cudaStream_t s);

// Reusable reduction scratch + device state of one Krylov solve.
template <typename S>
struct KrylovWork {
    int n = -1;
    DevBuf<S> xb[3], r, z, p, Ap, t, qt, bw;
    DevBuf<KState> st;
    DevBuf<double> hist;
    DevBuf<double2> partials, scal;
    DevBuf<unsigned int> ticket;
    void ensure(int n_, int hist_cap);
    RedBuf red() const { return RedBuf{partials.get(), ticket.get()}; }
};

// A CUDA graph of one iteration body, looped on the device by a WHILE
// conditional node (or, when SSV_GRAPH_MODE=chunk, a graph of `chunk` copies
// relaunched by the host until the state says done).
struct GraphLoop {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool cond = false;
    int chunk = 1;
    size_t body_nodes = 0;  // kernel nodes per iteration body
    std::string key;
    GraphLoop() = default;
    GraphLoop(const GraphLoop&) = delete;
    GraphLoop& operator=(const GraphLoop&) = delete;
    ~GraphLoop() { reset(); }
    void reset();
};

bool graph_while_mode();

// Ends a capture that a thrown exception interrupted (the stream leaves
// capture mode; the partial graph is dropped).
inline void abandon_capture(cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
        cudaGraph_t partial = nullptr;
        cudaStreamEndCapture(s, &partial);
        if (partial) cudaGraphDestroy(partial);
    }
    cudaGetLastError();
}

template <typename F>
void build_graph_loop_body(GraphLoop& g, cudaStream_t s, F& body) {
    if (graph_while_mode()) {
        SSV_CUDA(cudaGraphCreate(&g.graph, 0));
        cudaGraphConditionalHandle h;
        SSV_CUDA(cudaGraphConditionalHandleCreate(&h, g.graph, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        SSV_CUDA(cudaGraphAddNode(&node, g.graph, nullptr, 0, &cp));
        cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
        SSV_CUDA(cudaStreamBeginCaptureToGraph(s, bodyg, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal));
        body(h, 1);
        SSV_CUDA(cudaStreamEndCapture(s, &bodyg));
        SSV_CUDA(cudaGraphGetNodes(bodyg, nullptr, &g.body_nodes));
        SSV_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
        g.cond = true;
    } else {
        SSV_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        for (int c = 0; c < g.chunk; ++c) body(cudaGraphConditionalHandle(0), 0);
        SSV_CUDA(cudaStreamEndCapture(s, &g.graph));
        SSV_CUDA(cudaGraphGetNodes(g.graph, nullptr, &g.body_nodes));
        g.body_nodes /= (size_t)std::max(g.chunk, 1);
        SSV_CUDA(cudaGraphInstantiate(&g.exec, g.graph, 0));
        g.cond = false;
    }
}

template <typename F>
void build_graph_loop(GraphLoop& g, const std::string& key_in, F&& body) {
    const std::string key = key_in + (graph_while_mode() ? "|while" : "|chunk");
    if (g.exec && g.key == key) return;
    g.reset();
    cudaStream_t s = stream();
    try {
        build_graph_loop_body(g, s, body);
    } catch (...) {  // a failure inside the body (an allocation, a refused argument)
        abandon_capture(s);
        g.reset();
        throw;
    }
    g.key = key;
}


// Runs the loop until the device state reports done (bounded).
void run_graph_loop(GraphLoop& g, KState* d_st, int max_iters);
// Loop-body cap of a device-looped solve of maxiter iterations (see solver.cu).
int loop_guard(int maxiter);
void set_loop_guard(int loops);

// ---------------------------------------------------------------------------
// IC(0) preconditioner on the device (ic_preconditioner.hpp)
// ---------------------------------------------------------------------------
template <typename S>
struct ICDevice {
    using SL = typename ST<S>::lo;
    int n = 0;
    // pattern cache key (ICPreconditioner caches its ordering per pattern,
    // ic_preconditioner.hpp:74-81)
    bool built = false, abmc = false, rcm = false;
    int bs = 0, nct = 0;
    unsigned gen = 0;  // bumped on every pattern rebuild (part of graph keys)
    // schedule: launches in processing order, each a unit range
    std::vector<std::pair<int, int>> fwd_launch, bwd_launch;
    DevBuf<int> uoff, rows_f, rows_b;  // uoff: ABMC block row offsets
    int num_colors = 0, num_blocks = 0, num_levels_f = 0, num_levels_b = 0;
    std::vector<int> h_perm;           // ordering[old] = new (ABMC)
    std::vector<int> h_boff;           // ABMC block row offsets
    std::vector<int> sched_color_offsets;
    DevBuf<int> perm;
    // working matrix in ABMC numbering (values gathered through Asrc)
    std::vector<int> h_Arp;
    DevBuf<int> Arp, Aci, Asrc;
    DevBuf<S> Av;
    int lanes = 8;  // SpMV launch shape of the ABMC-ordered matrix (pick_shape)
    // factor L (diag last), U = L^T (diag first)
    std::vector<int> h_Lrp, h_Lci;
    DevBuf<int> Lrp, Lci, Lsrc, Urp, Uci, Usrc;
    DevBuf<S> Lv, Uv, inv;
    DevBuf<SL> Lv_lo, Uv_lo, inv_lo;
    DevBuf<double> scaling;
    DevBuf<int> flag;
    bool scaled_apply = false, lo = false;
    int missing_row = -1;
    double actual_shift = 0.0;
    DevBuf<S> tw;  // forward-sweep output
    // ABMC block-sweep layout (k_ic_fwd_blk / k_ic_bwd_blk): external parts of
    // L and U rows, packed strictly-lower intra-block table, diagonal
    bool blk = false;
    int blk_lanes = 0, tri = 1;
    // launches of the block sweeps in processing order: kind 0 = range of
    // ordinary blocks [a, b) (sub-warp kernels), kind 1 = range [a, b) of the
    // rows_f / rows_b lists (one level of an oversized block; factorisation),
    // kind 2 = an oversized block swept by one CTA over the level offsets
    // lev_f / lev_b [a, b] (apply)
    struct Launch { int kind, a, b, smem = 0, color = -1; };  // smem > 0: oversized block swept staged (bytes)
    std::vector<Launch> fwd_blk, bwd_blk, fwd_cta, bwd_cta;
    DevBuf<int> lev_f, lev_b;
    // staged sweeps of oversized blocks: per position in rows_f / rows_b, the
    // row's entries (value index, column, position in the block or -1)
    DevBuf<int> sf_rp, sf_src, sf_col, sf_loc, sb_rp, sb_src, sb_col, sb_loc;
    DevBuf<int> erp, eci, esrc, urpe, ucie, usrce, isrc, dsrc;
    DevBuf<S> ev, uev, iv, dv;
    DevBuf<SL> ev_lo, uev_lo, iv_lo, dv_lo;

    // Pattern set-up from the matrix pattern (host) for the given options.
    void build_pattern(int n, const std::vector<int>& rp, const std::vector<int>& ci,
                       const ssv_config& cfg);
    // Gathers values (vals = BC-modified matrix values, original numbering),
    // factorises with auto-shift on the device, builds U and the FP32 form.
    // Returns the number of kernels launched.
    int factorize(const S* vals, const ssv_config& cfg);
    // y = M^{-1} x in the working numbering (ABMC numbering or natural).
    void apply(const S* x, S* y, const KState* st, cudaStream_t s) const {
        apply_fwd(x, st, s);
        apply_bwd(y, st, s);
    }
    void apply_fwd(const S* x, const KState* st, cudaStream_t s) const;  // x -> tw
    void apply_bwd(S* y, const KState* st, cudaStream_t s) const;        // tw -> y
    int kernels_per_apply() const {
        if (blk)
            return (int)fwd_cta.size() + (int)bwd_cta.size() +
                   (scaled_apply ? 1 : 0);
        return (int)(fwd_launch.size() + bwd_launch.size()) + (scaled_apply ? 1 : 0);
    }
};

// Symmetric Gauss-Seidel preconditioner (sgs_preconditioner.hpp): level sets
// of the forward (j < i) and backward (j > i) sweeps over the full pattern,
// 1/a_ii, and the work vector between the sweeps.
template <typename S>
struct SgsDevice {
    bool built = false;
    unsigned gen = 0;
    std::vector<std::pair<int, int>> fwd_lev, bwd_lev;  // row ranges of rows_f / rows_b per level
    DevBuf<int> rows_f, rows_b;
    DevBuf<S> inv, tmp;
};

}  // namespace ssv

// ---------------------------------------------------------------------------
// Handles of the C ABI
// ---------------------------------------------------------------------------
struct ssv_matrix {
    int rows = 0, cols = 0;
    int64_t nnz = 0;
    int dtype = SSV_F64;
    std::vector<int> h_rp, h_ci;
    ssv::DevBuf<int> rp, ci;
    ssv::DevBuf<double> val;  // nnz (F64) or 2*nnz (C128) doubles
    int lanes = 8;  // SpMV launch shape (pick_shape)
    unsigned vgen = 0;  // bumped whenever the values change
    // sliced-ELL copy for the COCR iteration's SpMV of a large matrix (built on
    // first use, values gathered again after a value change)
    ssv::SellPattern sell;
    ssv::DevBuf<double> sell_v;
    unsigned sell_vgen = ~0u;
    bool sell_tried = false;
};

struct ssv_solver {
    ssv_matrix* A = nullptr;
    bool has_fd = false;
    std::vector<uint8_t> h_fd;
    ssv::DevBuf<uint8_t> fd;
    ssv::DevBuf<double> vals_bc;
    ssv::DevBuf<double> io_b, io_x;  // staging for host-pointer solves
    ssv::ICDevice<double> ic_d;
    ssv::ICDevice<ssv::zdouble> ic_z;
    ssv::SgsDevice<double> sgs_d;
    ssv::SgsDevice<ssv::zdouble> sgs_z;
    ssv::KrylovWork<double> w_d;
    ssv::KrylovWork<ssv::zdouble> w_z;
    ssv::GraphLoop loop;
};

namespace ssv {
struct AmsState;
void ams_free(AmsState* a);
struct AmgOnly;
void amg_free(AmgOnly* g);
}  // namespace ssv

struct ssv_precond {
    int kind = 0;    // 1 = IC, 2 = CompactAMS (real), 3 = ComplexCompactAMS, 4 = SGS, 5 = CompactAMG
    int vdtype = 0;  // scalar type of the vectors it applies to
    int n = 0;       // vector length
    ssv_matrix* A = nullptr;
    bool has_fd = false;
    std::vector<uint8_t> h_fd;
    ssv::DevBuf<uint8_t> fd;
    ssv::DevBuf<double> vals_bc;
    ssv_config cfg{};
    bool ready = false;
    ssv::ICDevice<double> ic_d;
    ssv::ICDevice<ssv::zdouble> ic_z;
    ssv::SgsDevice<double> sgs_d;
    ssv::SgsDevice<ssv::zdouble> sgs_z;
    ssv::DevBuf<double> xw, yw, io_x, io_y;
    std::unique_ptr<ssv::AmsState, void (*)(ssv::AmsState*)> ams{nullptr, ssv::ams_free};
    std::unique_ptr<ssv::AmgOnly, void (*)(ssv::AmgOnly*)> amg{nullptr, ssv::amg_free};
    virtual ~ssv_precond() = default;
};
