// amg_device.cu -- see amg_device.hpp. The host counterparts (amg_setup.cpp)
// fix the arithmetic: a thread per output row runs each row's loops in the
// host's order, products and sums rounded one at a time (__dmul_rn /
// __dadd_rn / __ddiv_rn), so the values are the host's bit for bit. Symbolic
// patterns (which columns a product row holds) come from a per-warp hash set
// in shared memory, sorted afterwards; their order never enters a sum.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <random>

#include "amg_device.hpp"

namespace ssv {
namespace {

constexpr int kT = 256;
constexpr int kHashBits = 11;
constexpr int kHash = 1 << kHashBits;  // per-warp slots of the symbolic hash set
constexpr int kSymWarps = 4;           // warps per block of the symbolic kernels
constexpr int kSymSmem = kSymWarps * kHash * (int)(sizeof(unsigned long long) + sizeof(int));  // 96 KB

inline int blocks_for(int64_t n, int t = kT) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + t - 1) / t, (int64_t)sm_count() * 16));
}

// ---- prefix sums -----------------------------------------------------------
// out[i] = sum cnt[0..i), out[n] = total (one block: set-up sizes only)
__global__ void __launch_bounds__(1024) k_scan(int n, const int* __restrict__ cnt, int* __restrict__ out) {
    __shared__ long long sh[1024];
    const int T = blockDim.x, t = threadIdx.x;
    const int chunk = (n + T - 1) / T;
    const int a = min(n, t * chunk), b = min(n, a + chunk);
    long long s = 0;
    for (int i = a; i < b; ++i) s += cnt[i];
    sh[t] = s;
    __syncthreads();
    for (int off = 1; off < T; off <<= 1) {
        const long long v = t >= off ? sh[t - off] : 0;
        __syncthreads();
        sh[t] += v;
        __syncthreads();
    }
    long long base = t ? sh[t - 1] : 0;
    for (int i = a; i < b; ++i) {
        out[i] = (int)base;
        base += cnt[i];
    }
    if (t == T - 1) out[n] = (int)sh[T - 1];
}

int scan(int n, const int* cnt, int* out, cudaStream_t s) {
    k_scan<<<1, 1024, 0, s>>>(n, cnt, out);
    SSV_LAUNCH_CHECK();
    int tot = 0;
    SSV_CUDA(cudaMemcpyAsync(&tot, out + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
    return tot;
}

__device__ __forceinline__ int lbound(const int* a, int len, int key) {
    int lo = 0, hi = len;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// ---- transpose ---------------------------------------------------------------
__global__ void k_col_count(int64_t nnz, const int* __restrict__ ci, int* __restrict__ cnt) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&cnt[ci[k]], 1);
}

__global__ void k_tr_scatter(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                             const double* __restrict__ v, const int* __restrict__ Trp, int* __restrict__ fill,
                             int* __restrict__ Tci, double* __restrict__ Tv, int* __restrict__ Tk) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int c = ci[k];
            const int p = Trp[c] + atomicAdd(&fill[c], 1);
            Tci[p] = i;
            if (Tv) Tv[p] = v[k];
            if (Tk) Tk[p] = k;
        }
}

// each row in increasing key (the source entry's index, i.e. the host's
// order); a and b move with the key
__global__ void k_row_sort(int n, const int* __restrict__ rp, int* __restrict__ key, int* __restrict__ a,
                           double* __restrict__ b) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int k0 = rp[r], k1 = rp[r + 1];
        for (int k = k0 + 1; k < k1; ++k) {
            const int kk = key[k], ka = a[k];
            const double kb = b ? b[k] : 0.0;
            int q = k - 1;
            while (q >= k0 && key[q] > kk) {
                key[q + 1] = key[q];
                a[q + 1] = a[q];
                if (b) b[q + 1] = b[q];
                --q;
            }
            key[q + 1] = kk;
            a[q + 1] = ka;
            if (b) b[q + 1] = kb;
        }
    }
}

// pattern-only transpose (row order not needed: PMIS reads counts and sets)
void graph_transpose(int n, int m, const int* rp, const int* ci, int64_t nnz, DevBuf<int>& Trp, DevBuf<int>& Tci,
                     cudaStream_t s) {
    DevBuf<int> cnt(std::max(m, 1)), fill(std::max(m, 1));
    cnt.zero(s);
    fill.zero(s);
    Trp.alloc(m + 1);
    if (nnz) k_col_count<<<blocks_for(nnz), kT, 0, s>>>(nnz, ci, cnt.get());
    scan(m, cnt.get(), Trp.get(), s);
    Tci.alloc(std::max<int64_t>(nnz, 1));
    if (nnz)
        k_tr_scatter<<<blocks_for(n), kT, 0, s>>>(n, rp, ci, nullptr, Trp.get(), fill.get(), Tci.get(), nullptr,
                                                   nullptr);
    SSV_LAUNCH_CHECK();
}

// ---- symbolic products --------------------------------------------------------
// Row `row` of X Y (Z): the distinct columns, counted (Cci == null) or written
// sorted at Crp[row]. X's entries in order, Y's strided over the lanes, Z's in
// order. A warp's hash set (kHash slots) holds the columns of one row; a slot
// stores (row + 1) << 32 | column, so the slots of earlier rows count as free
// and the table is cleared only once per block. Each column is appended to
// the warp's list as it is first inserted; more than kHash distinct columns
// in a row is an overflow.
template <bool THREE>
__global__ void __launch_bounds__(kSymWarps * 32)
k_sym(int rows, const int* __restrict__ Xrp, const int* __restrict__ Xci, const int* __restrict__ Yrp,
      const int* __restrict__ Yci, const int* __restrict__ Zrp, const int* __restrict__ Zci, int* __restrict__ cnt,
      const int* __restrict__ Crp, int* __restrict__ Cci, int* overflow) {
    extern __shared__ unsigned long long smem64[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long* tab = smem64 + warp * kHash;
    int* lst = reinterpret_cast<int*>(smem64 + kSymWarps * kHash) + warp * kHash;
    __shared__ int fillc[kSymWarps];
    for (int t = threadIdx.x; t < kSymWarps * kHash; t += blockDim.x) smem64[t] = 0ull;
    __syncthreads();
    for (int row = blockIdx.x * kSymWarps + warp; row < rows; row += gridDim.x * kSymWarps) {
        const unsigned long long tag = (unsigned long long)(row + 1) << 32;
        if (lane == 0) fillc[warp] = 0;
        __syncwarp();
        int mine = 0;
        bool ovf = false;
        auto insert = [&](int key) {
            const unsigned long long mark = tag | (unsigned)key;
            unsigned h = ((unsigned)key * 2654435761u) >> (32 - kHashBits);
            volatile unsigned long long* vt = tab;  // other lanes write through atomics
            for (int probe = 0; probe < 2 * kHash; ++probe) {
                const unsigned long long cur = vt[h];
                if ((cur & 0xffffffff00000000ull) == tag) {  // a column of this row
                    if (cur == mark) return;
                    h = (h + 1) & (kHash - 1);
                    continue;
                }
                if (atomicCAS(&tab[h], cur, mark) == cur) {  // claimed a free slot
                    const int pos = atomicAdd(&fillc[warp], 1);
                    if (pos < kHash) lst[pos] = key;
                    ++mine;
                    return;
                }
                // another lane took this slot first: look at it again
            }
            ovf = true;
        };
        for (int x = Xrp[row]; x < Xrp[row + 1]; ++x) {
            const int i = Xci[x];
            for (int y = Yrp[i] + lane; y < Yrp[i + 1]; y += 32) {
                const int j = Yci[y];
                if constexpr (THREE) {
                    for (int z = Zrp[j]; z < Zrp[j + 1]; ++z) insert(Zci[z]);
                } else {
                    insert(j);
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
        if (__any_sync(0xffffffffu, ovf) && lane == 0) atomicExch(overflow, 1);
        __syncwarp();
        if (!Cci) {
            if (lane == 0) cnt[row] = mine;
        } else {
            const int m = min(mine, kHash);
            int* out = Cci + Crp[row];
            for (int e = lane; e < m; e += 32) {
                const int key = lst[e];
                int r = 0;
                for (int f = 0; f < m; ++f) r += lst[f] < key;
                out[r] = key;
            }
        }
        __syncwarp();
    }
}

template <bool THREE>
bool symbolic(int rows, int cols, const int* Xrp, const int* Xci, const int* Yrp, const int* Yci, const int* Zrp,
              const int* Zci, DCsr& C, cudaStream_t s) {
    static std::once_flag once;
    std::call_once(once, [] {
        SSV_CUDA(cudaFuncSetAttribute(k_sym<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSymSmem));
        SSV_CUDA(cudaFuncSetAttribute(k_sym<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSymSmem));
    });
    DevBuf<int> cnt(std::max(rows, 1)), ovf(1);
    ovf.zero(s);
    const int grid = std::max(1, std::min((rows + kSymWarps - 1) / kSymWarps, sm_count() * 8));
    k_sym<THREE><<<grid, kSymWarps * 32, kSymSmem, s>>>(rows, Xrp, Xci, Yrp, Yci, Zrp, Zci, cnt.get(), nullptr,
                                                        nullptr, ovf.get());
    SSV_LAUNCH_CHECK();
    C.n = rows;
    C.m = cols;
    C.rp.alloc(rows + 1);
    C.nnz = scan(rows, cnt.get(), C.rp.get(), s);
    int h_ovf = 0;
    SSV_CUDA(cudaMemcpyAsync(&h_ovf, ovf.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
    if (h_ovf) return false;
    C.ci.alloc(std::max<int64_t>(C.nnz, 1));
    C.v.alloc(std::max<int64_t>(C.nnz, 1));
    C.v.zero(s);
    k_sym<THREE><<<grid, kSymWarps * 32, kSymSmem, s>>>(rows, Xrp, Xci, Yrp, Yci, Zrp, Zci, cnt.get(), C.rp.get(),
                                                        C.ci.get(), ovf.get());
    SSV_LAUNCH_CHECK();
    return true;
}

// ---- numeric products (host order, one thread per output row) ----------------
// csr_rap: for q in Pt row k, a in A row i, b in P row j:
// acc[l] += (Pt(k,i) * A(i,j)) * P(j,l)
__global__ void k_rap_num(int nc, const int* __restrict__ Ptrp, const int* __restrict__ Ptci,
                          const double* __restrict__ Ptv, const int* __restrict__ Arp, const int* __restrict__ Aci,
                          const double* __restrict__ Av, const int* __restrict__ Prp, const int* __restrict__ Pci,
                          const double* __restrict__ Pv, const int* __restrict__ Crp, const int* __restrict__ Cci,
                          double* __restrict__ Cv) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nc; k += gridDim.x * blockDim.x) {
        const int c0 = Crp[k], len = Crp[k + 1] - c0;
        const int* cc = Cci + c0;
        double* cv = Cv + c0;
        for (int q = Ptrp[k]; q < Ptrp[k + 1]; ++q) {
            const int i = Ptci[q];
            const double pki = Ptv[q];
            for (int a = Arp[i]; a < Arp[i + 1]; ++a) {
                const int j = Aci[a];
                const double pa = __dmul_rn(pki, Av[a]);
                for (int b = Prp[j]; b < Prp[j + 1]; ++b) {
                    const int pos = lbound(cc, len, Pci[b]);
                    cv[pos] = __dadd_rn(cv[pos], __dmul_rn(pa, Pv[b]));
                }
            }
        }
    }
}

// csr_mul: for a in A row i, b in B row j: acc[l] += A(i,j) * B(j,l)
__global__ void k_mul_num(int n, const int* __restrict__ Arp, const int* __restrict__ Aci,
                          const double* __restrict__ Av, const int* __restrict__ Brp, const int* __restrict__ Bci,
                          const double* __restrict__ Bv, const int* __restrict__ Crp, const int* __restrict__ Cci,
                          double* __restrict__ Cv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c0 = Crp[i], len = Crp[i + 1] - c0;
        const int* cc = Cci + c0;
        double* cv = Cv + c0;
        for (int a = Arp[i]; a < Arp[i + 1]; ++a) {
            const int j = Aci[a];
            const double av = Av[a];
            for (int b = Brp[j]; b < Brp[j + 1]; ++b) {
                const int pos = lbound(cc, len, Bci[b]);
                cv[pos] = __dadd_rn(cv[pos], __dmul_rn(av, Bv[b]));
            }
        }
    }
}

// csr_add: union of two sorted rows; per column 0 + a A(i,c) then + b B(i,c)
// (the host's stable sort of the concatenated row, summed in that order)
__global__ void k_add(int n, const int* __restrict__ Arp, const int* __restrict__ Aci, const double* __restrict__ Av,
                      double a, const int* __restrict__ Brp, const int* __restrict__ Bci,
                      const double* __restrict__ Bv, double b, int* __restrict__ cnt, const int* __restrict__ Crp,
                      int* __restrict__ Cci, double* __restrict__ Cv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int pa = Arp[i], ea = Arp[i + 1], pb = Brp[i], eb = Brp[i + 1];
        int c = 0, w = Crp ? Crp[i] : 0;
        while (pa < ea || pb < eb) {
            const int col = (pb >= eb || (pa < ea && Aci[pa] <= Bci[pb])) ? Aci[pa] : Bci[pb];
            double sum = 0.0;
            while (pa < ea && Aci[pa] == col) sum = __dadd_rn(sum, __dmul_rn(a, Av[pa++]));
            while (pb < eb && Bci[pb] == col) sum = __dadd_rn(sum, __dmul_rn(b, Bv[pb++]));
            if (Cci) {
                Cci[w] = col;
                Cv[w] = sum;
                ++w;
            }
            ++c;
        }
        if (cnt) cnt[i] = c;
    }
}

// ---- the small row-wise steps -------------------------------------------------
__global__ void k_bc(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                     const uint8_t* __restrict__ fd, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int j = ci[k];
            double x = v[k];
            if (fd) {
                if (!fd[i]) x = (j == i) ? 1.0 : 0.0;
                else if (!fd[j]) x = 0.0;
            }
            out[k] = x;
        }
}

// l1_norms (plain): sum |a_ik| in row order, 1 for a zero row
__global__ void k_l1(int n, const int* __restrict__ rp, const double* __restrict__ v, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) s = __dadd_rn(s, fabs(v[k]));
        out[i] = (s > 0) ? s : 1.0;
    }
}

__global__ void k_fix_zero_rows(int n, const int* __restrict__ rp, const int* __restrict__ ci, double* __restrict__ v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double l1 = 0.0;
        int dp = -1;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            l1 = __dadd_rn(l1, fabs(v[k]));
            if (ci[k] == i) dp = k;
        }
        if (l1 == 0.0 && dp >= 0) v[dp] = 1.0;
    }
}

__global__ void k_fine_l1(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                          double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double diag = 0.0, off = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            if (ci[k] == i) diag = fabs(v[k]);
            else off = __dadd_rn(off, fabs(v[k]));
        }
        const double t = __dadd_rn(diag, __dmul_rn(0.5, off));
        out[i] = (t <= __dmul_rn(4.0 / 3.0, diag)) ? ((diag > 0) ? diag : 1.0) : ((t > 0) ? t : 1.0);
    }
}

// ComputeStrength: count (Sci == null) or fill
__global__ void k_strength(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                           double theta, int* __restrict__ cnt, const int* __restrict__ Srp, int* __restrict__ Sci) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double max_neg = 0.0, max_abs = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] != i) {
                const double x = v[k];
                if (-x > max_neg) max_neg = -x;
                const double ax = fabs(x);
                if (ax > max_abs) max_abs = ax;
            }
        const bool neg = max_neg > 0;
        const double thr = __dmul_rn(theta, neg ? max_neg : max_abs);
        int c = 0, w = Srp ? Srp[i] : 0;
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] != i && (neg ? (-v[k] >= thr) : (fabs(v[k]) >= thr))) {
                if (Sci) Sci[w++] = ci[k];
                ++c;
            }
        if (cnt) cnt[i] = c;
    }
}

// ---- PMIS (CoarsenPMIS, compact_amg.hpp:378-454) --------------------------------
// The host visits the undecided rows of a round in order and makes row i a C
// point when no still-undecided neighbour has a larger measure; rows made C
// earlier in the same sweep no longer count as undecided. So i becomes C
// exactly when every neighbour j undecided at the round's start with
// measure[j] > measure[i] is a lower row that itself becomes C in this sweep.
// The device resolves that by fixpoint: a row is C once all such j are known
// C, not C as soon as one such j is higher or known not C; the lowest
// unresolved row is always resolvable, so every pass decides at least one.
enum : int { PM_OFF = 0, PM_UNK = 1, PM_C = 2, PM_NOTC = 3 };

__global__ void k_pmis_measure(int n, const int* __restrict__ Strp, const double* __restrict__ rnd,
                               double* __restrict__ measure, int* __restrict__ cf) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        measure[i] = __dadd_rn((double)(Strp[i + 1] - Strp[i]), rnd[i]);
        cf[i] = -1;
    }
}

__global__ void k_pmis_init(int n, const int* __restrict__ cf, int* __restrict__ state) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        state[i] = cf[i] == -1 ? PM_UNK : PM_OFF;
}

__global__ void k_pmis_resolve(int n, const int* __restrict__ Srp, const int* __restrict__ Sci,
                               const int* __restrict__ Trp, const int* __restrict__ Tci, const int* __restrict__ cf,
                               const double* __restrict__ measure, volatile int* state, int* unresolved) {
    int left = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (state[i] != PM_UNK) continue;
        const double mi = measure[i];
        bool blocked = false, pending = false;
        for (int pass = 0; pass < 2 && !blocked; ++pass) {
            const int* rp = pass ? Trp : Srp;
            const int* ci = pass ? Tci : Sci;
            for (int k = rp[i]; k < rp[i + 1]; ++k) {
                const int j = ci[k];
                if (cf[j] != -1 || !(measure[j] > mi)) continue;
                if (j > i) { blocked = true; break; }
                const int sj = state[j];
                if (sj == PM_NOTC) { blocked = true; break; }
                if (sj != PM_C) pending = true;
            }
        }
        if (blocked) state[i] = PM_NOTC;
        else if (!pending) state[i] = PM_C;
        else ++left;
    }
    if (left) atomicAdd(unresolved, left);
}

__global__ void k_pmis_commit(int n, const int* __restrict__ state, int* __restrict__ cf, int* changed) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (state[i] == PM_C) {
            cf[i] = 1;
            *changed = 1;
        }
}

// undecided neighbours of this round's C points become F
__global__ void k_pmis_fmark(int n, const int* __restrict__ Srp, const int* __restrict__ Sci,
                             const int* __restrict__ Trp, const int* __restrict__ Tci, const int* __restrict__ state,
                             volatile int* cf, int* changed) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (state[i] != PM_C) continue;
        for (int pass = 0; pass < 2; ++pass) {
            const int* rp = pass ? Trp : Srp;
            const int* ci = pass ? Tci : Sci;
            for (int k = rp[i]; k < rp[i + 1]; ++k)
                if (cf[ci[k]] == -1) {
                    cf[ci[k]] = 0;
                    *changed = 1;
                }
        }
    }
}

__global__ void k_pmis_finish(int n, int* __restrict__ cf, int* __restrict__ isc) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (cf[i] == -1) cf[i] = 1;
        isc[i] = cf[i] == 1 ? 1 : 0;
    }
}

// The first n draws of uniform_real_distribution<double>(0, 1) from a fresh
// std::mt19937(42), as the host's PMIS takes them (one per row, in row order);
// kept for the longest n asked so far (a prefix serves any shorter n).
const double* pmis_random(int n, cudaStream_t s) {
    // shared by concurrent set-ups: a grown table never frees the one that kernels
    // on other streams may still read, and it is allocated outside any
    // stream-ordered scope; the table is replaced only once its successor is
    // on the device (a failed allocation leaves the previous one in place)
    if (n <= 0) return nullptr;
    static std::mutex mu;
    static int have = 0;
    static std::vector<DevBuf<double>> dev;
    std::lock_guard<std::mutex> lk(mu);
    if (have < n) {
        std::vector<double> host(n);
        std::mt19937 rng(42);
        std::uniform_real_distribution<double> dist(0.0, 1.0);
        for (int i = 0; i < n; ++i) host[i] = dist(rng);
        AllocScope plain(nullptr);
        DevBuf<double> next;
        next.upload(host.data(), host.size(), s);
        SSV_CUDA(cudaStreamSynchronize(s));
        dev.push_back(std::move(next));
        have = n;
    }
    return dev.back().get();
}

// ---- direct interpolation (BuildClassicalInterp, compact_amg.hpp:488-612) ----------
__global__ void k_strong_flags(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                               const int* __restrict__ Srp, const int* __restrict__ Sci, uint8_t* __restrict__ strong) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int q = Srp[i];
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            uint8_t s = 0;
            if (q < Srp[i + 1] && ci[k] == Sci[q]) { s = 1; ++q; }
            strong[k] = s;
        }
    }
}

__global__ void k_interp_count(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                               const uint8_t* __restrict__ strong, const int* __restrict__ cf, int* __restrict__ cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int c = 0;
        if (cf[i] == 1) c = 1;
        else {
            for (int k = rp[i]; k < rp[i + 1]; ++k) c += (strong[k] && cf[ci[k]] == 1);
            if (c == 0) c = 1;
        }
        cnt[i] = c;
    }
}

__global__ void k_interp_fill(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                              const double* __restrict__ v, const uint8_t* __restrict__ strong,
                              const int* __restrict__ cf, const int* __restrict__ cidx, const int* __restrict__ Prp,
                              int* __restrict__ Pci, double* __restrict__ Pv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int p0 = Prp[i];
        if (cf[i] == 1) {
            Pci[p0] = cidx[i];
            Pv[p0] = 1.0;
            continue;
        }
        double aii = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i) { aii = v[k]; break; }
        double lump = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] != i && !(strong[k] && cf[ci[k]] == 1)) lump = __dadd_rn(lump, v[k]);
        double denom = __dadd_rn(aii, lump);
        if (fabs(denom) < 1e-30) denom = 1.0;
        int pos = 0;
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (strong[k] && cf[ci[k]] == 1) {
                Pci[p0 + pos] = cidx[ci[k]];
                Pv[p0 + pos] = __ddiv_rn(-v[k], denom);
                ++pos;
            }
        if (pos == 0) {  // inject to the largest C neighbour, else a zero row
            int best = -1;
            double bv = 0.0;
            for (int k = rp[i]; k < rp[i + 1]; ++k)
                if (cf[ci[k]] == 1 && fabs(v[k]) > bv) { bv = fabs(v[k]); best = cidx[ci[k]]; }
            Pci[p0] = best >= 0 ? best : 0;
            Pv[p0] = best >= 0 ? 1.0 : 0.0;
        }
    }
}

// ---- elementwise helpers ------------------------------------------------------
__global__ void k_scaled(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                         const double* __restrict__ rmul, const double* __restrict__ cmul, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            double f = 1.0;
            if (rmul) f = __dmul_rn(f, rmul[i]);
            if (cmul) f = __dmul_rn(f, cmul[ci[k]]);
            out[k] = __dmul_rn(v[k], f);
        }
}

// AD: A.v[k] / d[col]  (rows == false), or A.v[k] / d[row] (rows == true)
__global__ void k_div(int n, const int* __restrict__ rp, const int* __restrict__ ci, double* __restrict__ v,
                      const double* __restrict__ d, int rows) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = rp[i]; k < rp[i + 1]; ++k) v[k] = __ddiv_rn(v[k], rows ? d[i] : d[ci[k]]);
}

__global__ void k_diag_scale(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                             double* __restrict__ sc, double* __restrict__ isc) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 1.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (ci[k] == i && v[k] != 0.0) s = __dsqrt_rn(fabs(v[k]));
        sc[i] = s;
        isc[i] = __ddiv_rn(1.0, s);
    }
}

__global__ void k_scale_vec(int n, const double* __restrict__ in, const double* __restrict__ a,
                            const double* __restrict__ b, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double x = __dmul_rn(in[i], a[i]);
        if (b) x = __dmul_rn(x, b[i]);
        out[i] = x;
    }
}

__global__ void k_recip(int n, const double* __restrict__ in, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = __ddiv_rn(1.0, in[i]);
}

__global__ void k_to_float(int64_t n, const double* __restrict__ in, float* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = __double2float_rn(in[i]);
}

// the n x n identity pattern with 2.0 on the diagonal
__global__ void k_two_eye(int n, int* __restrict__ rp, int* __restrict__ ci, double* __restrict__ v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
        rp[i] = i;
        if (i < n) {
            ci[i] = i;
            v[i] = 2.0;
        }
    }
}

// U = [S | Q shifted by n]: row i = S's entries, then n + Q's columns
__global__ void k_concat_rows(int n, int shift, const int* __restrict__ Srp, const int* __restrict__ Sci,
                              const double* __restrict__ Sv, const int* __restrict__ Qrp, const int* __restrict__ Qci,
                              const double* __restrict__ Qv, const int* __restrict__ Urp, int* __restrict__ Uci,
                              double* __restrict__ Uv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int w = Urp[i];
        for (int k = Srp[i]; k < Srp[i + 1]; ++k, ++w) {
            Uci[w] = Sci[k];
            Uv[w] = Sv[k];
        }
        for (int k = Qrp[i]; k < Qrp[i + 1]; ++k, ++w) {
            Uci[w] = shift + Qci[k];
            Uv[w] = Qv[k];
        }
    }
}

__global__ void k_row_sum2(int n, const int* __restrict__ a, const int* __restrict__ b, int* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = (a[i + 1] - a[i]) + (b[i + 1] - b[i]);
}

bool d_mul(const DCsr& A, const DCsr& B, DCsr& C, cudaStream_t s) {
    if (!symbolic<false>(A.n, B.m, A.rp.get(), A.ci.get(), B.rp.get(), B.ci.get(), nullptr, nullptr, C, s))
        return false;
    if (A.n)
        k_mul_num<<<blocks_for(A.n), kT, 0, s>>>(A.n, A.rp.get(), A.ci.get(), A.v.get(), B.rp.get(), B.ci.get(),
                                                 B.v.get(), C.rp.get(), C.ci.get(), C.v.get());
    SSV_LAUNCH_CHECK();
    return true;
}

void d_add(const DCsr& A, double a, const DCsr& B, double b, DCsr& C, cudaStream_t s) {
    const int n = A.n;
    DevBuf<int> cnt(std::max(n, 1));
    k_add<<<blocks_for(n), kT, 0, s>>>(n, A.rp.get(), A.ci.get(), A.v.get(), a, B.rp.get(), B.ci.get(), B.v.get(),
                                       b, cnt.get(), nullptr, nullptr, nullptr);
    C.n = n;
    C.m = std::max(A.m, B.m);
    C.rp.alloc(n + 1);
    C.nnz = scan(n, cnt.get(), C.rp.get(), s);
    C.ci.alloc(std::max<int64_t>(C.nnz, 1));
    C.v.alloc(std::max<int64_t>(C.nnz, 1));
    k_add<<<blocks_for(n), kT, 0, s>>>(n, A.rp.get(), A.ci.get(), A.v.get(), a, B.rp.get(), B.ci.get(), B.v.get(),
                                       b, nullptr, C.rp.get(), C.ci.get(), C.v.get());
    SSV_LAUNCH_CHECK();
}

void d_l1(const DCsr& A, DevBuf<double>& out, cudaStream_t s) {
    out.alloc(std::max(A.n, 1));
    if (A.n) k_l1<<<blocks_for(A.n), kT, 0, s>>>(A.n, A.rp.get(), A.v.get(), out.get());
    SSV_LAUNCH_CHECK();
}

}  // namespace

// sliced-ELL offsets: off[s] = sum width[0..s), off[slices] = total; -1 when the
// total exceeds the int range (the caller then keeps no sliced-ELL copy)
__global__ void __launch_bounds__(1024) k_scan64(int n, const int* __restrict__ cnt, int* __restrict__ out,
                                                 long long* __restrict__ total) {
    __shared__ long long sh[1024];
    const int T = blockDim.x, t = threadIdx.x;
    const int chunk = (n + T - 1) / T;
    const int a = min(n, t * chunk), b = min(n, a + chunk);
    long long s = 0;
    for (int i = a; i < b; ++i) s += cnt[i];
    sh[t] = s;
    __syncthreads();
    for (int off = 1; off < T; off <<= 1) {
        const long long v = t >= off ? sh[t - off] : 0;
        __syncthreads();
        sh[t] += v;
        __syncthreads();
    }
    long long base = t ? sh[t - 1] : 0;
    for (int i = a; i < b; ++i) {
        out[i] = (int)min(base, (long long)INT32_MAX);
        base += cnt[i];
    }
    if (t == T - 1) {
        *total = sh[T - 1];
        out[n] = (int)min(sh[T - 1], (long long)INT32_MAX);
    }
}

int sell_offsets(int slices, const int* width, int* off, cudaStream_t s) {
    DevBuf<long long> tot(1);
    k_scan64<<<1, 1024, 0, s>>>(slices, width, off, tot.get());
    SSV_LAUNCH_CHECK();
    long long h = 0;
    SSV_CUDA(cudaMemcpyAsync(&h, tot.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    SSV_CUDA(cudaStreamSynchronize(s));
    return h > (long long)INT32_MAX - 4096 ? -1 : (int)h;
}

SetupLog::SetupLog(cudaStream_t st) : s(st) {
    static const bool env = std::getenv("SSV_AMS_SETUP_LOG") != nullptr;
    on = env;
    if (on) {
        SSV_CUDA(cudaStreamSynchronize(s));
        t = wall_seconds();
    }
}

void SetupLog::mark(const char* fmt, ...) {
    if (!on) return;
    SSV_CUDA(cudaStreamSynchronize(s));
    const double now = wall_seconds();
    std::fprintf(stderr, "ams setup: %8.3f ms  ", 1e3 * (now - t));
    va_list ap;
    va_start(ap, fmt);
    std::vfprintf(stderr, fmt, ap);
    va_end(ap);
    std::fprintf(stderr, "\n");
    t = now;
}

// ---- DCsr --------------------------------------------------------------------------
void DCsr::from_host(const HostCsr& H, cudaStream_t s) {
    n = H.n;
    m = H.m;
    nnz = H.nnz();
    rp.upload(H.rp.data(), H.rp.size(), s);
    ci.upload(H.ci.data(), std::max<size_t>(H.ci.size(), 0), s);
    v.upload(H.v.data(), H.v.size(), s);
}

HostCsr DCsr::to_host(cudaStream_t s) const {
    HostCsr H;
    H.n = n;
    H.m = m;
    H.rp.resize(n + 1);
    H.ci.resize(nnz);
    H.v.resize(nnz);
    SSV_CUDA(cudaMemcpyAsync(H.rp.data(), rp.get(), sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s));
    if (nnz) {
        SSV_CUDA(cudaMemcpyAsync(H.ci.data(), ci.get(), sizeof(int) * nnz, cudaMemcpyDeviceToHost, s));
        SSV_CUDA(cudaMemcpyAsync(H.v.data(), v.get(), sizeof(double) * nnz, cudaMemcpyDeviceToHost, s));
    }
    SSV_CUDA(cudaStreamSynchronize(s));
    return H;
}

void DCsr::copy_from(const DCsr& o, cudaStream_t s) {
    n = o.n;
    m = o.m;
    nnz = o.nnz;
    rp.alloc(n + 1);
    ci.alloc(std::max<int64_t>(nnz, 1));
    v.alloc(std::max<int64_t>(nnz, 1));
    SSV_CUDA(cudaMemcpyAsync(rp.get(), o.rp.get(), sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice, s));
    if (nnz) {
        SSV_CUDA(cudaMemcpyAsync(ci.get(), o.ci.get(), sizeof(int) * nnz, cudaMemcpyDeviceToDevice, s));
        SSV_CUDA(cudaMemcpyAsync(v.get(), o.v.get(), sizeof(double) * nnz, cudaMemcpyDeviceToDevice, s));
    }
}

// ---- public steps ---------------------------------------------------------------------
void d_bc_matrix(int n, int m, int64_t nnz, const int* rp, const int* ci, const double* vals, const uint8_t* d_fd,
                 DCsr& out, cudaStream_t s) {
    out.n = n;
    out.m = m;
    out.nnz = nnz;
    out.rp.alloc(n + 1);
    out.ci.alloc(std::max<int64_t>(nnz, 1));
    out.v.alloc(std::max<int64_t>(nnz, 1));
    SSV_CUDA(cudaMemcpyAsync(out.rp.get(), rp, sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice, s));
    if (nnz) SSV_CUDA(cudaMemcpyAsync(out.ci.get(), ci, sizeof(int) * nnz, cudaMemcpyDeviceToDevice, s));
    if (n) k_bc<<<blocks_for(n), kT, 0, s>>>(n, rp, ci, vals, d_fd, out.v.get());
    SSV_LAUNCH_CHECK();
}

void d_transpose(const DCsr& A, DCsr& T, cudaStream_t s) {
    DevBuf<int> cnt(std::max(A.m, 1)), fill(std::max(A.m, 1)), key(std::max<int64_t>(A.nnz, 1));
    cnt.zero(s);
    fill.zero(s);
    T.n = A.m;
    T.m = A.n;
    T.nnz = A.nnz;
    T.rp.alloc(A.m + 1);
    T.ci.alloc(std::max<int64_t>(A.nnz, 1));
    T.v.alloc(std::max<int64_t>(A.nnz, 1));
    if (A.nnz) k_col_count<<<blocks_for(A.nnz), kT, 0, s>>>(A.nnz, A.ci.get(), cnt.get());
    scan(A.m, cnt.get(), T.rp.get(), s);
    if (A.nnz) {
        k_tr_scatter<<<blocks_for(A.n), kT, 0, s>>>(A.n, A.rp.get(), A.ci.get(), A.v.get(), T.rp.get(), fill.get(),
                                                     T.ci.get(), T.v.get(), key.get());
        k_row_sort<<<blocks_for(T.n), kT, 0, s>>>(T.n, T.rp.get(), key.get(), T.ci.get(), T.v.get());
    }
    SSV_LAUNCH_CHECK();
}

bool d_rap(const DCsr& A, const DCsr& P, const DCsr& Pt, DCsr& C, cudaStream_t s) {
    if (!symbolic<true>(Pt.n, P.m, Pt.rp.get(), Pt.ci.get(), A.rp.get(), A.ci.get(), P.rp.get(), P.ci.get(), C, s))
        return false;
    if (Pt.n)
        k_rap_num<<<blocks_for(Pt.n, 128), 128, 0, s>>>(Pt.n, Pt.rp.get(), Pt.ci.get(), Pt.v.get(), A.rp.get(),
                                                         A.ci.get(), A.v.get(), P.rp.get(), P.ci.get(), P.v.get(),
                                                         C.rp.get(), C.ci.get(), C.v.get());
    SSV_LAUNCH_CHECK();
    return true;
}

void d_fix_zero_rows(DCsr& A, cudaStream_t s) {
    if (A.n) k_fix_zero_rows<<<blocks_for(A.n), kT, 0, s>>>(A.n, A.rp.get(), A.ci.get(), A.v.get());
    SSV_LAUNCH_CHECK();
}

void d_fine_l1(const DCsr& A, DevBuf<double>& out, cudaStream_t s) {
    out.alloc(std::max(A.n, 1));
    if (A.n) k_fine_l1<<<blocks_for(A.n), kT, 0, s>>>(A.n, A.rp.get(), A.ci.get(), A.v.get(), out.get());
    SSV_LAUNCH_CHECK();
}

void d_scaled(const DCsr& A, const double* rmul, const double* cmul, DCsr& out, cudaStream_t s) {
    out.copy_from(A, s);
    if (A.n)
        k_scaled<<<blocks_for(A.n), kT, 0, s>>>(A.n, A.rp.get(), A.ci.get(), A.v.get(), rmul, cmul, out.v.get());
    SSV_LAUNCH_CHECK();
}

void d_diag_scale(const DCsr& A, DevBuf<double>& sc, DevBuf<double>& isc, cudaStream_t s) {
    sc.alloc(std::max(A.n, 1));
    isc.alloc(std::max(A.n, 1));
    if (A.n) k_diag_scale<<<blocks_for(A.n), kT, 0, s>>>(A.n, A.rp.get(), A.ci.get(), A.v.get(), sc.get(), isc.get());
    SSV_LAUNCH_CHECK();
}

void d_scale_vec(int n, const double* in, const double* a, const double* b, double* out, cudaStream_t s) {
    if (n) k_scale_vec<<<blocks_for(n), kT, 0, s>>>(n, in, a, b, out);
    SSV_LAUNCH_CHECK();
}

void d_reciprocal(int n, const double* in, double* out, cudaStream_t s) {
    if (n) k_recip<<<blocks_for(n), kT, 0, s>>>(n, in, out);
    SSV_LAUNCH_CHECK();
}

void d_to_float(int64_t n, const double* in, float* out, cudaStream_t s) {
    if (n) k_to_float<<<blocks_for(n), kT, 0, s>>>(n, in, out);
    SSV_LAUNCH_CHECK();
}

bool d_fused_level(const DCsr& A, const DCsr& P, const DCsr& Pt, const double* d, DCsr& R, DCsr& U,
                   cudaStream_t s) {
    const int n = A.n;
    DCsr AD;
    AD.copy_from(A, s);
    if (n) k_div<<<blocks_for(n), kT, 0, s>>>(n, AD.rp.get(), AD.ci.get(), AD.v.get(), d, 0);  // A D^{-1}
    SSV_LAUNCH_CHECK();
    DCsr T1;
    if (!d_mul(Pt, AD, T1, s)) return false;
    d_add(Pt, 1.0, T1, -1.0, R, s);
    DCsr I2;  // 2 I
    I2.n = I2.m = n;
    I2.nnz = n;
    I2.rp.alloc(n + 1);
    I2.ci.alloc(std::max(n, 1));
    I2.v.alloc(std::max(n, 1));
    k_two_eye<<<blocks_for(n + 1), kT, 0, s>>>(n, I2.rp.get(), I2.ci.get(), I2.v.get());
    DCsr S;
    d_add(I2, 1.0, AD, -1.0, S, s);
    if (n) k_div<<<blocks_for(n), kT, 0, s>>>(n, S.rp.get(), S.ci.get(), S.v.get(), d, 1);  // rows by D^{-1}
    DCsr DAP;
    if (!d_mul(A, P, DAP, s)) return false;
    if (n) k_div<<<blocks_for(n), kT, 0, s>>>(n, DAP.rp.get(), DAP.ci.get(), DAP.v.get(), d, 1);
    SSV_LAUNCH_CHECK();
    DCsr Q;
    d_add(P, 1.0, DAP, -1.0, Q, s);
    DevBuf<int> cnt(std::max(n, 1));
    if (n) k_row_sum2<<<blocks_for(n), kT, 0, s>>>(n, S.rp.get(), Q.rp.get(), cnt.get());
    U.n = n;
    U.m = n + P.m;
    U.rp.alloc(n + 1);
    U.nnz = scan(n, cnt.get(), U.rp.get(), s);
    U.ci.alloc(std::max<int64_t>(U.nnz, 1));
    U.v.alloc(std::max<int64_t>(U.nnz, 1));
    if (n)
        k_concat_rows<<<blocks_for(n), kT, 0, s>>>(n, n, S.rp.get(), S.ci.get(), S.v.get(), Q.rp.get(), Q.ci.get(),
                                                   Q.v.get(), U.rp.get(), U.ci.get(), U.v.get());
    SSV_LAUNCH_CHECK();
    SSV_CUDA(cudaStreamSynchronize(s));  // the temporaries go out of scope
    return true;
}

bool d_amg_setup(const DCsr& A0, double theta, int max_levels, int min_coarse, std::vector<DAmgLevel>& out,
                 cudaStream_t s, WorkerThread* coarse) {
    SetupLog log(s);
    out.clear();
    out.emplace_back();
    out[0].A.copy_from(A0, s);
    d_l1(out[0].A, out[0].l1, s);
    for (int l = 0; l < max_levels - 1; ++l) {
        const int n = out[l].A.n;
        if (n <= min_coarse) break;
        log.mark("  level %d (%d rows, %lld nnz): start", l, n, (long long)out[l].A.nnz);
        const DCsr& A = out[l].A;
        // strength (ComputeStrength, compact_amg.hpp:292-372)
        DevBuf<int> cnt(n), Srp(n + 1), Sci;
        k_strength<<<blocks_for(n), kT, 0, s>>>(n, A.rp.get(), A.ci.get(), A.v.get(), theta, cnt.get(), nullptr,
                                                nullptr);
        const int snnz = scan(n, cnt.get(), Srp.get(), s);
        Sci.alloc(std::max(snnz, 1));
        k_strength<<<blocks_for(n), kT, 0, s>>>(n, A.rp.get(), A.ci.get(), A.v.get(), theta, nullptr, Srp.get(),
                                                Sci.get());
        SSV_LAUNCH_CHECK();
        DevBuf<int> Trp, Tci;
        graph_transpose(n, n, Srp.get(), Sci.get(), snnz, Trp, Tci, s);
        log.mark("    strength + transpose (%d strong)", snnz);
        int passes = 0, rounds = 0;
        // PMIS
        DevBuf<double> measure(n);
        DevBuf<int> cf(n), state(n), flags(2);
        k_pmis_measure<<<blocks_for(n), kT, 0, s>>>(n, Trp.get(), pmis_random(n, s), measure.get(), cf.get());
        SSV_LAUNCH_CHECK();
        for (int round = 0; round < 100; ++round) {
            ++rounds;
            k_pmis_init<<<blocks_for(n), kT, 0, s>>>(n, cf.get(), state.get());
            for (int pass = 0; pass <= n; ++pass) {  // each pass decides at least one row
                ++passes;
                flags.zero(s);
                k_pmis_resolve<<<blocks_for(n), kT, 0, s>>>(n, Srp.get(), Sci.get(), Trp.get(), Tci.get(), cf.get(),
                                                            measure.get(), state.get(), flags.get());
                SSV_LAUNCH_CHECK();
                int left = 0;
                SSV_CUDA(cudaMemcpyAsync(&left, flags.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
                SSV_CUDA(cudaStreamSynchronize(s));
                if (!left) break;
            }
            flags.zero(s);
            k_pmis_commit<<<blocks_for(n), kT, 0, s>>>(n, state.get(), cf.get(), flags.get() + 1);
            k_pmis_fmark<<<blocks_for(n), kT, 0, s>>>(n, Srp.get(), Sci.get(), Trp.get(), Tci.get(), state.get(),
                                                      cf.get(), flags.get() + 1);
            SSV_LAUNCH_CHECK();
            int changed = 0;
            SSV_CUDA(cudaMemcpyAsync(&changed, flags.get() + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
            SSV_CUDA(cudaStreamSynchronize(s));
            if (!changed) break;
        }
        DevBuf<int> isc(n), cidx(n + 1);
        k_pmis_finish<<<blocks_for(n), kT, 0, s>>>(n, cf.get(), isc.get());
        const int nc = scan(n, isc.get(), cidx.get(), s);
        log.mark("    PMIS: %d coarse, %d rounds, %d passes", nc, rounds, passes);
        if (nc == 0 || nc >= n) break;
        // interpolation
        DevBuf<uint8_t> strong(std::max<int64_t>(A.nnz, 1));
        k_strong_flags<<<blocks_for(n), kT, 0, s>>>(n, A.rp.get(), A.ci.get(), Srp.get(), Sci.get(), strong.get());
        k_interp_count<<<blocks_for(n), kT, 0, s>>>(n, A.rp.get(), A.ci.get(), strong.get(), cf.get(), cnt.get());
        SSV_LAUNCH_CHECK();
        DCsr P;
        P.n = n;
        P.m = nc;
        P.rp.alloc(n + 1);
        P.nnz = scan(n, cnt.get(), P.rp.get(), s);
        P.ci.alloc(std::max<int64_t>(P.nnz, 1));
        P.v.alloc(std::max<int64_t>(P.nnz, 1));
        k_interp_fill<<<blocks_for(n), kT, 0, s>>>(n, A.rp.get(), A.ci.get(), A.v.get(), strong.get(), cf.get(),
                                                   cidx.get(), P.rp.get(), P.ci.get(), P.v.get());
        SSV_LAUNCH_CHECK();
        log.mark("    interpolation (%lld nnz)", (long long)P.nnz);
        DCsr Pt, Ac;
        d_transpose(P, Pt, s);
        log.mark("    P transpose");
        if (!d_rap(A, P, Pt, Ac, s)) return false;
        log.mark("    RAP (%lld nnz)", (long long)Ac.nnz);
        SSV_CUDA(cudaStreamSynchronize(s));  // this level's temporaries go out of scope
        out[l].P = std::move(P);
        out[l].Pt = std::move(Pt);
        out.emplace_back();
        out.back().A = std::move(Ac);
        d_l1(out.back().A, out.back().l1, s);
    }
    DAmgLevel& co = out.back();
    if (co.A.n <= min_coarse * 10) {
        co.direct = true;
        if (coarse) {  // the level object stays where it is: out is not resized again
            coarse->start([&co, H = co.A.to_host(s)] {
                co.piv_min = dense_ldlt_pseudo(H, co.linv, co.linvt, co.piv);
            });
        } else {
            co.piv_min = dense_ldlt_pseudo(co.A.to_host(s), co.linv, co.linvt, co.piv);
            log.mark("  coarsest LDL^T (%d rows, host)", co.A.n);
        }
    }
    SSV_CUDA(cudaStreamSynchronize(s));
    return true;
}

}  // namespace ssv
