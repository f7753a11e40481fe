// FP64 masked (P)CG of one instance with one launch per iteration.
//
// Same solve as ConjGradCuda::solve (src/ConjGradCuda.cu:185-231) and as the
// two-kernel loop of cg.cu: r0 = m.(b - K x0), stop when (r, r) / (b, b) <=
// eps^2, the caller's x carries the last iterate. The iteration is arranged
// so that both inner products are taken together (Chronopoulos-Gear): with
// M the 2x2 block-Jacobi inverse (the Dirichlet mask without
// preconditioning), u = M r, w = K u, p the direction and kp = K p,
//   p' = u + beta p, kp' = w + beta kp, x += alpha p', r' = m.(r - alpha kp'),
//   u' = u - alpha (M w + beta M kp), w' = K u',
//   gamma' = (r', u'), beta' = gamma' / gamma,
//   alpha' = gamma' / (K p'', p''), (K p'', p'') = (w', u')
//            + beta' ((w', p') + (kp', u')) + beta'^2 (kp', p').
// K u' needs the neighbours' new u; each thread recomputes it from the
// neighbours' u, M w, M kp, kept in one 48-byte record per node and
// double-buffered by iteration parity, so an iteration is one kernel and one
// deterministic cross-block reduction (last block, index order). The
// scalars stay on the device; the loop runs in a CUDA graph with a WHILE
// node, as in cg.cu.
#include <cstddef>
#include <cstdlib>
#include <mutex>
#include <unordered_map>

#include "cg.h"
#include "common.cuh"
#include "internal.h"

namespace cp {

namespace {

constexpr int kThreads = 256;
constexpr int kSums = 6;

__device__ __forceinline__ double2 mvec(const double4& m, double2 v) {
    return make_double2(m.x * v.x + m.y * v.y, m.z * v.x + m.w * v.y);
}

__device__ __forceinline__ double2 apply_m(const FusedArgs& a, int n, double2 v) {
    if (a.precond) return mvec(a.minv[n], v);
    const uchar2 m = a.mask[n];
    return make_double2(m.x ? v.x : 0.0, m.y ? v.y : 0.0);
}

__device__ __forceinline__ double2 load_lo(const double* val, long long b) {
    return __ldg(reinterpret_cast<const double2*>(val + 4 * b));
}
__device__ __forceinline__ double2 load_hi(const double* val, long long b) {
    return __ldg(reinterpret_cast<const double2*>(val + 4 * b) + 1);
}

#define CPF_SLICE_LOOP                                                                          \
    const int lane = threadIdx.x & 31;                                                          \
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;                              \
    const int nwarps = (gridDim.x * blockDim.x) >> 5;                                           \
    for (int sl = warp; sl < (a.n + 31) / 32; sl += nwarps)

// Block sums of up to kSums values into partials[kSums * block]; true in the
// last block to arrive, which then holds the totals in out (thread 0).
__device__ __forceinline__ bool reduce_sums(const FusedArgs& a, double* v, int k, double* out, double* sh,
                                            bool* last) {
    for (int i = 0; i < k; i += 2) {
        const double2 s = block_sum2(v[i], i + 1 < k ? v[i + 1] : 0.0, sh);
        if (threadIdx.x == 0) {
            a.partials[kSums * blockIdx.x + i] = s.x;
            if (i + 1 < k) a.partials[kSums * blockIdx.x + i + 1] = s.y;
        }
    }
    if (!last_block_arrive(&a.sc->ticket, last)) return false;
    double t[kSums];
    for (int i = 0; i < k; ++i) t[i] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
        const volatile double* p = a.partials + kSums * b;
        for (int i = 0; i < k; ++i) t[i] += p[i];
    }
    for (int i = 0; i < k; i += 2) {
        const double2 s = block_sum2(t[i], i + 1 < k ? t[i + 1] : 0.0, sh);
        out[i] = s.x;
        if (i + 1 < k) out[i + 1] = s.y;
    }
    return true;
}

// Loads of vectors that other blocks write during the same launch. The
// one-launch-per-iteration kernels (P = false) read them through the
// read-only path; the persistent kernel (P = true) loads them at L2
// (ld.global.cg), since an SM's L1 is not coherent with the other SMs' stores.
template <bool P>
__device__ __forceinline__ double2 ld_other(const double2* p) {
    if (P) return __ldcg(p);
    return __ldg(p);
}

// r = m.(b - K x), block-Jacobi inverse, u = M r, p = kp = 0, the parity-0
// record (u, -, 0); sums (r, r), (b, b).
__device__ __forceinline__ void init_body(const FusedArgs& a, double* v) {
    CPF_SLICE_LOOP {
        const int n = 32 * sl + lane;
        if (n >= a.n) continue;
        const int base = a.slice_ptr[sl], wd = (a.slice_ptr[sl + 1] - base) >> 5;
        double k0 = 0.0, k1 = 0.0;
        for (int k = 0; k < wd; ++k) {
            const long long bi = base + 32LL * k + lane;
            const int col = __ldg(a.scol + bi);
            const double2 lo = load_lo(a.val, bi), hi = load_hi(a.val, bi);
            const double2 xc = a.x[col];
            k0 += lo.x * xc.x + lo.y * xc.y;
            k1 += hi.x * xc.x + hi.y * xc.y;
        }
        const double2 bb = a.b[n];
        const uchar2 m = a.mask[n];
        const double2 r = make_double2(m.x ? bb.x - k0 : 0.0, m.y ? bb.y - k1 : 0.0);
        a.r[n] = r;
        if (a.precond) {
            const double2 lo = load_lo(a.val, base + lane), hi = load_hi(a.val, base + lane);
            double i00 = 0, i01 = 0, i10 = 0, i11 = 0;
            if (m.x && m.y) {
                const double det = lo.x * hi.y - lo.y * hi.x;
                i00 = hi.y / det; i01 = -lo.y / det; i10 = -hi.x / det; i11 = lo.x / det;
            } else if (m.x) {
                i00 = 1.0 / lo.x;
            } else if (m.y) {
                i11 = 1.0 / hi.y;
            }
            a.minv[n] = make_double4(i00, i01, i10, i11);
        }
        const double2 u = apply_m(a, n, r);
        const double2 z = make_double2(0.0, 0.0);
        a.p[n] = z;
        a.kp[n] = z;
        a.gA[3 * (size_t)n] = u;
        a.gA[3 * (size_t)n + 2] = z;
        v[0] += r.x * r.x + r.y * r.y;
        v[1] += bb.x * bb.x + bb.y * bb.y;
    }
}

__device__ __forceinline__ void init_scalars(CgScalars* sc, const double* t, double eps2, long long max_iter) {
    const double rr = t[0], bb = t[1];
    sc->rr = rr;
    sc->bb = bb;
    sc->res64 = rr;
    sc->normB_inv = bb > 0.0 ? 1.0 / bb : 0.0;
    sc->eps2 = eps2;
    sc->iter = 0;
    sc->max_iter = max_iter;
    sc->status = 0;
    sc->lin_done = 0;
    sc->alpha = sc->beta = 0.0;
    sc->converged = (rr == 0.0 || rr * sc->normB_inv <= eps2) ? 1 : 0;
    if (!(rr == rr) || !(bb == bb)) sc->status = CP_ERR_BREAKDOWN;
    sc->ticket = 0;
}

// w = K u (u from the parity-0 records), M w into the record; gamma = (r, u),
// delta = (w, u): the first step.
template <bool P>
__device__ __forceinline__ void w_body(const FusedArgs& a, double* v) {
    CPF_SLICE_LOOP {
        const int n = 32 * sl + lane;
        if (n >= a.n) continue;
        const int base = a.slice_ptr[sl], wd = (a.slice_ptr[sl + 1] - base) >> 5;
        double k0 = 0.0, k1 = 0.0;
        for (int k = 0; k < wd; ++k) {
            const long long bi = base + 32LL * k + lane;
            const int col = __ldg(a.scol + bi);
            const double2 lo = load_lo(a.val, bi), hi = load_hi(a.val, bi);
            const double2 uc = P ? __ldcg(a.gA + 3 * (size_t)col) : a.gA[3 * (size_t)col];
            k0 += lo.x * uc.x + lo.y * uc.y;
            k1 += hi.x * uc.x + hi.y * uc.y;
        }
        const double2 w = make_double2(k0, k1);
        a.w[n] = w;
        a.gA[3 * (size_t)n + 1] = apply_m(a, n, w);
        const double2 u = a.gA[3 * (size_t)n], r = a.r[n];
        v[0] += r.x * u.x + r.y * u.y;
        v[1] += w.x * u.x + w.y * u.y;
    }
}

__device__ __forceinline__ void w_scalars(CgScalars* sc, const double* t) {
    const double g = t[0], d = t[1];
    sc->rho = g;
    sc->alpha = g / d;
    sc->beta = 0.0;
    if (!(d > 0.0) || !(sc->alpha == sc->alpha)) sc->status = CP_ERR_BREAKDOWN;
    sc->ticket = 0;
}

// One iteration (see the file comment); parity selects the record buffers.
// C > 0: the row's blocks are taken C at a time, their columns and values
// loaded together ahead of the C record gathers; C = 0: one unrolled loop.
template <bool P, int C = 0, bool ST = false>
__device__ __forceinline__ void iter_body(const FusedArgs& a, int parity, double al, double bt, double* v) {
    const double2* __restrict__ go = parity ? a.gB : a.gA;
    double2* __restrict__ gn = parity ? a.gA : a.gB;
    CPF_SLICE_LOOP {
        const int n = 32 * sl + lane;
        if (n >= a.n) continue;
        const int base = a.slice_ptr[sl], wd = (a.slice_ptr[sl + 1] - base) >> 5;
        const double2 u0 = ld_other<P>(go + 3 * (size_t)n), mw0 = ld_other<P>(go + 3 * (size_t)n + 1),
                      mk0 = ld_other<P>(go + 3 * (size_t)n + 2);
        const double2 pn = a.p[n], wn = a.w[n], kn = a.kp[n];
        const uchar2 m = a.mask[n];
        const double2 p = make_double2(u0.x + bt * pn.x, u0.y + bt * pn.y);
        const double2 kp = make_double2(wn.x + bt * kn.x, wn.y + bt * kn.y);
        const double2 u = make_double2(u0.x - al * (mw0.x + bt * mk0.x), u0.y - al * (mw0.y + bt * mk0.y));
        double2 x = a.x[n];
        x.x += al * p.x;
        x.y += al * p.y;
        double2 r = a.r[n];
        if (m.x) r.x -= al * kp.x;
        if (m.y) r.y -= al * kp.y;
        double k0 = 0.0, k1 = 0.0;
        if (C == 0) {
#pragma unroll 3
            for (int k = 0; k < wd; ++k) {
                const long long bi = base + 32LL * k + lane;
                const int col = __ldg(a.scol + bi);
                const double2 lo = load_lo(a.val, bi), hi = load_hi(a.val, bi);
                const double2 uc = ld_other<P>(go + 3 * (size_t)col), mwc = ld_other<P>(go + 3 * (size_t)col + 1),
                              mkc = ld_other<P>(go + 3 * (size_t)col + 2);
                const double ux = uc.x - al * (mwc.x + bt * mkc.x), uy = uc.y - al * (mwc.y + bt * mkc.y);
                k0 += lo.x * ux + lo.y * uy;
                k1 += hi.x * ux + hi.y * uy;
            }
        } else {
            for (int k0i = 0; k0i < wd; k0i += (C > 0 ? C : 1)) {
                int cc[C > 0 ? C : 1];
                double2 lo[C > 0 ? C : 1], hi[C > 0 ? C : 1];
#pragma unroll
                for (int j = 0; j < C; ++j) {
                    if (k0i + j < wd) {
                        const long long bi = base + 32LL * (k0i + j) + lane;
                        cc[j] = ld_stream<ST>(a.scol + bi);
                        const double2* vp = reinterpret_cast<const double2*>(a.val + 4 * bi);
                        lo[j] = ld_stream<ST>(vp);
                        hi[j] = ld_stream<ST>(vp + 1);
                    }
                }
#pragma unroll
                for (int j = 0; j < C; ++j) {
                    if (k0i + j < wd) {
                        const double2* rc = go + 3 * (size_t)cc[j];
                        const double2 uc = ld_other<P>(rc), mwc = ld_other<P>(rc + 1), mkc = ld_other<P>(rc + 2);
                        const double ux = uc.x - al * (mwc.x + bt * mkc.x), uy = uc.y - al * (mwc.y + bt * mkc.y);
                        k0 += lo[j].x * ux + lo[j].y * uy;
                        k1 += hi[j].x * ux + hi[j].y * uy;
                    }
                }
            }
        }
        const double2 w = make_double2(k0, k1);
        a.p[n] = p;
        a.kp[n] = kp;
        a.x[n] = x;
        a.r[n] = r;
        a.w[n] = w;
        gn[3 * (size_t)n] = u;
        gn[3 * (size_t)n + 1] = apply_m(a, n, w);
        gn[3 * (size_t)n + 2] = apply_m(a, n, kp);
        v[0] += r.x * u.x + r.y * u.y;
        v[1] += w.x * u.x + w.y * u.y;
        v[2] += r.x * r.x + r.y * r.y;
        v[3] += (w.x * p.x + w.y * p.y) + (kp.x * u.x + kp.y * u.y);
        v[4] += kp.x * p.x + kp.y * p.y;
    }
}

__device__ __forceinline__ void iter_scalars(CgScalars* sc, const double* t) {
    const double g = t[0], rn = t[2];
    const double beta = g / sc->rho;
    const double den = t[1] + beta * t[3] + beta * beta * t[4];
    sc->iter += 1;
    sc->rr = rn;
    sc->beta = beta;
    sc->alpha = g / den;
    sc->rho = g;
    if (rn * sc->normB_inv <= sc->eps2) sc->converged = 1;
    else if (sc->iter >= sc->max_iter) sc->status = CP_ERR_NOT_CONVERGED;
    else if (!(den > 0.0) || !(g > 0.0)) sc->status = CP_ERR_BREAKDOWN;
    if (!(rn == rn)) sc->status = CP_ERR_BREAKDOWN;
    sc->ticket = 0;
}

__global__ void __launch_bounds__(kThreads) k_f_init(FusedArgs a, double eps2, long long max_iter) {
    __shared__ double sh[2 * kThreads / 32];
    __shared__ bool last;
    double v[2] = {0.0, 0.0};
    init_body(a, v);
    double t[kSums];
    if (!reduce_sums(a, v, 2, t, sh, &last)) return;
    if (threadIdx.x == 0) init_scalars(a.sc, t, eps2, max_iter);
}

__global__ void __launch_bounds__(kThreads) k_f_w(FusedArgs a) {
    __shared__ double sh[2 * kThreads / 32];
    __shared__ bool last;
    CgScalars* sc = a.sc;
    if (sc->converged || sc->status) return;
    double v[2] = {0.0, 0.0};
    w_body<false>(a, v);
    double t[kSums];
    if (!reduce_sums(a, v, 2, t, sh, &last)) return;
    if (threadIdx.x == 0) w_scalars(sc, t);
}

template <int C, bool ST = false>
__device__ __forceinline__ void iter_kernel_body(const FusedArgs& a, int parity) {
    __shared__ double sh[2 * kThreads / 32];
    __shared__ bool last;
    pdl_enter();  // scheduled early by fused_launch_iteration
    CgScalars* sc = a.sc;
    if (sc->converged || sc->status) return;
    double v[kSums] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    iter_body<false, C, ST>(a, parity, sc->alpha, sc->beta, v);
    double t[kSums];
    if (!reduce_sums(a, v, 5, t, sh, &last)) return;
    if (threadIdx.x == 0) iter_scalars(sc, t);
}

// C and ST as in iter_body; k_f_iter4 asks the compiler for 4 resident
// blocks per SM (a 64-register cap).
template <int C, bool ST = false>
__global__ void __launch_bounds__(kThreads) k_f_iter(FusedArgs a, int parity) {
    iter_kernel_body<C, ST>(a, parity);
}
template <int C>
__global__ void __launch_bounds__(kThreads, 4) k_f_iter4(FusedArgs a, int parity) {
    iter_kernel_body<C>(a, parity);
}

// ---------------------------------------------------- persistent form --
//
// The whole linear solve in one cooperative launch: init, the first step and
// every iteration run back to back, separated by a grid barrier. The block
// that arrives last at a step (the reduction's last block) computes the
// scalars and releases the others by advancing sc->gen; the arithmetic, the
// block partition and the summation order are those of the kernels above, so
// the results are the same bit for bit. Co-residency of all blocks comes from
// the cooperative launch. Every wait is bounded in time: a block that gives up
// sets CP_ERR_TIMEOUT and returns, and so does every other waiting block.

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The last block of a step (thread 0): publish the scalars it has just
// written, then release the step.
__device__ __forceinline__ void grid_release(CgScalars* sc) {
    __threadfence();
    atomicAdd(&sc->gen, 1u);
}

// Waits until step `target` is released. Thread 0 polls and then reads the
// step's outcome once for the whole block (another block's time-out may
// change sc->status at any moment, and every thread of a block must take the
// same branch): true to go on, with alpha and beta in *view. Gives up after
// a.barrier_ns (2 s by default; one step takes microseconds) with
// CP_ERR_TIMEOUT set.
struct StepView {
    int go;
    double alpha, beta;
};

__device__ __forceinline__ bool grid_wait(const FusedArgs& a, unsigned int step, StepView* view) {
    CgScalars* sc = a.sc;
    const unsigned int target = step + a.barrier_skew;
    if (threadIdx.x == 0) {
        const volatile unsigned int* g = &sc->gen;
        int ok = 1;
        if (*g < target) {
            const unsigned long long t0 = global_ns();
            while (*g < target) {
                if (global_ns() - t0 > a.barrier_ns) {
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        if (!ok) atomicCAS(&sc->status, 0, CP_ERR_TIMEOUT);
        __threadfence();
        const volatile CgScalars* vs = sc;
        view->go = ok && !vs->converged && !vs->status;
        view->alpha = vs->alpha;
        view->beta = vs->beta;
    }
    __syncthreads();
    return view->go != 0;
}

template <int C>
__global__ void __launch_bounds__(kThreads) k_f_persistent(FusedArgs a, double eps2, long long max_iter) {
    __shared__ double sh[2 * kThreads / 32];
    __shared__ bool last;
    __shared__ StepView view;
    CgScalars* sc = a.sc;
    unsigned int step = 0;
    double t[kSums];
    {
        double v[2] = {0.0, 0.0};
        init_body(a, v);
        if (reduce_sums(a, v, 2, t, sh, &last) && threadIdx.x == 0) {
            init_scalars(sc, t, eps2, max_iter);
            grid_release(sc);
        }
        if (!grid_wait(a, ++step, &view)) return;
    }
    {
        double v[2] = {0.0, 0.0};
        w_body<true>(a, v);
        if (reduce_sums(a, v, 2, t, sh, &last) && threadIdx.x == 0) {
            w_scalars(sc, t);
            grid_release(sc);
        }
        if (!grid_wait(a, ++step, &view)) return;
    }
    for (int it = 0;; ++it) {
        double v[kSums] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        const double al = view.alpha, bt = view.beta;
        __syncthreads();  // everyone has read the view before thread 0 overwrites it
        iter_body<true, C>(a, it & 1, al, bt, v);
        if (reduce_sums(a, v, 5, t, sh, &last) && threadIdx.x == 0) {
            iter_scalars(sc, t);
            grid_release(sc);
        }
        if (!grid_wait(a, ++step, &view)) return;
    }
}

__global__ void k_f_condition(const CgScalars* sc, cudaGraphConditionalHandle h) {
    cudaGraphSetConditional(h, (sc->converged || sc->status) ? 0u : 1u);
}

template <typename K>
int fused_grid(K kernel, int n, int sm_count) {
    static std::mutex mu;
    static std::unordered_map<const void*, int> cache;
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find((const void*)kernel);
        if (it != cache.end()) per_sm = it->second;
    }
    if (per_sm == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0) != cudaSuccess || per_sm < 1)
            per_sm = 1;
        std::lock_guard<std::mutex> lock(mu);
        cache[(const void*)kernel] = per_sm;
    }
    long long g = (n + kThreads - 1) / kThreads;
    const long long cap = (long long)sm_count * per_sm;
    if (g > cap) g = cap;
    return g < 1 ? 1 : (int)g;
}

// The iteration kernel's form: CUPLAST_FUSED_FORM = 0 (one unrolled loop),
// 1 (blocks 3 at a time: the default, 20 % faster than 0 on the 2.1M-DOF
// plate), 2 (one loop, 4 blocks per SM), 3 (3 at a time, 4 blocks per SM),
// 4 / 5 (2 / 5 at a time), for measurements.
constexpr int kDefaultForm = 1;
using IterKernel = void (*)(FusedArgs, int);
using PersistentKernel = void (*)(FusedArgs, double, long long);

int form() {
    static const int f = [] {
        const char* e = std::getenv("CUPLAST_FUSED_FORM");
        const int v = e ? std::atoi(e) : kDefaultForm;
        return (v >= 0 && v <= 5) ? v : kDefaultForm;
    }();
    return f;
}

// the persistent form takes its blocks C at a time as the iteration kernel
// does, so that both sum in the same order
PersistentKernel persistent_kernel() {
    switch (form()) {
    case 0: case 2: return (PersistentKernel)k_f_persistent<0>;
    case 4: return (PersistentKernel)k_f_persistent<2>;
    case 5: return (PersistentKernel)k_f_persistent<5>;
    default: return (PersistentKernel)k_f_persistent<3>;
    }
}
IterKernel iter_kernel() {
    static const IterKernel k = [] {
        switch (form()) {
        case 0: return (IterKernel)k_f_iter<0>;
        case 2: return (IterKernel)k_f_iter4<0>;
        case 3: return (IterKernel)k_f_iter4<3>;
        case 4: return (IterKernel)k_f_iter<2>;
        case 5: return (IterKernel)k_f_iter<5>;
        default: return (IterKernel)k_f_iter<3>;
        }
    }();
    return k;
}

}  // namespace

void fused_launch_start(const FusedArgs& a, double eps2, long long max_iter, cudaStream_t s) {
    const int g1 = fused_grid(k_f_init, a.n, a.sm_count), g2 = fused_grid(k_f_w, a.n, a.sm_count);
    CP_CHECK(g1 <= a.max_blocks && g2 <= a.max_blocks, CP_ERR_INVALID, "partials buffer too small");
    k_f_init<<<g1, kThreads, 0, s>>>(a, eps2, max_iter);
    k_f_w<<<g2, kThreads, 0, s>>>(a);
    CP_CUDA(cudaGetLastError());
}

bool fused_persistent_fits(const FusedArgs& a) {
    const long long need = (a.n + kThreads - 1) / kThreads;
    return need <= fused_grid(persistent_kernel(), a.n, a.sm_count) && need <= fused_grid(iter_kernel(), a.n, a.sm_count);
}

void fused_launch_persistent(const FusedArgs& a, double eps2, long long max_iter, cudaStream_t s) {
    const int g = (a.n + kThreads - 1) / kThreads;  // the grid of k_f_init / k_f_w / k_f_iter when it fits
    CP_CHECK(fused_persistent_fits(a) && g <= a.max_blocks, CP_ERR_INVALID, "persistent CG: grid does not fit");
    // the reduction ticket and the barrier's release counter start at zero
    static_assert(offsetof(CgScalars, gen) == offsetof(CgScalars, ticket) + sizeof(unsigned int),
                  "ticket and gen must be adjacent");
    CP_CUDA(cudaMemsetAsync(&a.sc->ticket, 0, 2 * sizeof(unsigned int), s));
    FusedArgs args = a;
    void* params[] = {&args, &eps2, &max_iter};
    CP_CUDA(cudaLaunchCooperativeKernel((const void*)persistent_kernel(), dim3(g), dim3(kThreads), params, 0, s));
}

bool pdl_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("CUPLAST_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

void fused_launch_iteration(const FusedArgs& a, int parity, cudaStream_t s) {
    const IterKernel k = iter_kernel();
    const int g = fused_grid(k, a.n, a.sm_count);
    CP_CHECK(g <= a.max_blocks, CP_ERR_INVALID, "partials buffer too small");
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(g);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    CP_CUDA(cudaLaunchKernelEx(&cfg, k, a, parity));
}

// "while (!converged) { body_iters x iteration }" as a graph with a WHILE
// node; body_iters must be even (record parity).
cudaGraphExec_t fused_build_while_graph(const FusedArgs& a, int body_iters, cudaStream_t s) {
    cudaGraph_t g;
    CP_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    CP_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CP_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CP_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    for (int it = 0; it < body_iters; ++it) fused_launch_iteration(a, it & 1, s);
    k_f_condition<<<1, 1, 0, s>>>(a.sc, h);
    cudaGraph_t captured = nullptr;
    CP_CUDA(cudaStreamEndCapture(s, &captured));
    cudaGraphExec_t exec;
    CP_CUDA(cudaGraphInstantiate(&exec, g, 0));
    CP_CUDA(cudaGraphDestroy(g));
    return exec;
}

}  // namespace cp
