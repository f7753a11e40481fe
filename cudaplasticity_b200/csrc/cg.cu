// Masked conjugate gradients on the node-blocked CSR.
//
// Reference semantics (ConjGradSolver::solve, src/ConjGradSolver.h:52-101;
// ConjGradCuda::solve, src/ConjGradCuda.cu:185-231): unpreconditioned CG on the
// unmodified K, Dirichlet DOFs handled by a mask on the residual,
//   r0 = m.(b - K x0), z0 = r0, rr = (r, r)
//   alpha = rr / (K z, z); x += alpha z; r -= m.alpha K z
//   beta = (r', r') / rr; z = r' + beta z
// stop when (r, r) / (b, b) <= eps^2.
//
// One iteration = two kernels, no host round trip:
//   P: z' = v + beta z (own node), K z' gathered as K (v + beta z) from the
//      neighbours, (K z', z')          -- the SpMV reads each 2x2 block once
//   U: x += alpha z', r -= m.alpha K z', v' = M r (v' = r without the
//      preconditioner), (r, r)
// The neighbours' inputs of P are packed in one record per node, rec[n] =
// (v, z), double-buffered by iteration parity: P reads (v, z) of parity p and
// writes z' to a plain vector, U writes the whole record (v', z') of parity
// 1 - p (whole records: no partially written L2 sectors). A neighbour costs
// one gather (16 bytes in FP32, 32 in FP64).
// Scalars live on the device; every cross-block sum is reduced by the last
// block in index order (deterministic). The loop runs in a CUDA graph whose
// WHILE node re-launches the body until the device sets "converged".
//
// T is the type of K's values and of the CG recurrences (double, or float in
// the mixed-precision mode); the solution x always accumulates in FP64, and
// every dot product is accumulated and reduced in FP64.
#include <cstdlib>
#include <mutex>
#include <unordered_map>

#include "common.cuh"
#include "internal.h"
#include "cg.h"

namespace cp {

namespace {

constexpr int kThreads = 256;

// Block k of the node in lane l of slice sl: 4 values (K00 K01 K10 K11).
template <typename T>
__device__ __forceinline__ typename Vec4<T>::type load_block(const T* __restrict__ val, long long b) {
    using V4 = typename Vec4<T>::type;
    return *reinterpret_cast<const V4*>(val + 4 * b);
}
template <>
__device__ __forceinline__ double4 load_block<double>(const double* __restrict__ val, long long b) {
    // two 128-bit loads: lane l reads 32 B at 32 l, a warp reads 1 KB per block row
    const double2* p = reinterpret_cast<const double2*>(val + 4 * b);
    const double2 lo = __ldg(p), hi = __ldg(p + 1);
    return make_double4(lo.x, lo.y, hi.x, hi.y);
}
template <>
__device__ __forceinline__ float4 load_block<float>(const float* __restrict__ val, long long b) {
    return __ldg(reinterpret_cast<const float4*>(val + 4 * b));
}

// The same with the streaming hint of ld_stream.
template <typename T, bool ST>
__device__ __forceinline__ typename Vec4<T>::type load_block_st(const T* __restrict__ val, long long b) {
    using V4 = typename Vec4<T>::type;
    if constexpr (ST) return __ldcs(reinterpret_cast<const V4*>(val + 4 * b));
    else return load_block<T>(val, b);
}
template <>
__device__ __forceinline__ double4 load_block_st<double, true>(const double* __restrict__ val, long long b) {
    const double2* p = reinterpret_cast<const double2*>(val + 4 * b);
    const double2 lo = __ldcs(p), hi = __ldcs(p + 1);
    return make_double4(lo.x, lo.y, hi.x, hi.y);
}

// Node c's record (v, z) of the parity being read.
template <typename T>
__device__ __forceinline__ typename Vec4<T>::type load_rec(const typename Vec4<T>::type* rec, int c) {
    return rec[c];
}
template <>
__device__ __forceinline__ double4 load_rec<double>(const double4* rec, int c) {
    const double2* p = reinterpret_cast<const double2*>(rec + c);
    const double2 lo = p[0], hi = p[1];
    return make_double4(lo.x, lo.y, hi.x, hi.y);
}


// One warp per slice of 32 nodes, one thread per node: the loop over slices
// advances whole warps, so the trip count is warp-uniform.
#define CP_SLICE_LOOP(nvalid)                                                                    \
    const int lane = threadIdx.x & 31;                                                           \
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;                               \
    const int nwarps = (gridDim.x * blockDim.x) >> 5;                                            \
    for (int sl = warp; sl < (nvalid + 31) / 32; sl += nwarps)

// r = m.(b - K_A u) in FP64 arithmetic (A in VA precision), written in the
// recurrence type T; z = 0. Sums (r,r) in FP64 of the T-rounded values,
// (r64, r64) and (b, b). The last block sets up the scalars of the solve.
template <typename VA, typename T, bool PRE>
__global__ void __launch_bounds__(kThreads) k_cg_init(CgArgs<T> a, const VA* __restrict__ valA, double eps2,
                                                      long long max_iter, int relative_to_r0, double outer_eps2) {
    using V2 = typename Vec2<T>::type;
    __shared__ double sh[2 * kThreads / 32];
    __shared__ bool last;
    double s_rr = 0.0, s_r64 = 0.0, s_bb = 0.0, s_rho = 0.0;
    CP_SLICE_LOOP(a.n) {
        const int n = 32 * sl + lane;
        const int base = a.slice_ptr[sl], w = (a.slice_ptr[sl + 1] - base) >> 5;
        if (n < a.n) {
            double k0 = 0.0, k1 = 0.0;
#pragma unroll 3
            for (int k = 0; k < w; ++k) {
                const long long b = base + 32LL * k + lane;
                const int c = __ldg(a.scol + b);
                const auto v = load_block<VA>(valA, b);
                const double2 xc = a.x[c];
                k0 += (double)v.x * xc.x + (double)v.y * xc.y;
                k1 += (double)v.z * xc.x + (double)v.w * xc.y;
            }
            const double2 bb = a.b[n];
            const uchar2 m = a.mask[n];
            const double r0 = m.x ? bb.x - k0 : 0.0, r1 = m.y ? bb.y - k1 : 0.0;
            V2 rt;
            rt.x = (T)r0;
            rt.y = (T)r1;
            a.r[n] = rt;
            typename Vec4<T>::type rec;
            rec.x = rt.x;
            rec.y = rt.y;
            rec.z = (T)0;
            rec.w = (T)0;
            s_rr += (double)rt.x * (double)rt.x + (double)rt.y * (double)rt.y;
            if (PRE) {
                // inverse of the node's 2x2 diagonal block (block 0), restricted
                // to the free DOFs of the node
                const auto d = load_block<VA>(valA, base + lane);
                double i00 = 0, i01 = 0, i10 = 0, i11 = 0;
                if (m.x && m.y) {
                    const double det = (double)d.x * d.w - (double)d.y * d.z;
                    i00 = d.w / det; i01 = -d.y / det; i10 = -d.z / det; i11 = d.x / det;
                } else if (m.x) {
                    i00 = 1.0 / d.x;
                } else if (m.y) {
                    i11 = 1.0 / d.w;
                }
                typename Vec4<T>::type mi;
                mi.x = (T)i00; mi.y = (T)i01; mi.z = (T)i10; mi.w = (T)i11;
                a.minv[n] = mi;
                V2 sv;
                sv.x = mi.x * rt.x + mi.y * rt.y;
                sv.y = mi.z * rt.x + mi.w * rt.y;
                rec.x = sv.x;
                rec.y = sv.y;
                s_rho += (double)rt.x * (double)sv.x + (double)rt.y * (double)sv.y;
            }
            a.rec0[n] = rec;
            s_r64 += r0 * r0 + r1 * r1;
            s_bb += bb.x * bb.x + bb.y * bb.y;
        }
    }
    double2 p = block_sum2(s_rr, s_r64, sh);
    double2 q = block_sum2(s_bb, s_rho, sh);
    if (threadIdx.x == 0) {
        a.partials[4 * blockIdx.x] = p.x;
        a.partials[4 * blockIdx.x + 1] = p.y;
        a.partials[4 * blockIdx.x + 2] = q.x;
        a.partials[4 * blockIdx.x + 3] = q.y;
    }
    if (last_block_arrive(&a.sc->ticket, &last)) {
        double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
        for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
            const volatile double* pp = a.partials + 4 * i;
            t0 += pp[0];
            t1 += pp[1];
            t2 += pp[2];
            t3 += pp[3];
        }
        double2 x = block_sum2(t0, t1, sh);
        double2 yy = block_sum2(t2, t3, sh);
        const double y = yy.x;
        if (threadIdx.x == 0) {
            CgScalars* sc = a.sc;
            sc->rr = x.x;
            sc->rho = PRE ? yy.y : x.x;
            sc->res64 = x.y;
            sc->bb = y;
            sc->beta = 0.0;
            sc->alpha = 0.0;
            sc->iter = 0;
            sc->max_iter = max_iter;
            sc->eps2 = eps2;
            sc->status = 0;
            sc->normB_inv = relative_to_r0 ? (x.x > 0.0 ? 1.0 / x.x : 0.0) : (y > 0.0 ? 1.0 / y : 0.0);
            // outer_eps2 >= 0: the FP64 residual already meets the caller's
            // tolerance, no inner iterations needed
            const bool lin_done = outer_eps2 >= 0.0 && x.y <= outer_eps2 * y;
            sc->lin_done = lin_done ? 1 : 0;
            sc->converged = (lin_done || x.x == 0.0 || x.x * sc->normB_inv <= eps2) ? 1 : 0;
            if (!(x.x == x.x) || !(y == y)) sc->status = CP_ERR_BREAKDOWN;
            sc->ticket = 0;
        }
    }
}

// P: z' = v + beta z (own node); K z' gathered as K (v + beta z); (K z', z').
// C > 0: the blocks of a row are taken C at a time, their columns and values
// loaded together before the C record gathers; C = 0: one loop, unrolled.
template <typename T, bool PRE, int C, bool ST>
__global__ void __launch_bounds__(kThreads) k_cg_p(CgArgs<T> a, int parity) {
    using V2 = typename Vec2<T>::type;
    using V4 = typename Vec4<T>::type;
    __shared__ double sh[kThreads / 32];
    __shared__ bool last;
    CgScalars* sc = a.sc;
    if (sc->converged || sc->status) return;
    const V4* __restrict__ ro = parity ? a.rec1 : a.rec0;
    const T beta = (T)sc->beta;
    double dot = 0.0;
    CP_SLICE_LOOP(a.n) {
        const int n = 32 * sl + lane;
        const int base = a.slice_ptr[sl], w = (a.slice_ptr[sl + 1] - base) >> 5;
        if (n < a.n) {
            T k0 = (T)0, k1 = (T)0;
            if (C == 0) {
#pragma unroll 3
                for (int k = 0; k < w; ++k) {
                    const long long b = base + 32LL * k + lane;
                    const int c = ld_stream<ST>(a.scol + b);
                    const auto v = load_block_st<T, ST>(a.val, b);
                    const V4 g = load_rec<T>(ro, c);
                    const T wx = g.x + beta * g.z, wy = g.y + beta * g.w;
                    k0 += v.x * wx + v.y * wy;
                    k1 += v.z * wx + v.w * wy;
                }
            } else {
                for (int k0i = 0; k0i < w; k0i += (C > 0 ? C : 1)) {
                    int cc[C > 0 ? C : 1];
                    V4 vv[C > 0 ? C : 1];
#pragma unroll
                    for (int j = 0; j < C; ++j) {
                        if (k0i + j < w) {
                            const long long b = base + 32LL * (k0i + j) + lane;
                            cc[j] = ld_stream<ST>(a.scol + b);
                            vv[j] = load_block_st<T, ST>(a.val, b);
                        }
                    }
#pragma unroll
                    for (int j = 0; j < C; ++j) {
                        if (k0i + j < w) {
                            const V4 g = load_rec<T>(ro, cc[j]);
                            const T wx = g.x + beta * g.z, wy = g.y + beta * g.w;
                            k0 += vv[j].x * wx + vv[j].y * wy;
                            k1 += vv[j].z * wx + vv[j].w * wy;
                        }
                    }
                }
            }
            const V4 own = load_rec<T>(ro, n);
            V2 zz, qq;
            zz.x = own.x + beta * own.z;
            zz.y = own.y + beta * own.w;
            qq.x = k0;
            qq.y = k1;
            a.zn[n] = zz;
            a.q[n] = qq;
            dot += (double)k0 * (double)zz.x + (double)k1 * (double)zz.y;
        }
    }
    const double bs = block_sum(dot, sh);
    if (threadIdx.x == 0) a.partials[blockIdx.x] = bs;
    if (last_block_arrive(&sc->ticket, &last)) {
        const double pAz = block_reduce_array(a.partials, gridDim.x, sh);
        if (threadIdx.x == 0) {
            sc->pAz = pAz;
            sc->alpha = sc->rho / pAz;
            if (!(pAz > 0.0) || !(sc->alpha == sc->alpha)) sc->status = CP_ERR_BREAKDOWN;
            sc->ticket = 0;
        }
    }
}

// U: x += alpha z', r -= m.alpha K z', (r, r); the last block finishes the iteration.
template <typename T, bool PRE>
__global__ void __launch_bounds__(kThreads) k_cg_u(CgArgs<T> a, int parity) {
    using V2 = typename Vec2<T>::type;
    __shared__ bool last;
    CgScalars* sc = a.sc;
    if (sc->converged || sc->status) return;
    typename Vec4<T>::type* __restrict__ rn = parity ? a.rec0 : a.rec1;
    using V4 = typename Vec4<T>::type;
    const double alpha = sc->alpha;
    const T alpha_t = (T)alpha;
    double dot = 0.0, dot_s = 0.0;
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < a.n; n += gridDim.x * blockDim.x) {
        const V2 z = a.zn[n], q = a.q[n];
        const uchar2 m = a.mask[n];
        double2 x = a.x[n];
        x.x += alpha * (double)z.x;
        x.y += alpha * (double)z.y;
        a.x[n] = x;
        V2 r = a.r[n];
        if (m.x) r.x -= alpha_t * q.x;
        if (m.y) r.y -= alpha_t * q.y;
        a.r[n] = r;
        dot += (double)r.x * (double)r.x + (double)r.y * (double)r.y;
        V4 rec;
        rec.z = z.x;
        rec.w = z.y;
        if (PRE) {
            const auto mi = a.minv[n];
            V2 sv;
            sv.x = mi.x * r.x + mi.y * r.y;
            sv.y = mi.z * r.x + mi.w * r.y;
            rec.x = sv.x;
            rec.y = sv.y;
            dot_s += (double)r.x * (double)sv.x + (double)r.y * (double)sv.y;
        } else {
            rec.x = r.x;
            rec.y = r.y;
        }
        rn[n] = rec;
    }
    __shared__ double sh2[2 * kThreads / 32];
    const double2 bs = block_sum2(dot, dot_s, sh2);
    if (threadIdx.x == 0) {
        a.partials[2 * blockIdx.x] = bs.x;
        a.partials[2 * blockIdx.x + 1] = bs.y;
    }
    if (last_block_arrive(&sc->ticket, &last)) {
        const double2 t = block_reduce_array2(a.partials, gridDim.x, sh2);
        const double rn = t.x;
        if (threadIdx.x == 0) {
            const double rho_new = PRE ? t.y : rn;
            sc->beta = rho_new / sc->rho;
            sc->rho = rho_new;
            sc->rr = rn;
            sc->iter += 1;
            if (rn * sc->normB_inv <= sc->eps2) sc->converged = 1;
            else if (sc->iter >= sc->max_iter) sc->status = CP_ERR_NOT_CONVERGED;
            if (!(rn == rn)) sc->status = CP_ERR_BREAKDOWN;
            sc->ticket = 0;
        }
    }
}

__global__ void k_cg_condition(const CgScalars* sc, cudaGraphConditionalHandle h) {
    cudaGraphSetConditional(h, (sc->converged || sc->status) ? 0u : 1u);
}

// Grid = the blocks that can be resident at once (occupancy API), capped by
// the work: every kernel runs a grid-stride loop, one wave, no tail.
template <typename K>
int resident_grid(K kernel, long long units, int per_block, int sm_count) {
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
    long long g = (units + per_block - 1) / per_block;
    long long cap = (long long)sm_count * per_sm;
    if (g > cap) g = cap;
    return g < 1 ? 1 : (int)g;
}

}  // namespace

bool stream_loads() {
    static const bool v = [] {
        const char* e = std::getenv("CUPLAST_STREAM_LOADS");
        return !(e && e[0] == '0');
    }();
    return v;
}

template <typename T>
void cg_launch_init(const CgArgs<T>& a, const void* valA, bool valA_is_fp64, double eps2, long long max_iter,
                    int relative_to_r0, double outer_eps2, cudaStream_t s) {
#define CP_INIT(VA, PRE)                                                                                   \
    {                                                                                                      \
        auto k = k_cg_init<VA, T, PRE>;                                                                    \
        const int grid = resident_grid(k, a.n, kThreads, a.sm_count);                                     \
        CP_CHECK(grid <= a.max_blocks, CP_ERR_INVALID, "partials buffer too small");                       \
        k<<<grid, kThreads, 0, s>>>(a, (const VA*)valA, eps2, max_iter, relative_to_r0, outer_eps2);       \
    }
    if (valA_is_fp64) {
        if (a.precond) CP_INIT(double, true) else CP_INIT(double, false)
    } else {
        if (a.precond) CP_INIT(float, true) else CP_INIT(float, false)
    }
#undef CP_INIT
    CP_CUDA(cudaGetLastError());
}

// Blocks per gather chunk of P (0: the unrolled loop). CUPLAST_CG_CHUNK
// overrides the default, for measurements.
template <typename T>
int p_chunk() {
    static const int c = [] {
        const char* e = std::getenv("CUPLAST_CG_CHUNK");
        const int v = e ? std::atoi(e) : -1;
        return (v == 0 || v == 3 || v == 5 || v == 9) ? v : 0;
    }();
    return c;
}

template <typename T, bool PRE>
void (*p_kernel(int c))(CgArgs<T>, int) {
    if (stream_loads()) return k_cg_p<T, PRE, 0, true>;
    switch (c) {
    case 0: return k_cg_p<T, PRE, 0, false>;
    case 3: return k_cg_p<T, PRE, 3, false>;
    case 9: return k_cg_p<T, PRE, 9, false>;
    default: return k_cg_p<T, PRE, 5, false>;
    }
}

template <typename T>
void cg_launch_p(const CgArgs<T>& a, int parity, cudaStream_t s) {
    const int c = p_chunk<T>();
    auto kp = a.precond ? p_kernel<T, true>(c) : p_kernel<T, false>(c);
    const int gp = resident_grid(kp, a.n, kThreads, a.sm_count);
    CP_CHECK(gp <= a.max_blocks, CP_ERR_INVALID, "partials buffer too small");
    kp<<<gp, kThreads, 0, s>>>(a, parity);
    CP_CUDA(cudaGetLastError());
}

template <typename T>
void cg_launch_u(const CgArgs<T>& a, int parity, cudaStream_t s) {
    auto ku = a.precond ? k_cg_u<T, true> : k_cg_u<T, false>;
    const int gu = resident_grid(ku, a.n, kThreads, a.sm_count);
    CP_CHECK(gu <= a.max_blocks, CP_ERR_INVALID, "partials buffer too small");
    ku<<<gu, kThreads, 0, s>>>(a, parity);
    CP_CUDA(cudaGetLastError());
}

template <typename T>
void cg_launch_iteration(const CgArgs<T>& a, int parity, cudaStream_t s) {
    cg_launch_p<T>(a, parity, s);
    cg_launch_u<T>(a, parity, s);
}

// Captures "while (!converged) { body_iters x (P, U) }" as a graph with a
// conditional WHILE node. body_iters must be even (parity of z buffers).
template <typename T>
cudaGraphExec_t cg_build_while_graph(const CgArgs<T>& a, int body_iters, cudaStream_t s) {
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
    for (int it = 0; it < body_iters; ++it) cg_launch_iteration<T>(a, it & 1, s);
    k_cg_condition<<<1, 1, 0, s>>>(a.sc, h);
    cudaGraph_t captured = nullptr;
    CP_CUDA(cudaStreamEndCapture(s, &captured));
    cudaGraphExec_t exec;
    CP_CUDA(cudaGraphInstantiate(&exec, g, 0));
    CP_CUDA(cudaGraphDestroy(g));
    return exec;
}

template void cg_launch_init<double>(const CgArgs<double>&, const void*, bool, double, long long, int, double,
                                     cudaStream_t);
template void cg_launch_init<float>(const CgArgs<float>&, const void*, bool, double, long long, int, double,
                                    cudaStream_t);
template void cg_launch_iteration<double>(const CgArgs<double>&, int, cudaStream_t);
template void cg_launch_p<double>(const CgArgs<double>&, int, cudaStream_t);
template void cg_launch_p<float>(const CgArgs<float>&, int, cudaStream_t);
template void cg_launch_u<double>(const CgArgs<double>&, int, cudaStream_t);
template void cg_launch_u<float>(const CgArgs<float>&, int, cudaStream_t);
template void cg_launch_iteration<float>(const CgArgs<float>&, int, cudaStream_t);
template cudaGraphExec_t cg_build_while_graph<double>(const CgArgs<double>&, int, cudaStream_t);
template cudaGraphExec_t cg_build_while_graph<float>(const CgArgs<float>&, int, cudaStream_t);

}  // namespace cp
