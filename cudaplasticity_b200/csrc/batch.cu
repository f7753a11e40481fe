// Batched mixed-precision solves: many independent instances on one GPU.
//
// Every instance runs the single-instance algorithm of cp_solve in its
// mixed-precision form (outer secant iteration of the reference's
// PlasticitySolver::solveCUDA, src/PlasticitySolver.cu:469-512; masked CG of
// ConjGradCuda::solve, src/ConjGradCuda.cu:185-231, here with FP32 values and
// recurrences inside FP64 defect correction) as its own state machine on the
// device:
//
//   LEVEL -> ASM -> RES -> W -> ITER* [-> RES -> W -> ITER*] -> UPD -> RELAX -> ASM ...
//                           (level converged) -> LEVEL / PLASTIC -> DONE
//
// The linear solve is one preconditioned CG on the FP32 values with FP32
// recurrences ("reliable updates"): RES computes the residual b - K64 x in
// FP64 at the start; whenever the recursive FP32 residual has dropped by
// inner_tol since the last replacement, or meets the solve's tolerance, RES
// replaces it by the FP64 residual of the FP64 solution and the search
// direction carries on, so the Krylov space is kept; the solve ends when the
// FP64 residual meets the tolerance. One CG iteration is one launch (the
// Chronopoulos-Gear form, see the CG section).
//
// The instances' nodes and elements are cut into tiles; one work list holds
// every (instance, tile) pair. Three persistent kernels walk that list, each
// acting only on the tiles whose instance is in one of its phases:
//   k_batch_cg    RES (FP64 residual), W (w = K u), ITER (one CG iteration)
//   k_batch_asm   ASM (FP64 + FP32 values of K, node gather, no atomics)
//   k_batch_elem  LEVEL, UPD (strain / stress / secant / exit norm),
//                 RELAX (Aitken), PLASTIC
// Each tile writes one partial sum per 32-node slice or 32-element group; the
// last tile of an instance to arrive (per-instance ticket) reduces that
// instance's partials in index order with a fixed thread assignment and moves
// the instance to its next phase. The sums therefore do not depend on the
// tiling, on the grid, or on the other instances in the batch.
//
// One CUDA graph drives a run: a WHILE node whose body is
//   elem x E, asm, cg x C, condition
// and every launch advances every instance in a matching phase by one step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "common.cuh"
#include "elements.cuh"
#include "instance.h"
#include "internal.h"

namespace cp {
namespace {

constexpr int kThreads = 128;  // 4 warps; every kernel of the batch
constexpr int kWarps = kThreads / 32;
constexpr int kBuckets = 24;

enum : int {
    PH_FREE = 0,
    PH_LEVEL,
    PH_ASM,
    PH_RES,
    PH_W,
    PH_ITER,
    PH_UPD,
    PH_RELAX,
    PH_PLASTIC,
    PH_DONE,
    PH_COUNT
};

// Read-only description of one instance (written by the host at add).
struct BDesc {
    DevMesh m;
    int n_slices, n_groups;  // 32-node slices, 32-element groups
    const int* slice_ptr;
    const int* scol;
    const int* inc_pos;
    const int* inc;
    const uint32_t* inc_k;
    const uint32_t* inc_k8;
    double* val64;
    float* val32;
    double2* x;
    double2* b;
    const double2* b_full;
    const double2* u_full;
    const uchar2* mask;
    float2 *r, *w, *kp, *p;  // FP32 CG vectors, own node only
    float4 *gA, *gB;         // read by the neighbours, A/B by parity: node n's 32-byte record is
                             // g[2n] = (u, M w), g[2n+1] = (M kp, 0): one L2 sector per neighbour
    float4* minv;
    ElemState st;
    MaterialDev mat;
    double* part;  // 8 per slice / group
    double cg_tol, outer_tol, inner_tol;
    long long max_cg;
    int max_outer, levels, aitken, adaptive, precond;
    int predict;        // level predictor (cp_solve_opts.predict)
    double2* pred_u;    // the last level's u and psi (predict only)
    double* pred_psi;
};

// Mutable state of one instance.
struct BState {
    int phase, status, level, levels_done;
    int outer_it, outer_total, parity, res_kind;  // res_kind: 0 first residual of a solve, 1 replacement
    unsigned int ticket;
    int stalls;  // consecutive FP64 residual replacements without a 2x reduction
    long long iter, lin_iters, cg_total, fp64_spmv;
    double rr, gamma, alpha, beta, rr_ref, eps2_inner, bb, res64, res_last;
    double eps, rel_err, w_prev, omega, cg_rel_res;
    unsigned long long t_first, t_done;  // %globaltimer, ns
};

// Run control. The host writes it before every launch.
struct BCtl {
    int n_tiles;
    int active;
    int done;
    int exit_on_done;  // stop once done >= exit_on_done (0: never)
    long long trips, max_trips;
    int pop[PH_COUNT];  // instances per phase
    const volatile int* stop;  // host-mapped interrupt flag
    int go;                    // condition of the last trip (direct launches)
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void set_phase(BState* S, BCtl* c, int ph) {
    atomicSub(&c->pop[S->phase], 1);
    atomicAdd(&c->pop[ph], 1);
    S->phase = ph;
}

__device__ __forceinline__ void finish(BState* S, BCtl* c, int status) {
    if (status) S->status = status;
    S->t_done = global_ns();
    set_phase(S, c, PH_DONE);
    atomicAdd(&c->done, 1);
    atomicSub(&c->active, 1);
}

// Every thread of the block: true in the block whose tile is the instance's
// last to arrive in this launch.
__device__ __forceinline__ bool arrive(BState* S, int ntiles, int* sh_flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int t = atomicAdd(&S->ticket, 1u);
        *sh_flag = (t == (unsigned int)ntiles - 1u);
    }
    __syncthreads();
    const bool last = *sh_flag != 0;
    if (last) __threadfence();
    return last;
}

// Sums of the first K of the 8 partials per unit over units [0, n), fixed
// assignment (thread t takes units t, t + 128, ...) and a fixed tree.
// Results valid in thread 0.
constexpr int kPart = 8;
template <int K>
__device__ __forceinline__ void reduce_parts(const double* part, int n, double* out, double* sh) {
    double a[K];
#pragma unroll
    for (int k = 0; k < K; ++k) a[k] = 0.0;
    for (int i = threadIdx.x; i < n; i += kThreads) {
        const volatile double* p = part + kPart * (size_t)i;
#pragma unroll
        for (int k = 0; k < K; ++k) a[k] += p[k];
    }
#pragma unroll
    for (int k = 0; k < K; k += 2) {
        const double2 s = block_sum2(a[k], k + 1 < K ? a[k + 1] : 0.0, sh);
        out[k] = s.x;
        if (k + 1 < K) out[k + 1] = s.y;
    }
}

__device__ __forceinline__ int tile_phase(const BState* S, int* sh) {
    __syncthreads();
    if (threadIdx.x == 0) *sh = *(const volatile int*)&S->phase;
    __syncthreads();
    return *sh;
}

// Linear tolerance of the next solve, cp_solve's adaptive rules: 1 inexact
// early steps, tight within 10x of the outer tolerance; 2 looser, tight once
// the outer tolerance is met.
__device__ __forceinline__ double next_eps(const BDesc& d, double rel_err) {
    if (d.adaptive == 2) return rel_err > d.outer_tol ? fmax(d.cg_tol, kRule2Factor * rel_err) : d.cg_tol;
    return (d.adaptive && rel_err > 10.0 * d.outer_tol) ? fmax(d.cg_tol, 1e-2 * rel_err) : d.cg_tol;
}

// After the update (and Aitken): next level, plastic strains, or another
// outer iteration (cp_solve's loop body).
__device__ __forceinline__ void decide(const BDesc& d, BState* S, BCtl* c) {
    const bool conv = S->rel_err <= d.outer_tol && S->eps <= d.cg_tol;
    if (conv) {
        S->levels_done = S->level;
        if (S->level < d.levels) {
            S->level += 1;
            set_phase(S, c, PH_LEVEL);
        } else {
            set_phase(S, c, PH_PLASTIC);
        }
    } else if (S->outer_it >= d.max_outer) {
        S->levels_done = S->level;
        S->status = CP_ERR_NOT_CONVERGED;
        set_phase(S, c, PH_PLASTIC);
    } else {
        S->eps = next_eps(d, S->rel_err);
        set_phase(S, c, PH_ASM);
    }
}

// ------------------------------------------------------------ CG phases --
//
// The linear solve is preconditioned CG with one reduction per iteration
// (the Chronopoulos-Gear arrangement): with M the 2x2 block-Jacobi inverse
// (the Dirichlet mask without preconditioning), u = M r, w = K u, p the
// direction, kp = K p, an iteration is
//   p' = u + beta p, kp' = w + beta kp, x += alpha p', r' = m.(r - alpha kp'),
//   u' = u - alpha (M w + beta M kp), w' = K u',
//   gamma' = (r', u'), beta' = gamma' / gamma, alpha' = gamma' / (K p'', p'')
// with (K p'', p'') = (w', u') + beta' ((w', p') + (kp', u')) + beta'^2 (kp', p')
// expanded from this iteration's vectors, as standard CG computes its step.
// K u' needs the neighbours' new u, which each thread recomputes from the
// neighbours' u, M w and M kp, packed in one 32-byte record per node (one L2
// sector per neighbour; double-buffered by the instance's parity). The node
// itself uses the same formula, so every thread sees one vector u'.
// One iteration is one launch. RES (FP64 residual of the FP64 solution, at
// the start and at every replacement) and W (w = K u after it) bracket the
// iterations; r, u, w, kp, p are FP32, x and every sum are FP64.

__device__ __forceinline__ float2 mvec(const float4& m, float2 v) {
    return make_float2(m.x * v.x + m.y * v.y, m.z * v.x + m.w * v.y);
}
// M v: the block-Jacobi inverse, or the mask without preconditioning.
__device__ __forceinline__ float2 apply_m(const BDesc& d, int n, float2 v) {
    if (d.precond) return mvec(d.minv[n], v);
    const uchar2 m = d.mask[n];
    return make_float2(m.x ? v.x : 0.f, m.y ? v.y : 0.f);
}

// RES: r = m.(b - K64 x) in FP64 (stored in FP32), u = M r; at the start of
// a solve also the block-Jacobi inverse and p = kp = M kp = 0. Sums
// (r32, r32), (r64, r64), (b, b).
__device__ void tile_res(const BDesc& d, BState* S, BCtl* c, int4 tl, double* sh, int* shf) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int sl0 = tl.y * tl.z, sl1 = min(sl0 + tl.z, d.n_slices);
    const int pre = d.precond, first = S->res_kind == 0;
    const int par = S->parity;
    for (int sl = sl0 + w; sl < sl1; sl += kWarps) {
        const int n = 32 * sl + lane;
        const int base = d.slice_ptr[sl], wd = (d.slice_ptr[sl + 1] - base) >> 5;
        double s_rr = 0.0, s_r64 = 0.0, s_bb = 0.0;
        if (n < d.m.n_nodes) {
            double k0 = 0.0, k1 = 0.0;
            for (int k = 0; k < wd; ++k) {
                const long long bi = base + 32LL * k + lane;
                const int col = __ldg(d.scol + bi);
                const double2* vp = reinterpret_cast<const double2*>(d.val64 + 4 * bi);
                const double2 lo = __ldg(vp), hi = __ldg(vp + 1);
                const double2 xc = d.x[col];
                k0 += lo.x * xc.x + lo.y * xc.y;
                k1 += hi.x * xc.x + hi.y * xc.y;
            }
            const double2 bb = d.b[n];
            const uchar2 m = d.mask[n];
            const double r0 = m.x ? bb.x - k0 : 0.0, r1 = m.y ? bb.y - k1 : 0.0;
            const float2 rt = make_float2((float)r0, (float)r1);
            d.r[n] = rt;
            if (pre && first) {
                // inverse of the node's 2x2 diagonal block, restricted to its free DOFs
                const double2* dp = reinterpret_cast<const double2*>(d.val64 + 4 * ((long long)base + lane));
                const double2 dlo = __ldg(dp), dhi = __ldg(dp + 1);
                double i00 = 0, i01 = 0, i10 = 0, i11 = 0;
                if (m.x && m.y) {
                    const double det = dlo.x * dhi.y - dlo.y * dhi.x;
                    i00 = dhi.y / det; i01 = -dlo.y / det; i10 = -dhi.x / det; i11 = dlo.x / det;
                } else if (m.x) {
                    i00 = 1.0 / dlo.x;
                } else if (m.y) {
                    i11 = 1.0 / dhi.y;
                }
                d.minv[n] = make_float4((float)i00, (float)i01, (float)i10, (float)i11);
            }
            float4* g = par ? d.gB : d.gA;
            const float2 u = apply_m(d, n, rt);
            reinterpret_cast<float2*>(g + 2 * (size_t)n)[0] = u;
            if (first) {
                const float2 z = make_float2(0.f, 0.f);
                d.p[n] = z;
                d.kp[n] = z;
                g[2 * (size_t)n + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            s_rr = (double)rt.x * (double)rt.x + (double)rt.y * (double)rt.y;
            s_r64 = r0 * r0 + r1 * r1;
            s_bb = bb.x * bb.x + bb.y * bb.y;
        }
        s_rr = warp_sum(s_rr);
        s_r64 = warp_sum(s_r64);
        s_bb = warp_sum(s_bb);
        if (lane == 0) {
            double* p = d.part + kPart * (size_t)sl;
            p[0] = s_rr; p[1] = s_r64; p[2] = s_bb;
        }
    }
    if (!arrive(S, tl.w, shf)) return;
    double t[4];
    reduce_parts<3>(d.part, d.n_slices, t, sh);
    if (threadIdx.x == 0) {
        const double rr = t[0], res64 = t[1];
        S->ticket = 0;
        S->fp64_spmv += 1;
        if (first) S->bb = t[2];
        const double bb = S->bb;
        S->res64 = res64;
        S->cg_rel_res = bb > 0.0 ? sqrt(res64 / bb) : 0.0;
        // FP32 limit: on very ill-conditioned systems (kappa * eps32 >~ 1) the
        // recursive FP32 residual keeps falling while the FP64 residual no
        // longer does. Two replacements in a row without halving the FP64
        // residual norm end the linear solve with the best x so far (the
        // secant iteration goes on) instead of iterating to the cap.
        if (first) {
            S->stalls = 0;
        } else {
            S->stalls = res64 < 0.25 * S->res_last ? 0 : S->stalls + 1;
        }
        S->res_last = res64;
        if (!(rr == rr) || !(bb == bb) || !(res64 == res64)) {
            finish(S, c, CP_ERR_BREAKDOWN);
        } else if (res64 <= S->eps * S->eps * bb || rr == 0.0 || S->lin_iters >= d.max_cg || S->stalls >= 2) {
            set_phase(S, c, PH_UPD);  // the linear solve meets its tolerance (or its cap, or stalls)
        } else {
            S->rr = rr;
            S->rr_ref = rr;
            set_phase(S, c, PH_W);
        }
    }
}

// W: w = K32 u (u of RES, read from the neighbours), M w; gamma = (r, u),
// (w, u) and, for the direction that carries on after a replacement, (w, p),
// (kp, u), (kp, p): the step scalars of the next iteration.
__device__ void tile_w(const BDesc& d, BState* S, BCtl* c, int4 tl, double* sh, int* shf) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int sl0 = tl.y * tl.z, sl1 = min(sl0 + tl.z, d.n_slices);
    const int par = S->parity;
    float4* __restrict__ g = par ? d.gB : d.gA;
    for (int sl = sl0 + w; sl < sl1; sl += kWarps) {
        const int n = 32 * sl + lane;
        const int base = d.slice_ptr[sl], wd = (d.slice_ptr[sl + 1] - base) >> 5;
        double s_g = 0.0, s_d = 0.0, s_wp = 0.0, s_ku = 0.0, s_kp = 0.0;
        if (n < d.m.n_nodes) {
            float k0 = 0.f, k1 = 0.f;
#pragma unroll 3
            for (int k = 0; k < wd; ++k) {
                const long long bi = base + 32LL * k + lane;
                const int col = __ldg(d.scol + bi);
                const float4 v = __ldg(reinterpret_cast<const float4*>(d.val32 + 4 * bi));
                const float2 uc = reinterpret_cast<const float2*>(g + 2 * (size_t)col)[0];
                k0 += v.x * uc.x + v.y * uc.y;
                k1 += v.z * uc.x + v.w * uc.y;
            }
            const float2 wn = make_float2(k0, k1);
            d.w[n] = wn;
            const float2 un = reinterpret_cast<const float2*>(g + 2 * (size_t)n)[0];
            const float2 mw = apply_m(d, n, wn);
            g[2 * (size_t)n] = make_float4(un.x, un.y, mw.x, mw.y);
            const float2 rn = d.r[n], pn = d.p[n], kn = d.kp[n];
            s_g = (double)rn.x * (double)un.x + (double)rn.y * (double)un.y;
            s_d = (double)k0 * (double)un.x + (double)k1 * (double)un.y;
            s_wp = (double)k0 * (double)pn.x + (double)k1 * (double)pn.y;
            s_ku = (double)kn.x * (double)un.x + (double)kn.y * (double)un.y;
            s_kp = (double)kn.x * (double)pn.x + (double)kn.y * (double)pn.y;
        }
        s_g = warp_sum(s_g);
        s_d = warp_sum(s_d);
        s_wp = warp_sum(s_wp);
        s_ku = warp_sum(s_ku);
        s_kp = warp_sum(s_kp);
        if (lane == 0) {
            double* p = d.part + kPart * (size_t)sl;
            p[0] = s_g; p[1] = s_d; p[2] = 0.0; p[3] = s_wp; p[4] = s_ku; p[5] = s_kp;
        }
    }
    if (!arrive(S, tl.w, shf)) return;
    double t[6];
    reduce_parts<6>(d.part, d.n_slices, t, sh);
    if (threadIdx.x == 0) {
        const double g = t[0];
        S->ticket = 0;
        // the first solve starts with p = kp = 0; after a replacement the
        // direction carries on with beta from the replaced residual
        const double beta = S->res_kind != 0 ? g / S->gamma : 0.0;
        const double den = t[1] + beta * (t[3] + t[4]) + beta * beta * t[5];
        const double alpha = g / den;
        if (!(den > 0.0) || !(g > 0.0) || !(alpha == alpha)) {
            // at the start of a solve the FP32 system is not positive
            // definite: a breakdown; after a replacement only the FP32 step
            // degenerated, and the solve ends with the x it has
            if (S->res_kind == 0) finish(S, c, CP_ERR_BREAKDOWN);
            else set_phase(S, c, PH_UPD);
        } else {
            S->gamma = g;
            S->alpha = alpha;
            S->beta = beta;
            set_phase(S, c, PH_ITER);
        }
    }
}

// ITER: one CG iteration (see the section comment). C > 0: the row's blocks
// are taken C at a time, columns and values loaded together ahead of the C
// record gathers; C = 0: one unrolled loop.
template <int C, bool ST = false>
__device__ void tile_iter(const BDesc& d, BState* S, BCtl* c, int4 tl, double* sh, int* shf) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int sl0 = tl.y * tl.z, sl1 = min(sl0 + tl.z, d.n_slices);
    const int par = S->parity;
    const float4* __restrict__ go = par ? d.gB : d.gA;
    float4* __restrict__ gn = par ? d.gA : d.gB;
    const double alpha = S->alpha;
    const float a = (float)alpha, bt = (float)S->beta;
    for (int sl = sl0 + w; sl < sl1; sl += kWarps) {
        const int n = 32 * sl + lane;
        const int base = d.slice_ptr[sl], wd = (d.slice_ptr[sl + 1] - base) >> 5;
        double s_g = 0.0, s_d = 0.0, s_rr = 0.0, s_x = 0.0, s_kp = 0.0;
        if (n < d.m.n_nodes) {
            // own node
            const float4 g0 = __ldg(go + 2 * (size_t)n), g1 = __ldg(go + 2 * (size_t)n + 1);
            const float2 u0 = make_float2(g0.x, g0.y), mw0 = make_float2(g0.z, g0.w), mk0 = make_float2(g1.x, g1.y);
            const float2 pn = d.p[n], wn = d.w[n], kn = d.kp[n];
            const uchar2 m = d.mask[n];
            const float2 p = make_float2(u0.x + bt * pn.x, u0.y + bt * pn.y);
            const float2 kp = make_float2(wn.x + bt * kn.x, wn.y + bt * kn.y);
            const float2 u = make_float2(u0.x - a * (mw0.x + bt * mk0.x), u0.y - a * (mw0.y + bt * mk0.y));
            double2 x = d.x[n];
            x.x += alpha * (double)p.x;
            x.y += alpha * (double)p.y;
            float2 r = d.r[n];
            if (m.x) r.x -= a * kp.x;
            if (m.y) r.y -= a * kp.y;
            // w' = K u' with the neighbours' u' from their u, M w, M kp
            float k0 = 0.f, k1 = 0.f;
            if (C == 0) {
#pragma unroll 3
                for (int k = 0; k < wd; ++k) {
                    const long long bi = base + 32LL * k + lane;
                    const int col = __ldg(d.scol + bi);
                    const float4 v = __ldg(reinterpret_cast<const float4*>(d.val32 + 4 * bi));
                    const float4 c0 = __ldg(go + 2 * (size_t)col), c1 = __ldg(go + 2 * (size_t)col + 1);
                    const float ux = c0.x - a * (c0.z + bt * c1.x), uy = c0.y - a * (c0.w + bt * c1.y);
                    k0 += v.x * ux + v.y * uy;
                    k1 += v.z * ux + v.w * uy;
                }
            } else {
                for (int k0i = 0; k0i < wd; k0i += (C > 0 ? C : 1)) {
                    int cc[C > 0 ? C : 1];
                    float4 vv[C > 0 ? C : 1];
#pragma unroll
                    for (int j = 0; j < C; ++j) {
                        if (k0i + j < wd) {
                            const long long bi = base + 32LL * (k0i + j) + lane;
                            cc[j] = ld_stream<ST>(d.scol + bi);
                            vv[j] = ld_stream<ST>(reinterpret_cast<const float4*>(d.val32 + 4 * bi));
                        }
                    }
#pragma unroll
                    for (int j = 0; j < C; ++j) {
                        if (k0i + j < wd) {
                            const float4 c0 = __ldg(go + 2 * (size_t)cc[j]), c1 = __ldg(go + 2 * (size_t)cc[j] + 1);
                            const float ux = c0.x - a * (c0.z + bt * c1.x), uy = c0.y - a * (c0.w + bt * c1.y);
                            k0 += vv[j].x * ux + vv[j].y * uy;
                            k1 += vv[j].z * ux + vv[j].w * uy;
                        }
                    }
                }
            }
            const float2 w2 = make_float2(k0, k1);
            d.p[n] = p;
            d.kp[n] = kp;
            d.x[n] = x;
            d.r[n] = r;
            d.w[n] = w2;
            const float2 mw = apply_m(d, n, w2), mk = apply_m(d, n, kp);
            gn[2 * (size_t)n] = make_float4(u.x, u.y, mw.x, mw.y);
            gn[2 * (size_t)n + 1] = make_float4(mk.x, mk.y, 0.f, 0.f);
            s_g = (double)r.x * (double)u.x + (double)r.y * (double)u.y;
            s_d = (double)k0 * (double)u.x + (double)k1 * (double)u.y;
            s_rr = (double)r.x * (double)r.x + (double)r.y * (double)r.y;
            s_x = ((double)k0 * (double)p.x + (double)k1 * (double)p.y) +
                  ((double)kp.x * (double)u.x + (double)kp.y * (double)u.y);  // (w', p') + (kp', u')
            s_kp = (double)kp.x * (double)p.x + (double)kp.y * (double)p.y;
        }
        s_g = warp_sum(s_g);
        s_d = warp_sum(s_d);
        s_rr = warp_sum(s_rr);
        s_x = warp_sum(s_x);
        s_kp = warp_sum(s_kp);
        if (lane == 0) {
            double* p = d.part + kPart * (size_t)sl;
            p[0] = s_g; p[1] = s_d; p[2] = s_rr; p[3] = s_x; p[4] = 0.0; p[5] = s_kp;
        }
    }
    if (!arrive(S, tl.w, shf)) return;
    double t[6];
    reduce_parts<6>(d.part, d.n_slices, t, sh);
    if (threadIdx.x == 0) {
        const double g = t[0], rn = t[2];
        S->ticket = 0;
        S->parity ^= 1;
        S->iter += 1;
        S->lin_iters += 1;
        S->cg_total += 1;
        S->rr = rn;
        const double beta = g / S->gamma;
        const double den = t[1] + beta * (t[3] + t[4]) + beta * beta * t[5];
        if (!(rn == rn) || !(g == g)) {
            finish(S, c, CP_ERR_BREAKDOWN);
        } else if (rn <= S->eps * S->eps * S->bb || rn <= S->eps2_inner * S->rr_ref || !(den > 0.0) || !(g > 0.0)) {
            // converged in the FP32 recurrence (or its step degenerated): check
            // against the FP64 residual, which restarts the scalars
            S->res_kind = 1;
            set_phase(S, c, PH_RES);
        } else if (S->lin_iters >= d.max_cg) {
            set_phase(S, c, PH_UPD);
        } else {
            S->beta = beta;
            S->alpha = g / den;
            S->gamma = g;
            set_phase(S, c, PH_ITER);
        }
    }
}

// 8 resident blocks per SM (64 registers): the CG iteration is bound by the
// latency of its gathers, and the occupancy pays for the few spills. C: the
// ITER gather form (tile_iter).
template <int C, bool ST = false>
__global__ void __launch_bounds__(kThreads, 8) k_batch_cg(const BDesc* __restrict__ D, BState* SS,
                                                       const int4* __restrict__ tiles, BCtl* c) {
    __shared__ double sh[2 * kWarps];
    __shared__ int shf, shp;
    {
        const volatile int* pop = c->pop;
        if (pop[PH_RES] + pop[PH_W] + pop[PH_ITER] == 0) return;
    }
    const int nt = c->n_tiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int4 tl = tiles[t];
        BState* S = SS + tl.x;
        const int ph = tile_phase(S, &shp);
        if (ph == PH_ITER) tile_iter<C, ST>(D[tl.x], S, c, tl, sh, &shf);
        else if (ph == PH_W) tile_w(D[tl.x], S, c, tl, sh, &shf);
        else if (ph == PH_RES) tile_res(D[tl.x], S, c, tl, sh, &shf);
    }
}

// The work of an iteration for the autotuner, with the same per-tile costs
// as ITER: the phase read, the own-node and neighbour loads and arithmetic,
// the per-slice sums, a fence and a ticket per tile, and the last tile's
// pass over the slice sums. Everything it writes goes to scratch arrays of
// the batch (sink, one ticket per slot, sums), so the instances' state is
// left untouched whatever phase they are in.
__global__ void __launch_bounds__(kThreads) k_batch_probe(const BDesc* __restrict__ D, const BState* SS,
                                                          const int4* __restrict__ tiles, int nt, float a, float bt,
                                                          float2* sink, unsigned int* tickets, double* sums) {
    __shared__ double sh[2 * kWarps];
    __shared__ int shf, shp;
    float2 acc = make_float2(0.f, 0.f);
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int4 tl = tiles[t];
        const BDesc& d = D[tl.x];
        (void)tile_phase(SS + tl.x, &shp);
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        const int sl0 = tl.y * tl.z, sl1 = min(sl0 + tl.z, d.n_slices);
        const int par = SS[tl.x].parity;
        const float4* __restrict__ go = par ? d.gB : d.gA;
        for (int sl = sl0 + w; sl < sl1; sl += kWarps) {
            const int n = 32 * sl + lane;
            const int base = d.slice_ptr[sl], wd = (d.slice_ptr[sl + 1] - base) >> 5;
            double s0 = 0.0;
            if (n < d.m.n_nodes) {
                const float4 g0 = go[2 * (size_t)n], g1 = go[2 * (size_t)n + 1];
                const float2 u0 = make_float2(g0.x, g0.y), mw0 = make_float2(g0.z, g0.w), mk0 = make_float2(g1.x, g1.y);
                const float2 pn = d.p[n], wn = d.w[n], kn = d.kp[n], rn = d.r[n];
                const double2 xn = d.x[n];
                float k0 = 0.f, k1 = 0.f;
#pragma unroll 3
                for (int k = 0; k < wd; ++k) {
                    const long long bi = base + 32LL * k + lane;
                    const int col = __ldg(d.scol + bi);
                    const float4 v = __ldg(reinterpret_cast<const float4*>(d.val32 + 4 * bi));
                    const float4 c0 = go[2 * (size_t)col], c1 = go[2 * (size_t)col + 1];
                    const float ux = c0.x - a * (c0.z + bt * c1.x), uy = c0.y - a * (c0.w + bt * c1.y);
                    k0 += v.x * ux + v.y * uy;
                    k1 += v.z * ux + v.w * uy;
                }
                acc.x += k0 + u0.x + mw0.x + mk0.x + pn.x + wn.x + kn.x + rn.x + (float)xn.x;
                acc.y += k1 + u0.y + mw0.y + mk0.y + pn.y + wn.y + kn.y + rn.y + (float)xn.y;
                s0 = (double)k0 * (double)u0.x;
            }
            s0 = warp_sum(s0);
            if (lane == 0) sums[blockIdx.x] = s0;
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) shf = (atomicAdd(tickets + tl.x, 1u) % (unsigned)tl.w) == (unsigned)tl.w - 1u;
        __syncthreads();
        if (shf) {
            double r[6];
            reduce_parts<6>(d.part, d.n_slices, r, sh);  // reads only
            if (threadIdx.x == 0) sums[blockIdx.x] += r[0];
        }
    }
    sink[blockIdx.x * kThreads + threadIdx.x] = acc;
}

// ------------------------------------------------------ assembly phase --

// ASM: K(E_c, nu_c) in FP64 and FP32, one warp per 32-node slice, the
// slice's blocks accumulated in the warp's shared-memory region (each lane
// only touches its own node's blocks; element order) and written once,
// coalesced. Same arithmetic as the single-instance assembly.
template <bool Q8>
__global__ void __launch_bounds__(kThreads) k_batch_asm(const BDesc* __restrict__ D, BState* SS,
                                                        const int4* __restrict__ tiles, BCtl* c, int max_width) {
    extern __shared__ double sacc[];
    __shared__ int shf, shp;
    {
        const volatile int* pop = c->pop;
        if (pop[PH_ASM] == 0) return;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double* acc = sacc + (size_t)w * 128 * max_width;
    const int nt = c->n_tiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int4 tl = tiles[t];
        BState* S = SS + tl.x;
        if (tile_phase(S, &shp) != PH_ASM) continue;
        const BDesc& d = D[tl.x];
        const int sl0 = tl.y * tl.z, sl1 = min(sl0 + tl.z, d.n_slices);
        for (int sl = sl0 + w; sl < sl1; sl += kWarps) {
            const int base = d.slice_ptr[sl], wd = (d.slice_ptr[sl + 1] - base) >> 5;
            const int len = 128 * wd;
            for (int i = lane; i < len; i += 32) acc[i] = 0.0;
            __syncwarp();
            const int n = 32 * sl + lane;
            if (n < d.m.n_nodes) {
                double* nb = acc + 4 * lane;
                for (int q = d.inc_pos[n]; q < d.inc_pos[n + 1]; ++q) {
                    const int code = d.inc[q];
                    const int e = code >> 3, i = code & 7;
                    const Dmat dm = form_d(d.mat.plane, d.st.E_c[e], d.st.nu_c[e]);
                    element_rows<Q8>(d.m, e, i, d.inc_k[q], Q8 && d.inc_k8 ? d.inc_k8[q] : 0u, dm, d.mat.h, nb);
                }
            }
            __syncwarp();
            double* o64 = d.val64 + 4LL * base;
            float* o32 = d.val32 + 4LL * base;
            for (int i = lane; i < len; i += 32) {
                const double v = acc[i];
                o64[i] = v;
                o32[i] = (float)v;
            }
            __syncwarp();
        }
        if (arrive(S, tl.w, &shf) && threadIdx.x == 0) {
            S->ticket = 0;
            S->res_kind = 0;
            S->eps2_inner = d.inner_tol * d.inner_tol;
            set_phase(S, c, PH_RES);
        }
    }
}

// --------------------------------------------------- element phases --

template <bool Q8>
__global__ void __launch_bounds__(kThreads) k_batch_elem(const BDesc* __restrict__ D, BState* SS,
                                                         const int4* __restrict__ tiles, BCtl* c) {
    __shared__ double sh[2 * kWarps];
    __shared__ int shf, shp;
    {
        const volatile int* pop = c->pop;
        if (pop[PH_LEVEL] + pop[PH_UPD] + pop[PH_RELAX] + pop[PH_PLASTIC] == 0) return;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nt = c->n_tiles;
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int4 tl = tiles[t];
        BState* S = SS + tl.x;
        const int ph = tile_phase(S, &shp);
        if (ph != PH_LEVEL && ph != PH_UPD && ph != PH_RELAX && ph != PH_PLASTIC) continue;
        const BDesc& d = D[tl.x];
        const int ne = d.m.c3 + d.m.c4 + d.m.c8;
        const int g0 = tl.y * tl.z, g1 = min(g0 + tl.z, d.n_groups);
        if (ph == PH_LEVEL) {
            // k_set_level, the Aitken history reset and the level predictor
            // (k_predict) of cp_solve
            const double lam = (double)S->level / d.levels;
            const int lev = S->level;
            const bool rec = d.predict && lev >= 2, extra = d.predict && lev >= 3;
            const int s1 = min(g0 + tl.z, d.n_slices);
            for (int sl = g0 + w; sl < s1; sl += kWarps) {
                const int n = 32 * sl + lane;
                if (n < d.m.n_nodes) {
                    const double2 bf = d.b_full[n];
                    d.b[n] = make_double2(lam * bf.x, lam * bf.y);
                    const uchar2 m = d.mask[n];
                    double2 uu = d.x[n];
                    if (rec) {
                        const double2 cur = uu;
                        if (extra) {
                            const double2 pv = d.pred_u[n];
                            if (m.x) uu.x = 2.0 * cur.x - pv.x;
                            if (m.y) uu.y = 2.0 * cur.y - pv.y;
                        }
                        d.pred_u[n] = cur;
                    }
                    const double2 uf = d.u_full[n];
                    if (!m.x) uu.x = lam * uf.x;
                    if (!m.y) uu.y = lam * uf.y;
                    d.x[n] = uu;
                }
            }
            for (int g = g0 + w; g < g1; g += kWarps) {
                const int e = 32 * g + lane;
                if (e < ne) {
                    d.st.res_prev[e] = 0.0;
                    d.st.res_cur[e] = 0.0;
                    if (rec) {
                        const double cur = d.st.psi[e];
                        if (extra) {
                            double v = 2.0 * cur - d.pred_psi[e];
                            if (!(v >= 1.0)) v = 1.0;
                            d.st.psi[e] = v;
                            d.st.E_c[e] = d.mat.E / v;
                            d.st.nu_c[e] = 0.5 * (1. - (1. - 2. * d.mat.nu) / v);
                        }
                        d.pred_psi[e] = cur;
                    }
                }
            }
            if (arrive(S, tl.w, &shf) && threadIdx.x == 0) {
                S->ticket = 0;
                if (S->t_first == 0) S->t_first = global_ns();
                S->outer_it = 0;
                S->rel_err = 1.0;
                S->w_prev = 1.0;
                S->eps = next_eps(d, 1.0);
                set_phase(S, c, PH_ASM);
            }
        } else if (ph == PH_UPD) {
            for (int g = g0 + w; g < g1; g += kWarps) {
                const int e = 32 * g + lane;
                double s_num = 0.0, s_den = 0.0, s_an = 0.0, s_ad = 0.0;
                if (e < ne) update_element<Q8>(d.m, d.mat, d.x, d.st, e, d.aitken, s_num, s_den, s_an, s_ad);
                s_num = warp_sum(s_num);
                s_den = warp_sum(s_den);
                s_an = warp_sum(s_an);
                s_ad = warp_sum(s_ad);
                if (lane == 0) {
                    double* p = d.part + kPart * (size_t)g;
                    p[0] = s_num; p[1] = s_den; p[2] = s_an; p[3] = s_ad;
                }
            }
            if (arrive(S, tl.w, &shf)) {
                double r[4];
                reduce_parts<4>(d.part, d.n_groups, r, sh);
                if (threadIdx.x == 0) {
                    S->ticket = 0;
                    const double rel = sqrt(r[0] / r[1]);
                    S->rel_err = rel;
                    S->outer_it += 1;
                    S->outer_total += 1;
                    S->lin_iters = 0;
                    if (!isfinite(rel)) {
                        finish(S, c, CP_ERR_BREAKDOWN);
                    } else if (d.aitken) {
                        double om = 1.0;
                        if (S->outer_it > 1 && r[3] > 0) om = -S->w_prev * r[2] / r[3];
                        if (!(om >= 0.1)) om = 0.1;
                        if (om > 10.0) om = 10.0;
                        S->omega = om;
                        S->w_prev = om;
                        set_phase(S, c, PH_RELAX);
                    } else {
                        decide(d, S, c);
                    }
                }
            }
        } else if (ph == PH_RELAX) {
            const double om = S->omega;
            for (int g = g0 + w; g < g1; g += kWarps) {
                const int e = 32 * g + lane;
                if (e < ne) relax_element(d.mat, d.st, e, om);
            }
            if (arrive(S, tl.w, &shf) && threadIdx.x == 0) {
                S->ticket = 0;
                decide(d, S, c);
            }
        } else {  // PH_PLASTIC
            for (int g = g0 + w; g < g1; g += kWarps) {
                const int e = 32 * g + lane;
                if (e < ne) plastic_element(d.mat, d.st, e);
            }
            if (arrive(S, tl.w, &shf) && threadIdx.x == 0) {
                S->ticket = 0;
                finish(S, c, 0);
            }
        }
    }
}

__device__ __forceinline__ bool trip_condition(BCtl* c) {
    c->trips += 1;
    bool go = c->active > 0 && (c->max_trips <= 0 || c->trips < c->max_trips) &&
              !(c->exit_on_done > 0 && c->done >= c->exit_on_done);
    if (go && c->stop && *c->stop) go = false;
    c->go = go ? 1 : 0;
    return go;
}

__global__ void k_batch_cond(BCtl* c, cudaGraphConditionalHandle h) {
    cudaGraphSetConditional(h, trip_condition(c) ? 1u : 0u);
}

// The same condition for runs launched kernel by kernel (profilers cannot
// see kernel nodes of a graph with a conditional node).
__global__ void k_batch_cond_direct(BCtl* c) { trip_condition(c); }

// The batched CG kernel's ITER gather form: CUPLAST_BATCH_CHUNK = 3 (blocks
// 3 at a time: the default, 5 % faster per trip of 512 instances than one
// unrolled loop), 0 (one unrolled loop) or 5, for measurements.
using BatchCgKernel = void (*)(const BDesc*, BState*, const int4*, BCtl*);
BatchCgKernel batch_cg_kernel() {
    static const BatchCgKernel k = [] {
        const char* e = std::getenv("CUPLAST_BATCH_CHUNK");
        switch (e ? std::atoi(e) : 3) {
        case 0: return (BatchCgKernel)k_batch_cg<0>;
        case 5: return (BatchCgKernel)k_batch_cg<5>;
        default: return stream_loads() ? (BatchCgKernel)k_batch_cg<3, true> : (BatchCgKernel)k_batch_cg<3>;
        }
    }();
    return k;
}

int bucket_of(int n_slices) {
    int b = 0;
    while ((2 << b) <= n_slices && b + 1 < kBuckets) ++b;
    return b;
}

}  // namespace
}  // namespace cp

using namespace cp;

struct cp_batch {
    cp_context* ctx = nullptr;
    cp_batch_opts o{};
    int cap = 0;
    std::vector<cp_instance*> inst;      // per slot (nullptr: free)
    std::vector<BDesc> desc;             // host copies
    std::vector<BState> state;           // host copies, refreshed after each run
    std::vector<int> listed;             // slots in the batch, in admission order
    int tile_slices[kBuckets];
    BDesc* d_desc = nullptr;
    BState* d_state = nullptr;
    int4* d_tiles = nullptr;
    BCtl* d_ctl = nullptr;
    int tiles_cap = 0;
    int4* h_tiles = nullptr;  // pinned
    BState* h_state = nullptr;  // pinned
    BCtl* h_ctl = nullptr;  // pinned
    int* h_stop = nullptr;  // host-mapped
    int* d_stop = nullptr;
    cudaGraphExec_t graph = nullptr;
    int grid_cg = 0, grid_elem = 0, grid_asm = 0;
    float2* d_sink = nullptr;           // autotuner probe output
    unsigned int* d_ptickets = nullptr;  // autotuner probe tickets (one per slot)
    double* d_psums = nullptr;           // autotuner probe sums (one per block)
    size_t asm_smem = 0;
    bool running = false;
    bool use_graph = true;
    bool q8 = false;  // an 8-node instance joined: element kernels with the 8-node element  // false (CUPLAST_NO_GRAPH=1): trips launched kernel by kernel, for profilers
    int last_tiles = 0;
    long long trips = 0, launches = 0, runs = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // bracket each run on the batch's stream
    bool timed = false;
    double last_run_ms = 0.0;
};

namespace {

int bfail(cp_batch* b, const Error& e) {
    if (b && b->ctx) b->ctx->last_error = e.msg;
    return e.status;
}

template <typename F>
int bguard(cp_batch* b, F&& f) {
    try {
        f();
        return CP_OK;
    } catch (const Error& e) {
        return bfail(b, e);
    } catch (const std::bad_alloc&) {
        return bfail(b, Error{CP_ERR_NOMEM, "host allocation failed"});
    }
}

int default_tile(int bucket) {
    // 4 slices (one per warp) for small instances, up to 16 for large ones
    return bucket < 6 ? 4 : (bucket < 9 ? 8 : 16);
}

void ensure_tiles(cp_batch* b, int need) {
    if (need <= b->tiles_cap) return;
    int nc = std::max(need, 2 * b->tiles_cap);
    if (b->d_tiles) CP_CUDA(cudaFree(b->d_tiles));
    if (b->h_tiles) CP_CUDA(cudaFreeHost(b->h_tiles));
    b->d_tiles = nullptr;
    b->h_tiles = nullptr;
    CP_CUDA(cudaMalloc(&b->d_tiles, sizeof(int4) * (size_t)nc));
    CP_CUDA(cudaMallocHost(&b->h_tiles, sizeof(int4) * (size_t)nc));
    b->tiles_cap = nc;
    // the graph holds the work-list pointer: rebuild it
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
}

int tiles_of(const BDesc& d, int S) {
    const int a = (d.n_slices + S - 1) / S, g = (d.n_groups + S - 1) / S;
    return std::max(a, g);
}

// Work list of the listed, unfinished instances; returns the tile count.
// Tile sizes come from the table of the instance's size bucket; with
// `shrink`, when the active instances hold too few slices to give every
// block of the persistent grid a tile, tiles shrink (down to one slice per
// warp) so that the remaining work still spreads over the whole GPU.
int build_tiles(cp_batch* b, const std::vector<int>& slots, bool only_active, const int* S_override, bool shrink) {
    long long slices = 0;
    for (int sl : slots)
        if (!(only_active && b->state[sl].phase == PH_DONE)) slices += b->desc[sl].n_slices;
    int cap = 1 << 30;
    if (shrink && !S_override) {
        cap = kWarps;
        while ((long long)cap * 2 * b->grid_cg <= slices && cap < 64) cap *= 2;
    }
    auto S_of = [&](int sl) {
        if (S_override) return *S_override;
        return std::min(b->tile_slices[bucket_of(b->desc[sl].n_slices)], cap);
    };
    int total = 0;
    for (int sl : slots) {
        if (only_active && b->state[sl].phase == PH_DONE) continue;
        total += tiles_of(b->desc[sl], S_of(sl));
    }
    ensure_tiles(b, std::max(total, 1));
    int k = 0;
    for (int sl : slots) {
        if (only_active && b->state[sl].phase == PH_DONE) continue;
        const int S = S_of(sl);
        const int nt = tiles_of(b->desc[sl], S);
        for (int t = 0; t < nt; ++t) b->h_tiles[k++] = make_int4(sl, t, S, nt);
    }
    return k;
}

// Round-robin order across instances, so that the persistent grid's blocks
// take tiles of many instances at once (the last tile of a large instance is
// not left to run alone).
void interleave_tiles(cp_batch* b, int n) {
    std::vector<int4> out;
    out.reserve(n);
    std::vector<std::pair<int, int>> ranges;  // [begin, end) per instance
    int i = 0;
    while (i < n) {
        int j = i;
        while (j < n && b->h_tiles[j].x == b->h_tiles[i].x) ++j;
        ranges.push_back({i, j});
        i = j;
    }
    bool more = true;
    for (int r = 0; more; ++r) {
        more = false;
        for (auto& rg : ranges)
            if (rg.first + r < rg.second) {
                out.push_back(b->h_tiles[rg.first + r]);
                more = true;
            }
    }
    std::memcpy(b->h_tiles, out.data(), sizeof(int4) * (size_t)n);
}

// Grids of the element and assembly kernels: as many blocks as fit on the
// GPU. Q8 selects the instantiations with the 8-node element, used from the
// first 8-node instance on (they need more registers).
template <bool Q8>
void element_grids(cp_batch* b) {
    int per_sm = 0;
    CP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_elem<Q8>, kThreads, 0));
    b->grid_elem = b->ctx->sm_count * std::max(1, std::min(per_sm, 8));
    CP_CUDA(cudaFuncSetAttribute(k_batch_asm<Q8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->asm_smem));
    CP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_asm<Q8>, kThreads, b->asm_smem));
    b->grid_asm = b->ctx->sm_count * std::max(1, per_sm);
}

// One trip: element phases, assembly, CG launches.
void launch_body(cp_batch* b, cudaStream_t s) {
    for (int k = 0; k < b->o.elem_per_trip; ++k) {
        if (b->q8) k_batch_elem<true><<<b->grid_elem, kThreads, 0, s>>>(b->d_desc, b->d_state, b->d_tiles, b->d_ctl);
        else k_batch_elem<false><<<b->grid_elem, kThreads, 0, s>>>(b->d_desc, b->d_state, b->d_tiles, b->d_ctl);
    }
    if (b->q8)
        k_batch_asm<true><<<b->grid_asm, kThreads, b->asm_smem, s>>>(b->d_desc, b->d_state, b->d_tiles, b->d_ctl,
                                                                     b->o.max_width);
    else
        k_batch_asm<false><<<b->grid_asm, kThreads, b->asm_smem, s>>>(b->d_desc, b->d_state, b->d_tiles, b->d_ctl,
                                                                      b->o.max_width);
    for (int k = 0; k < b->o.cg_per_trip; ++k)
        batch_cg_kernel()<<<b->grid_cg, kThreads, 0, s>>>(b->d_desc, b->d_state, b->d_tiles, b->d_ctl);
}

// Direct launches: trip after trip with the condition read back each time.
void run_direct(cp_batch* b) {
    cudaStream_t s = b->ctx->stream;
    for (;;) {
        launch_body(b, s);
        k_batch_cond_direct<<<1, 1, 0, s>>>(b->d_ctl);
        CP_CUDA(cudaGetLastError());
        int go = 0;
        CP_CUDA(cudaMemcpyAsync(&go, &b->d_ctl->go, sizeof(int), cudaMemcpyDeviceToHost, s));
        CP_CUDA(cudaStreamSynchronize(s));
        if (!go) return;
    }
}

void build_graph(cp_batch* b) {
    cudaStream_t s = b->ctx->stream;
    cudaGraph_t g;
    CP_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    CP_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    CP_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &p));
    cudaGraph_t body = p.conditional.phGraph_out[0];
    CP_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    launch_body(b, s);
    k_batch_cond<<<1, 1, 0, s>>>(b->d_ctl, h);
    cudaGraph_t captured = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &captured);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        CP_CUDA(e);
    }
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    CP_CUDA(e);
}

cp_solve_report report_of(const BState& S) {
    cp_solve_report r{};
    r.status = S.status;
    r.outer_iters = S.outer_total;
    r.cg_iters = S.cg_total;
    r.fp64_spmv = S.fp64_spmv;
    r.rel_err = S.rel_err;
    r.cg_rel_res = S.cg_rel_res;
    r.levels_done = S.levels_done;
    r.seconds = (S.t_done > S.t_first && S.t_first) ? (double)(S.t_done - S.t_first) * 1e-9 : 0.0;
    r.kernel_launches = 0;
    return r;
}

}  // namespace

extern "C" {

CP_API void cp_batch_opts_default(cp_batch_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->max_instances = 1024;
    o->cg_per_trip = 16;
    o->elem_per_trip = 3;
    o->max_width = 16;
    o->cg_blocks_per_sm = 0;
}

CP_API int cp_batch_create(cp_context* ctx, const cp_batch_opts* opts, cp_batch** out) {
    if (!ctx || !out) return CP_ERR_INVALID;
    *out = nullptr;
    cp_batch_opts o;
    cp_batch_opts_default(&o);
    if (opts) o = *opts;
    if (o.max_instances <= 0 || o.max_instances > (1 << 20) || o.cg_per_trip <= 0 || o.elem_per_trip < 3 ||
        o.max_width < 1 || o.max_width > 48 || o.cg_blocks_per_sm < 0 || o.cg_blocks_per_sm > 16)
        return CP_ERR_INVALID;
    cp_batch* b = new (std::nothrow) cp_batch();
    if (!b) return CP_ERR_NOMEM;
    b->ctx = ctx;
    b->o = o;
    b->cap = o.max_instances;
    if (const char* g = std::getenv("CUPLAST_NO_GRAPH")) b->use_graph = !(g[0] == '1');
    for (int k = 0; k < kBuckets; ++k) b->tile_slices[k] = default_tile(k);
    int rc = bguard(b, [&] {
        CP_CUDA(cudaSetDevice(ctx->device));
        b->inst.assign(b->cap, nullptr);
        b->desc.assign(b->cap, BDesc{});
        b->state.assign(b->cap, BState{});
        CP_CUDA(cudaMalloc(&b->d_desc, sizeof(BDesc) * (size_t)b->cap));
        CP_CUDA(cudaMalloc(&b->d_state, sizeof(BState) * (size_t)b->cap));
        CP_CUDA(cudaMemset(b->d_state, 0, sizeof(BState) * (size_t)b->cap));
        CP_CUDA(cudaMalloc(&b->d_ctl, sizeof(BCtl)));
        CP_CUDA(cudaMemset(b->d_ctl, 0, sizeof(BCtl)));
        CP_CUDA(cudaMallocHost(&b->h_state, sizeof(BState) * (size_t)b->cap));
        CP_CUDA(cudaMallocHost(&b->h_ctl, sizeof(BCtl)));
        CP_CUDA(cudaHostAlloc(&b->h_stop, 64, cudaHostAllocMapped));
        *b->h_stop = 0;
        CP_CUDA(cudaHostGetDevicePointer((void**)&b->d_stop, b->h_stop, 0));
        ensure_tiles(b, 1024);
        int per_sm = 0;
        CP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_cg_kernel(), kThreads, 0));
        if (o.cg_blocks_per_sm > 0) per_sm = std::min(per_sm, o.cg_blocks_per_sm);
        b->grid_cg = ctx->sm_count * std::max(1, per_sm);
        b->asm_smem = (size_t)kWarps * 128 * o.max_width * sizeof(double);
        element_grids<false>(b);
        CP_CUDA(cudaEventCreate(&b->ev0));
        CP_CUDA(cudaEventCreate(&b->ev1));
        CP_CUDA(cudaMalloc(&b->d_sink, sizeof(float2) * (size_t)b->grid_cg * kThreads));
        CP_CUDA(cudaMalloc(&b->d_ptickets, sizeof(unsigned int) * (size_t)b->cap));
        CP_CUDA(cudaMemset(b->d_ptickets, 0, sizeof(unsigned int) * (size_t)b->cap));
        CP_CUDA(cudaMalloc(&b->d_psums, sizeof(double) * (size_t)b->grid_cg));
    });
    if (rc != CP_OK) {
        cp_batch_destroy(b);
        return rc;
    }
    *out = b;
    return CP_OK;
}

CP_API int cp_batch_destroy(cp_batch* b) {
    if (!b) return CP_ERR_INVALID;
    if (b->ctx) {
        cudaSetDevice(b->ctx->device);
        cudaStreamSynchronize(b->ctx->stream);
    }
    for (int sl : b->listed)
        if (b->inst[sl]) b->inst[sl]->in_batch = false;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->d_desc) cudaFree(b->d_desc);
    if (b->d_state) cudaFree(b->d_state);
    if (b->d_tiles) cudaFree(b->d_tiles);
    if (b->d_ctl) cudaFree(b->d_ctl);
    if (b->h_tiles) cudaFreeHost(b->h_tiles);
    if (b->h_state) cudaFreeHost(b->h_state);
    if (b->h_ctl) cudaFreeHost(b->h_ctl);
    if (b->h_stop) cudaFreeHost(b->h_stop);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->d_sink) cudaFree(b->d_sink);
    if (b->d_ptickets) cudaFree(b->d_ptickets);
    if (b->d_psums) cudaFree(b->d_psums);
    delete b;
    return CP_OK;
}

CP_API int cp_batch_add(cp_batch* b, cp_instance* I, const cp_solve_opts* opts, int* slot) {
    if (!b || !I || !opts) return CP_ERR_INVALID;
    if (b->running) return CP_ERR_BUSY;
    if (I->in_batch) return CP_ERR_BUSY;
    const cp_solve_opts o = *opts;
    if (o.precision != CP_PREC_MIXED) return CP_ERR_UNSUPPORTED;
    if (!(o.cg_tol > 0) || !(o.outer_tol > 0) || !(o.inner_tol > 0 && o.inner_tol < 1) || o.max_outer <= 0 ||
        o.levels <= 0 || o.max_cg <= 0 || (o.precond & ~1) || o.adaptive_cg < 0 || o.adaptive_cg > 2 ||
        (o.predict & ~1))
        return CP_ERR_INVALID;
    return bguard(b, [&] {
        CP_CHECK(I->loads_set, CP_ERR_INVALID, "loads not set");
        CP_CHECK(I->ctx && I->ctx->device == b->ctx->device, CP_ERR_INVALID, "instance on another device");
        CP_CHECK(I->csr.max_width <= b->o.max_width, CP_ERR_UNSUPPORTED,
                 "node degree above the batch's assembly width (cp_batch_opts.max_width)");
        int sl = -1;
        for (int k = 0; k < b->cap; ++k)
            if (!b->inst[k]) {
                sl = k;
                break;
            }
        CP_CHECK(sl >= 0, CP_ERR_BUSY, "no free batch slot");
        CP_CUDA(cudaSetDevice(b->ctx->device));
        if (I->mesh.c8 && !b->q8) {
            // the first 8-node instance: switch to the kernels that have the
            // 8-node element, and capture the trip again with them
            b->q8 = true;
            element_grids<true>(b);
            if (b->graph) {
                cudaGraphExecDestroy(b->graph);
                b->graph = nullptr;
            }
        }
        instance_prepare_mixed(I, o.precond);
        BDesc d{};
        d.m = I->mesh;
        d.n_slices = I->csr.n_slices;
        d.n_groups = (I->n_elem + 31) / 32;
        d.slice_ptr = I->csr.slice_ptr;
        d.scol = I->csr.scol;
        d.inc_pos = I->csr.inc_pos;
        d.inc = I->csr.inc;
        d.inc_k = I->csr.inc_k;
        d.inc_k8 = I->csr.inc_k8;
        d.val64 = I->csr.val64;
        d.val32 = I->csr.val32;
        d.x = I->u;
        d.b = I->b;
        d.b_full = I->b_full;
        d.u_full = I->u_full;
        d.mask = I->mask;
        {
            // the batch's own vectors, allocated once per instance (an
            // instance may be added again after it was harvested)
            const size_t nn = (size_t)I->n_nodes;
            if (!I->bt_vec) {
                I->bt_vec = I->alloc<float2>(4 * nn);
                I->bt_rec = I->alloc<float4>(4 * nn);
                I->bt_part = I->alloc<double>(kPart * (size_t)std::max(d.n_slices, d.n_groups));
            }
            float2* v = I->bt_vec;
            float4* g = I->bt_rec;
            CP_CUDA(cudaMemsetAsync(v, 0, sizeof(float2) * 4 * nn, I->s()));
            CP_CUDA(cudaMemsetAsync(g, 0, sizeof(float4) * 4 * nn, I->s()));
            d.r = v; d.w = v + nn; d.kp = v + 2 * nn; d.p = v + 3 * nn;
            d.gA = g; d.gB = g + 2 * nn;
        }
        d.minv = I->minv32;
        d.st = I->st;
        d.mat = I->mat;
        d.part = I->bt_part;
        d.cg_tol = o.cg_tol;
        d.outer_tol = o.outer_tol;
        d.inner_tol = o.inner_tol;
        d.max_cg = o.max_cg;
        d.max_outer = o.max_outer;
        d.levels = o.levels;
        d.aitken = o.aitken ? 1 : 0;
        d.adaptive = o.adaptive_cg;
        d.predict = o.predict ? 1 : 0;
        if (d.predict) {
            if (!I->pred_u) {
                I->pred_u = I->alloc<double2>(I->n_nodes);
                I->pred_psi = I->alloc<double>(I->n_elem);
            }
            d.pred_u = I->pred_u;
            d.pred_psi = I->pred_psi;
        }
        d.precond = o.precond;
        CP_CUDA(cudaStreamSynchronize(I->s()));  // buffers of the instance's own stream are ready
        BState S{};
        S.phase = PH_LEVEL;
        S.level = 1;
        S.rel_err = 1.0;
        S.w_prev = 1.0;
        b->desc[sl] = d;
        b->state[sl] = S;
        CP_CUDA(cudaMemcpyAsync(b->d_desc + sl, &b->desc[sl], sizeof(BDesc), cudaMemcpyHostToDevice, b->ctx->stream));
        CP_CUDA(cudaMemcpyAsync(b->d_state + sl, &b->state[sl], sizeof(BState), cudaMemcpyHostToDevice,
                                b->ctx->stream));
        CP_CUDA(cudaStreamSynchronize(b->ctx->stream));
        b->inst[sl] = I;
        I->in_batch = true;
        b->listed.push_back(sl);
        if (slot) *slot = sl;
    });
}

CP_API int cp_batch_launch(cp_batch* b, int until, long long max_trips) {
    if (!b || (until != CP_BATCH_RUN_ALL && until != CP_BATCH_RUN_ANY_DONE)) return CP_ERR_INVALID;
    if (b->running) return CP_ERR_BUSY;
    return bguard(b, [&] {
        cudaStream_t s = b->ctx->stream;
        CP_CUDA(cudaSetDevice(b->ctx->device));
        const int nt = build_tiles(b, b->listed, true, nullptr, true);
        interleave_tiles(b, nt);
        if (b->use_graph && !b->graph) build_graph(b);
        BCtl c{};
        c.n_tiles = nt;
        int active = 0, done = 0;
        for (int sl : b->listed) {
            const int ph = b->state[sl].phase;
            c.pop[ph] += 1;
            if (ph == PH_DONE) ++done;
            else ++active;
        }
        c.active = active;
        c.done = 0;
        c.exit_on_done = until == CP_BATCH_RUN_ANY_DONE ? 1 : 0;
        c.trips = 0;
        c.max_trips = max_trips;
        c.stop = b->d_stop;
        *b->h_ctl = c;
        *(volatile int*)b->h_stop = 0;
        if (nt > 0) CP_CUDA(cudaMemcpyAsync(b->d_tiles, b->h_tiles, sizeof(int4) * (size_t)nt, cudaMemcpyHostToDevice, s));
        CP_CUDA(cudaMemcpyAsync(b->d_ctl, b->h_ctl, sizeof(BCtl), cudaMemcpyHostToDevice, s));
        b->last_tiles = nt;
        b->timed = false;
        if (active > 0) {
            CP_CUDA(cudaEventRecord(b->ev0, s));
            if (b->use_graph) CP_CUDA(cudaGraphLaunch(b->graph, s));
            else run_direct(b);
            CP_CUDA(cudaEventRecord(b->ev1, s));
            b->timed = true;
            b->runs += 1;
        }
        CP_CUDA(cudaMemcpyAsync(b->h_ctl, b->d_ctl, sizeof(BCtl), cudaMemcpyDeviceToHost, s));
        // states of the listed slots (contiguous copy of the slot range in use)
        int lo = b->cap, hi = -1;
        for (int sl : b->listed) {
            lo = std::min(lo, sl);
            hi = std::max(hi, sl);
        }
        if (hi >= lo)
            CP_CUDA(cudaMemcpyAsync(b->h_state + lo, b->d_state + lo, sizeof(BState) * (size_t)(hi - lo + 1),
                                    cudaMemcpyDeviceToHost, s));
        b->running = true;
    });
}

CP_API int cp_batch_interrupt(cp_batch* b) {
    if (!b || !b->h_stop) return CP_ERR_INVALID;
    *(volatile int*)b->h_stop = 1;
    return CP_OK;
}

CP_API int cp_batch_wait(cp_batch* b, int* active, int* done) {
    if (!b) return CP_ERR_INVALID;
    if (!b->running) {
        int a = 0, d = 0;
        for (int sl : b->listed) (b->state[sl].phase == PH_DONE ? d : a) += 1;
        if (active) *active = a;
        if (done) *done = d;
        return CP_OK;
    }
    return bguard(b, [&] {
        b->running = false;
        CP_CUDA(cudaStreamSynchronize(b->ctx->stream));
        float ms = 0.f;
        if (b->timed) CP_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
        b->last_run_ms = ms;
        const long long trips = b->h_ctl->trips;
        b->trips += trips;
        b->launches += trips * (long long)(b->o.elem_per_trip + 1 + b->o.cg_per_trip + 1);
        int a = 0, d = 0;
        for (int sl : b->listed) {
            b->state[sl] = b->h_state[sl];
            (b->state[sl].phase == PH_DONE ? d : a) += 1;
        }
        if (active) *active = a;
        if (done) *done = d;
    });
}

CP_API int cp_batch_run(cp_batch* b, int until, long long max_trips, int* active, int* done) {
    int rc = cp_batch_launch(b, until, max_trips);
    if (rc != CP_OK) return rc;
    return cp_batch_wait(b, active, done);
}

CP_API int cp_batch_harvest(cp_batch* b, int cap, int* slots, cp_instance** insts, cp_solve_report* reports,
                            int* count) {
    if (!b || cap < 0 || !count) return CP_ERR_INVALID;
    if (b->running) return CP_ERR_BUSY;
    int k = 0;
    std::vector<int> keep;
    for (int sl : b->listed) {
        if (b->state[sl].phase == PH_DONE && k < cap) {
            if (slots) slots[k] = sl;
            if (insts) insts[k] = b->inst[sl];
            if (reports) reports[k] = report_of(b->state[sl]);
            b->inst[sl]->in_batch = false;
            b->inst[sl] = nullptr;
            b->state[sl] = BState{};
            ++k;
        } else {
            keep.push_back(sl);
        }
    }
    b->listed.swap(keep);
    *count = k;
    return CP_OK;
}

CP_API int cp_batch_set_tile(cp_batch* b, int bucket, int slices) {
    if (!b || bucket < 0 || bucket >= kBuckets || slices < 1 || slices > 1024) return CP_ERR_INVALID;
    b->tile_slices[bucket] = slices;
    return CP_OK;
}

CP_API int cp_batch_get_tile(const cp_batch* b, int bucket, int* slices) {
    if (!b || bucket < 0 || bucket >= kBuckets || !slices) return CP_ERR_INVALID;
    *slices = b->tile_slices[bucket];
    return CP_OK;
}

CP_API int cp_batch_autotune(cp_batch* b, double* ms_per_sweep) {
    if (!b) return CP_ERR_INVALID;
    if (b->running) return CP_ERR_BUSY;
    return bguard(b, [&] {
        cudaStream_t s = b->ctx->stream;
        CP_CUDA(cudaSetDevice(b->ctx->device));
        cudaEvent_t e0, e1;
        CP_CUDA(cudaEventCreate(&e0));
        CP_CUDA(cudaEventCreate(&e1));
        std::vector<int> active;
        for (int sl : b->listed)
            if (b->state[sl].phase != PH_DONE) active.push_back(sl);
        // one sweep of the probe over every active instance with the current table
        auto sweep = [&]() {
            const int nt = build_tiles(b, active, true, nullptr, false);
            interleave_tiles(b, nt);
            CP_CUDA(cudaMemcpyAsync(b->d_tiles, b->h_tiles, sizeof(int4) * (size_t)nt, cudaMemcpyHostToDevice, s));
            k_batch_probe<<<b->grid_cg, kThreads, 0, s>>>(b->d_desc, b->d_state, b->d_tiles, nt, 0.5f, 0.5f, b->d_sink,
                                                         b->d_ptickets, b->d_psums);  // warm
            const int reps = 3;
            CP_CUDA(cudaEventRecord(e0, s));
            for (int r = 0; r < reps; ++r)
                k_batch_probe<<<b->grid_cg, kThreads, 0, s>>>(b->d_desc, b->d_state, b->d_tiles, nt, 0.5f, 0.5f,
                                                             b->d_sink, b->d_ptickets, b->d_psums);
            CP_CUDA(cudaEventRecord(e1, s));
            CP_CUDA(cudaEventSynchronize(e1));
            CP_CUDA(cudaGetLastError());
            float ms = 0;
            CP_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            return (double)ms / reps;
        };
        bool present[kBuckets] = {};
        for (int sl : active) present[bucket_of(b->desc[sl].n_slices)] = true;
        // coordinate descent: one bucket at a time against the whole set,
        // largest buckets first (they carry most of the work)
        const int cands[] = {4, 8, 16, 32, 64};
        double best = active.empty() ? 0.0 : sweep();
        for (int pass = 0; pass < 2 && !active.empty(); ++pass)
            for (int bk = kBuckets - 1; bk >= 0; --bk) {
                if (!present[bk]) continue;
                const int keep = b->tile_slices[bk];
                int best_S = keep;
                for (int S : cands) {
                    if (S == keep) continue;
                    b->tile_slices[bk] = S;
                    const double t = sweep();
                    if (t < best) {
                        best = t;
                        best_S = S;
                    }
                }
                b->tile_slices[bk] = best_S;
            }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (ms_per_sweep) *ms_per_sweep = best;
    });
}

CP_API int cp_batch_progress(const cp_batch* b, int slot, int* phase, int* level, cp_solve_report* report) {
    if (!b || slot < 0 || slot >= b->cap || !b->inst[slot]) return CP_ERR_INVALID;
    if (b->running) return CP_ERR_BUSY;
    const BState& S = b->state[slot];
    if (phase) *phase = S.phase;
    if (level) *level = S.level;
    if (report) *report = report_of(S);
    return CP_OK;
}

CP_API int cp_batch_last_run_ms(const cp_batch* b, double* ms) {
    if (!b || !ms) return CP_ERR_INVALID;
    if (b->running) return CP_ERR_BUSY;
    *ms = b->last_run_ms;
    return CP_OK;
}

CP_API int cp_batch_stats(const cp_batch* b, long long* trips, long long* launches, long long* runs) {
    if (!b) return CP_ERR_INVALID;
    if (trips) *trips = b->trips;
    if (launches) *launches = b->launches;
    if (runs) *runs = b->runs;
    return CP_OK;
}

}  // extern "C"
