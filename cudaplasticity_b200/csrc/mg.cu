// Aggregation-multigrid preconditioned FP64 CG (see mg.h).
//
// No counterpart in the reference, whose linear solver is CG on the
// unmodified K with the Dirichlet DOFs masked (ConjGradSolver::solve,
// src/ConjGradSolver.h:52-101; ConjGradCuda::solve, src/ConjGradCuda.cu:185-231).
// The preconditioner changes the iterates, not the system: the linear solve
// stops on the same criterion ||r|| / ||b|| <= eps, with r = m.(b - K x) the
// masked residual of the same K.
//
// PCG (Hestenes-Stiefel) with z = M r one V-cycle:
//   P : p = z + beta p (own node; the neighbours' p gathered the same way),
//       q = K p, (p, q) -> alpha
//   U : x += alpha p, r -= m.alpha q, (r, r) -> converged?; pre-smoothing of
//       level 0 from zero: y0 = w0 D0^-1 r
//   R0: one block per level-0 node range: residuals r - K y0 restricted by
//       T0^T into each level-1 node; pre-smoothing y1 = w1 D1^-1 b1
//   R_l (l >= 1): the same one level down, on the 3x3 block CSR
//   C : coarsest correction e = A_c^-1 b_c (dense inverse)
//   S_l (l >= 1): prolongation fused into the post-smoothing sweep:
//       y' = y + T e, z = y' + w D^-1 (b - A y'), A y' gathered from the
//       neighbours' y and their aggregates' e
//   S0: the same on level 0; (r, z) -> rho, beta
// When level 1 is small, R_1 .. S_1 run in one block (k_mg_coarse_cycle), so
// an iteration is five kernels: P, U, R0, the coarse cycle, S0.
// Every kernel returns at once when the solve has converged or failed, so a
// graph body of several iterations stops doing work after convergence. Each
// value is produced by one thread in a fixed order and every cross-block sum
// is reduced by the last block in index order: the solve is deterministic.
#include <algorithm>
#include <cstdlib>
#include <vector>

#include "amg.h"
#include "common.cuh"
#include "instance.h"
#include "internal.h"
#include "mg.h"

namespace cp {

namespace {

constexpr int kThreads = 256;  // level-0 kernels (grid-stride, partial sums)
constexpr int kSmall = 128;    // coarse-level kernels (one thread per node or block)

__device__ __forceinline__ double4 ld_block(const double* __restrict__ val, long long b) {
    const double2* p = reinterpret_cast<const double2*>(val + 4 * b);
    const double2 lo = __ldg(p), hi = __ldg(p + 1);
    return make_double4(lo.x, lo.y, hi.x, hi.y);
}

// (K v)_i over node i's row of the sliced layout (padding blocks are zero).
__device__ __forceinline__ double2 k_row(const MgArgs& a, int i, const double2* __restrict__ v) {
    const int sl = i >> 5, lane = i & 31;
    const int base = a.slice_ptr[sl], w = (a.slice_ptr[sl + 1] - base) >> 5;
    double k0 = 0.0, k1 = 0.0;
    for (int k = 0; k < w; ++k) {
        const long long bi = base + 32LL * k + lane;
        const int c = __ldg(a.scol + bi);
        const double4 kv = ld_block(a.val, bi);
        const double2 vc = v[c];
        k0 += kv.x * vc.x + kv.y * vc.y;
        k1 += kv.z * vc.x + kv.w * vc.y;
    }
    return make_double2(k0, k1);
}

__device__ __forceinline__ double damping(const double* lam, int l, double omega) {
    const double b = lam[l];
    return b > 0.0 ? omega / b : 0.0;
}

// Largest value over the grid: warp maximum, then one atomic per warp on the
// bit pattern (non-negative doubles order like their bits). Called by every
// thread of the block.
__device__ __forceinline__ void max_to(double* dst, double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0 && v > 0.0)
        atomicMax(reinterpret_cast<unsigned long long*>(dst), (unsigned long long)__double_as_longlong(v));
}

// Inverse of a 3x3 block on the indices whose diagonal is nonzero; rows and
// columns of the others (prolongator columns that were dropped, which leave
// exact zero rows and columns) are zero.
__device__ __forceinline__ void inv3_masked(const double* __restrict__ d, double* o) {
    const bool on0 = d[0] != 0.0, on1 = d[4] != 0.0, on2 = d[8] != 0.0;
    const bool on[3] = {on0, on1, on2};
    double m[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) m[3 * r + c] = (on[r] && on[c]) ? d[3 * r + c] : (r == c ? 1.0 : 0.0);
    const double c00 = m[4] * m[8] - m[5] * m[7], c01 = m[5] * m[6] - m[3] * m[8], c02 = m[3] * m[7] - m[4] * m[6];
    const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
    const double id = det != 0.0 ? 1.0 / det : 0.0;
    o[0] = c00 * id;
    o[1] = (m[2] * m[7] - m[1] * m[8]) * id;
    o[2] = (m[1] * m[5] - m[2] * m[4]) * id;
    o[3] = c01 * id;
    o[4] = (m[0] * m[8] - m[2] * m[6]) * id;
    o[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    o[6] = c02 * id;
    o[7] = (m[1] * m[6] - m[0] * m[7]) * id;
    o[8] = (m[0] * m[4] - m[1] * m[3]) * id;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            if (!on[r] || !on[c]) o[3 * r + c] = 0.0;
}

// y' = y + T e of node j of a coarse level (3 DOFs), e the next level's correction.
__device__ __forceinline__ void prolonged3(const MgLevel& F, const MgLevel& C, int j, double* out) {
    const double* t = F.T + 9 * (size_t)j;
    const double* e = C.z + 3 * (size_t)F.agg[j];
    const double e0 = e[0], e1 = e[1], e2 = e[2];
#pragma unroll
    for (int r = 0; r < 3; ++r) out[r] = F.y[3 * (size_t)j + r] + t[3 * r] * e0 + t[3 * r + 1] * e1 + t[3 * r + 2] * e2;
}

// The same on level 0 (2 DOFs).
__device__ __forceinline__ double2 prolonged0(const MgLevel& L0, const MgLevel& L1, int j) {
    const double2 y = reinterpret_cast<const double2*>(L0.y)[j];
    const double* t = L0.T + 6 * (size_t)j;
    const double* e = L1.z + 3 * (size_t)L0.agg[j];
    const double e0 = e[0], e1 = e[1], e2 = e[2];
    return make_double2(y.x + t[0] * e0 + t[1] * e1 + t[2] * e2, y.y + t[3] * e0 + t[4] * e1 + t[5] * e2);
}

// ------------------------------------------------------------- set-up --

// Level 0: masked 2x2 inverse of every diagonal block and the Gershgorin
// bound of D0^-1 K over the free DOFs.
__global__ void __launch_bounds__(kThreads) k_mg_diag0(MgArgs a, MgLevel L0, double* lam) {
    double vmax = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const uchar2 m = a.mask[i];
        const int sl = i >> 5, lane = i & 31;
        const int base = a.slice_ptr[sl], w = (a.slice_ptr[sl + 1] - base) >> 5;
        const double4 d = ld_block(a.val, base + lane);  // block 0: the diagonal block
        double4 mi = make_double4(0.0, 0.0, 0.0, 0.0);
        if (m.x && m.y) {
            const double det = d.x * d.w - d.y * d.z;
            if (det != 0.0) mi = make_double4(d.w / det, -d.y / det, -d.z / det, d.x / det);
        } else if (m.x && d.x != 0.0) {
            mi.x = 1.0 / d.x;
        } else if (m.y && d.w != 0.0) {
            mi.w = 1.0 / d.w;
        }
        reinterpret_cast<double4*>(L0.dinv)[i] = mi;
        double s0 = 0.0, s1 = 0.0;
        for (int k = 0; k < w; ++k) {
            const long long bi = base + 32LL * k + lane;
            const uchar2 mc = a.mask[__ldg(a.scol + bi)];
            const double4 kv = ld_block(a.val, bi);
            const double a00 = mi.x * kv.x + mi.y * kv.z, a01 = mi.x * kv.y + mi.y * kv.w;
            const double a10 = mi.z * kv.x + mi.w * kv.z, a11 = mi.z * kv.y + mi.w * kv.w;
            if (mc.x) {
                s0 += fabs(a00);
                s1 += fabs(a10);
            }
            if (mc.y) {
                s0 += fabs(a01);
                s1 += fabs(a11);
            }
        }
        vmax = fmax(vmax, fmax(s0, s1));
    }
    max_to(lam, vmax);
}

// Coarse blocks of the next level: block c = sum over its map entries of
// T_i^T K_ij T_j (FB = the fine level's DOFs per node; level 0 reads the
// sliced values, 4 per block, coarse levels 9 per block).
template <int FB>
__global__ void __launch_bounds__(kSmall) k_mg_galerkin(int ncb, const int* __restrict__ gal_pos,
                                                        const int4* __restrict__ gal, const double* __restrict__ fval,
                                                        const double* __restrict__ T, double* __restrict__ cval) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncb; c += gridDim.x * blockDim.x) {
        double acc[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) acc[k] = 0.0;
        for (int q = gal_pos[c]; q < gal_pos[c + 1]; ++q) {
            const int4 g = gal[q];
            const double* K = fval + (size_t)FB * FB * g.x;
            const double* Ti = T + 3 * FB * (size_t)g.y;
            const double* Tj = T + 3 * FB * (size_t)g.z;
            double KT[FB * 3];
#pragma unroll
            for (int x = 0; x < FB; ++x)
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) {
                    double s = 0.0;
#pragma unroll
                    for (int y = 0; y < FB; ++y) s += K[FB * x + y] * Tj[3 * y + cc];
                    KT[3 * x + cc] = s;
                }
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) {
                    double s = 0.0;
#pragma unroll
                    for (int x = 0; x < FB; ++x) s += Ti[3 * x + r] * KT[3 * x + cc];
                    acc[3 * r + cc] += s;
                }
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) cval[9 * (size_t)c + k] = acc[k];
    }
}

// Coarse level: 3x3 block inverses and the Gershgorin bound of D^-1 A.
__global__ void __launch_bounds__(kSmall) k_mg_diag(MgLevel C, double* lam) {
    double vmax = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < C.n; i += gridDim.x * blockDim.x) {
        double di[9];
        inv3_masked(C.val + 9 * (size_t)C.rp[i], di);  // the row's first block is the diagonal one
#pragma unroll
        for (int k = 0; k < 9; ++k) C.dinv[9 * (size_t)i + k] = di[k];
        double s[3] = {0.0, 0.0, 0.0};
        for (int q = C.rp[i]; q < C.rp[i + 1]; ++q) {
            const double* A = C.val + 9 * (size_t)q;
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    s[r] += fabs(di[3 * r] * A[c] + di[3 * r + 1] * A[3 + c] + di[3 * r + 2] * A[6 + c]);
        }
        vmax = fmax(vmax, fmax(s[0], fmax(s[1], s[2])));
    }
    max_to(lam, vmax);
}

// Dense inverse of the coarsest operator by Gauss-Jordan elimination without
// pivoting (the operator is symmetric positive definite on its nonzero DOFs;
// a DOF whose row and column are zero gets a unit diagonal, and its
// right-hand side is always zero). One block; the matrix lives in shared
// memory when in_smem, else in `work`. The result is stored column-major.
__global__ void __launch_bounds__(1024) k_mg_coarse_inv(MgLevel C, int nc, double* __restrict__ cinv,
                                                        double* __restrict__ work, int in_smem) {
    extern __shared__ double sm_[];
    double* A = in_smem ? sm_ : work;
    double* colk = in_smem ? sm_ + (size_t)nc * nc : sm_;
    double* rowk = colk + nc;
    const int tid = threadIdx.x, nt = blockDim.x;
    const long long nn = (long long)nc * nc;
    for (long long e = tid; e < nn; e += nt) A[e] = 0.0;
    __syncthreads();
    for (int i = tid; i < C.n; i += nt)
        for (int q = C.rp[i]; q < C.rp[i + 1]; ++q) {
            const int j = C.ci[q];
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) A[(size_t)(3 * i + r) * nc + 3 * j + c] = C.val[9 * (size_t)q + 3 * r + c];
        }
    __syncthreads();
    for (int k = tid; k < nc; k += nt)
        if (A[(size_t)k * nc + k] == 0.0) A[(size_t)k * nc + k] = 1.0;
    __syncthreads();
    for (int k = 0; k < nc; ++k) {
        const double piv = A[(size_t)k * nc + k];
        const double p = piv != 0.0 ? 1.0 / piv : 0.0;
        for (int i = tid; i < nc; i += nt) {
            colk[i] = A[(size_t)i * nc + k];
            rowk[i] = A[(size_t)k * nc + i] * p;
        }
        __syncthreads();
        for (long long e = tid; e < nn; e += nt) {
            const int i = (int)(e / nc), j = (int)(e - (long long)i * nc);
            double v;
            if (i == k) v = (j == k) ? p : rowk[j];
            else if (j == k) v = -colk[i] * p;
            else v = A[e] - colk[i] * rowk[j];
            A[e] = v;
        }
        __syncthreads();
    }
    for (long long e = tid; e < nn; e += nt) {
        const int i = (int)(e / nc), j = (int)(e - (long long)i * nc);
        cinv[(size_t)j * nc + i] = A[e];
    }
}

// ----------------------------------------------------------- the solve --

// r = m.(b - K x), p = 0, y0 = w0 D0^-1 r; (r, r), (b, b); scalars.
__global__ void __launch_bounds__(kThreads) k_mg_init(MgArgs a, MgLevel L0, const double* lam, double omega,
                                                      double eps2, long long max_iter) {
    __shared__ double sh[2 * kThreads / 32];
    __shared__ bool last;
    const double w0 = damping(lam, 0, omega);
    double s_rr = 0.0, s_bb = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const double2 kx = k_row(a, i, a.x);
        const uchar2 m = a.mask[i];
        const double2 bb = a.b[i];
        const double2 r = make_double2(m.x ? bb.x - kx.x : 0.0, m.y ? bb.y - kx.y : 0.0);
        a.r[i] = r;
        a.p0[i] = make_double2(0.0, 0.0);
        a.p1[i] = make_double2(0.0, 0.0);
        const double4 mi = reinterpret_cast<const double4*>(L0.dinv)[i];
        reinterpret_cast<double2*>(L0.y)[i] = make_double2(w0 * (mi.x * r.x + mi.y * r.y), w0 * (mi.z * r.x + mi.w * r.y));
        s_rr += r.x * r.x + r.y * r.y;
        s_bb += bb.x * bb.x + bb.y * bb.y;
    }
    const double2 bs = block_sum2(s_rr, s_bb, sh);
    if (threadIdx.x == 0) {
        a.partials[2 * blockIdx.x] = bs.x;
        a.partials[2 * blockIdx.x + 1] = bs.y;
    }
    if (last_block_arrive(&a.sc->ticket, &last)) {
        const double2 t = block_reduce_array2(a.partials, gridDim.x, sh);
        if (threadIdx.x == 0) {
            CgScalars* sc = a.sc;
            sc->rr = t.x;
            sc->res64 = t.x;
            sc->bb = t.y;
            sc->normB_inv = t.y > 0.0 ? 1.0 / t.y : 0.0;
            sc->eps2 = eps2;
            sc->iter = 0;
            sc->max_iter = max_iter;
            sc->rho = 0.0;
            sc->beta = 0.0;
            sc->alpha = 0.0;
            sc->pAz = 0.0;
            sc->lin_done = 0;
            sc->status = 0;
            sc->converged = (t.x == 0.0 || t.x * sc->normB_inv <= eps2) ? 1 : 0;
            if (!(t.x == t.x) || !(t.y == t.y)) sc->status = CP_ERR_BREAKDOWN;
            sc->ticket = 0;
        }
    }
}

// P: p = z + beta p, q = K p, (p, q) -> alpha.
__global__ void __launch_bounds__(kThreads) k_mg_p(MgArgs a, MgLevel L0, int parity) {
    __shared__ double sh[kThreads / 32];
    __shared__ bool last;
    CgScalars* sc = a.sc;
    if (sc->converged || sc->status) return;
    const double2* __restrict__ po = parity ? a.p1 : a.p0;
    double2* __restrict__ pn = parity ? a.p0 : a.p1;
    const double2* __restrict__ z = reinterpret_cast<const double2*>(L0.z);
    const double beta = sc->beta;
    double dot = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const int sl = i >> 5, lane = i & 31;
        const int base = a.slice_ptr[sl], w = (a.slice_ptr[sl + 1] - base) >> 5;
        double k0 = 0.0, k1 = 0.0;
        for (int k = 0; k < w; ++k) {
            const long long bi = base + 32LL * k + lane;
            const int c = __ldg(a.scol + bi);
            const double4 kv = ld_block(a.val, bi);
            const double2 zc = z[c], pc = po[c];
            const double wx = zc.x + beta * pc.x, wy = zc.y + beta * pc.y;
            k0 += kv.x * wx + kv.y * wy;
            k1 += kv.z * wx + kv.w * wy;
        }
        const double2 zi = z[i], pi = po[i];
        const double2 pp = make_double2(zi.x + beta * pi.x, zi.y + beta * pi.y);
        pn[i] = pp;
        a.q[i] = make_double2(k0, k1);
        dot += k0 * pp.x + k1 * pp.y;
    }
    const double bs = block_sum(dot, sh);
    if (threadIdx.x == 0) a.partials[blockIdx.x] = bs;
    if (last_block_arrive(&sc->ticket, &last)) {
        const double pq = block_reduce_array(a.partials, gridDim.x, sh);
        if (threadIdx.x == 0) {
            sc->pAz = pq;
            sc->alpha = sc->rho / pq;
            if (!(pq > 0.0) || !(sc->alpha == sc->alpha)) sc->status = CP_ERR_BREAKDOWN;
            sc->ticket = 0;
        }
    }
}

// U: x += alpha p, r -= m.alpha q, y0 = w0 D0^-1 r; (r, r) -> iteration count
// and convergence.
__global__ void __launch_bounds__(kThreads) k_mg_u(MgArgs a, MgLevel L0, const double* lam, double omega,
                                                   int parity) {
    __shared__ double sh[kThreads / 32];
    __shared__ bool last;
    CgScalars* sc = a.sc;
    if (sc->converged || sc->status) return;
    const double2* __restrict__ pn = parity ? a.p0 : a.p1;
    const double alpha = sc->alpha;
    const double w0 = damping(lam, 0, omega);
    double dot = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const double2 p = pn[i], q = a.q[i];
        const uchar2 m = a.mask[i];
        double2 x = a.x[i];
        x.x += alpha * p.x;
        x.y += alpha * p.y;
        a.x[i] = x;
        double2 r = a.r[i];
        if (m.x) r.x -= alpha * q.x;
        if (m.y) r.y -= alpha * q.y;
        a.r[i] = r;
        const double4 mi = reinterpret_cast<const double4*>(L0.dinv)[i];
        reinterpret_cast<double2*>(L0.y)[i] = make_double2(w0 * (mi.x * r.x + mi.y * r.y), w0 * (mi.z * r.x + mi.w * r.y));
        dot += r.x * r.x + r.y * r.y;
    }
    const double bs = block_sum(dot, sh);
    if (threadIdx.x == 0) a.partials[blockIdx.x] = bs;
    if (last_block_arrive(&sc->ticket, &last)) {
        const double rn = block_reduce_array(a.partials, gridDim.x, sh);
        if (threadIdx.x == 0) {
            sc->rr = rn;
            sc->iter += 1;
            if (rn * sc->normB_inv <= sc->eps2) sc->converged = 1;
            else if (sc->iter >= sc->max_iter) sc->status = CP_ERR_NOT_CONVERGED;
            if (!(rn == rn)) sc->status = CP_ERR_BREAKDOWN;
            sc->ticket = 0;
        }
    }
}

// R0: per level-0 range of kMgPartNodes nodes (one block; no aggregate
// crosses a range), each thread the residual r - K y0 of one node, restricted
// by its prolongator block into shared memory; then per level-1 node of the
// range, the sum over its members in member order, and level 1's
// pre-smoothing from zero (unless it is the coarsest level).
__global__ void __launch_bounds__(kMgPartNodes) k_mg_restrict0(MgArgs a, MgLevel L0, MgLevel L1, const double* lam,
                                                               double omega, int coarsest) {
    __shared__ double tr[kMgPartNodes][3];
    if (a.sc->converged || a.sc->status) return;
    const int i0 = blockIdx.x * kMgPartNodes, i = i0 + threadIdx.x;
    if (i < a.n) {
        const double2 ky = k_row(a, i, reinterpret_cast<const double2*>(L0.y));
        const uchar2 m = a.mask[i];
        const double2 ri = a.r[i];
        const double rx = m.x ? ri.x - ky.x : 0.0, ry = m.y ? ri.y - ky.y : 0.0;
        const double* t = L0.T + 6 * (size_t)i;
#pragma unroll
        for (int c = 0; c < 3; ++c) tr[threadIdx.x][c] = t[c] * rx + t[3 + c] * ry;
    }
    __syncthreads();
    const double w1 = coarsest ? 0.0 : damping(lam, 1, omega);
    for (int A = L1.part_pos[blockIdx.x] + threadIdx.x; A < L1.part_pos[blockIdx.x + 1]; A += blockDim.x) {
        double c0 = 0.0, c1 = 0.0, c2 = 0.0;
        for (int q = L0.mem_pos[A]; q < L0.mem_pos[A + 1]; ++q) {
            const double* u = tr[L0.mem[q] - i0];
            c0 += u[0];
            c1 += u[1];
            c2 += u[2];
        }
        double* b = L1.b + 3 * (size_t)A;
        b[0] = c0;
        b[1] = c1;
        b[2] = c2;
        if (!coarsest) {
            const double* di = L1.dinv + 9 * (size_t)A;
            double* y = L1.y + 3 * (size_t)A;
#pragma unroll
            for (int r = 0; r < 3; ++r) y[r] = w1 * (di[3 * r] * c0 + di[3 * r + 1] * c1 + di[3 * r + 2] * c2);
        }
    }
}

// One node A of level l + 1 (C): the level-l (F) residual b - A y of its
// members, restricted, and C's pre-smoothing (wc = 0 on the coarsest).
__device__ __forceinline__ void restrict_node(const MgLevel& F, const MgLevel& C, int A, double wc, bool coarsest) {
    double c[3] = {0.0, 0.0, 0.0};
    for (int q = F.mem_pos[A]; q < F.mem_pos[A + 1]; ++q) {
        const int i = F.mem[q];
        double r[3] = {F.b[3 * (size_t)i], F.b[3 * (size_t)i + 1], F.b[3 * (size_t)i + 2]};
        for (int p = F.rp[i]; p < F.rp[i + 1]; ++p) {
            const double* Ab = F.val + 9 * (size_t)p;
            const double* yj = F.y + 3 * (size_t)F.ci[p];
            const double y0 = yj[0], y1 = yj[1], y2 = yj[2];
#pragma unroll
            for (int rr = 0; rr < 3; ++rr) r[rr] -= Ab[3 * rr] * y0 + Ab[3 * rr + 1] * y1 + Ab[3 * rr + 2] * y2;
        }
        const double* t = F.T + 9 * (size_t)i;
#pragma unroll
        for (int col = 0; col < 3; ++col) c[col] += t[col] * r[0] + t[3 + col] * r[1] + t[6 + col] * r[2];
    }
    double* b = C.b + 3 * (size_t)A;
    b[0] = c[0];
    b[1] = c[1];
    b[2] = c[2];
    if (!coarsest) {
        const double* di = C.dinv + 9 * (size_t)A;
        double* y = C.y + 3 * (size_t)A;
#pragma unroll
        for (int r = 0; r < 3; ++r) y[r] = wc * (di[3 * r] * c[0] + di[3 * r + 1] * c[1] + di[3 * r + 2] * c[2]);
    }
}

// Row r of the coarsest correction e = A_c^-1 b_c (column-major inverse).
__device__ __forceinline__ void coarse_row(const MgLevel& C, int nc, const double* __restrict__ cinv, int r) {
    double s = 0.0;
    for (int c = 0; c < nc; ++c) s += cinv[(size_t)c * nc + r] * C.b[c];
    C.z[r] = s;
}

// One node i of level l (F): z = y' + w D^-1 (b - A y'), y' = y + T e with e
// the next level's (C) correction, gathered for every column of the row.
__device__ __forceinline__ void smooth_node(const MgLevel& F, const MgLevel& C, int i, double w) {
    double s[3] = {F.b[3 * (size_t)i], F.b[3 * (size_t)i + 1], F.b[3 * (size_t)i + 2]};
    double yi[3] = {0.0, 0.0, 0.0};
    for (int p = F.rp[i]; p < F.rp[i + 1]; ++p) {
        double yj[3];
        prolonged3(F, C, F.ci[p], yj);
        const double* Ab = F.val + 9 * (size_t)p;
#pragma unroll
        for (int r = 0; r < 3; ++r) s[r] -= Ab[3 * r] * yj[0] + Ab[3 * r + 1] * yj[1] + Ab[3 * r + 2] * yj[2];
        if (p == F.rp[i]) {  // the diagonal block: column i itself
            yi[0] = yj[0];
            yi[1] = yj[1];
            yi[2] = yj[2];
        }
    }
    const double* di = F.dinv + 9 * (size_t)i;
#pragma unroll
    for (int r = 0; r < 3; ++r)
        F.z[3 * (size_t)i + r] = yi[r] + w * (di[3 * r] * s[0] + di[3 * r + 1] * s[1] + di[3 * r + 2] * s[2]);
}

// R_l (l >= 1), one thread per level-(l + 1) node.
__global__ void __launch_bounds__(kSmall) k_mg_restrict(MgLevel F, MgLevel C, const double* lam, int lc,
                                                        double omega, int coarsest, const CgScalars* sc) {
    if (sc->converged || sc->status) return;
    const double wc = coarsest ? 0.0 : damping(lam, lc, omega);
    for (int A = blockIdx.x * blockDim.x + threadIdx.x; A < C.n; A += gridDim.x * blockDim.x)
        restrict_node(F, C, A, wc, coarsest != 0);
}

// C: the coarsest correction (the threads of a warp read consecutive entries).
__global__ void __launch_bounds__(kSmall) k_mg_coarse(MgLevel C, int nc, const double* __restrict__ cinv,
                                                      const CgScalars* sc) {
    if (sc->converged || sc->status) return;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nc; r += gridDim.x * blockDim.x) coarse_row(C, nc, cinv, r);
}

// S_l (l >= 1), one thread per level-l node.
__global__ void __launch_bounds__(kSmall) k_mg_smooth(MgLevel F, MgLevel C, const double* lam, int l, double omega,
                                                      const CgScalars* sc) {
    if (sc->converged || sc->status) return;
    const double w = damping(lam, l, omega);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F.n; i += gridDim.x * blockDim.x) smooth_node(F, C, i, w);
}

// Levels 1 .. L-1 of the V-cycle in one block when level 1 is small: the
// restrictions R_1 .. R_{L-2}, the coarsest correction and the sweeps
// S_{L-2} .. S_1, separated by block barriers instead of kernel boundaries
// (the same per-node arithmetic as the kernels above).
__global__ void __launch_bounds__(1024) k_mg_coarse_cycle(MgDev m, const CgScalars* sc) {
    if (sc->converged || sc->status) return;
    const int L = m.L, tid = threadIdx.x, nt = blockDim.x;
    for (int l = 1; l + 1 < L; ++l) {
        const bool coarsest = l + 1 == L - 1;
        const double wc = coarsest ? 0.0 : damping(m.lam, l + 1, m.omega);
        for (int A = tid; A < m.lv[l + 1].n; A += nt) restrict_node(m.lv[l], m.lv[l + 1], A, wc, coarsest);
        __syncthreads();
    }
    for (int r = tid; r < m.nc; r += nt) coarse_row(m.lv[L - 1], m.nc, m.cinv, r);
    __syncthreads();
    for (int l = L - 2; l >= 1; --l) {
        const double w = damping(m.lam, l, m.omega);
        for (int i = tid; i < m.lv[l].n; i += nt) smooth_node(m.lv[l], m.lv[l + 1], i, w);
        __syncthreads();
    }
}

// S0: the same on level 0, giving z = M r; (r, z) -> rho, beta.
__global__ void __launch_bounds__(kThreads) k_mg_smooth0(MgArgs a, MgLevel L0, MgLevel L1, const double* lam,
                                                         double omega) {
    __shared__ double sh[kThreads / 32];
    __shared__ bool last;
    CgScalars* sc = a.sc;
    if (sc->converged || sc->status) return;
    const double w0 = damping(lam, 0, omega);
    double2* __restrict__ z = reinterpret_cast<double2*>(L0.z);
    double dot = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const int sl = i >> 5, lane = i & 31;
        const int base = a.slice_ptr[sl], w = (a.slice_ptr[sl + 1] - base) >> 5;
        const double2 ri = a.r[i];
        double s0 = ri.x, s1 = ri.y;
        double2 yi = make_double2(0.0, 0.0);
        for (int k = 0; k < w; ++k) {
            const long long bi = base + 32LL * k + lane;
            const int c = __ldg(a.scol + bi);
            const double4 kv = ld_block(a.val, bi);
            const double2 yc = prolonged0(L0, L1, c);
            s0 -= kv.x * yc.x + kv.y * yc.y;
            s1 -= kv.z * yc.x + kv.w * yc.y;
            if (k == 0) yi = yc;  // block 0: the diagonal block
        }
        const uchar2 m = a.mask[i];
        if (!m.x) s0 = 0.0;
        if (!m.y) s1 = 0.0;
        const double4 mi = reinterpret_cast<const double4*>(L0.dinv)[i];
        const double2 zi = make_double2(yi.x + w0 * (mi.x * s0 + mi.y * s1), yi.y + w0 * (mi.z * s0 + mi.w * s1));
        z[i] = zi;
        dot += ri.x * zi.x + ri.y * zi.y;
    }
    const double bs = block_sum(dot, sh);
    if (threadIdx.x == 0) a.partials[blockIdx.x] = bs;
    if (last_block_arrive(&sc->ticket, &last)) {
        const double rho_new = block_reduce_array(a.partials, gridDim.x, sh);
        if (threadIdx.x == 0) {
            sc->beta = sc->rho > 0.0 ? rho_new / sc->rho : 0.0;
            sc->rho = rho_new;
            if (!(rho_new > 0.0)) sc->status = CP_ERR_BREAKDOWN;  // M r must be a descent direction
            sc->ticket = 0;
        }
    }
}

__global__ void k_mg_condition(const CgScalars* sc, cudaGraphConditionalHandle h) {
    cudaGraphSetConditional(h, (sc->converged || sc->status) ? 0u : 1u);
}

int grid_nodes(const MgArgs& a) {
    const long long g = ((long long)a.n + kThreads - 1) / kThreads;
    return (int)std::max<long long>(1, std::min<long long>(g, a.max_blocks));
}

int grid_small(long long n, int sms) {
    const long long g = (n + kSmall - 1) / kSmall;
    return (int)std::max<long long>(1, std::min<long long>(g, 8LL * sms));
}

// Level 1 at most this many nodes: levels 1 .. L-1 run in one block.
constexpr int kMgOneBlockNodes = 4096;

// CUPLAST_MG_ONE_BLOCK=0 runs the coarse levels as one kernel per level step
// whatever their size (for measurements).
int one_block_limit() {
    static const int lim = [] {
        const char* e = std::getenv("CUPLAST_MG_ONE_BLOCK");
        return (e && e[0] == '0') ? 0 : kMgOneBlockNodes;
    }();
    return lim;
}

bool one_block_coarse(const MgDev& m) { return m.L >= 3 && m.lv[1].n <= one_block_limit(); }

// The V-cycle from U's y0 to S0's z, in three parts: R0, the coarse levels,
// S0. `ev` (optional): events recorded after R0 and after the coarse levels.
int launch_vcycle(const MgDev& m, const MgArgs& a, cudaStream_t s, cudaEvent_t* ev = nullptr) {
    const int L = m.L;
    const int sms = a.sm_count;
    const int parts = (a.n + kMgPartNodes - 1) / kMgPartNodes;
    k_mg_restrict0<<<parts, kMgPartNodes, 0, s>>>(a, m.lv[0], m.lv[1], m.lam, m.omega, L == 2);
    if (ev) CP_CUDA(cudaEventRecord(ev[0], s));
    int launches = 1;
    if (one_block_coarse(m)) {
        k_mg_coarse_cycle<<<1, 1024, 0, s>>>(m, a.sc);
        ++launches;
    } else {
        for (int l = 1; l + 1 < L; ++l)
            k_mg_restrict<<<grid_small(m.lv[l + 1].n, sms), kSmall, 0, s>>>(m.lv[l], m.lv[l + 1], m.lam, l + 1,
                                                                            m.omega, l + 1 == L - 1, a.sc);
        k_mg_coarse<<<grid_small(m.nc, sms), kSmall, 0, s>>>(m.lv[L - 1], m.nc, m.cinv, a.sc);
        for (int l = L - 2; l >= 1; --l)
            k_mg_smooth<<<grid_small(m.lv[l].n, sms), kSmall, 0, s>>>(m.lv[l], m.lv[l + 1], m.lam, l, m.omega, a.sc);
        launches += 2 * (L - 2) + 1;
    }
    if (ev) CP_CUDA(cudaEventRecord(ev[1], s));
    k_mg_smooth0<<<grid_nodes(a), kThreads, 0, s>>>(a, m.lv[0], m.lv[1], m.lam, m.omega);
    CP_CUDA(cudaGetLastError());
    return launches + 1;
}

}  // namespace

int mg_launches_per_iteration(const MgDev& m) { return 2 + (one_block_coarse(m) ? 3 : 2 * m.L - 1); }

int mg_launch_setup(const MgDev& m, const MgArgs& a, cudaStream_t s) {
    const int sms = a.sm_count;
    CP_CUDA(cudaMemsetAsync(m.lam, 0, sizeof(double) * kMgMaxLevels, s));
    k_mg_diag0<<<grid_nodes(a), kThreads, 0, s>>>(a, m.lv[0], m.lam);
    int launches = 1;
    for (int l = 0; l + 1 < m.L; ++l) {
        const MgLevel& F = m.lv[l];
        const MgLevel& C = m.lv[l + 1];
        if (l == 0)
            k_mg_galerkin<2><<<grid_small(C.nb, sms), kSmall, 0, s>>>(C.nb, F.gal_pos, F.gal, a.val, F.T, C.val);
        else
            k_mg_galerkin<3><<<grid_small(C.nb, sms), kSmall, 0, s>>>(C.nb, F.gal_pos, F.gal, F.val, F.T, C.val);
        ++launches;
        if (l + 1 < m.L - 1) {
            k_mg_diag<<<grid_small(C.n, sms), kSmall, 0, s>>>(C, m.lam + l + 1);
            ++launches;
        }
    }
    const bool in_smem = m.nc <= kMgMaxCoarse;
    const size_t smem = (in_smem ? (size_t)m.nc * m.nc + 2 * (size_t)m.nc : 2 * (size_t)m.nc) * sizeof(double);
    CP_CUDA(cudaFuncSetAttribute(k_mg_coarse_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_mg_coarse_inv<<<1, 1024, smem, s>>>(m.lv[m.L - 1], m.nc, m.cinv, m.work, in_smem ? 1 : 0);
    CP_CUDA(cudaGetLastError());
    return launches + 1;
}

int mg_launch_start(const MgDev& m, const MgArgs& a, double eps2, long long max_iter, cudaStream_t s) {
    k_mg_init<<<grid_nodes(a), kThreads, 0, s>>>(a, m.lv[0], m.lam, m.omega, eps2, max_iter);
    CP_CUDA(cudaGetLastError());
    return 1 + launch_vcycle(m, a, s);
}

int mg_launch_iteration(const MgDev& m, const MgArgs& a, int parity, cudaStream_t s, cudaEvent_t* ev) {
    if (ev) CP_CUDA(cudaEventRecord(ev[0], s));
    k_mg_p<<<grid_nodes(a), kThreads, 0, s>>>(a, m.lv[0], parity);
    if (ev) CP_CUDA(cudaEventRecord(ev[1], s));
    k_mg_u<<<grid_nodes(a), kThreads, 0, s>>>(a, m.lv[0], m.lam, m.omega, parity);
    if (ev) CP_CUDA(cudaEventRecord(ev[2], s));
    CP_CUDA(cudaGetLastError());
    const int n = 2 + launch_vcycle(m, a, s, ev ? ev + 3 : nullptr);
    if (ev) CP_CUDA(cudaEventRecord(ev[5], s));
    return n;
}

void mg_algorithmic_bytes(const MgDev& m, const MgArgs& a, long long blocks0, double* bytes) {
    // FP64 values; a level-0 block is 32 bytes of values and a 4-byte column,
    // a coarse block 72 bytes and a 4-byte column; vectors counted once each.
    const double n = a.n, K0 = 36.0 * (double)blocks0, n1 = m.lv[1].n;
    bytes[0] = K0 + 64 * n;                                // P: K, z, p; p', q
    bytes[1] = 146 * n;                                    // U: p, q, x, r, mask, D0^-1; x, r, y0
    bytes[2] = K0 + 90 * n + 124 * n1;                     // R0: K, y0, r, mask, T0, members; b1, y1, D1^-1
    double c = 0.0;
    for (int l = 1; l + 1 < m.L; ++l) {                    // restriction and sweep of every coarse level
        const double nl = m.lv[l].n, bl = m.lv[l].nb;
        c += 2 * 76 * bl + nl * (48 + 72 + 4 + 72 + 24 + 24) + 48.0 * m.lv[l + 1].n;
    }
    c += 8.0 * m.nc * m.nc + 16.0 * m.nc;                  // the coarsest inverse times b_c
    bytes[3] = c;
    bytes[4] = K0 + 134 * n + 24 * n1;                     // S0: K, y0, T0, agg, e1, r, mask, D0^-1; z
    double su = K0 + 2 * n + 32 * n;                       // diag0: K, mask; D0^-1
    for (int l = 0; l + 1 < m.L; ++l) {
        const double fb = l == 0 ? 36.0 : 76.0, bl = m.lv[l].nb;
        su += fb * bl + 16 * bl + 4.0 * (m.lv[l + 1].nb + 1) + 72.0 * m.lv[l + 1].nb;  // Galerkin: blocks, map; A_{l+1}
        if (l + 1 < m.L - 1) su += 76.0 * m.lv[l + 1].nb + 72.0 * m.lv[l + 1].n;       // diag: A, D^-1
    }
    su += 2 * 8.0 * m.nc * m.nc;                           // the coarsest inverse, written once
    bytes[5] = su;
}

cudaGraphExec_t mg_build_while_graph(const MgDev& m, const MgArgs& a, int body_iters, cudaStream_t s) {
    CP_CHECK(body_iters > 0 && body_iters % 2 == 0, CP_ERR_INVALID, "multigrid CG: graph body must be even");
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
    for (int it = 0; it < body_iters; ++it) mg_launch_iteration(m, a, it & 1, s);
    k_mg_condition<<<1, 1, 0, s>>>(a.sc, h);
    cudaGraph_t captured = nullptr;
    CP_CUDA(cudaStreamEndCapture(s, &captured));
    cudaGraphExec_t exec;
    CP_CUDA(cudaGraphInstantiate(&exec, g, 0));
    CP_CUDA(cudaGraphDestroy(g));
    return exec;
}

// ------------------------------------------------------ host set-up --

namespace {

template <typename T>
T* mg_alloc(cp_instance* I, size_t count) {
    void* p = nullptr;
    const size_t nb = std::max<size_t>(count, 1) * sizeof(T);
    CP_CUDA(cudaMallocAsync(&p, nb, I->s()));
    I->mg_allocs.push_back(p);
    I->bytes += nb;
    I->mg_bytes += nb;
    return static_cast<T*>(p);
}

template <typename T>
T* mg_upload(cp_instance* I, const std::vector<T>& v) {
    T* d = mg_alloc<T>(I, v.size());
    if (!v.empty()) CP_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, I->s()));
    return d;
}

}  // namespace

size_t mg_footprint(size_t n, size_t blocks) {
    // level 0: D0^-1, y, z, T0, aggregate, member (128 per node); one map
    // entry per block (16). Coarse levels: 3x3 values, column, map entry per
    // block (92) and D^-1, T, b, y, z, aggregate, member, ranges per node
    // (about 300), a geometric series of at most twice level 1, which has at
    // most half the nodes and blocks of level 0. The coarsest inverse and its
    // scratch: at most 2 x kMgMaxCoarsest^2 doubles = 1 MB (mg_prepare
    // rejects a coarser bottom level).
    return 128 * n + 16 * blocks + 2 * (300 * (n / 2) + 92 * (blocks / 2)) + (1u << 20);
}

void mg_release(cp_instance* I) {
    if (I->gmg) cudaGraphExecDestroy(I->gmg);
    I->gmg = nullptr;
    for (void* p : I->mg_allocs) cudaFreeAsync(p, I->s());
    I->mg_allocs.clear();
    I->bytes -= I->mg_bytes;
    I->mg_bytes = 0;
    I->mg = MgDev{};
    I->mg_ready = false;
}

void mg_prepare(cp_instance* I) {
    if (I->mg_ready && I->mg_mask == I->mask_host) return;
    mg_release(I);
    cudaStream_t s = I->s();
    const int n = I->n_nodes;
    const long long nadj = I->csr.nadj;
    std::vector<int> adj_pos(n + 1), adj(std::max<long long>(nadj, 1)), slice_ptr(I->csr.n_slices + 1);
    std::vector<double> xy(2 * (size_t)n);
    CP_CUDA(cudaMemcpyAsync(adj_pos.data(), I->csr.adj_pos, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s));
    if (nadj > 0) CP_CUDA(cudaMemcpyAsync(adj.data(), I->csr.adj, sizeof(int) * nadj, cudaMemcpyDeviceToHost, s));
    CP_CUDA(cudaMemcpyAsync(slice_ptr.data(), I->csr.slice_ptr, sizeof(int) * slice_ptr.size(), cudaMemcpyDeviceToHost, s));
    CP_CUDA(cudaMemcpyAsync(xy.data(), I->mesh.xy, sizeof(double2) * n, cudaMemcpyDeviceToHost, s));
    CP_CUDA(cudaStreamSynchronize(s));
    CP_CHECK(I->mask_host.size() == 2 * (size_t)n, CP_ERR_INVALID, "loads not set");
    amg::Hierarchy H = amg::build(n, adj_pos.data(), adj.data(), xy.data(), I->mask_host.data(), kMgMinCoarse,
                                  kMgPartNodes);
    if (H.levels.size() < 2)  // a mesh at or below the coarse size: coarsen while it shrinks
        H = amg::build(n, adj_pos.data(), adj.data(), xy.data(), I->mask_host.data(), 0, kMgPartNodes);
    CP_CHECK(H.levels.size() >= 2, CP_ERR_UNSUPPORTED, "multigrid: the node graph does not coarsen");
    const int L = std::min<int>((int)H.levels.size(), kMgMaxLevels);
    MgDev m;
    m.L = L;
    m.nc = 3 * H.levels[L - 1].n_nodes;
    CP_CHECK(m.nc <= kMgMaxCoarsest, CP_ERR_UNSUPPORTED, "multigrid: coarsest level too large");
    for (int l = 0; l < L; ++l) {
        const amg::Level& F = H.levels[l];
        MgLevel& D = m.lv[l];
        D.n = F.n_nodes;
        D.fb = F.fb;
        D.nb = F.n_nodes + F.adj_pos[F.n_nodes];
        const amg::DeviceMaps dm = amg::device_maps(H, l, slice_ptr.data());
        if (l == 0) {
            D.dinv = mg_alloc<double>(I, 4 * (size_t)D.n);
            D.y = mg_alloc<double>(I, 2 * (size_t)D.n);
            D.z = mg_alloc<double>(I, 2 * (size_t)D.n);
        } else {
            D.rp = mg_upload(I, dm.rp);
            D.ci = mg_upload(I, dm.ci);
            D.part_pos = mg_upload(I, F.part_pos);
            D.val = mg_alloc<double>(I, 9 * (size_t)D.nb);
            D.dinv = mg_alloc<double>(I, 9 * (size_t)D.n);
            D.b = mg_alloc<double>(I, 3 * (size_t)D.n);
            D.y = mg_alloc<double>(I, 3 * (size_t)D.n);
            D.z = mg_alloc<double>(I, 3 * (size_t)D.n);
        }
        if (l + 1 < L) {
            std::vector<int4> gal(dm.gal.size() / 4);
            for (size_t q = 0; q < gal.size(); ++q)
                gal[q] = make_int4(dm.gal[4 * q], dm.gal[4 * q + 1], dm.gal[4 * q + 2], dm.gal[4 * q + 3]);
            D.agg = mg_upload(I, F.agg);
            D.T = mg_upload(I, F.T);
            D.mem_pos = mg_upload(I, dm.mem_pos);
            D.mem = mg_upload(I, dm.mem);
            D.gal_pos = mg_upload(I, dm.gal_pos);
            D.gal = mg_upload(I, gal);
        }
    }
    m.cinv = mg_alloc<double>(I, (size_t)m.nc * m.nc);
    if (m.nc > kMgMaxCoarse) m.work = mg_alloc<double>(I, (size_t)m.nc * m.nc);
    m.lam = mg_alloc<double>(I, kMgMaxLevels);
    CP_CUDA(cudaStreamSynchronize(s));  // the host vectors above go out of scope
    I->mg = m;
    I->mg_mask = I->mask_host;
    I->mg_ready = true;
}

}  // namespace cp
