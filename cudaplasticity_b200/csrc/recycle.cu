// Initial guesses from the recent solution increments (recycle.h).
#include "common.cuh"
#include "internal.h"
#include "recycle.h"
#include "../../include/cuplast_host.h"

namespace cp {

namespace {

constexpr int kRecThreads = 256;

// The small system (W^T K W) y = W^T r0 by Cholesky of the diagonally scaled
// Gram matrix, dropping increments whose pivot is at most kDrop (or whose
// diagonal is not positive); dropped increments get y = 0. One thread.
constexpr double kDrop = 1e-10;

__host__ __device__ void small_solve(const double* t, int cnt, double* y) {
    double A[kRecycleMax][kRecycleMax], S[kRecycleMax][kRecycleMax], L[kRecycleMax][kRecycleMax];
    double h[kRecycleMax], d[kRecycleMax], z[kRecycleMax], yy[kRecycleMax];
    bool keep[kRecycleMax], ok[kRecycleMax];
    for (int j = 0; j < kRecycleMax; ++j) {
        for (int k = 0; k < kRecycleMax; ++k) {
            A[j][k] = 0.0;
            S[j][k] = 0.0;
            L[j][k] = 0.0;
        }
        h[j] = d[j] = z[j] = yy[j] = 0.0;
        keep[j] = ok[j] = false;
    }
    for (int j = 0; j < cnt; ++j) {
        for (int k = 0; k < cnt; ++k) A[j][k] = j <= k ? t[k * (k + 1) / 2 + j] : t[j * (j + 1) / 2 + k];
        h[j] = t[kRecycleGram + j];
        d[j] = A[j][j] > 0.0 ? sqrt(A[j][j]) : 0.0;
        keep[j] = d[j] > 0.0;
    }
    for (int j = 0; j < cnt; ++j)
        for (int k = 0; k < cnt; ++k) S[j][k] = (keep[j] && keep[k]) ? A[j][k] / (d[j] * d[k]) : 0.0;
    for (int j = 0; j < cnt; ++j) {
        if (!keep[j]) continue;
        double v = S[j][j];
        for (int k = 0; k < j; ++k)
            if (ok[k]) v -= L[j][k] * L[j][k];
        if (!(v > kDrop)) continue;
        L[j][j] = sqrt(v);
        ok[j] = true;
        for (int i = j + 1; i < cnt; ++i) {
            if (!keep[i]) continue;
            double s = S[i][j];
            for (int k = 0; k < j; ++k)
                if (ok[k]) s -= L[i][k] * L[j][k];
            L[i][j] = s / L[j][j];
        }
    }
    for (int j = 0; j < cnt; ++j) {
        if (!ok[j]) continue;
        double s = h[j] / d[j];
        for (int k = 0; k < j; ++k)
            if (ok[k]) s -= L[j][k] * z[k];
        z[j] = s / L[j][j];
    }
    for (int j = cnt - 1; j >= 0; --j) {
        if (!ok[j]) continue;
        double s = z[j];
        for (int k = j + 1; k < cnt; ++k)
            if (ok[k]) s -= L[k][j] * yy[k];
        yy[j] = s / L[j][j];
    }
    bool finite = true;
    for (int j = 0; j < kRecycleMax; ++j) {
        const double v = ok[j] ? yy[j] / d[j] : 0.0;
        yy[j] = v;
        if (!(v - v == 0.0)) finite = false;  // NaN or infinity
    }
    for (int j = 0; j < kRecycleMax; ++j) y[j] = finite ? yy[j] : 0.0;
}

// Per node: K u and K w_j gathered from the sliced blocks, r0 = m.(b - K u);
// partial sums w_j . K w_k (j <= k) and w_j . r0, reduced in a fixed order;
// the last block solves for y.
__global__ void __launch_bounds__(kRecThreads) k_recycle_sums(RecycleArgs a) {
    __shared__ double wpart[kRecThreads / 32][kRecycleStride];
    __shared__ double tot[kRecycleStride];
    __shared__ bool last;
    const int cnt = a.cnt;
    const double4* __restrict__ val4 = reinterpret_cast<const double4*>(a.val);
    double acc[kRecycleSums];
#pragma unroll
    for (int i = 0; i < kRecycleSums; ++i) acc[i] = 0.0;
    for (int nd = blockIdx.x * blockDim.x + threadIdx.x; nd < a.n; nd += gridDim.x * blockDim.x) {
        const int sl = nd >> 5, l = nd & 31;
        const int p0 = a.slice_ptr[sl], wd = (a.slice_ptr[sl + 1] - p0) >> 5;
        double2 ku = make_double2(0.0, 0.0);
        double2 kw[kRecycleMax];
#pragma unroll
        for (int j = 0; j < kRecycleMax; ++j) kw[j] = make_double2(0.0, 0.0);
        for (int k = 0; k < wd; ++k) {
            const int idx = p0 + 32 * k + l;
            const int c = __ldg(a.scol + idx);
            const double2 lo = __ldg(reinterpret_cast<const double2*>(val4 + idx));
            const double2 hi = __ldg(reinterpret_cast<const double2*>(val4 + idx) + 1);
            const double4 v = make_double4(lo.x, lo.y, hi.x, hi.y);
            const double2 uc = a.u[c];
            ku.x += v.x * uc.x + v.y * uc.y;
            ku.y += v.z * uc.x + v.w * uc.y;
#pragma unroll
            for (int j = 0; j < kRecycleMax; ++j)
                if (j < cnt) {
                    const double2 wc = a.w[(size_t)a.slot[j] * a.n + c];
                    kw[j].x += v.x * wc.x + v.y * wc.y;
                    kw[j].y += v.z * wc.x + v.w * wc.y;
                }
        }
        const uchar2 m = a.mask[nd];
        const double2 bb = a.b[nd];
        const double2 r = make_double2(m.x ? bb.x - ku.x : 0.0, m.y ? bb.y - ku.y : 0.0);
        double2 wn[kRecycleMax];
#pragma unroll
        for (int j = 0; j < kRecycleMax; ++j)
            wn[j] = j < cnt ? a.w[(size_t)a.slot[j] * a.n + nd] : make_double2(0.0, 0.0);
#pragma unroll
        for (int k = 0; k < kRecycleMax; ++k) {
#pragma unroll
            for (int j = 0; j <= k; ++j) acc[k * (k + 1) / 2 + j] += wn[j].x * kw[k].x + wn[j].y * kw[k].y;
            acc[kRecycleGram + k] += wn[k].x * r.x + wn[k].y * r.y;
        }
    }
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
#pragma unroll
    for (int i = 0; i < kRecycleSums; ++i) {
        const double v = warp_sum(acc[i]);
        if (lane == 0) wpart[wp][i] = v;
    }
    __syncthreads();
    if (threadIdx.x < kRecycleSums) {
        double t = 0.0;
        for (int q = 0; q < nwarps; ++q) t += wpart[q][threadIdx.x];
        a.partials[(size_t)blockIdx.x * kRecycleStride + threadIdx.x] = t;
    }
    if (last_block_arrive(a.ticket, &last)) {
        if (threadIdx.x < kRecycleSums) {
            const volatile double* p = a.partials;
            double t = 0.0;
            for (int q = 0; q < (int)gridDim.x; ++q) t += p[(size_t)q * kRecycleStride + threadIdx.x];
            tot[threadIdx.x] = t;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            small_solve(tot, cnt, a.y);
            *a.ticket = 0;
        }
    }
}

// u0 = u; u += sum_j y_j w_j (fixed order).
__global__ void __launch_bounds__(kRecThreads) k_recycle_apply(RecycleArgs a) {
    __shared__ double ys[kRecycleMax];
    if (threadIdx.x < kRecycleMax) ys[threadIdx.x] = (int)threadIdx.x < a.cnt ? a.y[threadIdx.x] : 0.0;
    __syncthreads();
    for (int nd = blockIdx.x * blockDim.x + threadIdx.x; nd < a.n; nd += gridDim.x * blockDim.x) {
        const double2 c = a.u[nd];
        a.u0[nd] = c;
        double2 x = c;
#pragma unroll
        for (int j = 0; j < kRecycleMax; ++j)
            if (j < a.cnt) {
                const double2 w = a.w[(size_t)a.slot[j] * a.n + nd];
                x.x += ys[j] * w.x;
                x.y += ys[j] * w.y;
            }
        a.u[nd] = x;
    }
}

__global__ void __launch_bounds__(kRecThreads) k_recycle_push(RecycleArgs a, int slot) {
    double2* __restrict__ w = a.w + (size_t)slot * a.n;
    for (int nd = blockIdx.x * blockDim.x + threadIdx.x; nd < a.n; nd += gridDim.x * blockDim.x) {
        const double2 c = a.u[nd], p = a.u0[nd];
        w[nd] = make_double2(c.x - p.x, c.y - p.y);
    }
}

int node_grid(int n, int sm_count) {
    const long long g = ((long long)n + kRecThreads - 1) / kRecThreads;
    const long long cap = 8LL * sm_count;
    return (int)std::max<long long>(1, std::min(g, cap));
}

}  // namespace

int recycle_grid(int n, int sm_count) {
    const long long g = ((long long)n + kRecThreads - 1) / kRecThreads;
    const long long cap = 4LL * sm_count;
    return (int)std::max<long long>(1, std::min(g, cap));
}

void recycle_project(const RecycleArgs& a, int sm_count, cudaStream_t s) {
    CP_CHECK(a.cnt >= 0 && a.cnt <= kRecycleMax, CP_ERR_INVALID, "recycle: bad increment count");
    for (int j = 0; j < a.cnt; ++j)
        CP_CHECK(a.slot[j] >= 0 && a.slot[j] < kRecycleMax, CP_ERR_INVALID, "recycle: bad slot");
    if (a.cnt > 0) {
        k_recycle_sums<<<recycle_grid(a.n, sm_count), kRecThreads, 0, s>>>(a);
        CP_CUDA(cudaGetLastError());
    }
    k_recycle_apply<<<node_grid(a.n, sm_count), kRecThreads, 0, s>>>(a);
    CP_CUDA(cudaGetLastError());
}

int recycle_solve_host(const double* sums, int cnt, double* y) {
    if (!sums || !y || cnt < 0 || cnt > kRecycleMax) return CP_ERR_INVALID;
    small_solve(sums, cnt, y);
    return CP_OK;
}

void recycle_push(const RecycleArgs& a, int slot, int sm_count, cudaStream_t s) {
    CP_CHECK(slot >= 0 && slot < kRecycleMax, CP_ERR_INVALID, "recycle: bad slot");
    k_recycle_push<<<node_grid(a.n, sm_count), kRecThreads, 0, s>>>(a, slot);
    CP_CUDA(cudaGetLastError());
}

}  // namespace cp

CP_API int cpx_recycle_solve(const double* sums, int cnt, double* y) { return cp::recycle_solve_host(sums, cnt, y); }
