// FP64 masked (P)CG of one small instance inside one thread-block cluster.
//
// Same solve as the single-launch iteration of cg_fused.cu (ConjGradCuda::solve,
// src/ConjGradCuda.cu:185-231, in the Chronopoulos-Gear arrangement described
// there), for instances small enough that one cluster of up to 16 CTAs holds
// the whole problem on chip:
//   - CTA `rank` owns the slices [rank spc, (rank + 1) spc) of 32 nodes, one
//     warp per slice and one node per thread; that thread keeps its node's x,
//     r, p, w, kp, u, M w, M kp, b and M in registers for the whole solve;
//   - the CTA's blocks of K (values and the neighbours' owner / local index)
//     are copied into its shared memory once per solve;
//   - each node publishes its record (u, M w, M kp) in its CTA's shared
//     memory, double-buffered by iteration parity; neighbours read it through
//     distributed shared memory;
//   - an iteration ends with one hardware cluster barrier, which also
//     publishes the records and the CTAs' partial sums; every CTA then reduces
//     the partial sums of all CTAs in rank order itself, so all of them hold
//     the same scalars and take the same branches (no second barrier, no
//     global memory round trip, no spin-wait).
// The summation order differs from the grid-wide kernels (other partition),
// so the iterates agree with them to rounding, not bit for bit.
#include <cooperative_groups.h>

#include <cstdlib>

#include "cg.h"
#include "common.cuh"
#include "internal.h"

namespace cp {

namespace {

namespace cgr = cooperative_groups;

constexpr int kMaxCluster = 16;
constexpr int kMaxWarps = 16;  // slices per CTA (512 threads)
constexpr int kSums = 5;
constexpr int kSmemCap = 220 * 1024;  // dynamic shared memory per CTA

__device__ __forceinline__ double2 mvec(const double4& m, double2 v) {
    return make_double2(m.x * v.x + m.y * v.y, m.z * v.x + m.w * v.y);
}

// Shared memory of one CTA (dynamic part):
//   kval [spc][wmax][32] double4  block values, 2x2 row-major
//   rec  [2][spc * 32][3] double2 published (u, M w, M kp) by parity
//   part [2][8] double            this CTA's partial sums by parity
//   kloc [spc][wmax][32] int      owner rank << 16 | owner-local node index
struct Smem {
    double4* kval;
    int* kloc;
    double2* rec;
    double* part;
};

__device__ __forceinline__ Smem carve(unsigned char* base, int spc, int wmax) {
    Smem s;
    const size_t nb = (size_t)spc * wmax * 32;
    s.kval = reinterpret_cast<double4*>(base);
    s.rec = reinterpret_cast<double2*>(base + nb * sizeof(double4));
    s.part = reinterpret_cast<double*>(base + nb * sizeof(double4) + 2 * (size_t)spc * 32 * 3 * sizeof(double2));
    s.kloc = reinterpret_cast<int*>(base + nb * sizeof(double4) + 2 * (size_t)spc * 32 * 3 * sizeof(double2) +
                                    16 * sizeof(double));
    return s;
}

size_t smem_bytes(int spc, int wmax) {
    const size_t nb = (size_t)spc * wmax * 32;
    return nb * sizeof(double4) + 2 * (size_t)spc * 32 * 3 * sizeof(double2) + 16 * sizeof(double) + nb * sizeof(int);
}

// Block-wide sums of kSums values per thread into part[0..kSums) of this CTA
// (thread 0 writes), same fixed tree in every CTA.
__device__ __forceinline__ void cta_sums(const double* v, double* part, double (*wsum)[8]) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int i = 0; i < kSums; ++i) {
        const double s = warp_sum(v[i]);
        if (lane == 0) wsum[w][i] = s;
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int i = 0; i < kSums; ++i) {
            const double s = warp_sum(lane < nw ? wsum[lane][i] : 0.0);
            if (lane == 0) part[i] = s;
        }
    }
}

// After the cluster barrier: totals over all CTAs, in rank order through a
// fixed shuffle tree (identical in every CTA), broadcast to the block.
__device__ __forceinline__ void cluster_totals(double* const* part_of, int ctas, double* tot) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (w == 0) {
#pragma unroll
        for (int i = 0; i < kSums; ++i) {
            const double s = warp_sum(lane < ctas ? part_of[lane][i] : 0.0);
            if (lane == 0) tot[i] = s;
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kMaxWarps * 32, 1)
    k_c_solve(FusedArgs a, ClusterPlan shp, double eps2, long long max_iter) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double wsum[kMaxWarps][8];
    __shared__ double tot[8];
    __shared__ double2* rec_of[kMaxCluster];
    __shared__ double* part_of[2][kMaxCluster];

    cgr::cluster_group cl = cgr::this_cluster();
    const int rank = (int)cl.block_rank();
    const int spc = shp.spc, wmax = shp.wmax, ctas = shp.ctas;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int n_slices = (a.n + 31) / 32;
    const int sl = rank * spc + w;
    const int n = 32 * sl + lane;
    const bool act = sl < n_slices && n < a.n;
    const int loc = w * 32 + lane;  // this node's index inside the CTA
    Smem S = carve(smem_raw, spc, wmax);
    if (threadIdx.x < ctas) {
        rec_of[threadIdx.x] = cl.map_shared_rank(S.rec, (int)threadIdx.x);
        part_of[0][threadIdx.x] = cl.map_shared_rank(S.part, (int)threadIdx.x);
        part_of[1][threadIdx.x] = cl.map_shared_rank(S.part + 8, (int)threadIdx.x);
    }
    const size_t rec_half = (size_t)spc * 32 * 3;  // double2 per parity buffer

    // ---- this thread's row blocks into shared memory
    int wd = 0;
    if (sl < n_slices) wd = (a.slice_ptr[sl + 1] - a.slice_ptr[sl]) >> 5;
    if (act) {
        const int base = a.slice_ptr[sl];
        for (int k = 0; k < wd; ++k) {
            const long long bi = base + 32LL * k + lane;
            const int col = __ldg(a.scol + bi);
            const double2 lo = __ldg(reinterpret_cast<const double2*>(a.val + 4 * bi));
            const double2 hi = __ldg(reinterpret_cast<const double2*>(a.val + 4 * bi) + 1);
            const int cr = (col >> 5) / spc;
            const size_t q = ((size_t)w * wmax + k) * 32 + lane;
            S.kval[q] = make_double4(lo.x, lo.y, hi.x, hi.y);
            S.kloc[q] = (cr << 16) | (col - cr * spc * 32);
        }
    }
    // ---- own data in registers
    double2 x = make_double2(0.0, 0.0), bb = x, r = x, p = x, kp = x, wv = x, u = x, mw = x, mk = x;
    uchar2 m = make_uchar2(0, 0);
    double4 minv = make_double4(0.0, 0.0, 0.0, 0.0);
    if (act) {
        x = a.x[n];
        bb = a.b[n];
        m = a.mask[n];
        // x goes out through the parity-1 buffer for the initial residual
        S.rec[rec_half + 3 * (size_t)loc] = x;
    }
    cl.sync();

    auto apply_m = [&](double2 v) {
        if (a.precond) return mvec(minv, v);
        return make_double2(m.x ? v.x : 0.0, m.y ? v.y : 0.0);
    };
    // sum_k K_k f(record of column k), f picking from the neighbour's record
    auto gather_x = [&](size_t half) {
        double k0 = 0.0, k1 = 0.0;
        for (int k = 0; k < wd; ++k) {
            const size_t q = ((size_t)w * wmax + k) * 32 + lane;
            const double4 kv = S.kval[q];
            const int lc = S.kloc[q];
            const double2 v = rec_of[lc >> 16][half + 3 * (size_t)(lc & 0xffff)];
            k0 += kv.x * v.x + kv.y * v.y;
            k1 += kv.z * v.x + kv.w * v.y;
        }
        return make_double2(k0, k1);
    };

    double v[kSums] = {0.0, 0.0, 0.0, 0.0, 0.0};
    // ---- init: r = m.(b - K x), M, u = M r, record parity 0 = (u, -, 0)
    if (act) {
        const double2 kx = gather_x(rec_half);
        r = make_double2(m.x ? bb.x - kx.x : 0.0, m.y ? bb.y - kx.y : 0.0);
        if (a.precond) {
            const double4 d = S.kval[((size_t)w * wmax) * 32 + lane];  // block 0: the diagonal block
            if (m.x && m.y) {
                const double det = d.x * d.w - d.y * d.z;
                minv = make_double4(d.w / det, -d.y / det, -d.z / det, d.x / det);
            } else if (m.x) {
                minv.x = 1.0 / d.x;
            } else if (m.y) {
                minv.w = 1.0 / d.w;
            }
        }
        u = apply_m(r);
        S.rec[3 * (size_t)loc] = u;
        S.rec[3 * (size_t)loc + 2] = make_double2(0.0, 0.0);
        v[0] = r.x * r.x + r.y * r.y;
        v[1] = bb.x * bb.x + bb.y * bb.y;
    }
    cta_sums(v, S.part, wsum);
    cl.sync();
    cluster_totals(part_of[0], ctas, tot);
    const double rr0 = tot[0], bnorm2 = tot[1];
    const double normB_inv = bnorm2 > 0.0 ? 1.0 / bnorm2 : 0.0;
    int status = 0, converged = (rr0 == 0.0 || rr0 * normB_inv <= eps2) ? 1 : 0;
    if (!(rr0 == rr0) || !(bnorm2 == bnorm2)) status = CP_ERR_BREAKDOWN;
    double rr = rr0, rho = 0.0, alpha = 0.0, beta = 0.0;
    long long iter = 0;
    // ---- first step: w = K u, M w into the record; gamma = (r, u), delta = (w, u)
    if (!converged && !status) {
        v[0] = v[1] = 0.0;
        if (act) {
            wv = gather_x(0);
            mw = apply_m(wv);
            S.rec[3 * (size_t)loc + 1] = mw;
            v[0] = r.x * u.x + r.y * u.y;
            v[1] = wv.x * u.x + wv.y * u.y;
        }
        cta_sums(v, S.part + 8, wsum);
        cl.sync();
        cluster_totals(part_of[1], ctas, tot);
        rho = tot[0];
        alpha = tot[0] / tot[1];
        if (!(tot[1] > 0.0) || !(alpha == alpha)) status = CP_ERR_BREAKDOWN;
    }
    // ---- iterations (see cg_fused.cu for the recurrences)
    int parity = 0;
    while (!converged && !status) {
        const size_t go = parity ? rec_half : 0, gn = parity ? 0 : rec_half;
        double t[kSums] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (act) {
            const double al = alpha, bt = beta;
            const double2 u0 = u;
            p = make_double2(u0.x + bt * p.x, u0.y + bt * p.y);
            kp = make_double2(wv.x + bt * kp.x, wv.y + bt * kp.y);
            u = make_double2(u0.x - al * (mw.x + bt * mk.x), u0.y - al * (mw.y + bt * mk.y));
            x.x += al * p.x;
            x.y += al * p.y;
            if (m.x) r.x -= al * kp.x;
            if (m.y) r.y -= al * kp.y;
            double k0 = 0.0, k1 = 0.0;
            for (int k = 0; k < wd; ++k) {
                const size_t q = ((size_t)w * wmax + k) * 32 + lane;
                const double4 kv = S.kval[q];
                const int lc = S.kloc[q];
                const double2* rc = rec_of[lc >> 16] + go + 3 * (size_t)(lc & 0xffff);
                const double2 uc = rc[0], mwc = rc[1], mkc = rc[2];
                const double ux = uc.x - al * (mwc.x + bt * mkc.x), uy = uc.y - al * (mwc.y + bt * mkc.y);
                k0 += kv.x * ux + kv.y * uy;
                k1 += kv.z * ux + kv.w * uy;
            }
            wv = make_double2(k0, k1);
            mw = apply_m(wv);
            mk = apply_m(kp);
            S.rec[gn + 3 * (size_t)loc] = u;
            S.rec[gn + 3 * (size_t)loc + 1] = mw;
            S.rec[gn + 3 * (size_t)loc + 2] = mk;
            t[0] = r.x * u.x + r.y * u.y;
            t[1] = wv.x * u.x + wv.y * u.y;
            t[2] = r.x * r.x + r.y * r.y;
            t[3] = (wv.x * p.x + wv.y * p.y) + (kp.x * u.x + kp.y * u.y);
            t[4] = kp.x * p.x + kp.y * p.y;
        }
        // this CTA's partials go to the buffer of this parity; the barrier
        // publishes them with the records
        cta_sums(t, S.part + 8 * parity, wsum);
        cl.sync();
        cluster_totals(part_of[parity], ctas, tot);
        const double g = tot[0], rn = tot[2];
        const double b2 = g / rho;
        const double den = tot[1] + b2 * tot[3] + b2 * b2 * tot[4];
        ++iter;
        rr = rn;
        beta = b2;
        alpha = g / den;
        rho = g;
        if (rn * normB_inv <= eps2) converged = 1;
        else if (iter >= max_iter) status = CP_ERR_NOT_CONVERGED;
        else if (!(den > 0.0) || !(g > 0.0)) status = CP_ERR_BREAKDOWN;
        if (!(rn == rn)) status = CP_ERR_BREAKDOWN;
        parity ^= 1;
    }
    // every CTA has read the others' shared memory for the last time
    cl.sync();
    if (act) a.x[n] = x;
    if (rank == 0 && threadIdx.x == 0) {
        CgScalars* sc = a.sc;
        sc->rr = rr;
        sc->bb = bnorm2;
        sc->res64 = rr0;
        sc->normB_inv = normB_inv;
        sc->eps2 = eps2;
        sc->iter = iter;
        sc->max_iter = max_iter;
        sc->converged = converged;
        sc->status = status;
        sc->lin_done = 0;
        sc->alpha = alpha;
        sc->beta = beta;
        sc->rho = rho;
        sc->ticket = 0;
    }
}

// Sets the launch attributes of kernel k and checks that a cluster of the
// shape can be scheduled.
template <typename K>
bool cluster_fits(K k, int ctas, int spc, size_t smem) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ctas);
    cfg.blockDim = dim3(32 * spc);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = ctas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (ctas > 8 && cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    // the cap, not this instance's size: the attribute is per function and
    // instances of other sizes launch the same kernel
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemCap) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, k, &cfg) != cudaSuccess || clusters < 1) {
        cudaGetLastError();
        return false;
    }
    return true;
}

template <typename K>
void launch_cluster(K k, const FusedArgs& a, const ClusterPlan& shp, double eps2, long long max_iter,
                    cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(shp.ctas);
    cfg.blockDim = dim3(32 * shp.spc);
    cfg.dynamicSmemBytes = shp.smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = shp.ctas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CP_CUDA(cudaLaunchKernelEx(&cfg, k, a, shp, eps2, max_iter));
}

}  // namespace

// The cluster shape for an instance, or ctas = 0 when it does not fit.
ClusterPlan cluster_cg_plan(const FusedArgs& a, int wmax) {
    ClusterPlan s;
    const int n_slices = (a.n + 31) / 32;
    // Cluster sizes tried in order: first the fewest CTAs whose share is at
    // most kPrefSlices slices (warps), then 16 and 8. Fewer, fuller CTAs keep
    // more neighbours in the CTA's own shared memory and sum fewer partials
    // across the cluster: on configuration 1 (130 slices) 11 CTAs of 12 warps
    // took 5.7 us per CG iteration against 6.1 with 16 CTAs of 9 (13: 6.1,
    // 9: 6.1). CUPLAST_CLUSTER_CTAS = 1..16 forces one size (measurements).
    constexpr int kPrefSlices = 12;
    int order[3] = {(n_slices + kPrefSlices - 1) / kPrefSlices, 16, 8}, n_order = 3;
    if (order[0] > kMaxCluster) {
        order[0] = 16;
        n_order = 2;  // too large for the preferred share: 16 CTAs, then 8
        order[1] = 8;
    }
    if (const char* e = std::getenv("CUPLAST_CLUSTER_CTAS")) {
        const int c = std::atoi(e);
        if (c >= 1 && c <= kMaxCluster) {
            order[0] = c;
            n_order = 1;
        }
    }
    for (int oi = 0; oi < n_order; ++oi) {
        const int ctas = order[oi];
        const int spc = (n_slices + ctas - 1) / ctas;
        if (spc > kMaxWarps) continue;
        const size_t smem = smem_bytes(spc, wmax);
        if (smem > (size_t)kSmemCap) continue;
        if (!cluster_fits(k_c_solve, ctas, spc, smem)) continue;
        s.ctas = ctas;
        s.spc = spc;
        s.wmax = wmax;
        s.smem = smem;
        return s;
    }
    return s;
}

void cluster_cg_launch(const FusedArgs& a, const ClusterPlan& shp, double eps2, long long max_iter, cudaStream_t s) {
    CP_CHECK(shp.ctas > 0 && shp.spc * 32 * shp.ctas >= a.n, CP_ERR_INVALID,
             "cluster CG: the instance does not fit one cluster");
    launch_cluster(k_c_solve, a, shp, eps2, max_iter, s);
}

}  // namespace cp
