// Element kernels: stiffness assembly into the node-blocked CSR, the fused
// strain / stress / secant update with the exit norm, Aitken relaxation of the
// secant iteration, and the plastic-strain post-processing.
//
// Element geometry is recomputed from node coordinates in every kernel (the
// reference stores B and detJ per Gauss point, 288 B per quad, computed once
// by calcBs4, src/PlasticitySolver.cu:139-144,1237-1246); reading 4 node
// coordinates costs less HBM traffic than reading B back.
#include <mutex>

#include "common.cuh"
#include "internal.h"

namespace cp {

namespace {

constexpr double kGp = 0.577350269189626;  // 2x2 Gauss points, src/PlasticitySolver.cu:14

// formC_plainStress / formC_plainStrain (src/PlasticitySolver.cu:226-242),
// same operation order. Only C00, C01, C11, C22 are non-zero.
struct Dmat {
    double c00, c01, c11, c22;
};
__device__ __forceinline__ Dmat form_d(int plane, double E, double nu) {
    Dmat d;
    if (plane == CP_PLANE_STRESS) {
        double coef = E / (1.0 - nu * nu);
        d.c00 = 1.0 * coef;
        d.c11 = 1.0 * coef;
        d.c01 = nu * coef;
        d.c22 = ((1.0 - nu) * 0.5) * coef;
    } else {
        double coef = E * (1. - nu) / ((1. + nu) * (1 - 2. * nu));
        d.c00 = 1.0 * coef;
        d.c11 = 1.0 * coef;
        d.c01 = (nu / (1. - nu)) * coef;
        d.c22 = ((1. - 2. * nu) * 0.5 / (1. - nu)) * coef;
    }
    return d;
}

// calcB4 (src/PlasticitySolver.cu:26-64) at Gauss point (r, s): shape-function
// gradients bx[k] = dN_k/dx, by[k] = dN_k/dy and detJ.
__device__ __forceinline__ double q4_grad(const double* x, const double* y, double r, double s, double* bx,
                                          double* by) {
    double J0 = 0.25 * ((1. + s) * x[0] - (1. + s) * x[1] - (1. - s) * x[2] + (1. - s) * x[3]);
    double J2 = 0.25 * ((1. + r) * x[0] + (1. - r) * x[1] - (1. - r) * x[2] - (1. + r) * x[3]);
    double J1 = 0.25 * ((1. + s) * y[0] - (1. + s) * y[1] - (1. - s) * y[2] + (1. - s) * y[3]);
    double J3 = 0.25 * ((1. + r) * y[0] + (1. - r) * y[1] - (1. - r) * y[2] - (1. + r) * y[3]);
    double det = J0 * J3 - J1 * J2;
    double inv = 1. / det;
    double i0 = J3 * inv, i1 = -J1 * inv, i2 = -J2 * inv, i3 = J0 * inv;
    bx[0] = 0.25 * ((1. + s) * i0 + (1. + r) * i1);
    by[0] = 0.25 * ((1. + s) * i2 + (1. + r) * i3);
    bx[1] = 0.25 * ((-1. - s) * i0 + (1. - r) * i1);
    by[1] = 0.25 * ((-1. - s) * i2 + (1. - r) * i3);
    bx[2] = 0.25 * ((-1. + s) * i0 - (1. - r) * i1);
    by[2] = 0.25 * ((-1. + s) * i2 - (1. - r) * i3);
    bx[3] = 0.25 * ((1. - s) * i0 - (1. + r) * i1);
    by[3] = 0.25 * ((1. - s) * i2 - (1. + r) * i3);
    return det;
}

// CST gradients (no reference counterpart: calcB3 is only declared,
// src/PlasticitySolver.cu:21-23). Returns the signed area.
__device__ __forceinline__ double t3_grad(const double* x, const double* y, double* bx, double* by) {
    double twoA = (x[1] - x[0]) * (y[2] - y[0]) - (x[2] - x[0]) * (y[1] - y[0]);
    double inv = 1.0 / twoA;
    bx[0] = (y[1] - y[2]) * inv;
    bx[1] = (y[2] - y[0]) * inv;
    bx[2] = (y[0] - y[1]) * inv;
    by[0] = (x[2] - x[1]) * inv;
    by[1] = (x[0] - x[2]) * inv;
    by[2] = (x[1] - x[0]) * inv;
    return 0.5 * twoA;
}

// Adds w * (B_i^T D B_j) to the 2x2 block acc. Written with the pair products
// first so that block (i,j) of one thread is exactly the transpose of block
// (j,i) of another: K stays bitwise symmetric.
// Explicitly rounded operations (no FMA contraction), so that the compiler
// cannot fuse the two mirrored expressions differently.
__device__ __forceinline__ double sym_term(double p, double c, double q, double e, double w) {
    return __dmul_rn(__dadd_rn(__dmul_rn(p, c), __dmul_rn(q, e)), w);
}
__device__ __forceinline__ void add_block(double* acc, double bxi, double byi, double bxj, double byj, const Dmat& d,
                                          double w) {
    const double pxx = __dmul_rn(bxi, bxj), pyy = __dmul_rn(byi, byj);
    const double pxy = __dmul_rn(bxi, byj), pyx = __dmul_rn(byi, bxj);
    acc[0] = __dadd_rn(acc[0], sym_term(pxx, d.c00, pyy, d.c22, w));
    acc[1] = __dadd_rn(acc[1], sym_term(pxy, d.c01, pyx, d.c22, w));
    acc[2] = __dadd_rn(acc[2], sym_term(pyx, d.c01, pxy, d.c22, w));
    acc[3] = __dadd_rn(acc[3], sym_term(pyy, d.c11, pxx, d.c22, w));
}

__device__ __forceinline__ int nth(const int4& v, int j) {
    return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w));
}

// Row-block (i, all j) of element e's stiffness, scaled by h, added into the
// owning node's 2x2 blocks through the slot bytes kk (block index k of local
// node j); block k of the node starts at nb + 128 k (sliced layout, 32 nodes
// x 4 values per block row).
__device__ __forceinline__ void add_scaled(double* b, const double* blk, double h) {
    b[0] = __dadd_rn(b[0], __dmul_rn(blk[0], h));
    b[1] = __dadd_rn(b[1], __dmul_rn(blk[1], h));
    b[2] = __dadd_rn(b[2], __dmul_rn(blk[2], h));
    b[3] = __dadd_rn(b[3], __dmul_rn(blk[3], h));
}

__device__ __forceinline__ void element_rows(const DevMesh& m, int e, int i, uint32_t kk, const Dmat& d, double h,
                                             double* nb) {
    double x[4], y[4];
    if (e < m.c3) {
        int4 el = m.e3[e];
        for (int a = 0; a < 3; ++a) {
            double2 p = m.xy[nth(el, a)];
            x[a] = p.x;
            y[a] = p.y;
        }
        double bx[3], by[3];
        double area = t3_grad(x, y, bx, by);
        double blk[3][4] = {};
#pragma unroll
        for (int j = 0; j < 3; ++j) add_block(blk[j], bx[i], by[i], bx[j], by[j], d, area);
#pragma unroll
        for (int j = 0; j < 3; ++j) add_scaled(nb + 128 * (int)((kk >> (8 * j)) & 0xffu), blk[j], h);
    } else {
        int4 el = m.e4[e - m.c3];
        for (int a = 0; a < 4; ++a) {
            double2 p = m.xy[nth(el, a)];
            x[a] = p.x;
            y[a] = p.y;
        }
        double blk[4][4] = {};
#pragma unroll
        for (int gi = 0; gi < 2; ++gi)
#pragma unroll
            for (int gj = 0; gj < 2; ++gj) {
                double bx[4], by[4];
                double r = gi ? kGp : -kGp, s = gj ? kGp : -kGp;
                double det = q4_grad(x, y, r, s, bx, by);
                double bxi = bx[0], byi = by[0];
                if (i == 1) { bxi = bx[1]; byi = by[1]; }
                else if (i == 2) { bxi = bx[2]; byi = by[2]; }
                else if (i == 3) { bxi = bx[3]; byi = by[3]; }
#pragma unroll
                for (int j = 0; j < 4; ++j) add_block(blk[j], bxi, byi, bx[j], by[j], d, det);
            }
#pragma unroll
        for (int j = 0; j < 4; ++j) add_scaled(nb + 128 * (int)((kk >> (8 * j)) & 0xffu), blk[j], h);
    }
}

constexpr int kAsmThreads = 128;  // = 4 slices of 32 nodes

// One thread per node, one block per tile of 4 slices. The tile's blocks are
// one contiguous range of values in the sliced layout, accumulated in shared
// memory (each thread only touches its own node's blocks: no atomics, and the
// summation order is the element order) and written out coalesced, once.
template <bool W64, bool W32>
__global__ void __launch_bounds__(kAsmThreads) k_assemble(DevMesh m, DevCsr csr, MaterialDev M, const double* E_c,
                                                          const double* nu_c) {
    extern __shared__ double sacc[];
    const int ntiles = (m.n_nodes + kAsmThreads - 1) / kAsmThreads;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int s0 = 4 * tile, s1 = min(s0 + 4, csr.n_slices);
        const long long B0 = csr.slice_ptr[s0], B1 = csr.slice_ptr[s1];
        const int len = (int)(4 * (B1 - B0));
        for (int t = threadIdx.x; t < len; t += blockDim.x) sacc[t] = 0.0;
        __syncthreads();
        const int n = tile * kAsmThreads + threadIdx.x;
        if (n < m.n_nodes) {
            double* nb = sacc + 4 * (csr.slice_ptr[n >> 5] - B0 + (n & 31));
            for (int q = csr.inc_pos[n]; q < csr.inc_pos[n + 1]; ++q) {
                const int code = csr.inc[q];
                const int e = code >> 2, i = code & 3;
                const Dmat d = form_d(M.plane, E_c[e], nu_c[e]);
                element_rows(m, e, i, csr.inc_k[q], d, M.h, nb);
            }
        }
        __syncthreads();
        double* out64 = csr.val64 + 4 * B0;
        float* out32 = W32 ? csr.val32 + 4 * B0 : nullptr;
        for (int t = threadIdx.x; t < len; t += blockDim.x) {
            double v = sacc[t];
            if (W64) out64[t] = v;
            if (W32) out32[t] = (float)v;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- diagram --
// sigma = f(eps_i): Material::f / dev_f (src/Material.cu:3-23) and the
// injected diagrams; compile-time dispatch on M.diagram (no device function
// pointers, cf. src/Material.cu:25-26).
__device__ double diagram_f(const MaterialDev& M, double eps) {
    const double E = M.E;
    switch (M.diagram) {
    case CP_DIAGRAM_LINEAR: {
        double epsT = M.sigma_t / E;
        return eps < epsT ? eps * E : M.sigma_t + (eps - epsT) * M.k_t;
    }
    case CP_DIAGRAM_POWER: {
        double epsT = M.sigma_t / E, A = M.a, mm = M.m;
        return eps < epsT ? eps * E
                          : M.sigma_t + A * pow(eps - epsT + pow(E / (A * mm), 1. / (mm - 1.)), mm) -
                                A * pow(E / (A * mm), mm / (mm - 1.));
    }
    case CP_DIAGRAM_HOLLOMON: {
        // eps = s/E + eps0((s/sy)^(1/n) - 1), inverted by Newton from s = sy
        double sy = M.sigma_t, e0 = M.eps0, n = M.n, s = sy;
        if (eps < sy / E) return eps * E;
        for (int it = 0; it < 200; ++it) {
            double t = pow(s / sy, 1.0 / n);
            double g = s / E + e0 * (t - 1.0) - eps;
            double dg = 1.0 / E + e0 * t / (n * s);
            double ds = g / dg;
            s -= ds;
            if (fabs(ds) <= 1e-15 * s) break;
        }
        return s;
    }
    case CP_DIAGRAM_PIECEWISE: {
        if (eps < M.pw_eps[0]) return eps * E;
        int k = 0;
        while (k + 1 < M.n_points - 1 && eps >= M.pw_eps[k + 1]) ++k;
        double slope = (M.pw_sig[k + 1] - M.pw_sig[k]) / (M.pw_eps[k + 1] - M.pw_eps[k]);
        return M.pw_sig[k] + (eps - M.pw_eps[k]) * slope;
    }
    default:
        return eps * E;
    }
}

}  // namespace
constexpr int kElemThreads = 256;

// strain4 + plastStress + exitNorm2 (src/PlasticitySolver.cu:1517-1549,
// 1590-1610, 1664-1691) fused: element-mean strain, stress from the C of the
// last assembly, stress intensity, secant update, and the two exit-norm sums
// (reduced deterministically by the last block). With Aitken on, the raw
// secant target psi is stored as a residual and the relax kernel moves psi.
__global__ void __launch_bounds__(kElemThreads) k_update(DevMesh m, MaterialDev M, const double2* __restrict__ u,
                                                         ElemState st, OuterScalars* sc, double* partials, int aitken) {
    __shared__ double sh[2 * kElemThreads / 32];
    __shared__ bool last;
    const int ne = m.c3 + m.c4;
    double s_num = 0.0, s_den = 0.0, s_an = 0.0, s_ad = 0.0;
    const double E0 = M.E, nu0 = M.nu;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
        double ex, ey, g;
        if (e < m.c3) {
            int4 el = m.e3[e];
            double x[3], y[3], uu[3], vv[3], bx[3], by[3];
            for (int a = 0; a < 3; ++a) {
                int nd = nth(el, a);
                double2 p = m.xy[nd], w = u[nd];
                x[a] = p.x; y[a] = p.y; uu[a] = w.x; vv[a] = w.y;
            }
            t3_grad(x, y, bx, by);
            ex = uu[0] * bx[0] + uu[1] * bx[1] + uu[2] * bx[2];
            ey = vv[0] * by[0] + vv[1] * by[1] + vv[2] * by[2];
            g = uu[0] * by[0] + uu[1] * by[1] + uu[2] * by[2] + vv[0] * bx[0] + vv[1] * bx[1] + vv[2] * bx[2];
        } else {
            int4 el = m.e4[e - m.c3];
            double x[4], y[4], uu[4], vv[4];
            for (int a = 0; a < 4; ++a) {
                int nd = nth(el, a);
                double2 p = m.xy[nd], w = u[nd];
                x[a] = p.x; y[a] = p.y; uu[a] = w.x; vv[a] = w.y;
            }
            ex = 0.0; ey = 0.0; g = 0.0;
#pragma unroll
            for (int gi = 0; gi < 2; ++gi)
#pragma unroll
                for (int gj = 0; gj < 2; ++gj) {
                    double bx[4], by[4];
                    q4_grad(x, y, gi ? kGp : -kGp, gj ? kGp : -kGp, bx, by);
                    ex += uu[0] * bx[0] + uu[1] * bx[1] + uu[2] * bx[2] + uu[3] * bx[3];
                    ey += vv[0] * by[0] + vv[1] * by[1] + vv[2] * by[2] + vv[3] * by[3];
                    g += uu[0] * by[0] + uu[1] * by[1] + uu[2] * by[2] + uu[3] * by[3] + vv[0] * bx[0] +
                         vv[1] * bx[1] + vv[2] * bx[2] + vv[3] * bx[3];
                }
            ex *= 0.25; ey *= 0.25; g *= 0.25;
        }
        const double Ec = st.E_c[e];
        const Dmat d = form_d(M.plane, Ec, st.nu_c[e]);
        const double sx = d.c00 * ex + d.c01 * ey;
        const double sy = d.c01 * ex + d.c11 * ey;
        const double t = d.c22 * g;
        const double sI = sqrt(0.5 * (sx * sx + sy * sy + (sx - sy) * (sx - sy) + 6. * (t * t)));
        const double eI = sI / Ec;
        const double tab = diagram_f(M, eI);
        const double ps = E0 * eI / tab;
        st.exx[e] = ex; st.eyy[e] = ey; st.gam[e] = g;
        st.sxx[e] = sx; st.syy[e] = sy; st.tau[e] = t;
        st.sig_i[e] = sI; st.eps_i[e] = eI; st.table_s[e] = tab;
        const double diff = sI - tab;
        s_num += diff * diff;
        s_den += tab * tab;
        if (!aitken) {
            st.psi[e] = ps;
            st.E_c[e] = E0 / ps;
            st.nu_c[e] = 0.5 * (1. - (1. - 2. * nu0) / ps);
        } else {
            const double r = (ps == ps) ? ps - st.psi[e] : 0.0;
            const double dr = r - st.res_prev[e];
            st.res_cur[e] = r;
            s_an += st.res_prev[e] * dr;
            s_ad += dr * dr;
        }
    }
    double2 a = block_sum2(s_num, s_den, sh);
    double2 b = aitken ? block_sum2(s_an, s_ad, sh) : make_double2(0.0, 0.0);
    if (threadIdx.x == 0) {
        partials[4 * blockIdx.x + 0] = a.x;
        partials[4 * blockIdx.x + 1] = a.y;
        partials[4 * blockIdx.x + 2] = b.x;
        partials[4 * blockIdx.x + 3] = b.y;
    }
    if (last_block_arrive(&sc->ticket, &last)) {
        double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
        for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
            const volatile double* p = partials + 4 * i;
            t0 += p[0]; t1 += p[1]; t2 += p[2]; t3 += p[3];
        }
        double2 x = block_sum2(t0, t1, sh);
        double2 y = block_sum2(t2, t3, sh);
        if (threadIdx.x == 0) {
            sc->num = x.x;
            sc->den = x.y;
            sc->rel_err = sqrt(x.x / x.y);
            sc->a_num = y.x;
            sc->a_den = y.y;
            sc->ticket = 0;
        }
    }
}

namespace {

// Aitken (Irons-Tuck) relaxation of the secant iteration on psi:
// psi_{k+1} = psi_k + w_k r_k, w_k = -w_{k-1} (r_{k-1}, r_k - r_{k-1}) / |r_k - r_{k-1}|^2.
// The fixed point (r = 0) is the reference's.
__global__ void k_aitken(DevMesh m, MaterialDev M, ElemState st, const OuterScalars* sc, double w) {
    const int ne = m.c3 + m.c4;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
        const double r = st.res_cur[e];
        double ps = st.psi[e] + w * r;
        if (!(ps >= 1.0)) ps = 1.0;  // the secant modulus never exceeds E on a hardening diagram
        st.psi[e] = ps;
        st.E_c[e] = M.E / ps;
        st.nu_c[e] = 0.5 * (1. - (1. - 2. * M.nu) / ps);
        st.res_prev[e] = r;
    }
}

// plastDeform (src/PlasticitySolver.cu:1641-1653); the reference's guard is
// e > count (one past the end), here e < count.
__global__ void k_plastic(int ne, MaterialDev M, ElemState st) {
    const double E = M.E, G = M.E * 0.5 / (1. + M.nu);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
        const double Ec = st.E_c[e];
        const double xp = (1. / Ec - 1. / E) * st.sxx[e];
        const double yp = (1. / Ec - 1. / E) * st.syy[e];
        const double Gc = Ec * 0.5 / (1. + st.nu_c[e]);
        const double gp = (1. / Gc - 1. / G) * st.tau[e];
        st.exx_p[e] = xp;
        st.eyy_p[e] = yp;
        st.gam_p[e] = gp;
        st.eps_p_i[e] = sqrt(2.) / 3. * sqrt((xp - yp) * (xp - yp) + 6. * gp * gp);
        st.psi[e] = E / Ec;
    }
}

}  // namespace

void launch_assemble(const DevMesh& m, const DevCsr& csr, const MaterialDev& mat, const double* E_c,
                     const double* nu_c, bool want64, bool want32, cudaStream_t s, int sm_count) {
    const int ntiles = (m.n_nodes + kAsmThreads - 1) / kAsmThreads;
    const size_t smem = (size_t)kAsmThreads * 4 * csr.max_width * sizeof(double);
    CP_CHECK(smem <= 200 * 1024, CP_ERR_UNSUPPORTED, "node degree too large for the assembly tile");
    int grid = ntiles < sm_count * 8 ? ntiles : sm_count * 8;
    if (grid < 1) grid = 1;
    if (want64 && want32) {
        CP_CUDA(cudaFuncSetAttribute(k_assemble<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_assemble<true, true><<<grid, kAsmThreads, smem, s>>>(m, csr, mat, E_c, nu_c);
    } else if (want64) {
        CP_CUDA(cudaFuncSetAttribute(k_assemble<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_assemble<true, false><<<grid, kAsmThreads, smem, s>>>(m, csr, mat, E_c, nu_c);
    } else {
        CP_CUDA(cudaFuncSetAttribute(k_assemble<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_assemble<false, true><<<grid, kAsmThreads, smem, s>>>(m, csr, mat, E_c, nu_c);
    }
    CP_CUDA(cudaGetLastError());
}

int update_grid(int ne, int sm_count) {
    int g = (ne + kElemThreads - 1) / kElemThreads;
    int cap = sm_count * 4;
    return g < 1 ? 1 : (g < cap ? g : cap);
}

void launch_update(const DevMesh& m, const MaterialDev& mat, const double2* u, ElemState& st, OuterScalars* sc,
                   double* partials, int aitken, cudaStream_t s, int sm_count) {
    const int ne = m.c3 + m.c4;
    k_update<<<update_grid(ne, sm_count), kElemThreads, 0, s>>>(m, mat, u, st, sc, partials, aitken);
    CP_CUDA(cudaGetLastError());
}

void launch_aitken_relax(const DevMesh& m, const MaterialDev& mat, ElemState& st, const OuterScalars* sc, double w,
                         cudaStream_t s, int sm_count) {
    const int ne = m.c3 + m.c4;
    k_aitken<<<update_grid(ne, sm_count), kElemThreads, 0, s>>>(m, mat, st, sc, w);
    CP_CUDA(cudaGetLastError());
}

void launch_plastic(const DevMesh& m, const MaterialDev& mat, ElemState& st, cudaStream_t s, int sm_count) {
    const int ne = m.c3 + m.c4;
    k_plastic<<<update_grid(ne, sm_count), kElemThreads, 0, s>>>(ne, mat, st);
    CP_CUDA(cudaGetLastError());
}

}  // namespace cp

// ------------------------------------------------ allocation-free update --
//
// Some callers cannot allocate device memory: code that runs while a CUDA
// graph is being captured (cudaMalloc is not a capturable operation), code
// inside a framework that owns the whole device memory pool through its own
// allocator, and real-time loops whose memory budget is fixed up front. For
// them cp_secant_update_noalloc runs the fused strain / stress / secant-update
// kernel (k_update above) on buffers the caller already owns. Its only scratch
// -- the block partial sums of the exit norm and the reduction's scalars --
// lives in the file-scope array below, which every GPU that loads this library
// keeps until the process exits.
namespace {

constexpr int kNoAllocMaxBlocks = 4096;  // one partial-sum slot per block of 256 elements
constexpr int kNoAllocScalarBytes = 256;  // cp::OuterScalars, padded
static_assert(sizeof(cp::OuterScalars) <= kNoAllocScalarBytes, "scalars do not fit the scratch header");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScalarBytes + 4 * 8 * kNoAllocMaxBlocks];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device. In host code the
// array's name is only a host-side stand-in, so the address is looked up once
// per device (with that device current) and cached.
int noalloc_scratch(int device, unsigned char** out) {
    if (device < 0 || device >= kNoAllocMaxDevices) return CP_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return CP_ERR_CUDA;
        g_noalloc_ptr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_noalloc_ptr[device]);
    return CP_OK;
}

}  // namespace

extern "C" CP_API int cp_secant_update_noalloc(void* stream, const cp_material* mat, int node_count,
                                               const double* d_node_xy, int count4, const int* d_elem4,
                                               const double* d_uv, double* d_E_c, double* d_nu_c, double* d_psi,
                                               double* d_fields, double* rel_err) {
    if (!mat || !d_node_xy || !d_elem4 || !d_uv || !d_E_c || !d_nu_c || !d_psi || !d_fields || !rel_err)
        return CP_ERR_INVALID;
    if (node_count <= 0 || count4 <= 0) return CP_ERR_INVALID;
    if ((long long)count4 > (long long)kNoAllocMaxBlocks * cp::kElemThreads) return CP_ERR_INVALID;  // > 1,048,576
    if (((uintptr_t)d_node_xy | (uintptr_t)d_elem4 | (uintptr_t)d_uv) & 15u) return CP_ERR_INVALID;
    if (!(mat->E > 0) || !(mat->nu > -1.0 && mat->nu < 0.5) || mat->diagram < CP_DIAGRAM_ELASTIC ||
        mat->diagram > CP_DIAGRAM_PIECEWISE || (mat->diagram == CP_DIAGRAM_PIECEWISE &&
                                                 (mat->n_points < 2 || mat->n_points > CP_MAX_PW)))
        return CP_ERR_INVALID;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return CP_ERR_NO_DEVICE;
    unsigned char* scratch = nullptr;
    int st = noalloc_scratch(device, &scratch);
    if (st != CP_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cp::OuterScalars* sc = reinterpret_cast<cp::OuterScalars*>(scratch);
    double* partials = reinterpret_cast<double*>(scratch + kNoAllocScalarBytes);
    // the array keeps the previous call's contents: the reduction ticket must start at zero
    if (cudaMemsetAsync(sc, 0, sizeof(cp::OuterScalars), s) != cudaSuccess) return CP_ERR_CUDA;
    cp::MaterialDev M{};
    M.E = mat->E; M.nu = mat->nu; M.h = mat->h; M.plane = mat->plane; M.diagram = mat->diagram;
    M.sigma_t = mat->sigma_t; M.k_t = mat->k_t; M.a = mat->a; M.m = mat->m; M.eps0 = mat->eps0; M.n = mat->n;
    M.n_points = mat->n_points;
    for (int i = 0; i < CP_MAX_PW; ++i) { M.pw_eps[i] = mat->pw_eps[i]; M.pw_sig[i] = mat->pw_sig[i]; }
    cp::DevMesh m;
    m.n_nodes = node_count;
    m.c3 = 0;
    m.c4 = count4;
    m.xy = reinterpret_cast<double2*>(const_cast<double*>(d_node_xy));
    m.e4 = reinterpret_cast<int4*>(const_cast<int*>(d_elem4));
    cp::ElemState es{};
    const size_t ne = (size_t)count4;
    es.exx = d_fields; es.eyy = d_fields + ne; es.gam = d_fields + 2 * ne; es.eps_i = d_fields + 3 * ne;
    es.sxx = d_fields + 4 * ne; es.syy = d_fields + 5 * ne; es.tau = d_fields + 6 * ne; es.sig_i = d_fields + 7 * ne;
    es.table_s = d_fields + 8 * ne;
    es.psi = d_psi; es.E_c = d_E_c; es.nu_c = d_nu_c;
    const int grid = (count4 + cp::kElemThreads - 1) / cp::kElemThreads;  // <= kNoAllocMaxBlocks
    cp::k_update<<<grid, cp::kElemThreads, 0, s>>>(m, M, reinterpret_cast<const double2*>(d_uv), es, sc, partials, 0);
    if (cudaGetLastError() != cudaSuccess) return CP_ERR_CUDA;
    double host_err = 0.0;
    if (cudaMemcpyAsync(&host_err, &sc->rel_err, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return CP_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return CP_ERR_CUDA;
    *rel_err = host_err;
    return CP_OK;
}
