// Element-level device arithmetic shared by the single-instance kernels
// (elements.cu) and the batched kernels (batch.cu): geometry, D, the row
// blocks of B^T D B, the hardening diagrams, and the per-element secant
// update, Aitken relaxation and plastic strains. Every kernel that uses
// these computes bit-identical values for the same element.
#pragma once

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

// calcB8 (src/PlasticitySolver.cu:67-134) at (r, s): gradients and detJ of the
// 8-node serendipity quad. Local nodes: corners (1,1), (-1,1), (-1,-1), (1,-1),
// then the mid-sides of the edges s = 1, r = -1, s = -1, r = 1. Corner shape
// functions (1 + r ri)(1 + s si)(r ri + s si - 1)/4, mid-side ones
// (1 - r^2)(1 + s si)/2 and (1 + r ri)(1 - s^2)/2, differentiated in factored
// form. The 3x3 Gauss rule uses sqrt(3/5), 5/9 and 8/9 to full precision.
__device__ __forceinline__ double q8_grad(const double* x, const double* y, double r, double s, double* bx,
                                          double* by) {
    double dr[8], ds[8];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double ri = (k == 0 || k == 3) ? 1. : -1., si = k < 2 ? 1. : -1.;
        dr[k] = 0.25 * ri * (1. + s * si) * (2. * r * ri + s * si);
        ds[k] = 0.25 * si * (1. + r * ri) * (r * ri + 2. * s * si);
    }
    dr[4] = -r * (1. + s);        ds[4] = 0.5 * (1. - r * r);     // s = 1
    dr[5] = -0.5 * (1. - s * s);  ds[5] = -s * (1. - r);          // r = -1
    dr[6] = -r * (1. - s);        ds[6] = -0.5 * (1. - r * r);    // s = -1
    dr[7] = 0.5 * (1. - s * s);   ds[7] = -s * (1. + r);          // r = 1
    double xr = 0., yr = 0., xs = 0., ys = 0.;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        xr += dr[k] * x[k]; yr += dr[k] * y[k];
        xs += ds[k] * x[k]; ys += ds[k] * y[k];
    }
    const double det = xr * ys - yr * xs;
    const double inv = 1. / det;
    const double rx = ys * inv, sx = -yr * inv, ry = -xs * inv, sy = xr * inv;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        bx[k] = dr[k] * rx + ds[k] * sx;
        by[k] = dr[k] * ry + ds[k] * sy;
    }
    return det;
}

__device__ __forceinline__ double q8_point(int g) { return g == 0 ? -0.7745966692414834 : (g == 1 ? 0.0 : 0.7745966692414834); }
__device__ __forceinline__ double q8_weight(int g) { return g == 1 ? 8.0 / 9.0 : 5.0 / 9.0; }

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
// node j; kk8 for local nodes 4..7 of an 8-node element); block k of the node
// starts at nb + 128 k (sliced layout, 32 nodes x 4 values per block row).
// Q8 = false compiles the 8-node branch out (it needs about 50 registers
// more), for meshes without 8-node elements.
__device__ __forceinline__ void add_scaled(double* b, const double* blk, double h) {
    b[0] = __dadd_rn(b[0], __dmul_rn(blk[0], h));
    b[1] = __dadd_rn(b[1], __dmul_rn(blk[1], h));
    b[2] = __dadd_rn(b[2], __dmul_rn(blk[2], h));
    b[3] = __dadd_rn(b[3], __dmul_rn(blk[3], h));
}

template <bool Q8>
__device__ __forceinline__ void element_rows(const DevMesh& m, int e, int i, uint32_t kk, uint32_t kk8, const Dmat& d,
                                             double h, double* nb) {
    if (Q8 && e >= m.c3 + m.c4) {
        // formKe8 (src/PlasticitySolver.cu:189-224), one Gauss point at a
        // time: each point's block h (B_i^T D B_j) w detJ goes straight into
        // the node's accumulator (the mirrored thread adds the transposed
        // values in the same order, so K stays bitwise symmetric)
        const int le = e - m.c3 - m.c4;
        const int4 c = m.e8[2 * le], md = m.e8[2 * le + 1];
        double x[8], y[8];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const double2 p = m.xy[nth(c, a)], q = m.xy[nth(md, a)];
            x[a] = p.x; y[a] = p.y;
            x[4 + a] = q.x; y[4 + a] = q.y;
        }
        for (int g = 0; g < 9; ++g) {
            double bx[8], by[8];
            const int gi = g / 3, gj = g - 3 * gi;
            const double det = q8_grad(x, y, q8_point(gi), q8_point(gj), bx, by);
            const double w = q8_weight(gi) * q8_weight(gj) * det;
            double bxi = bx[0], byi = by[0];
#pragma unroll
            for (int a = 1; a < 8; ++a)
                if (i == a) { bxi = bx[a]; byi = by[a]; }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                double blk[4] = {0.0, 0.0, 0.0, 0.0};
                add_block(blk, bxi, byi, bx[j], by[j], d, w);
                const uint32_t k = j < 4 ? (kk >> (8 * j)) & 0xffu : (kk8 >> (8 * (j - 4))) & 0xffu;
                add_scaled(nb + 128 * (int)k, blk, h);
            }
        }
        return;
    }
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


// strain4 / strain8 + plastStress (src/PlasticitySolver.cu:1517-1610) for
// element e: element-mean strain, stress from the C of the last assembly,
// stress intensity, diagram value and the secant target psi. Adds the exit
// norm terms (sig_i - table_s)^2, table_s^2 to num / den. Without Aitken psi,
// E_c, nu_c move to the secant target; with Aitken the target is stored as a
// residual and the Aitken sums are added to an / ad. Q8 as for element_rows.
template <bool Q8>
__device__ __forceinline__ void update_element(const DevMesh& m, const MaterialDev& M, const double2* __restrict__ u,
                                               const ElemState& st, int e, int aitken, double& s_num, double& s_den,
                                               double& s_an, double& s_ad) {
    const double E0 = M.E, nu0 = M.nu;
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
    } else if (Q8 && e >= m.c3 + m.c4) {
        // strain8 (src/PlasticitySolver.cu:1551-1588): the Gauss-weighted
        // mean over the reference square, (1/4) sum w_i w_j eps(r_i, s_j)
        const int le = e - m.c3 - m.c4;
        const int4 c = m.e8[2 * le], md = m.e8[2 * le + 1];
        double x[8], y[8], uu[8], vv[8];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int n0 = nth(c, a), n1 = nth(md, a);
            const double2 p = m.xy[n0], q = m.xy[n1], w0 = u[n0], w1 = u[n1];
            x[a] = p.x; y[a] = p.y; uu[a] = w0.x; vv[a] = w0.y;
            x[4 + a] = q.x; y[4 + a] = q.y; uu[4 + a] = w1.x; vv[4 + a] = w1.y;
        }
        ex = 0.0; ey = 0.0; g = 0.0;
        for (int gp = 0; gp < 9; ++gp) {
            double bx[8], by[8];
            const int gi = gp / 3, gj = gp - 3 * gi;
            q8_grad(x, y, q8_point(gi), q8_point(gj), bx, by);
            double exl = 0.0, eyl = 0.0, gl = 0.0;
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                exl += uu[a] * bx[a];
                eyl += vv[a] * by[a];
                gl += uu[a] * by[a] + vv[a] * bx[a];
            }
            const double w = q8_weight(gi) * q8_weight(gj);
            ex += exl * w; ey += eyl * w; g += gl * w;
        }
        ex *= 0.25; ey *= 0.25; g *= 0.25;
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

// Aitken (Irons-Tuck) relaxation of the secant iteration on psi for element e:
// psi_{k+1} = psi_k + w_k r_k, w_k = -w_{k-1} (r_{k-1}, r_k - r_{k-1}) / |r_k - r_{k-1}|^2.
// The fixed point (r = 0) is the reference's.
__device__ __forceinline__ void relax_element(const MaterialDev& M, const ElemState& st, int e, double w) {
    const double r = st.res_cur[e];
    double ps = st.psi[e] + w * r;
    if (!(ps >= 1.0)) ps = 1.0;  // the secant modulus never exceeds E on a hardening diagram
    st.psi[e] = ps;
    st.E_c[e] = M.E / ps;
    st.nu_c[e] = 0.5 * (1. - (1. - 2. * M.nu) / ps);
    st.res_prev[e] = r;
}

// plastDeform (src/PlasticitySolver.cu:1641-1653) for element e.
__device__ __forceinline__ void plastic_element(const MaterialDev& M, const ElemState& st, int e) {
    const double E = M.E, G = M.E * 0.5 / (1. + M.nu);
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

}  // namespace

}  // namespace cp
