// Host orchestration of one problem instance and the extern "C" entry points
// declared in include/cuplast.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "cg.h"
#include "instance.h"
#include "internal.h"

using cp::Error;

namespace {

__global__ void k_set_level(int n, double lam, const double2* b_full, const double2* u_full, const uchar2* mask,
                            double2* b, double2* u) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double2 bf = b_full[i];
        b[i] = make_double2(lam * bf.x, lam * bf.y);
        const uchar2 m = mask[i];
        double2 uu = u[i];
        const double2 uf = u_full[i];
        if (!m.x) uu.x = lam * uf.x;
        if (!m.y) uu.y = lam * uf.y;
        u[i] = uu;
    }
}

__global__ void k_reset_state(int ne, double E, double nu, cp::ElemState st) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
        st.psi[e] = 1.0;
        st.E_c[e] = E;
        st.nu_c[e] = nu;
        st.res_prev[e] = 0.0;
        st.res_cur[e] = 0.0;
        st.sig_i[e] = 0.0;
        st.table_s[e] = 0.0;
    }
}

// Level predictor: keeps the last level's u and psi in u_prev / psi_prev and,
// with extrapolate, starts the next level from 2 (last) - (one before) on the
// free DOFs (k_set_level then sets the prescribed ones), with psi >= 1 and
// E_c, nu_c from psi as the secant update sets them.
__global__ void k_predict(int n, int ne, const uchar2* mask, double2* u, double2* u_prev, double E, double nu,
                          cp::ElemState st, double* psi_prev, int extrapolate) {
    const int m = n > ne ? n : ne;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        if (i < n) {
            const double2 c = u[i];
            if (extrapolate) {
                const double2 p = u_prev[i];
                const uchar2 f = mask[i];
                u[i] = make_double2(f.x ? 2.0 * c.x - p.x : c.x, f.y ? 2.0 * c.y - p.y : c.y);
            }
            u_prev[i] = c;
        }
        if (i < ne) {
            const double c = st.psi[i];
            if (extrapolate) {
                double v = 2.0 * c - psi_prev[i];
                if (!(v >= 1.0)) v = 1.0;
                st.psi[i] = v;
                st.E_c[i] = E / v;
                st.nu_c[i] = 0.5 * (1. - (1. - 2. * nu) / v);
            }
            psi_prev[i] = c;
        }
    }
}

__global__ void k_zero_double(double* p, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        p[i] = 0.0;
}

__global__ void k_widen(const float* in, double* out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

cp::MaterialDev to_dev(const cp_material& m) {
    cp::MaterialDev d{};
    d.E = m.E;
    d.nu = m.nu;
    d.h = m.h;
    d.plane = m.plane;
    d.diagram = m.diagram;
    d.sigma_t = m.sigma_t;
    d.k_t = m.k_t;
    d.a = m.a;
    d.m = m.m;
    d.eps0 = m.eps0;
    d.n = m.n;
    d.n_points = m.n_points;
    for (int i = 0; i < CP_MAX_PW; ++i) {
        d.pw_eps[i] = m.pw_eps[i];
        d.pw_sig[i] = m.pw_sig[i];
    }
    return d;
}

void validate_material(const cp_material& m) {
    CP_CHECK(m.E > 0 && std::isfinite(m.E), CP_ERR_INVALID, "material: E must be positive");
    CP_CHECK(m.nu > -1.0 && m.nu < 0.5, CP_ERR_INVALID, "material: nu must be in (-1, 0.5)");
    CP_CHECK(m.h > 0, CP_ERR_INVALID, "material: thickness h must be positive");
    CP_CHECK(m.plane == CP_PLANE_STRESS || m.plane == CP_PLANE_STRAIN, CP_ERR_INVALID, "material: bad plane condition");
    CP_CHECK(m.diagram >= CP_DIAGRAM_ELASTIC && m.diagram <= CP_DIAGRAM_PIECEWISE, CP_ERR_INVALID,
             "material: unknown diagram");
    if (m.diagram == CP_DIAGRAM_PIECEWISE) {
        CP_CHECK(m.n_points >= 2 && m.n_points <= CP_MAX_PW, CP_ERR_INVALID, "material: piecewise needs 2..16 points");
        for (int i = 1; i < m.n_points; ++i)
            CP_CHECK(m.pw_eps[i] > m.pw_eps[i - 1], CP_ERR_INVALID, "material: piecewise strains must increase");
    }
    if (m.diagram == CP_DIAGRAM_HOLLOMON)
        CP_CHECK(m.eps0 > 0 && m.n > 0 && m.sigma_t > 0, CP_ERR_INVALID, "material: Hollomon needs sy, eps0, n > 0");
}

}  // namespace

template <>
cp::CgArgs<double> cp_instance::cg_args<double>(int precond) {
    cp::CgArgs<double> a;
    if (precond && !minv64) minv64 = alloc<double4>(n_nodes);
    if (!rec64a) {
        rec64a = alloc<double4>(n_nodes);
        rec64b = alloc<double4>(n_nodes);
    }
    a.precond = precond;
    a.minv = minv64;
    a.n = n_nodes;
    a.sm_count = sms();
    a.max_blocks = max_blocks;
    a.slice_ptr = csr.slice_ptr;
    a.scol = csr.scol;
    a.val = csr.val64;
    a.b = b;
    a.mask = mask;
    a.x = u;
    a.r = r64;
    a.rec0 = rec64a;
    a.rec1 = rec64b;
    a.zn = z64a;  // shared with the multigrid solve, which never runs at the same time
    a.q = q64;
    a.sc = sc;
    a.partials = partials;
    return a;
}

template <>
cp::CgArgs<float> cp_instance::cg_args<float>(int precond) {
    cp::CgArgs<float> a;
    if (precond && !minv32) minv32 = alloc<float4>(n_nodes);
    a.precond = precond;
    a.minv = minv32;
    a.n = n_nodes;
    a.sm_count = sms();
    a.max_blocks = max_blocks;
    a.slice_ptr = csr.slice_ptr;
    a.scol = csr.scol;
    a.val = csr.val32;
    a.b = b;
    a.mask = mask;
    a.x = u;
    a.r = r32;
    a.rec0 = rec32a;
    a.rec1 = rec32b;
    a.zn = z32;
    a.q = q32;
    a.sc = sc;
    a.partials = partials;
    return a;
}

namespace {

// Adaptive rule 2's factor (the linear tolerance is factor x relErr until
// the outer tolerance is met): kRule2Factor, or CUPLAST_RULE2_FACTOR for
// measurements.
double rule2_factor() {
    static const double f = [] {
        const char* e = std::getenv("CUPLAST_RULE2_FACTOR");
        const double v = e ? std::atof(e) : 0.0;
        return (v > 0.0 && v < 1.0) ? v : cp::kRule2Factor;
    }();
    return f;
}

int fail(cp_context* ctx, const Error& e) {
    if (ctx) ctx->last_error = e.msg;
    return e.status;
}

template <typename F>
int guarded(cp_context* ctx, F&& f) {
    try {
        f();
        return CP_OK;
    } catch (const Error& e) {
        return fail(ctx, e);
    } catch (const std::bad_alloc&) {
        return fail(ctx, Error{CP_ERR_NOMEM, "host allocation failed"});
    }
}

void grid1d(long long n, int sms, int& grid) {
    long long g = (n + 255) / 256;
    long long cap = (long long)sms * 8;
    grid = (int)std::max<long long>(1, std::min(g, cap));
}

void ensure_fp32(cp_instance* I) {
    if (I->csr.val32) return;
    I->csr.val32 = I->alloc<float>(4 * (size_t)I->csr.sell_blocks);
    I->r32 = I->alloc<float2>(I->n_nodes);
    I->rec32a = I->alloc<float4>(I->n_nodes);
    I->rec32b = I->alloc<float4>(I->n_nodes);
    I->z32 = I->alloc<float2>(I->n_nodes);
    I->q32 = I->alloc<float2>(I->n_nodes);
}

void assemble(cp_instance* I, int precision) {
    const bool want32 = precision == CP_PREC_MIXED;
    if (want32) ensure_fp32(I);
    cp::launch_assemble(I->mesh, I->csr, I->mat, I->st.E_c, I->st.nu_c, true, want32, I->s(), I->sms());
    I->last_assembly = precision;
    I->launches += 1;
}

// Runs CG iterations until the device flags convergence or an error: one
// graph launch (WHILE node), or -- with graphs off, e.g. to profile the
// kernels one by one -- chunks of direct launches with a host poll between.
template <typename T>
void run_cg_loop(cp_instance* I, const cp::CgArgs<T>& a, cudaGraphExec_t g) {
    I->launches += 1;  // the init kernel launched before the loop
    if (I->use_graph) {
        CP_CUDA(cudaGraphLaunch(g, I->s()));
        CP_CUDA(cudaMemcpyAsync(I->sc_h, I->sc, sizeof(cp::CgScalars), cudaMemcpyDeviceToHost, I->s()));
        CP_CUDA(cudaStreamSynchronize(I->s()));
        // the WHILE body (body_iters x (P, U) + the condition kernel) ran
        // until the iteration that converged, at least once
        const long long trips = std::max<long long>(1, (I->sc_h->iter + I->body_iters - 1) / I->body_iters);
        I->launches += trips * (2LL * I->body_iters + 1);
        return;
    }
    for (;;) {
        for (int it = 0; it < I->body_iters; ++it) cp::cg_launch_iteration<T>(a, it & 1, I->s());
        I->launches += 2LL * I->body_iters;
        CP_CUDA(cudaMemcpyAsync(I->sc_h, I->sc, sizeof(cp::CgScalars), cudaMemcpyDeviceToHost, I->s()));
        CP_CUDA(cudaStreamSynchronize(I->s()));
        if (I->sc_h->converged || I->sc_h->status) return;
    }
}

// Arguments of the one-launch FP64 CG (cg_fused.cu) of this instance; its
// vectors are allocated on first use.
cp::FusedArgs fused_args(cp_instance* I, int precond) {
    const int n = I->n_nodes;
    if (!I->f_r) {
        I->f_r = I->alloc<double2>(n);
        I->f_w = I->alloc<double2>(n);
        I->f_p = I->alloc<double2>(n);
        I->f_kp = I->alloc<double2>(n);
        I->f_g = I->alloc<double2>(6 * (size_t)n);
        I->f_partials = I->alloc<double>(6 * (size_t)I->max_blocks);
    }
    if (precond && !I->minv64) (void)I->cg_args<double>(1);  // allocates the block-Jacobi inverse
    cp::FusedArgs a;
    a.n = n;
    a.sm_count = I->sms();
    a.max_blocks = I->max_blocks;
    a.slice_ptr = I->csr.slice_ptr;
    a.scol = I->csr.scol;
    a.val = I->csr.val64;
    a.b = I->b;
    a.mask = I->mask;
    a.x = I->u;
    a.r = I->f_r;
    a.w = I->f_w;
    a.p = I->f_p;
    a.kp = I->f_kp;
    a.gA = I->f_g;
    a.gB = I->f_g + 3 * (size_t)n;
    a.minv = precond ? I->minv64 : nullptr;
    a.precond = precond;
    a.sc = I->sc;
    a.partials = I->f_partials;
    return a;
}

// FP64 CG, one launch per iteration (cg_fused.cu), or the whole solve in one
// thread-block cluster where the instance fits.
void cg_fp64_fused(cp_instance* I, double eps, long long max_iter, int precond) {
    cp::FusedArgs a = fused_args(I, precond);
    if (I->cluster_fp64) {
        if (!I->cluster_planned) {
            I->cluster_plan = cp::cluster_cg_plan(a, I->csr.max_width);
            I->cluster_planned = 1;
        }
        if (I->cluster_plan.ctas > 0) {
            // one cluster holds the whole solve
            cp::cluster_cg_launch(a, I->cluster_plan, eps * eps, max_iter, I->s());
            I->launches += 1;
            CP_CUDA(cudaMemcpyAsync(I->sc_h, I->sc, sizeof(cp::CgScalars), cudaMemcpyDeviceToHost, I->s()));
            CP_CUDA(cudaStreamSynchronize(I->s()));
            return;
        }
    }
    if (I->persistent_fp64 && cp::fused_persistent_fits(a)) {
        // one cooperative launch for the whole solve
        if (I->test_barrier_ns) {
            a.barrier_ns = I->test_barrier_ns;
            a.barrier_skew = 1;
        }
        cp::fused_launch_persistent(a, eps * eps, max_iter, I->s());
        I->launches += 1;
        CP_CUDA(cudaMemcpyAsync(I->sc_h, I->sc, sizeof(cp::CgScalars), cudaMemcpyDeviceToHost, I->s()));
        CP_CUDA(cudaStreamSynchronize(I->s()));
        if (I->sc_h->status == CP_ERR_TIMEOUT) throw Error{CP_ERR_TIMEOUT, "persistent CG: grid barrier timed out"};
        return;
    }
    if (I->use_graph && !I->gf[precond]) I->gf[precond] = cp::fused_build_while_graph(a, I->body_iters, I->s());
    cp::fused_launch_start(a, eps * eps, max_iter, I->s());
    I->launches += 2;
    if (I->use_graph) {
        CP_CUDA(cudaGraphLaunch(I->gf[precond], I->s()));
        CP_CUDA(cudaMemcpyAsync(I->sc_h, I->sc, sizeof(cp::CgScalars), cudaMemcpyDeviceToHost, I->s()));
        CP_CUDA(cudaStreamSynchronize(I->s()));
        const long long trips = std::max<long long>(1, (I->sc_h->iter + I->body_iters - 1) / I->body_iters);
        I->launches += trips * (I->body_iters + 1);
        return;
    }
    for (;;) {
        for (int it = 0; it < I->body_iters; ++it) cp::fused_launch_iteration(a, it & 1, I->s());
        I->launches += I->body_iters;
        CP_CUDA(cudaMemcpyAsync(I->sc_h, I->sc, sizeof(cp::CgScalars), cudaMemcpyDeviceToHost, I->s()));
        CP_CUDA(cudaStreamSynchronize(I->s()));
        if (I->sc_h->converged || I->sc_h->status) return;
    }
}

// FP64 CG preconditioned by one aggregation-multigrid V-cycle (mg.cu), from
// the current u: coarse operators from the current K, then the PCG loop.
cp::MgArgs mg_args(cp_instance* I) {
    cp::MgArgs a;
    a.n = I->n_nodes;
    a.sm_count = I->sms();
    a.max_blocks = I->max_blocks;
    a.slice_ptr = I->csr.slice_ptr;
    a.scol = I->csr.scol;
    a.val = I->csr.val64;
    a.b = I->b;
    a.mask = I->mask;
    a.x = I->u;
    a.r = I->r64;
    a.q = I->q64;
    a.p0 = I->z64a;
    a.p1 = I->z64b;
    a.sc = I->sc;
    a.partials = I->partials;
    return a;
}

int mg_body(const cp_instance* I) { return std::max(2, I->body_iters + (I->body_iters & 1)); }

// Kernel count of the WHILE graph once sc_h holds the solve's scalars.
void mg_count_graph_launches(cp_instance* I) {
    const int body = mg_body(I);
    const long long trips = std::max<long long>(1, (I->sc_h->iter + body - 1) / body);
    I->launches += trips * (body * (long long)cp::mg_launches_per_iteration(I->mg) + 1);
}

// defer (graph loop only): enqueue the scalars' copy to sc_h and return
// without waiting; the caller synchronises later (after the secant update,
// which then follows the solve on the stream with no host round trip in
// between) and calls mg_count_graph_launches.
void cg_fp64_mg(cp_instance* I, double eps, long long max_iter, bool defer = false) {
    cp::mg_prepare(I);
    const cp::MgArgs a = mg_args(I);
    const int body = mg_body(I);
    I->launches += cp::mg_launch_setup(I->mg, a, I->s());
    if (I->use_graph && !I->gmg) I->gmg = cp::mg_build_while_graph(I->mg, a, body, I->s());
    I->launches += cp::mg_launch_start(I->mg, a, eps * eps, max_iter, I->s());
    const long long per_iter = cp::mg_launches_per_iteration(I->mg);
    if (I->use_graph) {
        CP_CUDA(cudaGraphLaunch(I->gmg, I->s()));
        CP_CUDA(cudaMemcpyAsync(I->sc_h, I->sc, sizeof(cp::CgScalars), cudaMemcpyDeviceToHost, I->s()));
        if (defer) return;
        CP_CUDA(cudaStreamSynchronize(I->s()));
        mg_count_graph_launches(I);
        return;
    }
    for (;;) {
        for (int it = 0; it < body; ++it) cp::mg_launch_iteration(I->mg, a, it & 1, I->s());
        I->launches += body * per_iter;
        CP_CUDA(cudaMemcpyAsync(I->sc_h, I->sc, sizeof(cp::CgScalars), cudaMemcpyDeviceToHost, I->s()));
        CP_CUDA(cudaStreamSynchronize(I->s()));
        if (I->sc_h->converged || I->sc_h->status) return;
    }
}

// Reference-semantics FP64 CG from the current u.
void cg_fp64(cp_instance* I, double eps, long long max_iter, int precond = 0) {
    if (I->fused_fp64) {
        cg_fp64_fused(I, eps, max_iter, precond);
        return;
    }
    auto a = I->cg_args<double>(precond);
    if (I->use_graph && !I->g64[precond]) I->g64[precond] = cp::cg_build_while_graph<double>(a, I->body_iters, I->s());
    cp::cg_launch_init<double>(a, I->csr.val64, true, eps * eps, max_iter, 0, -1.0, I->s());
    run_cg_loop(I, a, I->g64[precond]);
}

// Initial guesses from the level's solution increments (recycle.h): the
// arguments with the m-slot ring's increments newest first.
cp::RecycleArgs recycle_args(cp_instance* I, int m) {
    if (!I->rec_w) {
        I->rec_w = I->alloc<double2>((size_t)cp::kRecycleMax * I->n_nodes);
        I->rec_u0 = I->alloc<double2>(I->n_nodes);
        I->rec_part = I->alloc<double>((size_t)cp::recycle_grid(I->n_nodes, I->sms()) * cp::kRecycleStride);
        I->rec_y = I->alloc<double>(cp::kRecycleMax);
        I->rec_ticket = I->alloc<unsigned int>(1);
        CP_CUDA(cudaMemsetAsync(I->rec_ticket, 0, sizeof(unsigned int), I->s()));
        CP_CUDA(cudaMemsetAsync(I->rec_y, 0, cp::kRecycleMax * sizeof(double), I->s()));
    }
    cp::RecycleArgs a;
    a.n = I->n_nodes;
    a.slice_ptr = I->csr.slice_ptr;
    a.scol = I->csr.scol;
    a.val = I->csr.val64;
    a.u = I->u;
    a.b = I->b;
    a.mask = I->mask;
    a.w = I->rec_w;
    a.u0 = I->rec_u0;
    a.partials = I->rec_part;
    a.ticket = I->rec_ticket;
    a.y = I->rec_y;
    a.cnt = std::min(I->rec_cnt, m);
    for (int i = 0; i < a.cnt; ++i) a.slot[i] = ((I->rec_head - 1 - i) % m + m) % m;
    return a;
}

// Before a linear solve: u0 = u and, with increments in the ring, u += W y.
void recycle_before(cp_instance* I, int m) {
    const cp::RecycleArgs a = recycle_args(I, m);
    cp::recycle_project(a, I->sms(), I->s());
    I->launches += a.cnt > 0 ? 2 : 1;
}

// After it: the increment u - u0 goes into the ring.
void recycle_after(cp_instance* I, int m) {
    const cp::RecycleArgs a = recycle_args(I, m);
    cp::recycle_push(a, I->rec_head, I->sms(), I->s());
    I->launches += 1;
    I->rec_head = (I->rec_head + 1) % m;
    I->rec_cnt = std::min(I->rec_cnt + 1, m);
}

// Mixed precision: FP64 defect correction around FP32 CG. Each step computes
// r = m.(b - K64 u) in FP64 and runs CG on K32 from that residual (FP32
// recurrences, u accumulated in FP64) to a relative reduction inner_tol; stops
// when ||r64|| / ||b|| <= eps.
void cg_mixed(cp_instance* I, double eps, double inner_tol, long long max_iter, long long* inner_total,
              long long* fp64_spmv, double* rel_res, int precond = 0) {
    auto a = I->cg_args<float>(precond);
    if (I->use_graph && !I->g32[precond]) I->g32[precond] = cp::cg_build_while_graph<float>(a, I->body_iters, I->s());
    long long total = 0;
    for (int step = 0; step < 200; ++step) {
        cp::cg_launch_init<float>(a, I->csr.val64, true, inner_tol * inner_tol, max_iter, 1, eps * eps, I->s());
        ++*fp64_spmv;
        run_cg_loop(I, a, I->g32[precond]);
        const cp::CgScalars& h = *I->sc_h;
        *rel_res = h.bb > 0 ? std::sqrt(h.res64 / h.bb) : 0.0;
        if (h.lin_done) break;
        total += h.iter;
        if (h.status == CP_ERR_BREAKDOWN) throw Error{CP_ERR_BREAKDOWN, "FP32 inner CG broke down"};
        if (total >= max_iter) break;
    }
    *inner_total += total;
}

}  // namespace

void cp::instance_prepare_mixed(cp_instance* I, int precond) {
    const bool fresh = !I->csr.val32;
    ensure_fp32(I);
    if (fresh) {
        CP_CUDA(cudaMemsetAsync(I->rec32a, 0, sizeof(float4) * I->n_nodes, I->s()));
        CP_CUDA(cudaMemsetAsync(I->rec32b, 0, sizeof(float4) * I->n_nodes, I->s()));
    }
    if (precond) (void)I->cg_args<float>(1);  // allocates minv32 once
}

// ------------------------------------------------------------------ C ABI --

extern "C" {

CP_API const char* cp_version(void) { return "cuplast-b200 0.1.0 (sm_100a)"; }

CP_API const char* cp_status_string(int s) {
    switch (s) {
    case CP_OK: return "ok";
    case CP_ERR_INVALID: return "invalid argument";
    case CP_ERR_CUDA: return "CUDA error";
    case CP_ERR_NOMEM: return "out of device memory";
    case CP_ERR_NOT_CONVERGED: return "iteration limit reached";
    case CP_ERR_BREAKDOWN: return "numerical breakdown (NaN/Inf or non-positive curvature)";
    case CP_ERR_MESH: return "malformed mesh";
    case CP_ERR_UNSUPPORTED: return "unsupported";
    case CP_ERR_BUSY: return "busy";
    case CP_ERR_NO_DEVICE: return "no CUDA device";
    case CP_ERR_CANCELLED: return "cancelled";
    case CP_ERR_TIMEOUT: return "a bounded device-side wait gave up";
    default: return "unknown status";
    }
}

CP_API int cp_device_count(int* count) {
    if (!count) return CP_ERR_INVALID;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    *count = (e == cudaSuccess) ? n : 0;
    return CP_OK;
}

CP_API int cp_context_create(int device, cp_context** out) {
    if (!out) return CP_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return CP_ERR_NO_DEVICE;
    if (device < 0 || device >= n) return CP_ERR_INVALID;
    cp_context* c = new (std::nothrow) cp_context();
    if (!c) return CP_ERR_NOMEM;
    c->device = device;
    int rc = guarded(c, [&] {
        CP_CUDA(cudaSetDevice(device));
        CP_CUDA(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device));
        CP_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        CP_CUDA(cudaEventCreate(&c->ev0));
        CP_CUDA(cudaEventCreate(&c->ev1));
    });
    if (rc != CP_OK) {
        delete c;
        return rc;
    }
    *out = c;
    return CP_OK;
}

CP_API int cp_context_destroy(cp_context* ctx) {
    if (!ctx) return CP_ERR_INVALID;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return CP_OK;
}

CP_API const char* cp_context_last_error(const cp_context* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

CP_API const char* cp_instance_last_error(const cp_instance* inst) {
    return inst && inst->ctx ? inst->ctx->last_error.c_str() : "";
}

CP_API int cp_context_synchronize(cp_context* ctx) {
    if (!ctx) return CP_ERR_INVALID;
    return guarded(ctx, [&] { CP_CUDA(cudaStreamSynchronize(ctx->stream)); });
}

CP_API int cp_instance_footprint(const cp_mesh_view* m, int precision, size_t* bytes) {
    if (!m || !bytes || m->node_count <= 0 || m->count3 < 0 || m->count4 < 0 || m->count8 < 0) return CP_ERR_INVALID;
    const size_t n = (size_t)m->node_count, ne = (size_t)m->count3 + (size_t)m->count4 + (size_t)m->count8;
    const size_t incs = 3 * (size_t)m->count3 + 4 * (size_t)m->count4 + 8 * (size_t)m->count8;
    // upper bound of the neighbour count: the reference's link capacity
    const size_t nadj = 2 * (size_t)m->count3 + 3 * (size_t)m->count4 + 7 * (size_t)m->count8;
    const size_t nadj_est = std::min(nadj, incs * 3);
    const size_t nnz = 4 * (nadj_est + n);
    size_t b = n * 16 + ne * 16 + (size_t)m->count8 * 16 + incs * (m->count8 ? 12 : 8) + (2 * n + 2) * 4 +
               nadj_est * 4;                                                   // mesh + structure
    b += nnz * 8;                                                              // K (FP64)
    b += n * (16 * 8 + 2);                                                     // u, b, b_full, u_full, r, z, z, q, mask
    b += ne * 18 * 8;                                                          // element state
    b += n * 2 * 32;                                                           // (v, z) records, FP64 two-kernel form
    if (precision != CP_PREC_FP64) b += nnz * 4 + n * 8 * 4 + n * 2 * 16;
    b += n * 16 * (cp::kRecycleMax + 1);                                       // solution increments (recycle)
    b += 1 << 20;                                                              // scalars, partials, graphs
    *bytes = b;
    return CP_OK;
}

CP_API int cp_instance_create(cp_context* ctx, const cp_mesh_view* mv, const cp_material* mat, cp_instance** out) {
    if (!ctx || !mv || !mat || !out) return CP_ERR_INVALID;
    *out = nullptr;
    cp_instance* I = new (std::nothrow) cp_instance();
    if (!I) return CP_ERR_NOMEM;
    I->ctx = ctx;
    if (const char* g = std::getenv("CUPLAST_NO_GRAPH")) I->use_graph = !(g[0] == '1');
    // FP64 CG form: one thread-block cluster when the instance fits (default),
    // else one launch per iteration in a graph; CUPLAST_FP64_CG=fused keeps
    // the graph loop, =persistent makes it one cooperative launch, =classic
    // selects the two-kernel loop of cg.cu.
    if (const char* g = std::getenv("CUPLAST_FP64_CG")) {
        I->fused_fp64 = std::strcmp(g, "classic") != 0;
        I->persistent_fp64 = std::strcmp(g, "persistent") == 0;
        I->cluster_fp64 = std::strcmp(g, "cluster") == 0;
    }
    if (const char* g = std::getenv("CUPLAST_TEST_BARRIER_NS")) I->test_barrier_ns = std::strtoull(g, nullptr, 10);
    int rc = guarded(ctx, [&] {
        CP_CHECK(mv->node_count > 0 && mv->node_xy, CP_ERR_INVALID, "mesh: no nodes");
        CP_CHECK(mv->count3 >= 0 && mv->count4 >= 0 && mv->count8 >= 0 &&
                     (long long)mv->count3 + mv->count4 + mv->count8 > 0,
                 CP_ERR_INVALID, "mesh: no elements");
        CP_CHECK(mv->count3 == 0 || mv->elem3, CP_ERR_INVALID, "mesh: elem3 missing");
        CP_CHECK(mv->count4 == 0 || mv->elem4, CP_ERR_INVALID, "mesh: elem4 missing");
        CP_CHECK(mv->count8 == 0 || mv->elem8, CP_ERR_INVALID, "mesh: elem8 missing");
        CP_CHECK((long long)mv->count3 + mv->count4 + mv->count8 < (1LL << 28), CP_ERR_UNSUPPORTED,
                 "mesh: too many elements");
        validate_material(*mat);
        CP_CUDA(cudaSetDevice(ctx->device));
        I->mat_host = *mat;
        I->mat = to_dev(*mat);
        I->n_nodes = mv->node_count;
        I->n_elem = mv->count3 + mv->count4 + mv->count8;
        cudaStream_t s = I->s();
        // mesh upload (the reference's meshToGPU, src/Mesh.cu:678-717)
        I->mesh.n_nodes = mv->node_count;
        I->mesh.c3 = mv->count3;
        I->mesh.c4 = mv->count4;
        I->mesh.c8 = mv->count8;
        I->mesh.xy = I->alloc<double2>(I->n_nodes);
        std::vector<int4> e3((size_t)mv->count3), e4((size_t)mv->count4);
        for (int e = 0; e < mv->count3; ++e)
            e3[e] = make_int4(mv->elem3[3 * e], mv->elem3[3 * e + 1], mv->elem3[3 * e + 2], -1);
        for (int e = 0; e < mv->count4; ++e)
            e4[e] = make_int4(mv->elem4[4 * e], mv->elem4[4 * e + 1], mv->elem4[4 * e + 2], mv->elem4[4 * e + 3]);
        std::vector<int4> e8(2 * (size_t)mv->count8);
        for (size_t q = 0; q < e8.size(); ++q)
            e8[q] = make_int4(mv->elem8[4 * q], mv->elem8[4 * q + 1], mv->elem8[4 * q + 2], mv->elem8[4 * q + 3]);
        I->mesh.e3 = I->alloc<int4>(e3.size());
        I->mesh.e4 = I->alloc<int4>(e4.size());
        I->mesh.e8 = I->alloc<int4>(e8.size());
        CP_CUDA(cudaMemcpyAsync(I->mesh.xy, mv->node_xy, sizeof(double2) * I->n_nodes, cudaMemcpyHostToDevice, s));
        if (!e3.empty()) CP_CUDA(cudaMemcpyAsync(I->mesh.e3, e3.data(), sizeof(int4) * e3.size(), cudaMemcpyHostToDevice, s));
        if (!e4.empty()) CP_CUDA(cudaMemcpyAsync(I->mesh.e4, e4.data(), sizeof(int4) * e4.size(), cudaMemcpyHostToDevice, s));
        if (!e8.empty()) CP_CUDA(cudaMemcpyAsync(I->mesh.e8, e8.data(), sizeof(int4) * e8.size(), cudaMemcpyHostToDevice, s));
        // sparsity structure + slot map on the device
        cp::setup_csr(I->mesh, I->csr, s, I->sms());
        I->allocs.push_back(I->csr.inc_pos);
        I->allocs.push_back(I->csr.adj_pos);
        I->allocs.push_back(I->csr.inc);
        I->allocs.push_back(I->csr.inc_k);
        if (I->csr.inc_k8) I->allocs.push_back(I->csr.inc_k8);
        I->allocs.push_back(I->csr.adj);
        I->bytes += (size_t)(2 * (I->n_nodes + 1)) * 4 +
                    (3ull * mv->count3 + 4ull * mv->count4 + 8ull * mv->count8) * (mv->count8 ? 12 : 8) +
                    I->csr.nadj * 4;
        CP_CHECK(I->csr.nnz < (1LL << 31), CP_ERR_UNSUPPORTED, "matrix too large for 32-bit CSR offsets");
        I->allocs.push_back(I->csr.slice_ptr);
        I->allocs.push_back(I->csr.scol);
        I->bytes += ((size_t)I->csr.n_slices + 1 + (size_t)I->csr.sell_blocks) * 4;
        I->csr.val64 = I->alloc<double>(4 * (size_t)I->csr.sell_blocks);
        const int n = I->n_nodes, ne = I->n_elem;
        I->u = I->alloc<double2>(n);
        I->b = I->alloc<double2>(n);
        I->b_full = I->alloc<double2>(n);
        I->u_full = I->alloc<double2>(n);
        I->mask = I->alloc<uchar2>(n);
        I->r64 = I->alloc<double2>(n);
        I->z64a = I->alloc<double2>(n);
        I->z64b = I->alloc<double2>(n);
        I->q64 = I->alloc<double2>(n);
        CP_CUDA(cudaMemsetAsync(I->u, 0, sizeof(double2) * n, s));
        CP_CUDA(cudaMemsetAsync(I->b, 0, sizeof(double2) * n, s));
        CP_CUDA(cudaMemsetAsync(I->b_full, 0, sizeof(double2) * n, s));
        CP_CUDA(cudaMemsetAsync(I->u_full, 0, sizeof(double2) * n, s));
        CP_CUDA(cudaMemsetAsync(I->mask, 1, sizeof(uchar2) * n, s));
        CP_CUDA(cudaMemsetAsync(I->z64a, 0, sizeof(double2) * n, s));
        CP_CUDA(cudaMemsetAsync(I->z64b, 0, sizeof(double2) * n, s));
        // element state: 18 arrays in one block
        I->st_block = I->alloc<double>(18 * (size_t)ne);
        double** f[] = {&I->st.exx, &I->st.eyy, &I->st.gam, &I->st.eps_i, &I->st.sxx, &I->st.syy,
                        &I->st.tau, &I->st.sig_i, &I->st.table_s, &I->st.psi, &I->st.E_c, &I->st.nu_c,
                        &I->st.exx_p, &I->st.eyy_p, &I->st.gam_p, &I->st.eps_p_i, &I->st.res_prev, &I->st.res_cur};
        for (int k = 0; k < 18; ++k) *f[k] = I->st_block + (size_t)k * ne;
        {
            int g;
            grid1d(18LL * ne, I->sms(), g);
            k_zero_double<<<g, 256, 0, s>>>(I->st_block, 18LL * ne);
        }
        I->sc = I->alloc<cp::CgScalars>(1);
        I->osc = I->alloc<cp::OuterScalars>(1);
        CP_CUDA(cudaMemsetAsync(I->sc, 0, sizeof(cp::CgScalars), s));
        CP_CUDA(cudaMemsetAsync(I->osc, 0, sizeof(cp::OuterScalars), s));
        I->max_blocks = I->sms() * 8;
        I->partials = I->alloc<double>(4 * (size_t)I->max_blocks);  // <= 4 sums per block
        CP_CUDA(cudaMallocHost(&I->sc_h, sizeof(cp::CgScalars)));
        CP_CUDA(cudaMallocHost(&I->osc_h, sizeof(cp::OuterScalars)));
        {
            int g;
            grid1d(ne, I->sms(), g);
            k_reset_state<<<g, 256, 0, s>>>(ne, I->mat.E, I->mat.nu, I->st);
        }
        CP_CUDA(cudaGetLastError());
        CP_CUDA(cudaStreamSynchronize(s));
    });
    if (rc != CP_OK) {
        cp_instance_destroy(I);
        return rc;
    }
    *out = I;
    return CP_OK;
}

CP_API int cp_instance_destroy(cp_instance* I) {
    if (I && I->in_batch) return CP_ERR_BUSY;  // owned by a batch until harvested
    if (!I) return CP_ERR_INVALID;
    if (I->ctx) {
        cudaSetDevice(I->ctx->device);
        cudaStreamSynchronize(I->ctx->stream);
    }
    for (int k = 0; k < 2; ++k) {
        if (I->g64[k]) cudaGraphExecDestroy(I->g64[k]);
        if (I->g32[k]) cudaGraphExecDestroy(I->g32[k]);
        if (I->gf[k]) cudaGraphExecDestroy(I->gf[k]);
    }
    if (I->ctx) cp::mg_release(I);
    for (void* p : I->allocs) cudaFreeAsync(p, I->ctx->stream);
    if (I->sc_h) cudaFreeHost(I->sc_h);
    if (I->osc_h) cudaFreeHost(I->osc_h);
    if (I->ctx) cudaStreamSynchronize(I->ctx->stream);
    delete I;
    return CP_OK;
}

CP_API int cp_instance_sizes(const cp_instance* I, int* nodes, int* elems, long long* nnz, long long* nadj) {
    if (!I) return CP_ERR_INVALID;
    if (nodes) *nodes = I->n_nodes;
    if (elems) *elems = I->n_elem;
    if (nnz) *nnz = I->csr.nnz;
    if (nadj) *nadj = I->csr.nadj;
    return CP_OK;
}

CP_API int cp_instance_set_loads(cp_instance* I, const double* rp, const unsigned char* mask, const double* uv) {
    if (I && I->in_batch) return CP_ERR_BUSY;  // owned by a batch until harvested
    if (!I || !rp || !mask) return CP_ERR_INVALID;
    return guarded(I->ctx, [&] {
        const int n = I->n_nodes;
        cudaStream_t s = I->s();
        std::vector<unsigned char> m(2 * (size_t)n);
        for (size_t i = 0; i < m.size(); ++i) m[i] = mask[i] ? 1 : 0;
        CP_CUDA(cudaMemcpyAsync(I->b_full, rp, sizeof(double2) * n, cudaMemcpyHostToDevice, s));
        CP_CUDA(cudaMemcpyAsync(I->mask, m.data(), 2 * (size_t)n, cudaMemcpyHostToDevice, s));
        if (uv) {
            CP_CUDA(cudaMemcpyAsync(I->u_full, uv, sizeof(double2) * n, cudaMemcpyHostToDevice, s));
            CP_CUDA(cudaMemcpyAsync(I->u, uv, sizeof(double2) * n, cudaMemcpyHostToDevice, s));
        } else {
            CP_CUDA(cudaMemsetAsync(I->u_full, 0, sizeof(double2) * n, s));
            CP_CUDA(cudaMemsetAsync(I->u, 0, sizeof(double2) * n, s));
        }
        int g;
        grid1d(n, I->sms(), g);
        k_set_level<<<g, 256, 0, s>>>(n, 1.0, I->b_full, I->u_full, I->mask, I->b, I->u);
        CP_CUDA(cudaGetLastError());
        CP_CUDA(cudaStreamSynchronize(s));
        I->mask_host = m;
        I->loads_set = true;
    });
}

CP_API int cp_instance_set_level(cp_instance* I, double lam) {
    if (I && I->in_batch) return CP_ERR_BUSY;  // owned by a batch until harvested
    if (!I) return CP_ERR_INVALID;
    return guarded(I->ctx, [&] {
        int g;
        grid1d(I->n_nodes, I->sms(), g);
        k_set_level<<<g, 256, 0, I->s()>>>(I->n_nodes, lam, I->b_full, I->u_full, I->mask, I->b, I->u);
        CP_CUDA(cudaGetLastError());
    });
}

CP_API int cp_instance_reset_state(cp_instance* I) {
    if (I && I->in_batch) return CP_ERR_BUSY;  // owned by a batch until harvested
    if (!I) return CP_ERR_INVALID;
    return guarded(I->ctx, [&] {
        int g;
        grid1d(I->n_elem, I->sms(), g);
        k_reset_state<<<g, 256, 0, I->s()>>>(I->n_elem, I->mat.E, I->mat.nu, I->st);
        CP_CUDA(cudaGetLastError());
    });
}

CP_API int cp_assemble(cp_instance* I, int precision) {
    if (I && I->in_batch) return CP_ERR_BUSY;  // owned by a batch until harvested
    if (!I || (precision != CP_PREC_FP64 && precision != CP_PREC_MIXED)) return CP_ERR_INVALID;
    return guarded(I->ctx, [&] {
        assemble(I, precision);
        CP_CUDA(cudaStreamSynchronize(I->s()));
    });
}

CP_API int cp_cg_solve(cp_instance* I, double eps, long long max_iter, long long* iters, double* rel_res) {
    if (I && I->in_batch) return CP_ERR_BUSY;  // owned by a batch until harvested
    if (!I || !(eps > 0) || max_iter <= 0) return CP_ERR_INVALID;
    int st = CP_OK;
    int rc = guarded(I->ctx, [&] {
        CP_CHECK(I->loads_set, CP_ERR_INVALID, "loads not set");
        CP_CHECK(I->last_assembly >= 0, CP_ERR_INVALID, "matrix not assembled");
        cg_fp64(I, eps, max_iter);
        if (iters) *iters = I->sc_h->iter;
        if (rel_res) *rel_res = std::sqrt(I->sc_h->rr * I->sc_h->normB_inv);
        st = I->sc_h->status;
    });
    return rc != CP_OK ? rc : st;
}

CP_API int cp_secant_update(cp_instance* I, double* rel_err) {
    if (I && I->in_batch) return CP_ERR_BUSY;  // owned by a batch until harvested
    if (!I) return CP_ERR_INVALID;
    return guarded(I->ctx, [&] {
        cp::launch_update(I->mesh, I->mat, I->u, I->st, I->osc, I->partials, 0, I->s(), I->sms());
        CP_CUDA(cudaMemcpyAsync(I->osc_h, I->osc, sizeof(cp::OuterScalars), cudaMemcpyDeviceToHost, I->s()));
        CP_CUDA(cudaStreamSynchronize(I->s()));
        if (rel_err) *rel_err = I->osc_h->rel_err;
    });
}

CP_API int cp_plastic_strains(cp_instance* I) {
    if (I && I->in_batch) return CP_ERR_BUSY;  // owned by a batch until harvested
    if (!I) return CP_ERR_INVALID;
    return guarded(I->ctx, [&] {
        cp::launch_plastic(I->mesh, I->mat, I->st, I->s(), I->sms());
        CP_CUDA(cudaStreamSynchronize(I->s()));
    });
}

CP_API void cp_solve_opts_default(cp_solve_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->precision = CP_PREC_FP64;
    o->cg_tol = 1e-7;
    o->outer_tol = 1e-5;
    o->max_outer = 50;
    o->max_cg = 200000;
    o->levels = 1;
    o->aitken = 0;
    o->inner_tol = 1e-4;
    o->adaptive_cg = 0;
    o->precond = 0;
}

CP_API int cp_solve(cp_instance* I, const cp_solve_opts* opts, cp_solve_report* rep) {
    if (I && I->in_batch) return CP_ERR_BUSY;  // owned by a batch until harvested
    if (!I || !opts) return CP_ERR_INVALID;
    cp_solve_report R{};
    const cp_solve_opts o = *opts;
    if (!(o.cg_tol > 0) || !(o.outer_tol > 0) || o.max_outer <= 0 || o.levels <= 0 || o.max_cg <= 0)
        return CP_ERR_INVALID;
    if (o.precision != CP_PREC_FP64 && o.precision != CP_PREC_MIXED && o.precision != CP_PREC_FLOAT_BOOST)
        return CP_ERR_INVALID;
    if (o.precond < 0 || o.precond > 2) return CP_ERR_INVALID;
    if (o.precond == 2 && o.precision != CP_PREC_FP64) return CP_ERR_UNSUPPORTED;  // multigrid: FP64 only
    if (o.adaptive_cg < 0 || o.adaptive_cg > 2 || o.predict < 0 || o.predict > 1) return CP_ERR_INVALID;
    if (o.recycle < 0 || o.recycle > cp::kRecycleMax) return CP_ERR_INVALID;
    // the increments' ring holds o.recycle slots; FP64 linear solves with precond 0 or 1 only
    const int m_rec = o.precond == 2 ? 0 : o.recycle;
    // floatBoost's first phase (solveCUDA_FD, src/PlasticitySolver.cu:660-679):
    // CG 1e-4 and relErr 1e-4 in reduced precision
    constexpr double kBoostTol = 1e-4;
    int rc = guarded(I->ctx, [&] {
        CP_CHECK(I->loads_set, CP_ERR_INVALID, "loads not set");
        cudaStream_t s = I->s();
        CP_CUDA(cudaEventRecord(I->ctx->ev0, s));
        const long long launches0 = I->launches;
        R.status = CP_OK;
        for (int lev = 1; lev <= o.levels; ++lev) {
            const double lam = (double)lev / o.levels;
            int g;
            if (o.predict && lev >= 2) {
                // level 2 records level 1; from level 3 on, extrapolate
                if (!I->pred_u) {
                    I->pred_u = I->alloc<double2>(I->n_nodes);
                    I->pred_psi = I->alloc<double>(I->n_elem);
                }
                grid1d(std::max(I->n_nodes, I->n_elem), I->sms(), g);
                k_predict<<<g, 256, 0, s>>>(I->n_nodes, I->n_elem, I->mask, I->u, I->pred_u, I->mat.E, I->mat.nu,
                                            I->st, I->pred_psi, lev >= 3 ? 1 : 0);
                I->launches += 1;
            }
            grid1d(I->n_nodes, I->sms(), g);
            k_set_level<<<g, 256, 0, s>>>(I->n_nodes, lam, I->b_full, I->u_full, I->mask, I->b, I->u);
            grid1d(2LL * I->n_elem, I->sms(), g);
            k_zero_double<<<g, 256, 0, s>>>(I->st.res_prev, 2LL * I->n_elem);  // res_prev, res_cur adjacent
            I->launches += 2;
            I->rec_cnt = 0;  // increments of this level only
            I->rec_head = 0;
            double rel_err = 1.0, w_prev = 1.0;
            bool converged = false;
            // floatBoost: the reduced-precision phase, then FP64 from its state
            bool boost = o.precision == CP_PREC_FLOAT_BOOST;
            int prec = boost ? CP_PREC_MIXED : o.precision;
            for (int it = 0; it < o.max_outer; ++it) {
                CP_CHECK(!I->cancel.load(std::memory_order_relaxed), CP_ERR_CANCELLED, "solve cancelled");
                if (cudaStream_t ns = I->ctx->restream.exchange(nullptr)) {
                    CP_CUDA(cudaStreamSynchronize(s));  // nothing of this solve left on the old stream
                    I->ctx->stream = ns;
                    s = ns;
                }
                // linear tolerance: tight once the secant iteration is close
                double eps = boost ? std::max(o.cg_tol, kBoostTol) : o.cg_tol;
                if (!boost && o.adaptive_cg == 1 && rel_err > 10.0 * o.outer_tol) eps = std::max(o.cg_tol, 1e-2 * rel_err);
                if (!boost && o.adaptive_cg == 2 && rel_err > o.outer_tol)
                    eps = std::max(o.cg_tol, rule2_factor() * rel_err);
                assemble(I, prec);
                // the multigrid graph loop leaves its scalars for after the update
                const bool mg_deferred = prec == CP_PREC_FP64 && o.precond == 2 && I->use_graph;
                if (mg_deferred) {
                    cg_fp64_mg(I, eps, o.max_cg, true);
                } else if (prec == CP_PREC_FP64) {
                    if (o.precond == 2) {
                        cg_fp64_mg(I, eps, o.max_cg);
                    } else {
                        if (m_rec > 0) recycle_before(I, m_rec);
                        cg_fp64(I, eps, o.max_cg, o.precond ? 1 : 0);
                        if (m_rec > 0) recycle_after(I, m_rec);
                    }
                    R.cg_iters += I->sc_h->iter;
                    R.cg_rel_res = std::sqrt(I->sc_h->rr * I->sc_h->normB_inv);
                    if (I->sc_h->status == CP_ERR_BREAKDOWN) throw Error{CP_ERR_BREAKDOWN, "CG broke down"};
                } else {
                    double rr = 0;
                    cg_mixed(I, eps, o.inner_tol, o.max_cg, &R.cg_iters, &R.fp64_spmv, &rr, o.precond ? 1 : 0);
                    R.cg_rel_res = rr;
                }
                cp::launch_update(I->mesh, I->mat, I->u, I->st, I->osc, I->partials, o.aitken, s, I->sms());
                I->launches += 1;
                CP_CUDA(cudaMemcpyAsync(I->osc_h, I->osc, sizeof(cp::OuterScalars), cudaMemcpyDeviceToHost, s));
                CP_CUDA(cudaStreamSynchronize(s));
                if (mg_deferred) {
                    mg_count_graph_launches(I);
                    R.cg_iters += I->sc_h->iter;
                    R.cg_rel_res = std::sqrt(I->sc_h->rr * I->sc_h->normB_inv);
                    if (I->sc_h->status == CP_ERR_BREAKDOWN) throw Error{CP_ERR_BREAKDOWN, "CG broke down"};
                }
                rel_err = I->osc_h->rel_err;
                R.outer_iters += 1;
                CP_CHECK(std::isfinite(rel_err), CP_ERR_BREAKDOWN, "secant iteration produced NaN");
                if (o.aitken) {
                    double w = 1.0;
                    if (it > 0 && I->osc_h->a_den > 0) w = -w_prev * I->osc_h->a_num / I->osc_h->a_den;
                    if (!(w >= 0.1)) w = 0.1;
                    if (w > 10.0) w = 10.0;
                    cp::launch_aitken_relax(I->mesh, I->mat, I->st, I->osc, w, s, I->sms());
                    I->launches += 1;
                    w_prev = w;
                }
                if (boost) {
                    if (rel_err <= kBoostTol) {
                        // switch to FP64 (copyFloatToDouble keeps u, E_c, nu_c;
                        // the Aitken history starts afresh); the FP64 phase
                        // gets its own max_outer and takes at least one step
                        boost = false;
                        prec = CP_PREC_FP64;
                        w_prev = 1.0;
                        I->rec_cnt = 0;
                        I->rec_head = 0;
                        int g2;
                        grid1d(2LL * I->n_elem, I->sms(), g2);
                        k_zero_double<<<g2, 256, 0, s>>>(I->st.res_prev, 2LL * I->n_elem);
                        I->launches += 1;
                        it = -1;
                    }
                    continue;
                }
                if (rel_err <= o.outer_tol && eps <= o.cg_tol) {
                    converged = true;
                    break;
                }
            }
            R.rel_err = rel_err;
            R.levels_done = lev;
            if (!converged) {
                R.status = CP_ERR_NOT_CONVERGED;
                break;
            }
        }
        cp::launch_plastic(I->mesh, I->mat, I->st, s, I->sms());
        I->launches += 1;
        R.kernel_launches = I->launches - launches0;
        CP_CUDA(cudaEventRecord(I->ctx->ev1, s));
        CP_CUDA(cudaEventSynchronize(I->ctx->ev1));
        float ms = 0;
        CP_CUDA(cudaEventElapsedTime(&ms, I->ctx->ev0, I->ctx->ev1));
        R.seconds = ms * 1e-3;
    });
    if (rep) *rep = R;
    if (rc != CP_OK) return rc;
    return R.status;
}

CP_API int cp_bench_mg(cp_instance* I, int iters, double* ms, double* bytes) {
    if (I && I->in_batch) return CP_ERR_BUSY;
    if (!I || iters <= 0 || !ms) return CP_ERR_INVALID;
    return guarded(I->ctx, [&] {
        CP_CHECK(I->loads_set, CP_ERR_INVALID, "loads not set");
        cudaStream_t s = I->s();
        assemble(I, CP_PREC_FP64);
        cp::mg_prepare(I);
        const cp::MgArgs a = mg_args(I);
        std::vector<cudaEvent_t> ev(6 * (size_t)iters + 2);
        for (auto& e : ev) CP_CUDA(cudaEventCreate(&e));
        CP_CUDA(cudaEventRecord(ev[0], s));
        cp::mg_launch_setup(I->mg, a, s);
        CP_CUDA(cudaEventRecord(ev[1], s));
        // a tolerance no iteration reaches, so every kernel does its work
        cp::mg_launch_start(I->mg, a, 0.0, (long long)iters + 8, s);
        for (int it = 0; it < iters; ++it) cp::mg_launch_iteration(I->mg, a, it & 1, s, &ev[2 + 6 * (size_t)it]);
        CP_CUDA(cudaEventSynchronize(ev.back()));
        double t[5] = {0, 0, 0, 0, 0};
        for (int it = 0; it < iters; ++it)
            for (int k = 0; k < 5; ++k) {
                float x = 0;
                CP_CUDA(cudaEventElapsedTime(&x, ev[2 + 6 * (size_t)it + k], ev[2 + 6 * (size_t)it + k + 1]));
                t[k] += x;
            }
        float su = 0;
        CP_CUDA(cudaEventElapsedTime(&su, ev[0], ev[1]));
        for (auto& e : ev) cudaEventDestroy(e);
        CP_CUDA(cudaMemcpy(I->sc_h, I->sc, sizeof(cp::CgScalars), cudaMemcpyDeviceToHost));
        CP_CHECK(I->sc_h->status == 0 && I->sc_h->iter == iters, CP_ERR_BREAKDOWN,
                 "multigrid bench: the iterations stopped early");
        for (int k = 0; k < 5; ++k) ms[k] = t[k] / iters;
        ms[5] = su;
        if (bytes) cp::mg_algorithmic_bytes(I->mg, a, I->csr.nadj + I->n_nodes, bytes);
    });
}

CP_API int cp_bench_cg(cp_instance* I, int precision, int precond, int iters, double* ms_p, double* ms_u,
                       double* bytes_p, double* bytes_u) {
    if (I && I->in_batch) return CP_ERR_BUSY;
    if (!I || iters <= 0 || (precision != CP_PREC_FP64 && precision != CP_PREC_MIXED) || (precond & ~1)) return CP_ERR_INVALID;
    return guarded(I->ctx, [&] {
        CP_CHECK(I->loads_set, CP_ERR_INVALID, "loads not set");
        cudaStream_t s = I->s();
        assemble(I, precision);
        std::vector<cudaEvent_t> ev(2 * (size_t)iters + 1);
        for (auto& e : ev) CP_CUDA(cudaEventCreate(&e));
        auto time_it = [&](auto a, const void* valA) {
            using T = typename std::remove_cv<typename std::remove_reference<decltype(*a.val)>::type>::type;
            cp::cg_launch_init<T>(a, valA, true, 0.0, (long long)iters + 8, precision == CP_PREC_MIXED, -1.0, s);
            for (int it = 0; it < iters; ++it) {
                CP_CUDA(cudaEventRecord(ev[2 * it], s));
                cp::cg_launch_p<T>(a, it & 1, s);
                CP_CUDA(cudaEventRecord(ev[2 * it + 1], s));
                cp::cg_launch_u<T>(a, it & 1, s);
            }
            CP_CUDA(cudaEventRecord(ev[2 * (size_t)iters], s));
        };
        const double n = I->n_nodes, nnz = (double)I->csr.nnz;
        double sv, sx;
        if (precision == CP_PREC_FP64) {
            time_it(I->cg_args<double>(precond), I->csr.val64);
            sv = 8;
            sx = 8;
        } else {
            time_it(I->cg_args<float>(precond), I->csr.val64);
            sv = 4;
            sx = 4;
        }
        CP_CUDA(cudaEventSynchronize(ev.back()));
        double tp = 0, tu = 0;
        for (int it = 0; it < iters; ++it) {
            float a = 0, b = 0;
            CP_CUDA(cudaEventElapsedTime(&a, ev[2 * it], ev[2 * it + 1]));
            CP_CUDA(cudaEventElapsedTime(&b, ev[2 * it + 1], ev[2 * it + 2]));
            tp += a;
            tu += b;
        }
        for (auto& e : ev) cudaEventDestroy(e);
        // algorithmic bytes per launch (2 DOFs per node, N = 2n):
        //  P: values nnz*sv + block columns nnz/4*4 + read r, z + write z', Kz' (4 N sx)
        //  U: read x (16 n), z', r, Kz' (3 N sx), mask (2 n); write x, r (16 n + N sx)
        //     and the record (v', z') (2 N sx) [+ block Jacobi: read M^-1 (4 n sx)]
        const double N = 2 * n;
        if (ms_p) *ms_p = tp / iters;
        if (ms_u) *ms_u = tu / iters;
        if (bytes_p) *bytes_p = nnz * sv + nnz + 4 * N * sx;
        if (bytes_u) *bytes_u = 32 * n + 4 * N * sx + 2 * n + (precond ? 4 * n * sx : 0.0) + 2 * N * sx;
    });
}

CP_API int cp_bench_cg_fused(cp_instance* I, int precond, int iters, double* ms_iter, double* bytes_iter) {
    if (I && I->in_batch) return CP_ERR_BUSY;
    if (!I || iters <= 0 || (precond & ~1)) return CP_ERR_INVALID;
    return guarded(I->ctx, [&] {
        CP_CHECK(I->loads_set, CP_ERR_INVALID, "loads not set");
        cudaStream_t s = I->s();
        assemble(I, CP_PREC_FP64);
        cp::FusedArgs a = fused_args(I, precond);
        std::vector<cudaEvent_t> ev((size_t)iters + 1);
        for (auto& e : ev) CP_CUDA(cudaEventCreate(&e));
        cp::fused_launch_start(a, 0.0, (long long)iters + 8, s);
        for (int it = 0; it < iters; ++it) {
            CP_CUDA(cudaEventRecord(ev[it], s));
            cp::fused_launch_iteration(a, it & 1, s);
        }
        CP_CUDA(cudaEventRecord(ev[iters], s));
        CP_CUDA(cudaEventSynchronize(ev.back()));
        double t = 0;
        for (int it = 0; it < iters; ++it) {
            float x = 0;
            CP_CUDA(cudaEventElapsedTime(&x, ev[it], ev[it + 1]));
            t += x;
        }
        for (auto& e : ev) cudaEventDestroy(e);
        // algorithmic bytes of one iteration: 8 per value and one 4-byte
        // column per 2x2 block; per node read r, w, p, kp, x and the own
        // 48-byte record, write them back (256), the mask and the
        // block-Jacobi inverse (34 with, 2 without)
        const double n = I->n_nodes, nnz = (double)I->csr.nnz;
        if (ms_iter) *ms_iter = t / iters;
        if (bytes_iter) *bytes_iter = nnz * 8 + nnz + n * (256 + (precond ? 34 : 2));
    });
}

CP_API int cp_bench_assemble(cp_instance* I, int precision, int iters, double* ms, double* bytes) {
    if (I && I->in_batch) return CP_ERR_BUSY;
    if (!I || iters <= 0 || (precision != CP_PREC_FP64 && precision != CP_PREC_MIXED)) return CP_ERR_INVALID;
    return guarded(I->ctx, [&] {
        cudaStream_t s = I->s();
        assemble(I, precision);  // warm, and allocates the FP32 values if asked
        cudaEvent_t e0, e1;
        CP_CUDA(cudaEventCreate(&e0));
        CP_CUDA(cudaEventCreate(&e1));
        CP_CUDA(cudaEventRecord(e0, s));
        for (int it = 0; it < iters; ++it)
            cp::launch_assemble(I->mesh, I->csr, I->mat, I->st.E_c, I->st.nu_c, true, precision == CP_PREC_MIXED, s,
                                I->sms());
        CP_CUDA(cudaEventRecord(e1, s));
        CP_CUDA(cudaEventSynchronize(e1));
        float t = 0;
        CP_CUDA(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        I->launches += iters + 1;
        const double incs = 3.0 * I->mesh.c3 + 4.0 * I->mesh.c4 + 8.0 * I->mesh.c8;
        if (ms) *ms = t / iters;
        // values written once (sliced layout, padding included); the
        // connectivity (4 per node of an element) and E_c, nu_c (16 per
        // element); per incidence its code and slot bytes (8, 12 with 8-node
        // elements); the node coordinates once (16 per node)
        if (bytes)
            *bytes = 4.0 * I->csr.sell_blocks * (precision == CP_PREC_MIXED ? 12.0 : 8.0) + incs * 4.0 +
                     16.0 * I->n_elem + incs * (I->mesh.c8 ? 12.0 : 8.0) + 16.0 * I->n_nodes;
    });
}

CP_API int cp_get_csr(cp_instance* I, int* rows, int* cols, int* adj_pos, int* adj, double* values) {
    if (!I) return CP_ERR_INVALID;
    return guarded(I->ctx, [&] {
        cudaStream_t s = I->s();
        const int n = I->n_nodes;
        const long long nnz = I->csr.nnz;
        int *d_rows = nullptr, *d_cols = nullptr;
        if (rows || cols) {
            CP_CUDA(cudaMallocAsync(&d_rows, sizeof(int) * (2 * (size_t)n + 1), s));
            if (cols) CP_CUDA(cudaMallocAsync(&d_cols, sizeof(int) * (size_t)nnz, s));
            cp::csr_rows_cols(I->mesh, I->csr, d_rows, d_cols, s);
            if (rows) CP_CUDA(cudaMemcpyAsync(rows, d_rows, sizeof(int) * (2 * (size_t)n + 1), cudaMemcpyDeviceToHost, s));
            if (cols) CP_CUDA(cudaMemcpyAsync(cols, d_cols, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToHost, s));
        }
        if (adj_pos) CP_CUDA(cudaMemcpyAsync(adj_pos, I->csr.adj_pos, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s));
        if (adj) CP_CUDA(cudaMemcpyAsync(adj, I->csr.adj, sizeof(int) * (size_t)I->csr.nadj, cudaMemcpyDeviceToHost, s));
        double* d_vals = nullptr;
        if (values) {
            CP_CUDA(cudaMallocAsync(&d_vals, sizeof(double) * (size_t)nnz, s));
            cp::csr_export_values(I->mesh, I->csr, d_vals, s);
            CP_CUDA(cudaMemcpyAsync(values, d_vals, sizeof(double) * (size_t)nnz, cudaMemcpyDeviceToHost, s));
        }
        CP_CUDA(cudaStreamSynchronize(s));
        if (d_rows) cudaFreeAsync(d_rows, s);
        if (d_cols) cudaFreeAsync(d_cols, s);
        if (d_vals) cudaFreeAsync(d_vals, s);
        CP_CUDA(cudaStreamSynchronize(s));
    });
}

CP_API int cp_get_slot_map(cp_instance* I, int* slots) {
    if (!I || !slots) return CP_ERR_INVALID;
    return guarded(I->ctx, [&] {
        cudaStream_t s = I->s();
        const size_t ns = 9 * (size_t)I->mesh.c3 + 16 * (size_t)I->mesh.c4 + 64 * (size_t)I->mesh.c8;
        int* d = nullptr;
        CP_CUDA(cudaMallocAsync(&d, sizeof(int) * std::max<size_t>(ns, 1), s));
        cp::csr_slot_map(I->mesh, I->csr, d, s);
        CP_CUDA(cudaMemcpyAsync(slots, d, sizeof(int) * ns, cudaMemcpyDeviceToHost, s));
        CP_CUDA(cudaStreamSynchronize(s));
        cudaFreeAsync(d, s);
        CP_CUDA(cudaStreamSynchronize(s));
    });
}

static double* field_ptr(cp_instance* I, const char* name, size_t* count) {
    struct F {
        const char* n;
        double* p;
    } fs[] = {{"exx", I->st.exx},       {"eyy", I->st.eyy},     {"gamma", I->st.gam},    {"eps_i", I->st.eps_i},
              {"sxx", I->st.sxx},       {"syy", I->st.syy},     {"tau", I->st.tau},      {"sig_i", I->st.sig_i},
              {"table_s", I->st.table_s}, {"psi", I->st.psi},   {"E_c", I->st.E_c},      {"nu_c", I->st.nu_c},
              {"exx_p", I->st.exx_p},   {"eyy_p", I->st.eyy_p}, {"gamma_p", I->st.gam_p}, {"eps_p_i", I->st.eps_p_i}};
    if (!std::strcmp(name, "uv")) {
        *count = 2 * (size_t)I->n_nodes;
        return reinterpret_cast<double*>(I->u);
    }
    if (!std::strcmp(name, "rp")) {
        *count = 2 * (size_t)I->n_nodes;
        return reinterpret_cast<double*>(I->b);
    }
    for (auto& f : fs)
        if (!std::strcmp(name, f.n)) {
            *count = (size_t)I->n_elem;
            return f.p;
        }
    return nullptr;
}

CP_API int cp_get_field(cp_instance* I, const char* name, double* out) {
    if (!I || !name || !out) return CP_ERR_INVALID;
    size_t count = 0;
    double* p = field_ptr(I, name, &count);
    if (!p) return CP_ERR_INVALID;
    return guarded(I->ctx, [&] {
        CP_CUDA(cudaMemcpyAsync(out, p, sizeof(double) * count, cudaMemcpyDeviceToHost, I->s()));
        CP_CUDA(cudaStreamSynchronize(I->s()));
    });
}

CP_API int cp_set_field(cp_instance* I, const char* name, const double* in) {
    if (I && I->in_batch) return CP_ERR_BUSY;  // owned by a batch until harvested
    if (!I || !name || !in) return CP_ERR_INVALID;
    size_t count = 0;
    double* p = field_ptr(I, name, &count);
    if (!p) return CP_ERR_INVALID;
    return guarded(I->ctx, [&] {
        CP_CUDA(cudaMemcpyAsync(p, in, sizeof(double) * count, cudaMemcpyHostToDevice, I->s()));
        CP_CUDA(cudaStreamSynchronize(I->s()));
    });
}

}  // extern "C"
