// Host-side definitions of the opaque handles cp_context and cp_instance
// (include/cuplast.h), shared by the translation units that drive them.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <string>
#include <vector>

#include "cg.h"
#include "internal.h"
#include "mg.h"
#include "recycle.h"

struct cp_context {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string last_error;
    // Set from another thread (the solve service's oldest-first priorities):
    // cp_solve moves to this stream at its next outer iteration, after the
    // current one has drained.
    std::atomic<cudaStream_t> restream{nullptr};
};

struct cp_instance {
    cp_context* ctx = nullptr;
    cp::DevMesh mesh;
    cp::DevCsr csr;
    cp_material mat_host{};
    cp::MaterialDev mat{};
    int n_nodes = 0, n_elem = 0;
    double2 *u = nullptr, *b = nullptr, *b_full = nullptr, *u_full = nullptr;
    uchar2* mask = nullptr;
    double2 *r64 = nullptr, *z64a = nullptr, *z64b = nullptr, *q64 = nullptr;
    float2 *r32 = nullptr, *z32 = nullptr, *q32 = nullptr;
    double4 *rec64a = nullptr, *rec64b = nullptr;  // (v, z) records of the two-kernel CG (cg.cu), by parity
    float4 *rec32a = nullptr, *rec32b = nullptr;
    double4* minv64 = nullptr;
    float4* minv32 = nullptr;
    cp::ElemState st{};
    double* st_block = nullptr;
    cp::CgScalars* sc = nullptr;
    cp::OuterScalars* osc = nullptr;
    double* partials = nullptr;
    int max_blocks = 0;
    cp::CgScalars* sc_h = nullptr;     // pinned
    cp::OuterScalars* osc_h = nullptr;  // pinned
    cudaGraphExec_t g64[2] = {nullptr, nullptr}, g32[2] = {nullptr, nullptr};  // [precond]
    int body_iters = 8;
    bool use_graph = true;  // CG loop as a CUDA graph with a device-side WHILE condition
    bool loads_set = false;
    bool in_batch = false;  // owned by a cp_batch until harvested: no other call may touch it
    std::atomic<int> cancel{0};  // set from another thread: cp_solve stops at its next outer iteration
    // single-launch FP64 CG (cg_fused.cu), allocated on first use
    bool fused_fp64 = true;        // false (CUPLAST_FP64_CG=classic): the two-kernel loop of cg.cu
    bool persistent_fp64 = false;  // CUPLAST_FP64_CG=persistent: one cooperative launch per linear solve
    // CUPLAST_TEST_BARRIER_NS=<ns> (failure-path tests of the persistent CG):
    // each grid-barrier wait gives up after <ns> and waits for a step that is
    // never released, so every wait runs out and the solve ends with
    // CP_ERR_TIMEOUT
    unsigned long long test_barrier_ns = 0;
    bool cluster_fp64 = true;      // one thread-block cluster when the instance fits (CUPLAST_FP64_CG other than cluster: off)
    int cluster_planned = 0;       // cluster_plan below is computed (once per instance)
    double2* pred_u = nullptr;     // level predictor (cp_solve_opts.predict): the last level's u and psi
    double* pred_psi = nullptr;
    // initial guesses from the level's solution increments (cp_solve_opts.recycle, recycle.h), allocated on
    // first use: the increments (a ring of kRecycleMax), the warm start before the correction, partial sums,
    // the coefficients and a ticket; rec_cnt increments in use, rec_head the next slot to write
    double2 *rec_w = nullptr, *rec_u0 = nullptr;
    double *rec_part = nullptr, *rec_y = nullptr;
    unsigned int* rec_ticket = nullptr;
    int rec_cnt = 0, rec_head = 0;
    cp::ClusterPlan cluster_plan;
    double2 *f_r = nullptr, *f_w = nullptr, *f_p = nullptr, *f_kp = nullptr, *f_g = nullptr;
    double* f_partials = nullptr;
    cudaGraphExec_t gf[2] = {nullptr, nullptr};  // [precond]
    // batched engine (batch.cu): FP32 CG vectors, neighbour records, partial sums
    float2* bt_vec = nullptr;
    float4* bt_rec = nullptr;
    double* bt_part = nullptr;
    // aggregation-multigrid PCG (mg.cu, cp_solve_opts.precond 2), built on first use
    std::vector<unsigned char> mask_host;  // the Dirichlet mask of the last cp_instance_set_loads
    std::vector<unsigned char> mg_mask;    // the mask the hierarchy was built for
    bool mg_ready = false;
    cp::MgDev mg;
    std::vector<void*> mg_allocs;
    size_t mg_bytes = 0;  // the part of `bytes` the hierarchy holds
    cudaGraphExec_t gmg = nullptr;
    long long launches = 0;  // kernels launched (graph nodes included)
    int last_assembly = -1;  // precision of the last assembly
    size_t bytes = 0;
    std::vector<void*> allocs;

    template <typename T>
    T* alloc(size_t count) {
        void* p = nullptr;
        size_t nb = std::max<size_t>(count, 1) * sizeof(T);
        CP_CUDA(cudaMallocAsync(&p, nb, ctx->stream));
        allocs.push_back(p);
        bytes += nb;
        return static_cast<T*>(p);
    }

    cudaStream_t s() const { return ctx->stream; }
    int sms() const { return ctx->sm_count; }

    template <typename T>
    cp::CgArgs<T> cg_args(int precond = 0);
};


namespace cp {
// Allocates (once) what the mixed-precision solve needs beyond the FP64
// instance: FP32 values and recurrence vectors, and with precond the FP32
// block-Jacobi vectors. Stream-ordered on the instance's context stream.
void instance_prepare_mixed(cp_instance* I, int precond);
}  // namespace cp
