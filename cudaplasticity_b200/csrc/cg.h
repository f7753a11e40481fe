// CG launch interface (kernels in cg.cu).
#pragma once

#include "internal.h"

namespace cp {

template <typename T>
struct Vec2;
template <>
struct Vec2<double> {
    using type = double2;
};
template <>
struct Vec2<float> {
    using type = float2;
};
template <typename T>
struct Vec4;
template <>
struct Vec4<double> {
    using type = double4;
};
template <>
struct Vec4<float> {
    using type = float4;
};

// Everything the CG kernels touch, passed by value.
template <typename T>
struct CgArgs {
    using V2 = typename Vec2<T>::type;
    int n = 0;            // nodes (2 DOFs each)
    int sm_count = 148;
    int max_blocks = 0;   // capacity of the partials buffer (blocks)
    const int* slice_ptr = nullptr;  // sliced layout (see DevCsr)
    const int* scol = nullptr;
    const T* val = nullptr;         // K in the recurrence type, 4 values per block
    const double2* b = nullptr;     // right-hand side (FP64)
    const uchar2* mask = nullptr;   // 1 = free DOF
    double2* x = nullptr;           // solution, accumulated in FP64
    V2* r = nullptr;
    typename Vec4<T>::type* minv = nullptr;  // inverse 2x2 diagonal blocks (block Jacobi only)
    int precond = 0;                // 0: plain CG (reference), 1: 2x2 block-Jacobi PCG
    // per node (v, z): v = M^-1 r (r without the preconditioner), z the
    // direction; by iteration parity
    typename Vec4<T>::type* rec0 = nullptr;
    typename Vec4<T>::type* rec1 = nullptr;
    V2* zn = nullptr;               // z' from P to U
    V2* q = nullptr;
    CgScalars* sc = nullptr;
    double* partials = nullptr;     // >= 3 * max_blocks doubles
};

// The single-launch FP64 iteration of cg_fused.cu.
struct FusedArgs {
    int n = 0;
    int sm_count = 148;
    int max_blocks = 0;              // capacity of partials (blocks, 6 sums each)
    const int* slice_ptr = nullptr;
    const int* scol = nullptr;
    const double* val = nullptr;
    const double2* b = nullptr;
    const uchar2* mask = nullptr;
    double2* x = nullptr;
    double2 *r = nullptr, *w = nullptr, *p = nullptr, *kp = nullptr;
    double2 *gA = nullptr, *gB = nullptr;  // per node: u, M w, M kp (by parity)
    double4* minv = nullptr;
    int precond = 0;
    CgScalars* sc = nullptr;
    double* partials = nullptr;
    // persistent form only: time limit of each grid-barrier wait, and the
    // number of extra steps every wait asks for (0; 1 makes each wait ask for
    // a step that is never released, so that every wait runs out: the
    // time-out path's test)
    unsigned long long barrier_ns = 2000000000ull;
    unsigned int barrier_skew = 0;
};

void fused_launch_start(const FusedArgs& a, double eps2, long long max_iter, cudaStream_t s);
void fused_launch_iteration(const FusedArgs& a, int parity, cudaStream_t s);
// The whole solve (init, first step, iterations) as one cooperative launch;
// only when its grid is that of the kernels above (fused_persistent_fits).
bool fused_persistent_fits(const FusedArgs& a);
void fused_launch_persistent(const FusedArgs& a, double eps2, long long max_iter, cudaStream_t s);
cudaGraphExec_t fused_build_while_graph(const FusedArgs& a, int body_iters, cudaStream_t s);

// The same solve inside one thread-block cluster (cg_cluster.cu), for
// instances whose blocks of K and records fit the cluster's shared memory.
struct ClusterPlan {
    int ctas = 0;      // cluster size (0: does not fit)
    int spc = 0;       // slices of 32 nodes per CTA (one warp each)
    int wmax = 0;      // widest node row, in blocks
    size_t smem = 0;   // dynamic shared memory per CTA
};
ClusterPlan cluster_cg_plan(const FusedArgs& a, int max_width);
void cluster_cg_launch(const FusedArgs& a, const ClusterPlan& plan, double eps2, long long max_iter, cudaStream_t s);

template <typename T>
void cg_launch_init(const CgArgs<T>& a, const void* valA, bool valA_is_fp64, double eps2, long long max_iter,
                    int relative_to_r0, double outer_eps2, cudaStream_t s);
template <typename T>
void cg_launch_iteration(const CgArgs<T>& a, int parity, cudaStream_t s);
template <typename T>
void cg_launch_p(const CgArgs<T>& a, int parity, cudaStream_t s);
template <typename T>
void cg_launch_u(const CgArgs<T>& a, int parity, cudaStream_t s);
template <typename T>
cudaGraphExec_t cg_build_while_graph(const CgArgs<T>& a, int body_iters, cudaStream_t s);

}  // namespace cp
