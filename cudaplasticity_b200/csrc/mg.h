// Aggregation-multigrid preconditioned FP64 CG (mg.cu): device side of the
// hierarchy built on the host by amg_setup.cpp.
//
// Level 0 is the instance's own K (sliced layout, 2x2 blocks); every coarser
// level l >= 1 is a block CSR with 3x3 blocks whose rows hold the diagonal
// block first. Per outer iteration the coarse operators are recomputed from
// the new K through the fixed Galerkin maps, with the smoother's block
// inverses, its damping (a Gershgorin bound of D^-1 A, so the damped Jacobi
// sweep always converges) and the dense inverse of the coarsest level.
// The preconditioner is one V-cycle: one damped block-Jacobi sweep before and
// one after the coarse correction on every level but the coarsest, which is
// solved exactly; pre- and post-smoothers are the same symmetric sweep, so
// the V-cycle is a symmetric positive definite operator and plain PCG
// applies.
#pragma once

#include "internal.h"

struct cp_instance;

namespace cp {

constexpr int kMgMaxLevels = 16;
constexpr int kMgMaxCoarsest = 256;  // coarsest DOFs accepted: its inverse and scratch stay within 1 MB
constexpr int kMgMaxCoarse = 160;  // coarsest DOFs whose inversion runs in shared memory
constexpr int kMgMinCoarse = 150;  // coarsening stops at this many DOFs
constexpr int kMgPartNodes = 256;  // level-0 node ranges that no aggregate crosses
constexpr double kMgOmega = 1.8;   // damping, relative to the Gershgorin bound

struct MgLevel {
    int n = 0, fb = 2, nb = 0;  // nodes, DOFs per node, blocks
    // operator (levels >= 1; level 0 is the instance's K)
    int* rp = nullptr;          // n + 1 block offsets
    int* ci = nullptr;          // column node of every block
    double* val = nullptr;      // 9 per block, row-major
    double* dinv = nullptr;     // smoother: fb x fb inverse of the diagonal block per node
    int* part_pos = nullptr;    // levels >= 1: the nodes of level-0 range p are part_pos[p] .. part_pos[p+1]
    // transfer to the next level (not on the coarsest)
    int* agg = nullptr;         // next-level node of every node
    double* T = nullptr;        // fb x 3 prolongator block per node, row-major
    int* mem_pos = nullptr;     // members of every next-level node: mem[mem_pos[a] .. mem_pos[a+1])
    int* mem = nullptr;
    int* gal_pos = nullptr;     // next level's block c gathers gal[gal_pos[c] .. gal_pos[c+1])
    int4* gal = nullptr;        // (this level's block index, row node, column node, 0)
    // V-cycle vectors, fb per node (level 0: y and z only)
    double* b = nullptr;        // restricted residual
    double* y = nullptr;        // after the pre-smoothing sweep
    double* z = nullptr;        // correction handed to the level above
};

struct MgDev {
    int L = 0;                  // levels
    int nc = 0;                 // DOFs of the coarsest level
    MgLevel lv[kMgMaxLevels];
    double* cinv = nullptr;     // nc x nc inverse of the coarsest operator, column-major
    double* work = nullptr;     // nc x nc scratch when nc > kMgMaxCoarse (inverted in global memory)
    double* lam = nullptr;      // per level: Gershgorin bound of D^-1 A
    double omega = kMgOmega;
};

// The CG side (level 0), passed by value.
struct MgArgs {
    int n = 0;
    int sm_count = 148;
    int max_blocks = 0;         // capacity of partials (blocks, 2 sums each)
    const int* slice_ptr = nullptr;
    const int* scol = nullptr;
    const double* val = nullptr;
    const double2* b = nullptr;
    const uchar2* mask = nullptr;
    double2* x = nullptr;
    double2* r = nullptr;
    double2* q = nullptr;
    double2* p0 = nullptr;      // search direction, by iteration parity
    double2* p1 = nullptr;
    CgScalars* sc = nullptr;
    double* partials = nullptr;
};

// Coarse operators, smoother data and the coarsest inverse from the current K.
int mg_launch_setup(const MgDev& m, const MgArgs& a, cudaStream_t s);
// r = m.(b - K x), the first V-cycle and the scalars of a solve.
int mg_launch_start(const MgDev& m, const MgArgs& a, double eps2, long long max_iter, cudaStream_t s);
// One PCG iteration (search direction, update, V-cycle). `ev` (optional, 6
// events): recorded before P and after P, U, R0, the coarse levels and S0.
int mg_launch_iteration(const MgDev& m, const MgArgs& a, int parity, cudaStream_t s, cudaEvent_t* ev = nullptr);
// Algorithmic bytes per launch of P, U, R0, the coarse levels (all of their
// kernels), S0 and the per-outer-iteration set-up (all of its kernels).
void mg_algorithmic_bytes(const MgDev& m, const MgArgs& a, long long blocks0, double* bytes);
// Kernels launched by one iteration.
int mg_launches_per_iteration(const MgDev& m);
// while (!converged) { body_iters iterations } as one graph (body_iters even).
cudaGraphExec_t mg_build_while_graph(const MgDev& m, const MgArgs& a, int body_iters, cudaStream_t s);

// Upper estimate of the device bytes a hierarchy adds to an instance of
// n_nodes nodes and `blocks` level-0 blocks (nodes + graph edges): level 0's
// maps and vectors, and coarse levels of at most half the nodes each time.
size_t mg_footprint(size_t n_nodes, size_t blocks);

// Builds the hierarchy of an instance (host set-up, uploaded once) unless the
// one it holds was built for the same Dirichlet mask; mg_release frees it.
void mg_prepare(cp_instance* I);
void mg_release(cp_instance* I);

}  // namespace cp
