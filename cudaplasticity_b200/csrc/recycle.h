// Initial guesses from the recent solution increments ("recycling") for the
// FP64 linear solves of the secant iteration (cp_solve_opts.recycle).
//
// Within one load level the outer iterations solve K_k u_k = b with K_k
// changing a little from one iteration to the next. Before each solve the
// warm start u (the last solution) is corrected by the Galerkin projection
// of the error onto W = [d_1 .. d_m], the last m increments d = u_k - u_{k-1}
// of the same level, newest first:
//     x0 = u + W y,   (W^T K W) y = W^T m.(b - K u)
// (m the Dirichlet mask; the increments are zero on fixed DOFs). The CG then
// starts from a smaller residual and stops on the same criterion, so the
// converged iterate meets the same tolerance and the secant fixed point is
// unchanged. The small system is solved by a Cholesky factorisation of the
// diagonally scaled Gram matrix that drops the increments whose pivot falls
// below 1e-10 (nearly dependent directions), in a fixed order, so the result
// is deterministic.
#pragma once

#include <cuda_runtime.h>

namespace cp {

constexpr int kRecycleMax = 6;
// Gram entries (j <= k) at k (k + 1) / 2 + j, then the right-hand sides.
constexpr int kRecycleGram = kRecycleMax * (kRecycleMax + 1) / 2;
constexpr int kRecycleSums = kRecycleGram + kRecycleMax;
constexpr int kRecycleStride = kRecycleSums + 1;  // doubles per block partial

struct RecycleArgs {
    int n = 0;  // nodes
    const int* slice_ptr = nullptr;
    const int* scol = nullptr;
    const double* val = nullptr;  // FP64 sliced 2x2 blocks
    double2* u = nullptr;
    const double2* b = nullptr;
    const uchar2* mask = nullptr;
    double2* w = nullptr;   // kRecycleMax x n increments
    double2* u0 = nullptr;  // the warm start before the correction
    int slot[kRecycleMax] = {0, 0, 0, 0, 0, 0};  // increments in use, newest first
    int cnt = 0;
    double* partials = nullptr;  // grid x kRecycleStride
    unsigned int* ticket = nullptr;
    double* y = nullptr;  // kRecycleMax coefficients
};

// Blocks of the sums kernel for n nodes (the partials buffer holds that many).
int recycle_grid(int n, int sm_count);
// u0 = u, then (cnt > 0) the Gram sums, the small solve and u += W y.
void recycle_project(const RecycleArgs& a, int sm_count, cudaStream_t s);
// The small solve on the host (the device's code; cpx_recycle_solve).
int recycle_solve_host(const double* sums, int cnt, double* y);
// w[slot] = u - u0 after the linear solve.
void recycle_push(const RecycleArgs& a, int slot, int sm_count, cudaStream_t s);

}  // namespace cp
