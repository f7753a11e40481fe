// Shared device helpers for the cuplast kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define CP_WARP 32

// Work-list / grid sizing: every kernel in the library runs a grid-stride
// loop over its units, so grids are sized in multiples of the SM count.
namespace cp {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over groups of G consecutive lanes (G a power of two <= 32); every lane
// of the group receives the group's sum.
template <int G>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, G);
    return v;
}
template <int G>
__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, G);
    return v;
}

// Block-wide sum of one double per thread, deterministic (fixed tree).
// Result valid in thread 0. `sh` needs blockDim.x/32 doubles.
__device__ __forceinline__ double block_sum(double v, double* sh) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) sh[w] = v;
    __syncthreads();
    int nw = (blockDim.x + 31) >> 5;
    double s = 0.0;
    if (w == 0) {
        s = lane < nw ? sh[lane] : 0.0;
        s = warp_sum(s);
    }
    __syncthreads();
    return s;
}

// Two sums at once (same determinism). Results valid in thread 0.
__device__ __forceinline__ double2 block_sum2(double a, double b, double* sh) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    if (lane == 0) { sh[2 * w] = a; sh[2 * w + 1] = b; }
    __syncthreads();
    int nw = (blockDim.x + 31) >> 5;
    double2 s = make_double2(0.0, 0.0);
    if (w == 0) {
        s.x = warp_sum(lane < nw ? sh[2 * lane] : 0.0);
        s.y = warp_sum(lane < nw ? sh[2 * lane + 1] : 0.0);
    }
    __syncthreads();
    return s;
}

// "Last block finishes": every block stores its partial(s), fences, and takes
// a ticket; the block that draws the final ticket reduces all partials in
// index order (so the result does not depend on which block came last) and
// resets the ticket. Returns true in all threads of the last block.
__device__ __forceinline__ bool last_block_arrive(unsigned int* ticket, bool* sh_flag) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int t = atomicAdd(ticket, 1u);
        *sh_flag = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (*sh_flag) __threadfence();
    return *sh_flag;
}

// Deterministic sum of n doubles by one block (fixed assignment + tree).
__device__ __forceinline__ double block_reduce_array(const volatile double* p, int n, double* sh) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += p[i];
    return block_sum(s, sh);
}
__device__ __forceinline__ double2 block_reduce_array2(const volatile double* p, int n, double* sh) {
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) { a += p[2 * i]; b += p[2 * i + 1]; }
    return block_sum2(a, b, sh);
}

// Loads of data a kernel streams through once (matrix values, block
// columns): ST = true marks them evict-first (ld.global.cs), so that they do
// not push the gathered neighbour records out of L1 / L2; ST = false reads
// them through the read-only path.
template <bool ST, typename V>
__device__ __forceinline__ V ld_stream(const V* p) {
    if constexpr (ST) return __ldcs(p);
    else return __ldg(p);
}

// Whether the two-kernel and the batched CG take the ST = true forms (the
// default: FP32 k_cg_p 53.1 -> 47.3 us and FP64 84.6 -> 76.5 us on the
// 2.1M-DOF plate, the batch 3.7 % per trip); CUPLAST_STREAM_LOADS=0 turns it
// off for measurements. The one-launch FP64 iteration gained nothing from it
// (345 against 347 ms for 3000 iterations) and keeps the read-only path.
bool stream_loads();

// Whether the one-launch FP64 CG iterations (cg_fused.cu) launch with
// programmatic stream serialization: the next grid is scheduled while the current one finishes
// and waits for it on the device (cudaGridDependencySynchronize), hiding the
// launch gap of latency-bound iterations. CUPLAST_PDL=0 launches them
// plainly (measurements).
bool pdl_enabled();

// The first statements of a kernel launched that way: nothing of the
// previous grid is read before it has completed and its writes are visible;
// then the next grid may be scheduled. Without the launch attribute both
// return at once.
__device__ __forceinline__ void pdl_enter() {
    cudaGridDependencySynchronize();
    cudaTriggerProgrammaticLaunchCompletion();
}

}  // namespace cp
