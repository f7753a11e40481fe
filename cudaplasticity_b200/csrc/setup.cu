// Device-side set-up of the sparsity structure, in the reference's ordering.
//
// The reference builds SparseSLAE(Mesh&, 2) on the host (src/SparseSLAE.h:60-196,
// and CudaSparseSLAE::constructorByCPU, src/CudaSparseSLAE.cuh:303-458): per node,
// the distinct other nodes of its elements in first-occurrence order over the
// traversal "triangles, then 4-node quads, then 8-node quads; element order;
// own local index i; local j != i". Here the same order comes out of a
// per-node walk over its incident elements sorted by element id:
//   1. count incidences per node           (integer atomics, counts only)
//   2. exclusive scan -> inc_pos, cap_pos  (cap = sum of (nen - 1), the
//                                            reference's linkCounts)
//   3. scatter incidences, then sort each node's few entries by element id
//   4. per node: neighbour list in first-occurrence order + for every
//      incidence the block index of each local node in this node's row
//      (the element-to-CSR slot map, one byte per local node)
//   5. scan neighbour counts -> adj_pos; compact the lists -> adj
// All of it is deterministic: atomics only count, and each node's entries are
// sorted before they are used.
#include "common.cuh"
#include "internal.h"

namespace cp {

namespace {

constexpr int kMaxInc = 64;       // incident elements per node
constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int elem_nen(const DevMesh& m, int e) { return e < m.c3 ? 3 : (e < m.c3 + m.c4 ? 4 : 8); }

__device__ __forceinline__ int nth(const int4& v, int j) {
    return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w));
}

// Local node j (0 .. nen-1) of element e.
__device__ __forceinline__ int elem_node(const DevMesh& m, int e, int j) {
    if (e < m.c3) return nth(m.e3[e], j);
    if (e < m.c3 + m.c4) return nth(m.e4[e - m.c3], j);
    return nth(m.e8[2 * (e - m.c3 - m.c4) + (j >> 2)], j & 3);
}

__device__ __forceinline__ long long incidence_count(const DevMesh& m) {
    return 3LL * m.c3 + 4LL * m.c4 + 8LL * m.c8;
}

// Incidence t (element order, then local index) -> element and local index.
__device__ __forceinline__ void incidence(const DevMesh& m, long long t, int& e, int& i) {
    if (t < 3LL * m.c3) { e = (int)(t / 3); i = (int)(t % 3); return; }
    t -= 3LL * m.c3;
    if (t < 4LL * m.c4) { e = m.c3 + (int)(t / 4); i = (int)(t % 4); return; }
    t -= 4LL * m.c4;
    e = m.c3 + m.c4 + (int)(t / 8);
    i = (int)(t % 8);
}

__global__ void k_count(DevMesh m, int* inc_cnt, int* cap_cnt, int* err) {
    const long long total = incidence_count(m);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int e, i;
        incidence(m, t, e, i);
        const int nen = elem_nen(m, e);
        const int n = elem_node(m, e, i);
        if (n < 0 || n >= m.n_nodes) { atomicExch(err, 1); continue; }
        for (int j = 0; j < nen; ++j)
            if (j != i && elem_node(m, e, j) == n) atomicExch(err, 2);  // degenerate element
        atomicAdd(&inc_cnt[n], 1);
        atomicAdd(&cap_cnt[n], nen - 1);
    }
}

// Exclusive scan, three passes (tile scan, scan of tile totals, add).
__global__ void k_scan_tiles(const int* in, int* out, int* tile_tot, int n) {
    __shared__ int sh[kScanThreads / 32];
    const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int v[kScanItems], run = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        int t = v[k];
        v[k] = run;
        run += t;
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5, inc = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) sh[w] = inc;
    __syncthreads();
    if (w == 0) {
        int x = lane < kScanThreads / 32 ? sh[lane] : 0, xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) xi += y;
        }
        if (lane < kScanThreads / 32) sh[lane] = xi - x;
        if (lane == kScanThreads / 32 - 1) tile_tot[blockIdx.x] = xi;
    }
    __syncthreads();
    int off = sh[w] + inc - run;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) out[base + k] = off + v[k];
}

__global__ void k_scan_totals(int* tile_tot, int ntiles, int* total_out) {
    __shared__ int carry;
    __shared__ int sh[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int s = 0; s < ntiles; s += blockDim.x) {
        int i = s + threadIdx.x;
        int x = i < ntiles ? tile_tot[i] : 0, xi = x;
        int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) xi += y;
        }
        if (lane == 31) sh[w] = xi;
        __syncthreads();
        if (w == 0) {
            int nw = blockDim.x / 32;
            int z = lane < nw ? sh[lane] : 0, zi = z;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, zi, o);
                if (lane >= o) zi += y;
            }
            if (lane < nw) sh[lane] = zi - z;
        }
        __syncthreads();
        int excl = carry + sh[w] + xi - x;
        if (i < ntiles) tile_tot[i] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total_out = carry;
}

__global__ void k_scan_add(int* out, const int* tile_off, int n, const int* total, int* out_last) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += tile_off[i / kScanTile];
    if (i == 0) *out_last = *total;
}

void exclusive_scan(const int* in, int* out /* n+1 */, int n, int* scratch /* tiles+1 */, cudaStream_t s) {
    int ntiles = (n + kScanTile - 1) / kScanTile;
    if (ntiles < 1) ntiles = 1;
    k_scan_tiles<<<ntiles, kScanThreads, 0, s>>>(in, out, scratch, n);
    k_scan_totals<<<1, 1024, 0, s>>>(scratch, ntiles, scratch + ntiles);
    k_scan_add<<<(n + 255) / 256 + 1, 256, 0, s>>>(out, scratch, n, scratch + ntiles, out + n);
}

__global__ void k_fill(DevMesh m, const int* inc_pos, int* cursor, int* inc) {
    const long long total = incidence_count(m);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int e, i;
        incidence(m, t, e, i);
        const int n = elem_node(m, e, i);
        if (n < 0 || n >= m.n_nodes) continue;
        int slot = inc_pos[n] + atomicAdd(&cursor[n], 1);
        inc[slot] = (e << 3) | i;
    }
}

__global__ void k_adjacency(DevMesh m, const int* inc_pos, int* inc, const int* cap_pos, int* links, int* adj_cnt,
                            uint32_t* inc_k, uint32_t* inc_k8, int* max_deg, int* err) {
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < m.n_nodes; n += gridDim.x * blockDim.x) {
        const int b = inc_pos[n], cnt = inc_pos[n + 1] - b;
        if (cnt > kMaxInc) { atomicExch(err, 3); adj_cnt[n] = 0; continue; }
        // insertion sort of this node's incidences by (element, local index)
        for (int a = b + 1; a < b + cnt; ++a) {
            int key = inc[a], c = a - 1;
            while (c >= b && inc[c] > key) { inc[c + 1] = inc[c]; --c; }
            inc[c + 1] = key;
        }
        int* L = links + cap_pos[n];
        int s = 0;
        for (int q = b; q < b + cnt; ++q) {
            const int e = inc[q] >> 3, i = inc[q] & 7;
            const int nen = elem_nen(m, e);
            uint32_t packed = 0, packed8 = 0;
            for (int j = 0; j < nen; ++j) {
                uint32_t k = 0;
                if (j != i) {
                    const int mj = elem_node(m, e, j);
                    int pos = -1;
                    for (int t = 0; t < s; ++t)
                        if (L[t] == mj) { pos = t; break; }
                    if (pos < 0) { pos = s; L[s++] = mj; }
                    k = (uint32_t)(pos + 1);
                }
                if (k > 255u) { atomicExch(err, 4); k = 255u; }
                if (j < 4) packed |= k << (8 * j);
                else packed8 |= k << (8 * (j - 4));
            }
            inc_k[q] = packed;
            if (inc_k8) inc_k8[q] = packed8;
        }
        adj_cnt[n] = s;
        atomicMax(max_deg, s);
    }
}

__global__ void k_adj_write(int n_nodes, const int* cap_pos, const int* links, const int* adj_pos, int* adj) {
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_nodes; n += gridDim.x * blockDim.x) {
        const int* L = links + cap_pos[n];
        const int b = adj_pos[n], s = adj_pos[n + 1] - b;
        for (int t = 0; t < s; ++t) adj[b + t] = L[t];
    }
}

__global__ void k_rows_cols(int n_nodes, const int* adj_pos, const int* adj, int* rows, int* cols) {
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_nodes; n += gridDim.x * blockDim.x) {
        const int begin = adj_pos[n], size = adj_pos[n + 1] - begin;
        // rows[2n + r + 1] = 4 begin + 2 (r + 1) size + 2 (2n + r + 1), SparseSLAE.h:170
        if (n == 0) rows[0] = 0;
        for (int r = 0; r < 2; ++r) rows[2 * n + r + 1] = begin * 4 + (r + 1) * size * 2 + (2 * n + r + 1) * 2;
        if (cols) {
            for (int r = 0; r < 2; ++r) {
                int base = 4 * (begin + n) + r * 2 * (size + 1);
                cols[base] = 2 * n;
                cols[base + 1] = 2 * n + 1;
                for (int k = 0; k < size; ++k) {
                    cols[base + 2 * (k + 1)] = 2 * adj[begin + k];
                    cols[base + 2 * (k + 1) + 1] = 2 * adj[begin + k] + 1;
                }
            }
        }
    }
}

__global__ void k_slot_map(DevMesh m, const int* inc_pos, const int* inc, const uint32_t* inc_k,
                           const uint32_t* inc_k8, const int* adj_pos, int* slots) {
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < m.n_nodes; n += gridDim.x * blockDim.x) {
        const int base = 4 * (adj_pos[n] + n);
        for (int q = inc_pos[n]; q < inc_pos[n + 1]; ++q) {
            const int e = inc[q] >> 3, i = inc[q] & 7, nen = elem_nen(m, e);
            const long long off = e < m.c3 ? 9LL * e
                                : e < m.c3 + m.c4 ? 9LL * m.c3 + 16LL * (e - m.c3)
                                                  : 9LL * m.c3 + 16LL * m.c4 + 64LL * (e - m.c3 - m.c4);
            const uint64_t kk = (uint64_t)inc_k[q] | (nen == 8 ? (uint64_t)inc_k8[q] << 32 : 0);
            for (int j = 0; j < nen; ++j) slots[off + i * nen + j] = base + 2 * (int)((kk >> (8 * j)) & 0xffu);
        }
    }
}

__global__ void k_slice_width(int n_nodes, int n_slices, const int* adj_pos, int* width32) {
    for (int sl = blockIdx.x * blockDim.x + threadIdx.x; sl < n_slices; sl += gridDim.x * blockDim.x) {
        int w = 1;
        for (int l = 0; l < 32; ++l) {
            int n = 32 * sl + l;
            if (n < n_nodes) w = max(w, adj_pos[n + 1] - adj_pos[n] + 1);
        }
        width32[sl] = 32 * w;
    }
}

__global__ void k_sell_cols(int n_nodes, int n_slices, const int* adj_pos, const int* adj, const int* slice_ptr,
                            int* scol) {
    const long long total = 32LL * n_slices;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int sl = (int)(t >> 5), l = (int)(t & 31), n = 32 * sl + l;
        const int base = slice_ptr[sl], w = (slice_ptr[sl + 1] - base) >> 5;
        const int s = n < n_nodes ? adj_pos[n + 1] - adj_pos[n] : -1;
        for (int k = 0; k < w; ++k) {
            int c = 0;
            if (n < n_nodes) c = (k >= 1 && k <= s) ? adj[adj_pos[n] + k - 1] : n;
            scol[base + 32 * k + l] = c;
        }
    }
}

__global__ void k_export_values(int n_nodes, const int* adj_pos, const int* slice_ptr, const double* val,
                                double* data) {
    for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_nodes; n += gridDim.x * blockDim.x) {
        const int s = adj_pos[n + 1] - adj_pos[n], L = 2 * (s + 1);
        const long long r0 = 4LL * (adj_pos[n] + n);
        const int sl = n >> 5, l = n & 31;
        for (int k = 0; k <= s; ++k) {
            const double* b = val + 4LL * (slice_ptr[sl] + 32 * k + l);
            data[r0 + 2 * k] = b[0];
            data[r0 + 2 * k + 1] = b[1];
            data[r0 + L + 2 * k] = b[2];
            data[r0 + L + 2 * k + 1] = b[3];
        }
    }
}

}  // namespace

void setup_csr(DevMesh& m, DevCsr& csr, cudaStream_t s, int sm_count) {
    const int n = m.n_nodes;
    const int ntiles = (n + kScanTile - 1) / kScanTile + 1;
    // one scratch allocation: counts, cursors, cap offsets, scan tiles, flags
    size_t words = 4 * (size_t)(n + 1) + 2 * (size_t)(ntiles + 1) + 8;
    int* scratch = nullptr;
    CP_CUDA(cudaMallocAsync(&scratch, words * sizeof(int), s));
    CP_CUDA(cudaMemsetAsync(scratch, 0, words * sizeof(int), s));
    int* inc_cnt = scratch;
    int* cap_cnt = inc_cnt + (n + 1);
    int* cap_pos = cap_cnt + (n + 1);
    int* cursor = cap_pos + (n + 1);
    int* tiles = cursor + (n + 1);
    int* flags = tiles + 2 * (ntiles + 1);  // [0] error, [1] max degree
    const long long incs = 3LL * m.c3 + 4LL * m.c4 + 8LL * m.c8;
    CP_CHECK(incs < (1LL << 31), CP_ERR_UNSUPPORTED, "mesh too large for 32-bit incidence offsets");
    CP_CHECK((long long)m.c3 + m.c4 + m.c8 < (1LL << 28), CP_ERR_UNSUPPORTED, "mesh: too many elements");
    CP_CUDA(cudaMallocAsync(&csr.inc_pos, (n + 1) * sizeof(int), s));
    CP_CUDA(cudaMallocAsync(&csr.adj_pos, (n + 1) * sizeof(int), s));
    CP_CUDA(cudaMallocAsync(&csr.inc, (incs + 1) * sizeof(int), s));
    CP_CUDA(cudaMallocAsync(&csr.inc_k, (incs + 1) * sizeof(uint32_t), s));
    if (m.c8) CP_CUDA(cudaMallocAsync(&csr.inc_k8, (incs + 1) * sizeof(uint32_t), s));
    const int grid = sm_count * 8;
    k_count<<<grid, 256, 0, s>>>(m, inc_cnt, cap_cnt, flags);
    exclusive_scan(inc_cnt, csr.inc_pos, n, tiles, s);
    exclusive_scan(cap_cnt, cap_pos, n, tiles, s);
    k_fill<<<grid, 256, 0, s>>>(m, csr.inc_pos, cursor, csr.inc);
    int cap_total = 0, err = 0;
    CP_CUDA(cudaMemcpyAsync(&cap_total, cap_pos + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    CP_CUDA(cudaMemcpyAsync(&err, flags, sizeof(int), cudaMemcpyDeviceToHost, s));
    CP_CUDA(cudaStreamSynchronize(s));
    if (err) {
        cudaFreeAsync(scratch, s);
        throw Error{CP_ERR_MESH, err == 1 ? "element references a node outside [0, node_count)"
                                          : "degenerate element (a node repeated)"};
    }
    int* links = nullptr;
    CP_CUDA(cudaMallocAsync(&links, ((size_t)cap_total + 1) * sizeof(int), s));
    int* adj_cnt = cursor;  // reuse
    k_adjacency<<<(n + 127) / 128, 128, 0, s>>>(m, csr.inc_pos, csr.inc, cap_pos, links, adj_cnt, csr.inc_k,
                                                csr.inc_k8, flags + 1, flags);
    exclusive_scan(adj_cnt, csr.adj_pos, n, tiles, s);
    int nadj = 0, maxdeg = 0;
    CP_CUDA(cudaMemcpyAsync(&nadj, csr.adj_pos + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    CP_CUDA(cudaMemcpyAsync(&maxdeg, flags + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    CP_CUDA(cudaMemcpyAsync(&err, flags, sizeof(int), cudaMemcpyDeviceToHost, s));
    CP_CUDA(cudaStreamSynchronize(s));
    if (err) {
        cudaFreeAsync(links, s);
        cudaFreeAsync(scratch, s);
        throw Error{CP_ERR_MESH, err == 3 ? "a node has more than 64 incident elements"
                                          : "a node has more than 254 neighbours"};
    }
    csr.nadj = nadj;
    csr.nnz = 4LL * ((long long)nadj + n);
    csr.max_deg = maxdeg;
    CP_CUDA(cudaMallocAsync(&csr.adj, ((size_t)nadj + 1) * sizeof(int), s));
    k_adj_write<<<grid, 256, 0, s>>>(n, cap_pos, links, csr.adj_pos, csr.adj);
    CP_CUDA(cudaFreeAsync(links, s));
    // sliced layout for the SpMV
    csr.n_slices = (n + 31) / 32;
    int* width32 = cap_cnt;  // reuse (n + 1 >= n_slices + 1 entries)
    k_slice_width<<<(csr.n_slices + 255) / 256, 256, 0, s>>>(n, csr.n_slices, csr.adj_pos, width32);
    CP_CUDA(cudaMallocAsync(&csr.slice_ptr, (csr.n_slices + 1) * sizeof(int), s));
    exclusive_scan(width32, csr.slice_ptr, csr.n_slices, tiles, s);
    int blocks = 0;
    CP_CUDA(cudaMemcpyAsync(&blocks, csr.slice_ptr + csr.n_slices, sizeof(int), cudaMemcpyDeviceToHost, s));
    CP_CUDA(cudaStreamSynchronize(s));
    csr.sell_blocks = blocks;
    csr.max_width = maxdeg + 1;
    CP_CUDA(cudaMallocAsync(&csr.scol, ((size_t)blocks + 1) * sizeof(int), s));
    k_sell_cols<<<grid, 256, 0, s>>>(n, csr.n_slices, csr.adj_pos, csr.adj, csr.slice_ptr, csr.scol);
    CP_CUDA(cudaFreeAsync(scratch, s));
}

void csr_export_values(const DevMesh& m, const DevCsr& csr, double* data, cudaStream_t s) {
    k_export_values<<<(m.n_nodes + 255) / 256, 256, 0, s>>>(m.n_nodes, csr.adj_pos, csr.slice_ptr, csr.val64, data);
}

void csr_rows_cols(const DevMesh& m, const DevCsr& csr, int* rows, int* cols, cudaStream_t s) {
    k_rows_cols<<<(m.n_nodes + 255) / 256, 256, 0, s>>>(m.n_nodes, csr.adj_pos, csr.adj, rows, cols);
}

void csr_slot_map(const DevMesh& m, const DevCsr& csr, int* slots, cudaStream_t s) {
    k_slot_map<<<(m.n_nodes + 255) / 256, 256, 0, s>>>(m, csr.inc_pos, csr.inc, csr.inc_k, csr.inc_k8, csr.adj_pos,
                                                        slots);
}

}  // namespace cp
