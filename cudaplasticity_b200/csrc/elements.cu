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
#include "elements.cuh"
#include "internal.h"

namespace cp {

namespace {


constexpr int kAsmThreads = 128;  // = 4 slices of 32 nodes

// One thread per node, one block per tile of 4 slices. The tile's blocks are
// one contiguous range of values in the sliced layout, accumulated in shared
// memory (each thread only touches its own node's blocks: no atomics, and the
// summation order is the element order) and written out coalesced, once.
template <bool W64, bool W32, bool Q8>
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
                const int e = code >> 3, i = code & 7;
                const Dmat d = form_d(M.plane, E_c[e], nu_c[e]);
                element_rows<Q8>(m, e, i, csr.inc_k[q], Q8 ? csr.inc_k8[q] : 0u, d, M.h, nb);
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


}  // namespace
constexpr int kElemThreads = 256;

// strain4 + plastStress + exitNorm2 (src/PlasticitySolver.cu:1517-1549,
// 1590-1610, 1664-1691) fused: element-mean strain, stress from the C of the
// last assembly, stress intensity, secant update, and the two exit-norm sums
// (reduced deterministically by the last block). With Aitken on, the raw
// secant target psi is stored as a residual and the relax kernel moves psi.
template <bool Q8>
__global__ void __launch_bounds__(kElemThreads) k_update(DevMesh m, MaterialDev M, const double2* __restrict__ u,
                                                         ElemState st, OuterScalars* sc, double* partials, int aitken) {
    __shared__ double sh[2 * kElemThreads / 32];
    __shared__ bool last;
    const int ne = m.c3 + m.c4 + m.c8;
    double s_num = 0.0, s_den = 0.0, s_an = 0.0, s_ad = 0.0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x)
        update_element<Q8>(m, M, u, st, e, aitken, s_num, s_den, s_an, s_ad);
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
    const int ne = m.c3 + m.c4 + m.c8;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x)
        relax_element(M, st, e, w);
}

// plastDeform (src/PlasticitySolver.cu:1641-1653); the reference's guard is
// e > count (one past the end), here e < count.
__global__ void k_plastic(int ne, MaterialDev M, ElemState st) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x)
        plastic_element(M, st, e);
}

}  // namespace

template <bool Q8>
void assemble_as(const DevMesh& m, const DevCsr& csr, const MaterialDev& mat, const double* E_c, const double* nu_c,
                 bool want64, bool want32, int grid, size_t smem, cudaStream_t s) {
    if (want64 && want32) {
        CP_CUDA(cudaFuncSetAttribute(k_assemble<true, true, Q8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_assemble<true, true, Q8><<<grid, kAsmThreads, smem, s>>>(m, csr, mat, E_c, nu_c);
    } else if (want64) {
        CP_CUDA(cudaFuncSetAttribute(k_assemble<true, false, Q8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_assemble<true, false, Q8><<<grid, kAsmThreads, smem, s>>>(m, csr, mat, E_c, nu_c);
    } else {
        CP_CUDA(cudaFuncSetAttribute(k_assemble<false, true, Q8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_assemble<false, true, Q8><<<grid, kAsmThreads, smem, s>>>(m, csr, mat, E_c, nu_c);
    }
}

void launch_assemble(const DevMesh& m, const DevCsr& csr, const MaterialDev& mat, const double* E_c,
                     const double* nu_c, bool want64, bool want32, cudaStream_t s, int sm_count) {
    const int ntiles = (m.n_nodes + kAsmThreads - 1) / kAsmThreads;
    const size_t smem = (size_t)kAsmThreads * 4 * csr.max_width * sizeof(double);
    CP_CHECK(smem <= 200 * 1024, CP_ERR_UNSUPPORTED, "node degree too large for the assembly tile");
    int grid = ntiles < sm_count * 8 ? ntiles : sm_count * 8;
    if (grid < 1) grid = 1;
    if (m.c8)
        assemble_as<true>(m, csr, mat, E_c, nu_c, want64, want32, grid, smem, s);
    else
        assemble_as<false>(m, csr, mat, E_c, nu_c, want64, want32, grid, smem, s);
    CP_CUDA(cudaGetLastError());
}

int update_grid(int ne, int sm_count) {
    int g = (ne + kElemThreads - 1) / kElemThreads;
    int cap = sm_count * 4;
    return g < 1 ? 1 : (g < cap ? g : cap);
}

void launch_update(const DevMesh& m, const MaterialDev& mat, const double2* u, ElemState& st, OuterScalars* sc,
                   double* partials, int aitken, cudaStream_t s, int sm_count) {
    const int ne = m.c3 + m.c4 + m.c8;
    if (m.c8)
        k_update<true><<<update_grid(ne, sm_count), kElemThreads, 0, s>>>(m, mat, u, st, sc, partials, aitken);
    else
        k_update<false><<<update_grid(ne, sm_count), kElemThreads, 0, s>>>(m, mat, u, st, sc, partials, aitken);
    CP_CUDA(cudaGetLastError());
}

void launch_aitken_relax(const DevMesh& m, const MaterialDev& mat, ElemState& st, const OuterScalars* sc, double w,
                         cudaStream_t s, int sm_count) {
    const int ne = m.c3 + m.c4 + m.c8;
    k_aitken<<<update_grid(ne, sm_count), kElemThreads, 0, s>>>(m, mat, st, sc, w);
    CP_CUDA(cudaGetLastError());
}

void launch_plastic(const DevMesh& m, const MaterialDev& mat, ElemState& st, cudaStream_t s, int sm_count) {
    const int ne = m.c3 + m.c4 + m.c8;
    k_plastic<<<update_grid(ne, sm_count), kElemThreads, 0, s>>>(ne, mat, st);
    CP_CUDA(cudaGetLastError());
}

}  // namespace cp

// ------------------------------------------------ allocation-free update --
//
// Some callers cannot allocate device memory: code inside a framework that
// owns the whole device memory pool through its own caching allocator (a
// cudaMalloc beside it fails or fragments that pool), and embedded or
// real-time loops whose memory budget is fixed up front. For
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
    cp::k_update<false><<<grid, cp::kElemThreads, 0, s>>>(m, M, reinterpret_cast<const double2*>(d_uv), es, sc, partials, 0);
    if (cudaGetLastError() != cudaSuccess) return CP_ERR_CUDA;
    double host_err = 0.0;
    if (cudaMemcpyAsync(&host_err, &sc->rel_err, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return CP_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return CP_ERR_CUDA;
    *rel_err = host_err;
    return CP_OK;
}
