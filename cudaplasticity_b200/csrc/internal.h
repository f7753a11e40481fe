// Internal declarations shared by the cuplast translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/cuplast.h"

namespace cp {

// ----------------------------------------------------------------- errors --
struct Error {
    int status;
    std::string msg;
};

#define CP_CUDA(call)                                                                           \
    do {                                                                                        \
        cudaError_t _e = (call);                                                                \
        if (_e != cudaSuccess)                                                                  \
            throw ::cp::Error{CP_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)}; \
    } while (0)

#define CP_CHECK(cond, code, text)                       \
    do {                                                 \
        if (!(cond)) throw ::cp::Error{(code), (text)}; \
    } while (0)

// Adaptive rule 2 (cp_solve_opts.adaptive_cg = 2): the linear tolerance is
// max(cg_tol, kRule2Factor x relErr) until relErr meets the outer tolerance.
// 0.2 measured best on configuration 1 (40.8k CG iterations per solve against
// 46.5k at 0.1; 0.3 and 0.5 add more outer iterations than they save).
constexpr double kRule2Factor = 0.2;

// ------------------------------------------------------------- device data --
// Elements are numbered triangles first, then 4-node quads, then 8-node quads
// (the reference's element order, elemPos, src/Mesh.cuh:60).
struct DevMesh {
    int n_nodes = 0, c3 = 0, c4 = 0, c8 = 0;
    double2* xy = nullptr;
    int4* e3 = nullptr;  // (n1, n2, n3, -1)
    int4* e4 = nullptr;
    int4* e8 = nullptr;  // two per element: the corners, then the mid-sides
};

// Node-blocked CSR in the reference's layout: node n owns rows 2n and 2n+1,
// which start at 4 * (adj_pos[n] + n) and hold 2 * (s + 1) values each, the
// 2x2 blocks of the columns (n, adj[adj_pos[n]], ..., adj[adj_pos[n+1]-1]).
struct DevCsr {
    long long nadj = 0, nnz = 0;
    int max_deg = 0;
    int* adj_pos = nullptr;   // n+1
    int* adj = nullptr;       // nadj
    int* inc_pos = nullptr;   // n+1, incidences of node n (element order)
    int* inc = nullptr;       // (global element id << 3) | local node index
    uint32_t* inc_k = nullptr;  // packed block index (byte j) of local node j in node n's row
    uint32_t* inc_k8 = nullptr;  // 8-node meshes: the same for local nodes 4..7 (byte j - 4)
    // Values live in a sliced layout for the SpMV (the reference-ordered CSR
    // above is exported on demand): nodes in slices of 32, slice s padded to
    // width w_s = max(deg + 1) over its nodes; block k (2x2: K00 K01 K10 K11)
    // of node 32 s + l sits at 4 * (slice_ptr[s] + 32 k + l). Block 0 is the
    // diagonal block, block k >= 1 the k-th neighbour in reference order,
    // padding blocks are zero with column = the node itself.
    int n_slices = 0;
    int max_width = 0;
    long long sell_blocks = 0;
    int* slice_ptr = nullptr;  // n_slices + 1, in blocks
    int* scol = nullptr;       // column node of every block
    double* val64 = nullptr;   // 4 * sell_blocks
    float* val32 = nullptr;    // 4 * sell_blocks
};

struct ElemState {
    double *exx, *eyy, *gam, *eps_i, *sxx, *syy, *tau, *sig_i, *table_s, *psi, *E_c, *nu_c;
    double *exx_p, *eyy_p, *gam_p, *eps_p_i;
    double *res_prev, *res_cur;  // Aitken history: secant residual of psi
};

// Device-resident scalars of one linear solve.
struct CgScalars {
    double rr;          // (r, r) of the recurrence residual
    double rho;         // (r, M^-1 r); equals rr without preconditioner
    double alpha, beta;
    double pAz;         // (K z, z)
    double normB_inv;   // stop when rr * normB_inv <= eps2
    double eps2;
    double res64;       // (r, r) of the FP64 residual computed at init
    double bb;          // (b, b)
    long long iter, max_iter;
    int converged;
    int status;         // 0 running/ok, CP_ERR_BREAKDOWN, CP_ERR_NOT_CONVERGED
    int lin_done;       // init found the FP64 residual already below the caller's tolerance
    unsigned int ticket;
    unsigned int gen;   // persistent CG: grid-barrier steps released so far
};

struct OuterScalars {
    double num, den;      // sum (sig_i - table_s)^2, sum table_s^2
    double rel_err;
    double aitken_omega;  // relaxation factor of the last step
    double a_num, a_den;  // Aitken sums
    int iter;
    unsigned int ticket;
};

// Launch helpers (defined in the .cu files).
void setup_csr(DevMesh& m, DevCsr& csr, cudaStream_t s, int sm_count);
void csr_rows_cols(const DevMesh& m, const DevCsr& csr, int* rows, int* cols, cudaStream_t s);
void csr_slot_map(const DevMesh& m, const DevCsr& csr, int* slots, cudaStream_t s);
void csr_export_values(const DevMesh& m, const DevCsr& csr, double* data, cudaStream_t s);

struct MaterialDev {
    double E, nu, h;
    int plane;
    int diagram;
    double sigma_t, k_t, a, m, eps0, n;
    int n_points;
    double pw_eps[CP_MAX_PW], pw_sig[CP_MAX_PW];
};

void launch_assemble(const DevMesh& m, const DevCsr& csr, const MaterialDev& mat, const double* E_c,
                     const double* nu_c, bool want64, bool want32, cudaStream_t s, int sm_count);
void launch_update(const DevMesh& m, const MaterialDev& mat, const double2* u, ElemState& st, OuterScalars* sc,
                   double* partials, int aitken, cudaStream_t s, int sm_count);
void launch_aitken_relax(const DevMesh& m, const MaterialDev& mat, ElemState& st, const OuterScalars* sc, double w,
                         cudaStream_t s, int sm_count);
void launch_plastic(const DevMesh& m, const MaterialDev& mat, ElemState& st, cudaStream_t s, int sm_count);

}  // namespace cp
