/*
 * cuplast.h -- C ABI of the B200 (sm_100a) implementation of CudaPlasticity's
 * 2D elasto-plastic FEM hot path: element B / B^T D B stiffness, CSR sparsity
 * and slot-map assembly, masked conjugate gradients, and the secant
 * ("variable elastic parameters") plastic update inside the outer iterations.
 *
 * The reference exposes this path only through C++ classes (no C ABI). Each
 * entry point below names the reference code it replaces; the C++ drop-in
 * classes with the reference's names (the headers in include/cuplast/) are
 * written on top of these functions.
 *
 * Conventions: every function returns a cp_status (0 = CP_OK); on error the
 * context keeps a message (cp_context_last_error). All array arguments are
 * plain HOST pointers with the sizes stated; nothing here exposes CUDA or
 * PyTorch types. DOF order is the reference's: (u_0, v_0, u_1, v_1, ...).
 * Element numbering is the reference's: triangles first, then quads
 * (Mesh::elemPos, src/Mesh.cuh:26-30).
 */
#ifndef CUPLAST_H
#define CUPLAST_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define CP_API __attribute__((visibility("default")))
#else
#define CP_API
#endif

typedef enum {
    CP_OK = 0,
    CP_ERR_INVALID = 1,        /* bad argument */
    CP_ERR_CUDA = 2,           /* a CUDA call failed */
    CP_ERR_NOMEM = 3,          /* device memory exhausted / above the admission limit */
    CP_ERR_NOT_CONVERGED = 4,  /* iteration cap reached */
    CP_ERR_BREAKDOWN = 5,      /* NaN/Inf or a non-positive curvature in CG */
    CP_ERR_MESH = 6,           /* malformed mesh (bad node index, degenerate element) */
    CP_ERR_UNSUPPORTED = 7,
    CP_ERR_BUSY = 8,
    CP_ERR_NO_DEVICE = 9,      /* no CUDA device visible */
    CP_ERR_CANCELLED = 10,
    CP_ERR_TIMEOUT = 11        /* a bounded device-side wait gave up (grid barrier of the persistent CG) */
} cp_status;

typedef struct cp_context cp_context;
typedef struct cp_instance cp_instance;

enum { CP_PLANE_STRESS = 0, CP_PLANE_STRAIN = 1 };           /* plainCondition, src/PlasticitySolver.cuh:15 */
enum {
    CP_DIAGRAM_ELASTIC = 0,   /* sigma = E eps */
    CP_DIAGRAM_LINEAR = 1,    /* Material::setLinearPlast, src/Material.cu:14-17,29-35 */
    CP_DIAGRAM_POWER = 2,     /* Material::setPowerPlast, src/Material.cu:19-23,37-43 */
    CP_DIAGRAM_HOLLOMON = 3,  /* sigma = sigma_y (1 + eps_p / eps0)^n (new) */
    CP_DIAGRAM_PIECEWISE = 4  /* elastic to (pw_eps[0], pw_sig[0]), then piecewise linear (new) */
};
/* CP_PREC_FLOAT_BOOST: the reference's floatBoost (solveCUDA_FD,
 * src/PlasticitySolver.cu:631-708): each load level first iterates in mixed
 * precision with loose tolerances (CG and relErr 1e-4), then goes on in FP64
 * from that state to the caller's tolerances (at least one FP64 step). */
enum { CP_PREC_FP64 = 0, CP_PREC_MIXED = 1, CP_PREC_FLOAT_BOOST = 2 };
#define CP_MAX_PW 16

/* Material and hardening diagram (class Material, src/Material.cuh:9-40). */
typedef struct {
    double E, nu, h, rho;
    int plane;
    int diagram;
    double sigma_t;   /* yield stress: sigmaT (linear/power) or sigma_y (Hollomon) */
    double k_t;       /* linear: hardening modulus K_T */
    double a, m;      /* power: A, m */
    double eps0, n;   /* Hollomon */
    int n_points;     /* piecewise: breakpoints, pw_eps ascending, pw_sig[k] = f(pw_eps[k]) */
    double pw_eps[CP_MAX_PW], pw_sig[CP_MAX_PW];
} cp_material;

/* A mesh as the public arrays of class Mesh (src/Mesh.cuh:42-66). Elements
 * are numbered triangles, then 4-node quads, then 8-node quads; per-element
 * fields follow that order. */
typedef struct {
    int node_count;
    const double* node_xy;  /* 2 * node_count */
    int count3;
    const int* elem3;       /* 3 * count3 */
    int count4;
    const int* elem4;       /* 4 * count4 */
    int count8;
    const int* elem8;       /* 8 * count8: corners, then the mid-sides of edges 1-2, 2-3, 3-4, 4-1
                               (Mesh::remapOrder, src/Mesh.cu:443-503) */
} cp_mesh_view;

typedef struct {
    int precision;       /* CP_PREC_FP64: FP64 throughout; CP_PREC_MIXED: FP32 matrix + inner CG, FP64 defect correction;
                            CP_PREC_FLOAT_BOOST: mixed to 1e-4, then FP64 (the reference's floatBoost) */
    double cg_tol;       /* linear solve: stop when ||r|| / ||b|| <= cg_tol (reference: 1e-7) */
    double outer_tol;    /* secant iteration: stop when relErr <= outer_tol (reference: 1e-5) */
    int max_outer;       /* per load level (reference CPU path: 50) */
    long long max_cg;    /* per linear solve */
    int levels;          /* load levels lambda_k = k / levels, k = 1..levels, each warm-started */
    int aitken;          /* 1: Aitken-relaxed secant iteration (same fixed point) */
    double inner_tol;    /* mixed precision: relative tolerance of each FP32 inner solve */
    int adaptive_cg;     /* linear tolerance follows the outer error (inexact early steps; the converged result
                            meets the same criterion): 1: max(cg_tol, 1e-2 relErr) while relErr > 10 outer_tol;
                            2: max(cg_tol, 0.2 relErr) while relErr > outer_tol (fewer CG iterations, a few
                            more outer ones) */
    int precond;         /* 0: unpreconditioned CG as the reference; 1: 2x2 block-Jacobi PCG (same solution);
                            2: PCG with one aggregation-multigrid V-cycle (CP_PREC_FP64 only, else
                            CP_ERR_UNSUPPORTED; the hierarchy is built on first use and kept while the
                            Dirichlet mask stays the same) */
    int predict;         /* 1: from the third load level on, start from the linear extrapolation of the last two
                            levels' displacements and secant moduli (a predictor; each level still converges to
                            the same criterion) */
    int recycle;         /* 0..6, CP_PREC_FP64 with precond 0 or 1: each linear solve of a load level starts
                            from the last solution corrected by the Galerkin projection of the error onto the
                            level's last `recycle` solution increments (fewer CG iterations; each solve stops on
                            the same criterion, so the fixed point is unchanged). 0: off (the reference).
                            cp_solve only; a batch ignores it */
} cp_solve_opts;

typedef struct {
    int status;
    int outer_iters;      /* summed over levels */
    long long cg_iters;   /* summed over all linear solves (FP32 inner iterations in mixed mode) */
    long long fp64_spmv;  /* FP64 residual evaluations (mixed mode) */
    double rel_err;       /* final relErr of the secant iteration */
    double cg_rel_res;    /* final ||r|| / ||b|| of the last linear solve (FP64) */
    double seconds;       /* device time of the solve (CUDA events) */
    int levels_done;
    long long kernel_launches;  /* kernels launched by the solve (graph nodes included) */
} cp_solve_report;

/* ------------------------------------------------------------ library --- */
CP_API const char* cp_version(void);
CP_API const char* cp_status_string(int status);
CP_API int cp_device_count(int* count);

/* ------------------------------------------------------------ context --- */
/* One context per device and stream; all instances of a context run on its
 * stream. Replaces the reference's implicit device 0 (src/Mesh.cuh:86-104). */
CP_API int cp_context_create(int device, cp_context** out);
CP_API int cp_context_destroy(cp_context* ctx);
CP_API const char* cp_context_last_error(const cp_context* ctx);
/* The message of the last error on the context an instance belongs to (for
 * instances a solve service hands back, whose contexts are the service's;
 * no counterpart in the reference). */
CP_API const char* cp_instance_last_error(const cp_instance* inst);
CP_API int cp_context_synchronize(cp_context* ctx);

/* ----------------------------------------------------------- instance --- */
/* Uploads the mesh, builds on the device the reference CSR structure of
 * SparseSLAE(Mesh&, 2) (src/SparseSLAE.h:60-196) and the element-to-CSR slot
 * map, and allocates the per-element secant state. Replaces the set-up part
 * of PlasticitySolver::PlasticitySolver + solveCUDA
 * (src/PlasticitySolver.cuh:236-338, src/PlasticitySolver.cu:469-485). */
CP_API int cp_instance_create(cp_context* ctx, const cp_mesh_view* mesh, const cp_material* mat, cp_instance** out);
CP_API int cp_instance_destroy(cp_instance* inst);
/* Device bytes an instance of this mesh holds (for admission control). */
CP_API int cp_instance_footprint(const cp_mesh_view* mesh, int precision, size_t* bytes);
CP_API int cp_instance_sizes(const cp_instance* inst, int* node_count, int* elem_count, long long* nnz,
                             long long* nadj);
/* Right-hand side, Dirichlet mask (1 = free DOF, 0 = prescribed) and the
 * prescribed/initial displacements, all of length 2 * node_count, as built by
 * initConditions (src/PlasticitySolver.cu:812-1005). Resets uv. */
CP_API int cp_instance_set_loads(cp_instance* inst, const double* rp, const unsigned char* mask, const double* uv);
/* psi = 1, E_c = E, nu_c = nu (initPlastParams, src/PlasticitySolver.cu:385-415). */
CP_API int cp_instance_reset_state(cp_instance* inst);
/* Scales the loads to level lam: rp = lam * rp_full, uv[prescribed] = lam * uv_full. */
CP_API int cp_instance_set_level(cp_instance* inst, double lam);

/* ------------------------------------------------------------- phases --- */
/* K(E_c, nu_c) into the CSR values: fillGlobalStiffness + insertKe4
 * (src/PlasticitySolver.cu:1413-1499), no band matrix and no atomics. */
CP_API int cp_assemble(cp_instance* inst, int precision);
/* Masked CG from the current uv: ConjGradCuda::solve (src/ConjGradCuda.cu:185-231). */
CP_API int cp_cg_solve(cp_instance* inst, double eps, long long max_iter, long long* iters, double* rel_res);
/* Strain, stress, secant update and exit norm: strain4 + plastStress +
 * exitCondition (src/PlasticitySolver.cu:1517-1549,1590-1610,1722-1735). */
CP_API int cp_secant_update(cp_instance* inst, double* rel_err);
/* Plastic strains: plastDeform (src/PlasticitySolver.cu:1641-1662). */
CP_API int cp_plastic_strains(cp_instance* inst);
/* The whole outer loop: solveCUDA (src/PlasticitySolver.cu:469-512). */
CP_API void cp_solve_opts_default(cp_solve_opts* opts);
CP_API int cp_solve(cp_instance* inst, const cp_solve_opts* opts, cp_solve_report* report);

/* Kernel timing of the linear solver (no reference counterpart; the
 * reference times whole solves only, src/Main.cpp:458-902): assembles K at
 * the current state, starts a CG from the current uv and runs `iters`
 * iterations as direct launches, with CUDA events around every SpMV (P) and
 * update (U) kernel. Outputs the mean duration of each in milliseconds and
 * the algorithmic bytes each must move per launch: P reads the values, one
 * 4-byte column per 2x2 block, r and z, and writes z' and K z'; U reads x,
 * z', r, K z' and the mask and writes x and r (plus M^-1 and s with block
 * Jacobi). Leaves uv changed. */
CP_API int cp_bench_cg(cp_instance* inst, int precision, int precond, int iters, double* ms_spmv, double* ms_update,
                       double* bytes_spmv, double* bytes_update);
/* Measurement entry point of the FP64 CG form that instances too large for
 * one thread-block cluster run (one launch per iteration; no counterpart in
 * the reference, whose ConjGradCuda::solve, src/ConjGradCuda.cu:185-231,
 * launches three kernels and synchronises per iteration): assembles K at the
 * current state, starts a (block-Jacobi with precond 1) CG from the current
 * uv and runs `iters` iterations as direct launches with CUDA events around
 * each. Outputs the mean duration of one iteration in milliseconds and the
 * algorithmic bytes one iteration moves: the values and one 4-byte column per
 * 2x2 block, and per node the vectors read and written once. Leaves uv
 * changed. */
CP_API int cp_bench_cg_fused(cp_instance* inst, int precond, int iters, double* ms_iter, double* bytes_iter);
/* Measurement entry point: runs the assembly (fillGlobalStiffness) `iters`
 * times as direct launches with CUDA events around each, from the current
 * secant moduli. Outputs the mean duration in milliseconds and the
 * algorithmic bytes one assembly moves: the values written (FP64, plus FP32
 * for CP_PREC_MIXED), the connectivity, E_c and nu_c of every element, the
 * incidence codes and slot bytes, and the node coordinates once. */
CP_API int cp_bench_assemble(cp_instance* inst, int precision, int iters, double* ms, double* bytes);
/* Measurement entry point of the multigrid PCG (precond 2): assembles K from
 * the current secant moduli, runs the per-outer-iteration set-up once and
 * `iters` PCG iterations as direct launches, with CUDA events around each
 * part. ms[0..4]: mean duration of P, U, R0, the coarse levels (all of their
 * kernels) and S0 per iteration; ms[5]: the set-up. bytes[0..5] (may be
 * NULL): the algorithmic bytes each part moves (FP64 values, vectors counted
 * once). Leaves uv changed. */
CP_API int cp_bench_mg(cp_instance* inst, int iters, double* ms, double* bytes);

/* Allocation-free secant update (no counterpart in the reference). For
 * callers that cannot allocate device memory -- code inside a framework whose
 * caching allocator owns the device memory (a cudaMalloc of its own would
 * fail or fragment that pool), embedded and real-time loops whose memory
 * budget is fixed up front -- this runs the same fused
 * strain / stress / secant-update / exit-norm kernel as cp_secant_update on
 * buffers the caller owns, and allocates nothing (no cudaMalloc, no cudaFree,
 * no allocating library call). Every pointer except mat and rel_err is a
 * DEVICE pointer on the current device; node_xy, elem4 and uv must be 16-byte
 * aligned. Quad meshes only: count4 <= 1,048,576 elements, larger meshes
 * return CP_ERR_INVALID. Every elem4 entry must lie in [0, node_count): the
 * kernel gathers node_xy and uv at those indices unchecked. The call ends
 * with a stream synchronisation and a copy of the exit norm to the host.
 * In: node_xy (2 * node_count), elem4 (4 * count4), uv
 * (2 * node_count), E_c / nu_c (count4, the moduli K was assembled with).
 * Out: E_c, nu_c, psi updated; fields = 9 * count4 doubles, one block of
 * count4 each: exx, eyy, gamma, eps_i, sxx, syy, tau, sig_i, table_s; *rel_err
 * = the exit norm; the call returns when the result is on the host.
 * Its scratch (the exit norm's per-block partial sums and scalars) is a
 * file-scope device array of 131,328 bytes that every GPU loading the library holds
 * until exit. The first call on each device looks up that array's address
 * (with the device current); make that first call before any stream capture.
 * All calls share the array: calls that overlap on the GPU, on any stream,
 * race and must be serialised by the caller. stream may be NULL. */
CP_API int cp_secant_update_noalloc(void* stream, const cp_material* mat, int node_count, const double* node_xy,
                                    int count4, const int* elem4, const double* uv, double* E_c, double* nu_c,
                                    double* psi, double* fields, double* rel_err);

/* ------------------------------------------------------------- batch --- */
/* Many independent instances solved together on one GPU (no counterpart in
 * the reference, which solves one mesh per process, src/Main.cpp:1193-1227).
 * Each instance runs cp_solve's outer algorithm (load levels, assembly,
 * linear solve, secant update, optional Aitken relaxation) in mixed
 * precision: FP32 values and FP32 CG recurrences, with the solution u
 * accumulated in FP64, every dot product reduced in FP64, and the recursive
 * residual replaced by the FP64 residual b - K64 u whenever it has dropped by
 * inner_tol since the last replacement or meets cg_tol (the linear solve ends
 * on the FP64 residual); CG runs in the Chronopoulos-Gear form, one reduction
 * and one kernel launch per iteration; the secant update is FP64. Every instance is its own
 * device-side state machine. One captured CUDA graph drives all of them: a
 * device WHILE loop over a body of phase-filtered kernels that walk a work
 * list of (instance, tile) entries, so instances of different sizes advance
 * concurrently with no host round trip; an instance that finishes its linear
 * solve continues while others are still iterating. Every cross-tile sum is
 * reduced per instance in a fixed order, so an instance's result does not
 * depend on what else is in the batch. Instances are added between runs and
 * harvested when done. */
typedef struct cp_batch cp_batch;

typedef struct {
    int max_instances;   /* slots */
    int cg_per_trip;     /* CG kernel launches per graph trip (each advances every CG instance by half an iteration) */
    int elem_per_trip;   /* element-phase launches per trip (>= 3: update, Aitken, next level) */
    int max_width;       /* assembly limit on blocks per node row (node degree + 1) */
    int cg_blocks_per_sm;  /* persistent grid of the CG kernel: 0 = occupancy limit */
} cp_batch_opts;

enum { CP_BATCH_RUN_ALL = 0, CP_BATCH_RUN_ANY_DONE = 1 };

CP_API void cp_batch_opts_default(cp_batch_opts* opts);
CP_API int cp_batch_create(cp_context* ctx, const cp_batch_opts* opts, cp_batch** out);
CP_API int cp_batch_destroy(cp_batch* b);
/* Adds an instance (loads set; it may belong to another context on the same
 * device) with its solve options; opts->precision must be CP_PREC_MIXED.
 * From here until it is harvested the batch owns the instance: every other
 * call on it returns CP_ERR_BUSY. Not allowed while a run is in flight. */
CP_API int cp_batch_add(cp_batch* b, cp_instance* inst, const cp_solve_opts* opts, int* slot);
/* Starts a run on the batch's stream and returns: the graph loops until every
 * listed instance is done (CP_BATCH_RUN_ALL), or until at least one finishes
 * (CP_BATCH_RUN_ANY_DONE), or after max_trips trips (<= 0: no limit), or when
 * cp_batch_interrupt is called. */
CP_API int cp_batch_launch(cp_batch* b, int until, long long max_trips);
/* Waits for the run; *active = instances still running, *done = instances
 * ready to harvest. */
CP_API int cp_batch_wait(cp_batch* b, int* active, int* done);
/* Asks a run in flight to stop at the end of its current trip (thread-safe,
 * through host-mapped memory; used by schedulers that have new work). */
CP_API int cp_batch_interrupt(cp_batch* b);
CP_API int cp_batch_run(cp_batch* b, int until, long long max_trips, int* active, int* done);
/* Removes up to cap finished instances: their slots, handles and reports
 * (report->seconds = device time from the instance's first to its last phase). */
CP_API int cp_batch_harvest(cp_batch* b, int cap, int* slots, cp_instance** insts, cp_solve_report* reports,
                            int* count);
/* Slices (32 nodes) per work-list tile for instances whose slice count lies
 * in [2^bucket, 2^(bucket+1)); buckets 0..23. */
CP_API int cp_batch_set_tile(cp_batch* b, int bucket, int slices);
CP_API int cp_batch_get_tile(const cp_batch* b, int bucket, int* slices);
/* Autotuner: times the CG kernel's SpMV over the listed instances of each
 * size bucket for every candidate tile size (4..64 slices; state is left
 * unchanged) and keeps the fastest per bucket. ms_per_sweep (may be NULL):
 * the tuned time of one SpMV sweep over all listed instances. */
CP_API int cp_batch_autotune(cp_batch* b, double* ms_per_sweep);
/* Progress of the instance in a slot as of the end of the last run: phase
 * (1 level set-up, 2 assembly, 3 FP64 residual (first or replacement),
 * 4 w = K u, 5 CG iteration, 6 secant update, 7 Aitken, 8 plastic strains,
 * 9 done), load level, and the counters of its report so far. */
CP_API int cp_batch_progress(const cp_batch* b, int slot, int* phase, int* level, cp_solve_report* report);
/* Device time of the last completed run in milliseconds (CUDA events
 * recorded on the batch's stream around the run's graph). */
CP_API int cp_batch_last_run_ms(const cp_batch* b, double* ms);
/* Counters of the batch since creation: graph trips and kernel launches. */
CP_API int cp_batch_stats(const cp_batch* b, long long* trips, long long* kernel_launches, long long* runs);

/* ------------------------------------------------------------ server --- */
/* A solve service on one GPU (no counterpart in the reference): requests of
 * uneven sizes (mesh, material / hardening diagram, loads, load levels) are
 * submitted from any thread as they arrive; a scheduler thread admits them
 * in arrival order while their device footprint (cp_instance_footprint) fits
 * into the free device memory minus a reserve and a batch slot is free, sets
 * each one up on its own stream while the batch's graph keeps running, then
 * makes the running graph stop at its next trip so that the new instances
 * join, and harvests finished ones. Every request's matrix, displacements and
 * plastic state stay on the device from admission to completion; requests
 * that arrive while others are on the GPU overlap with them (continuous
 * batching). Each result is the one the same request gives alone. */
typedef struct cp_server cp_server;

typedef struct {
    int device;
    double hbm_reserve;      /* fraction of the device memory kept free (admission limit) */
    size_t max_bytes;        /* limit on the sum of admitted footprints (0: free memory only) */
    int max_inflight;        /* requests on the device at once (<= batch slots) */
    long long trip_quantum;  /* graph trips per run before the scheduler looks again (<= 0: until one finishes) */
    cp_batch_opts batch;
    int fp64_lanes;          /* CP_PREC_FP64 / CP_PREC_FLOAT_BOOST requests: each is solved by cp_solve on one of
                                this many lane threads, each with its own stream, concurrently with the other
                                lanes and the batch (0: such requests are refused) */
} cp_server_opts;

typedef struct {
    long long submitted, admitted, completed, failed, rejected;
    long long inflight, pending;
    long long runs, trips;
    double busy_seconds;     /* host time with a run in flight */
    size_t peak_bytes;       /* largest sum of admitted footprints */
} cp_server_stats;

CP_API void cp_server_opts_default(cp_server_opts* opts);
CP_API int cp_server_create(const cp_server_opts* opts, cp_server** out);
/* Stops the scheduler; requests not yet completed are cancelled
 * (CP_ERR_CANCELLED to their waiters); instances not yet taken are freed. */
CP_API int cp_server_destroy(cp_server* s);
/* Copies the request and returns at once; *id identifies it. CP_PREC_MIXED
 * requests join the batch; CP_PREC_FP64 and CP_PREC_FLOAT_BOOST ones go to the
 * FP64 lanes (CP_ERR_UNSUPPORTED when there are none). A request larger than
 * the whole admission limit is rejected here with CP_ERR_NOMEM. */
CP_API int cp_server_submit(cp_server* s, const cp_mesh_view* mesh, const cp_material* mat, const double* rp,
                            const unsigned char* mask, const double* uv, const cp_solve_opts* opts, long long* id);
/* Waits (timeout_s < 0: without limit) until request id completes; returns
 * CP_ERR_BUSY on timeout. On completion hands over the instance with the
 * results (read them with cp_get_field; free it with cp_instance_destroy
 * before cp_server_destroy: it lives on the server's streams),
 * its report (report->status: the solve's own status) and the latency from
 * submission to completion in seconds. Each id can be taken once. */
CP_API int cp_server_wait(cp_server* s, long long id, double timeout_s, cp_instance** inst, cp_solve_report* report,
                          double* latency_s);
CP_API int cp_server_get_stats(cp_server* s, cp_server_stats* stats);

/* ---------------------------------------------------------- read-back --- */
/* Reference CSR arrays (SparseSLAE::rows/cols/adjPos/adj/data); any pointer
 * may be NULL. values: the last assembly (FP64, or FP32 widened). */
CP_API int cp_get_csr(cp_instance* inst, int* rows, int* cols, int* adj_pos, int* adj, double* values);
/* slots[off_e + i*nen + j] = index in values of K(2*node_i, 2*node_j) of
 * element e; off_e = 9e for triangles, 9*count3 + 16(e - count3) for quads. */
CP_API int cp_get_slot_map(cp_instance* inst, int* slots);
/* Fields by name: "uv" (2 * node_count) or per element "exx", "eyy", "gamma",
 * "eps_i", "sxx", "syy", "tau", "sig_i", "table_s", "psi", "E_c", "nu_c",
 * "exx_p", "eyy_p", "gamma_p", "eps_p_i" (PlasticitySolver::dataToRAM). */
CP_API int cp_get_field(cp_instance* inst, const char* name, double* out);
CP_API int cp_set_field(cp_instance* inst, const char* name, const double* in);

#ifdef __cplusplus
}
#endif
#endif
