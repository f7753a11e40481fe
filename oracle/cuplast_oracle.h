/*
 * cuplast_oracle.h -- CPU restatement of CudaPlasticity's 2D elasto-plastic
 * hot path, used ONLY as the checker of the CUDA product (tests/, smoke(),
 * bench.py's CPU-baseline leg). It is never linked into the product library.
 *
 * Every step cites the reference function it restates (paths relative to the
 * reference project). It is pinned against the reference itself (the harness
 * in ref_harness.cu and the reference's shipped golden data) by the CPU tests.
 */
#ifndef CUPLAST_ORACLE_H
#define CUPLAST_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Runs a job file with the same syntax as the reference harness (see the
 * comment block at the top of ref_harness.cu; meshes come as "mesh file"),
 * writing CPBIN01 records with the same names. Returns 0 on success. */
int orc_run_job(const char* job_path, const char* out_path);

/* Reference CSR structure of SparseSLAE(Mesh&, 2) (src/SparseSLAE.h:60-196).
 * Call once with rows == NULL to get *nnz and *nadj, then with buffers of
 * size 2n+1 (rows), nnz (cols), n+1 (adj_pos), nadj (adj). */
int orc_csr_build(int n_nodes, int c3, const int* e3, int c4, const int* e4, int c8, const int* e8,
                  int* rows, int* cols, int* adj_pos, int* adj, long long* nnz, long long* nadj);

/* Element-to-CSR slot map: for element e (T3 first, then Q4, then Q8, the
 * reference's element order) and local nodes (i, j), the index in data[] of
 * K(2*node_i, 2*node_j). Laid out as slots[off_e + i*nen + j] with
 * off_e = 9*e for T3, 9*c3 + 16*(e - c3) for Q4 and
 * 9*c3 + 16*c4 + 64*(e - c3 - c4) for Q8. */
int orc_slot_map(int n_nodes, int c3, const int* e3, int c4, const int* e4, int c8, const int* e8,
                 const int* rows, const int* adj_pos, const int* adj, int* slots);

#ifdef __cplusplus
}
#endif
#endif
