/*
 * cuplast_host.h -- C ABI over the host-side half of the drop-in API (the
 * C++ classes Mesh and LoadConditions of include/cuplast/*.hpp), so that
 * non-C++ callers (the Python package, tests, benchmarks) use the same mesh
 * generators and the same right-hand-side / Dirichlet-mask construction as
 * C++ users. No function here touches the GPU.
 */
#ifndef CUPLAST_HOST_H
#define CUPLAST_HOST_H

#include "cuplast.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cpx_mesh cpx_mesh;
typedef struct cpx_loads cpx_loads;

CP_API int cpx_mesh_create(cpx_mesh** out);
CP_API int cpx_mesh_destroy(cpx_mesh* m);
/* The generators take the reference's element order: 1 (4-node quads) or 2
 * (8-node quads: Mesh::remapOrder, src/Mesh.cu:443-505). The device solver
 * takes order-1 meshes; order-2 meshes serve the host side (load building,
 * I/O) and the C++ classes. */
/* Mesh::genRectangle (src/Mesh.cu:17-110) */
CP_API int cpx_mesh_gen_rect(cpx_mesh* m, double x1, double x2, double y1, double y2, int n1, int n2, int order);
/* Mesh::genRectWithHole (src/Mesh.cu:112-246); rad_n > 0 overrides the reference's radial count */
CP_API int cpx_mesh_gen_rect_with_hole(cpx_mesh* m, double x1, double x2, double y1, double y2, double hole_rad,
                                       int n1, int n2, int rad_n, int order);
/* Mesh::genRing (src/Mesh.cu:249-329) */
CP_API int cpx_mesh_gen_ring(cpx_mesh* m, double a, double b, int n_phi, int n_r, int order);
/* Mesh::loadFromFile (src/Mesh.cu:725-937): an .inp file with *NODE, *ELEMENT
 * (TYPE=S3, S4, S8R) and *MPC border blocks. CP_ERR_INVALID for a bad file. */
CP_API int cpx_mesh_load_inp(cpx_mesh* m, const char* path);
/* Mesh::renumByDirection (src/Mesh.cu:537-636): nodes renumbered by their
 * projection on (dx, dy) */
CP_API int cpx_mesh_renum_by_direction(cpx_mesh* m, double dx, double dy);
/* Mesh::smoothRing (src/Mesh.cu:386-416) of an O-grid with border_n columns */
CP_API int cpx_mesh_smooth_ring(cpx_mesh* m, int border_n);
/* Mesh::aspectRatio / skewAngleSin per 4-node element (count4 each, either
 * may be NULL) and Mesh::avrElemSize (src/Mesh.cuh:279-317) */
CP_API int cpx_mesh_quality(const cpx_mesh* m, double* aspect, double* skew_sin, double* avr_size);
/* every quad (n1,n2,n3,n4) -> triangles (n1,n2,n3), (n1,n3,n4) (extension) */
CP_API int cpx_mesh_split_t3(cpx_mesh* m);
/* Mesh from arrays; elem8 (8 * count8, may be NULL when count8 = 0) marks its
 * mid-side nodes as second-order nodes, as the reference's generators do. */
CP_API int cpx_mesh_set(cpx_mesh* m, int node_count, const double* xy, int count3, const int* elem3, int count4,
                        const int* elem4, int n_borders, const int* border_len, const int* border_nodes, int count8,
                        const int* elem8);
CP_API int cpx_mesh_counts(const cpx_mesh* m, int* node_count, int* count3, int* count4, int* n_borders,
                           int* border_total, int* count8);
/* elem8: 8 * count8 node indices, corners 0..3 then mid-side nodes 4..7 */
CP_API int cpx_mesh_get(const cpx_mesh* m, double* xy, int* elem3, int* elem4, int* border_len, int* border_nodes,
                        int* elem8);
CP_API int cpx_mesh_max_index_diff(const cpx_mesh* m, int* out);

CP_API int cpx_loads_create(cpx_loads** out);
CP_API int cpx_loads_destroy(cpx_loads* l);
/* LoadConditions setters (src/LoadConditions.cuh:70-179), constant-valued */
CP_API int cpx_loads_set_force(cpx_loads* l, int border, double fx, double fy, int normal);
CP_API int cpx_loads_set_displacement(cpx_loads* l, int border, double ux, double uy, int fix_mid_x, int fix_mid_y);
CP_API int cpx_loads_fix_border(cpx_loads* l, int border);
CP_API int cpx_loads_fix_border_vert(cpx_loads* l, int border);
CP_API int cpx_loads_fix_border_hor(cpx_loads* l, int border);
CP_API int cpx_loads_fix_vert_axis(cpx_loads* l, double x);
CP_API int cpx_loads_fix_hor_axis(cpx_loads* l, double y);
CP_API int cpx_loads_fix_point(cpx_loads* l, double x, double y);
CP_API int cpx_loads_set_displ_point(cpx_loads* l, double x, double y, double ux, double uy);
CP_API int cpx_loads_set_force_point(cpx_loads* l, double x, double y, double fx, double fy);
CP_API int cpx_loads_set_gravity(cpx_loads* l, double g, double dx, double dy);
CP_API int cpx_loads_set_rotation(cpx_loads* l, double omega, double ax, double ay);
CP_API int cpx_loads_fix_dof(cpx_loads* l, int dof);
/* initConditions (src/PlasticitySolver.cu:812-1005): rp, mask (1 = free) and
 * the prescribed displacements, each 2 * node_count long. */
CP_API int cpx_loads_build(const cpx_mesh* m, const cpx_loads* l, double h, double rho, double* rp,
                           unsigned char* mask, double* uv);

/* Aggregation multigrid hierarchy of the node graph (host set-up; the
 * solver keeps one per instance for the whole solve). adj_pos / adj: node
 * graph without the node itself (cp_get_csr's adj_pos / adj); xy: 2 per
 * node; mask: 2 per node, 1 = free DOF. Coarsening stops at
 * min_coarse_dofs DOFs or when a level stops shrinking. Level 0 has 2 DOFs
 * per node, coarser levels 3 (the rigid-body modes of an aggregate).
 * part_nodes > 0 cuts level 0 into ranges of that many nodes that no level-0
 * aggregate crosses (0: one range); level 1's partition bounds then give the
 * aggregates of each range, and coarser levels aggregate without ranges. */
typedef struct cpx_amg cpx_amg;
CP_API int cpx_amg_build(int node_count, const int* adj_pos, const int* adj, const double* xy,
                         const unsigned char* mask, int min_coarse_dofs, int part_nodes, cpx_amg** out);
/* Partition bounds of level l: part_pos[p] .. part_pos[p + 1] are the nodes
 * of partition p (n_parts + 1 values; one partition from level 2 on). */
CP_API int cpx_amg_level_parts(const cpx_amg* h, int level, int* n_parts, int* part_pos);
CP_API int cpx_amg_destroy(cpx_amg* h);
CP_API int cpx_amg_levels(const cpx_amg* h, int* n_levels);
/* Level l: its node count, DOFs per node and blocks (node count + graph
 * edges: row n holds n itself, then its neighbours), and the aggregate count
 * of the next level (0 on the coarsest). */
CP_API int cpx_amg_level_sizes(const cpx_amg* h, int level, int* node_count, int* dofs_per_node, int* n_blocks,
                               int* n_aggregates);
/* Level l's graph (adj_pos: node_count + 1; adj: n_blocks - node_count), the
 * aggregate of every node and the prolongator blocks (dofs_per_node x 3 per
 * node, row-major). agg and T are left untouched on the coarsest level; any
 * output may be NULL. */
CP_API int cpx_amg_level_get(const cpx_amg* h, int level, int* adj_pos, int* adj, int* agg, double* T);
/* Galerkin operator of level l + 1 from level l's blocks: fine holds
 * dofs_per_node^2 values per block (row-major, blocks in row order: node n's
 * row starts at block adj_pos[n] + n with the diagonal block), coarse
 * receives 9 per block of level l + 1 in the same order. */
CP_API int cpx_amg_galerkin(const cpx_amg* h, int level, const double* fine, double* coarse);
/* The index arrays the device kernels of level l read: counts[6] receives the
 * lengths of rp, ci (block CSR of levels >= 1, diagonal block first), mem_pos,
 * mem (members of every next-level node), gal_pos and gal (the Galerkin map,
 * 4 ints per entry: the fine block's storage index -- at level 0 its position
 * in the sliced layout slice_ptr describes -- its row node, its column node,
 * 0). Arrays may be NULL (counts only); slice_ptr is needed at level 0. */
CP_API int cpx_amg_device_maps(const cpx_amg* h, int level, const int* slice_ptr, int* counts, int* rp, int* ci,
                               int* mem_pos, int* mem, int* gal_pos, int* gal);

/* The small solve of the recycled initial guesses (cp_solve_opts.recycle),
 * the same code the device runs: sums holds the Gram entries d_j . K d_k
 * (j <= k) at k (k + 1) / 2 + j, then the right-hand sides d_j . r0 at 21 + j;
 * cnt (0..6) increments; y receives 6 coefficients (0 for dropped ones). */
CP_API int cpx_recycle_solve(const double* sums, int cnt, double* y);

#ifdef __cplusplus
}
#endif
#endif
