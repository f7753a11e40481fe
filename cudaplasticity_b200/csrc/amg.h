// Aggregation multigrid hierarchy for the secant-stiffness systems (host-side
// set-up). No counterpart in the reference, which solves with plain CG
// (src/ConjGradSolver.h:52-101).
//
// The hierarchy is built once per instance from the node graph and the node
// coordinates, and kept for the whole solve ("frozen"): per outer iteration
// only the Galerkin coarse operators A_{l+1} = T_l^T A_l T_l are recomputed,
// through the fixed maps stored here. Level 0 is the FE system in 2x2 node
// blocks; every coarser level has 3x3 blocks, one "node" per aggregate of the
// level below with the three rigid-body modes (two translations, the
// rotation) as its degrees of freedom.
//   - aggregation: greedy on the level's node graph (a node whose neighbours
//     are all free starts an aggregate of itself and its neighbours; the rest
//     join their first aggregated neighbour, or start a singleton), never
//     across partitions: level 0 may be cut into ranges of part_nodes nodes
//     (the nodes one thread block restricts on the device), and every level-0
//     aggregate belongs to its members' range; level-1 nodes are numbered
//     range by range, and level 1's part_pos records where each range's
//     aggregates lie; coarser levels aggregate without ranges;
//   - tentative prolongator T_l: for each aggregate, the near-null-space rows
//     of its members (at level 0 the rigid-body modes about the aggregate's
//     centroid, with zero rows for prescribed DOFs; at coarser levels the R
//     factors of the level below) orthonormalised by modified Gram-Schmidt;
//     columns that vanish are dropped (left zero);
//   - coarse structure: aggregate I's row holds I itself, then the other
//     aggregates reached from its members' rows, in first-occurrence order.
#pragma once

#include <vector>

namespace cp {
namespace amg {

struct Level {
    int n_nodes = 0;  // nodes of this level (level 0: mesh nodes; else aggregates of the level below)
    int fb = 2;       // DOFs per node (2 at level 0, 3 above)
    std::vector<int> adj_pos, adj;  // node graph: row n holds n, then adj[adj_pos[n] .. adj_pos[n+1])
    std::vector<int> part_pos;      // level 0: range p owns nodes [part_pos[p], part_pos[p+1]); level 1: the
                                    // aggregates of range p; coarser levels: one range
    // to the next level (empty on the coarsest)
    int n_aggs = 0;
    std::vector<int> agg;           // aggregate of every node
    std::vector<double> T;          // per node: fb x 3 block (row-major) of the prolongator
    std::vector<double> nullspace;  // per node: fb x 3 near-null-space rows (input of T)
    // Galerkin map: coarse block b (row I, slot s: s = 0 the diagonal block,
    // s >= 1 the s-th coarse neighbour) gathers the fine blocks listed in
    // gal_src[gal_pos[b] .. gal_pos[b+1]) (fine block = fine row start of node i
    // + slot k, numbered as in this level's rows)
    std::vector<int> gal_pos, gal_src;
    std::vector<int> block_pos;  // first block of every node row of this level (n_nodes + 1)
};

struct Hierarchy {
    std::vector<Level> levels;  // levels[0] fine ... levels.back() coarsest (no aggregation)
};

// Builds the hierarchy. adj_pos / adj: the mesh node graph (node n's
// neighbours, without n); xy: 2 per node; mask: 2 per node, 1 = free DOF;
// part_nodes: nodes per level-0 partition (0: one partition). Coarsening
// stops when a level has at most min_coarse_dofs DOFs or stops shrinking.
Hierarchy build(int n_nodes, const int* adj_pos, const int* adj, const double* xy, const unsigned char* mask,
                int min_coarse_dofs, int part_nodes = 0);

// The index arrays the device kernels of level l use (mg.cu):
//   rp, ci   -- block CSR of level l >= 1 (diagonal block first in every row);
//   mem_pos, mem -- members of every level l + 1 node (not on the coarsest);
//   gal_pos, gal -- the Galerkin map with 4 ints per entry: the fine block's
//      storage index (level 0: its position in the sliced layout given by
//      slice_ptr, in blocks of 32 nodes, slice s of width w_s holding block k
//      of node 32 s + t at slice_ptr[s] + 32 k + t; coarser levels: its block
//      CSR position), its row node, its column node, 0.
struct DeviceMaps {
    std::vector<int> rp, ci, mem_pos, mem, gal_pos, gal;
};
DeviceMaps device_maps(const Hierarchy& h, int l, const int* slice_ptr);

// A_{l+1} from A_l (host restatement of the map the device applies):
// fine: per block of level l, fb*fb values row-major, blocks in row order;
// coarse: the same for level l+1 (3x3 blocks).
void galerkin(const Hierarchy& h, int l, const double* fine, double* coarse);

}  // namespace amg
}  // namespace cp
