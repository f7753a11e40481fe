// Host-side set-up of the aggregation multigrid hierarchy (see amg.h).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "amg.h"

namespace cp {
namespace amg {

namespace {

constexpr int kMinRange = 16;  // coarse levels: fewest nodes of a range aggregated on its own

// Greedy aggregation of a node graph inside each partition (nodes
// [part_pos[p], part_pos[p+1]) form partition p; edges between partitions are
// ignored): pass 1 makes an aggregate of every node whose neighbours are all
// still free (the node and its neighbours); pass 2 puts each remaining node
// into the aggregate of its first aggregated neighbour, or into a new
// singleton. Aggregates are then numbered partition by partition, in order of
// creation within a partition, and the next level's partition bounds are
// returned in cpart.
int aggregate(int n, const std::vector<int>& adj_pos, const std::vector<int>& adj, const std::vector<int>& part_pos,
              std::vector<int>& agg, std::vector<int>& cpart) {
    const int np = (int)part_pos.size() - 1;
    std::vector<int> part_of(n);
    for (int p = 0; p < np; ++p)
        for (int i = part_pos[p]; i < part_pos[p + 1]; ++i) part_of[i] = p;
    agg.assign(n, -1);
    int na = 0;
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        bool free_all = true;
        for (int q = adj_pos[i]; q < adj_pos[i + 1]; ++q)
            if (part_of[adj[q]] == part_of[i] && agg[adj[q]] >= 0) {
                free_all = false;
                break;
            }
        if (!free_all) continue;
        agg[i] = na;
        for (int q = adj_pos[i]; q < adj_pos[i + 1]; ++q)
            if (part_of[adj[q]] == part_of[i]) agg[adj[q]] = na;
        ++na;
    }
    for (int i = 0; i < n; ++i) {
        if (agg[i] >= 0) continue;
        int a = -1;
        for (int q = adj_pos[i]; q < adj_pos[i + 1]; ++q)
            if (part_of[adj[q]] == part_of[i] && agg[adj[q]] >= 0) {
                a = agg[adj[q]];
                break;
            }
        agg[i] = a >= 0 ? a : na++;
    }
    // partition of every aggregate (its members share one), then renumber
    std::vector<int> apart(na), cnt(np + 1, 0);
    for (int i = 0; i < n; ++i) apart[agg[i]] = part_of[i];
    for (int a = 0; a < na; ++a) ++cnt[apart[a] + 1];
    for (int p = 0; p < np; ++p) cnt[p + 1] += cnt[p];
    cpart = cnt;
    std::vector<int> renum(na);
    for (int a = 0; a < na; ++a) renum[a] = cnt[apart[a]]++;
    for (int i = 0; i < n; ++i) agg[i] = renum[agg[i]];
    return na;
}

// Modified Gram-Schmidt of the columns of B (rows x 3, row-major) in place:
// B becomes Q (orthonormal columns, dropped ones zero), R (3x3) its factor.
void mgs(std::vector<double>& B, int rows, double R[9]) {
    for (int i = 0; i < 9; ++i) R[i] = 0.0;
    double ref[3];
    for (int c = 0; c < 3; ++c) {
        double s = 0.0;
        for (int r = 0; r < rows; ++r) s += B[3 * r + c] * B[3 * r + c];
        ref[c] = std::sqrt(s);
    }
    for (int c = 0; c < 3; ++c) {
        for (int p = 0; p < c; ++p) {
            double d = 0.0;
            for (int r = 0; r < rows; ++r) d += B[3 * r + p] * B[3 * r + c];
            R[3 * p + c] = d;
            for (int r = 0; r < rows; ++r) B[3 * r + c] -= d * B[3 * r + p];
        }
        double s = 0.0;
        for (int r = 0; r < rows; ++r) s += B[3 * r + c] * B[3 * r + c];
        const double nrm = std::sqrt(s);
        if (!(nrm > 1e-10 * ref[c]) || nrm == 0.0) {  // dependent (or empty) column: dropped
            for (int r = 0; r < rows; ++r) B[3 * r + c] = 0.0;
            continue;
        }
        R[3 * c + c] = nrm;
        for (int r = 0; r < rows; ++r) B[3 * r + c] /= nrm;
    }
}

}  // namespace

Hierarchy build(int n_nodes, const int* adj_pos, const int* adj, const double* xy, const unsigned char* mask,
                int min_coarse_dofs, int part_nodes) {
    if (n_nodes <= 0 || !adj_pos || !adj || !xy || !mask || part_nodes < 0)
        throw std::invalid_argument("amg: empty input");
    Hierarchy h;
    Level L0;
    L0.n_nodes = n_nodes;
    L0.fb = 2;
    L0.adj_pos.assign(adj_pos, adj_pos + n_nodes + 1);
    L0.adj.assign(adj, adj + adj_pos[n_nodes]);
    if (part_nodes == 0 || part_nodes >= n_nodes) {
        L0.part_pos = {0, n_nodes};
    } else {
        for (int b = 0; b < n_nodes; b += part_nodes) L0.part_pos.push_back(b);
        L0.part_pos.push_back(n_nodes);
    }
    // level-0 near-null space: rigid-body modes, centred per aggregate below
    L0.nullspace.assign(6 * (size_t)n_nodes, 0.0);
    h.levels.push_back(std::move(L0));
    for (;;) {
        Level& F = h.levels.back();
        const int fb = F.fb;
        F.block_pos.assign(F.n_nodes + 1, 0);
        for (int i = 0; i < F.n_nodes; ++i) F.block_pos[i + 1] = F.block_pos[i] + 1 + (F.adj_pos[i + 1] - F.adj_pos[i]);
        if (F.n_nodes * fb <= min_coarse_dofs) break;
        // Level 0 aggregates inside its ranges. A coarser level aggregates
        // inside the ranges it inherits, merged with their successors until
        // each holds at least kMinRange nodes: small ranges keep the coarse
        // aggregates small (gentle coarsening), merging keeps coarsening going.
        const bool fine = h.levels.size() == 1;
        std::vector<int> ranges = {0};
        if (fine) {
            ranges = F.part_pos;
        } else {
            for (size_t p = 1; p < F.part_pos.size(); ++p)
                if (F.part_pos[p] - ranges.back() >= kMinRange || p + 1 == F.part_pos.size()) ranges.push_back(F.part_pos[p]);
            if (ranges.size() > 2 && ranges[ranges.size() - 1] - ranges[ranges.size() - 2] < kMinRange)
                ranges.erase(ranges.end() - 2);  // a short last range joins the one before
        }
        std::vector<int> agg, cpart;
        const int na = aggregate(F.n_nodes, F.adj_pos, F.adj, ranges, agg, cpart);
        if (na >= F.n_nodes) break;  // no longer shrinking
        F.agg = agg;
        F.n_aggs = na;
        // members of every aggregate, in node order
        std::vector<int> mpos(na + 1, 0), mem(F.n_nodes);
        for (int i = 0; i < F.n_nodes; ++i) ++mpos[agg[i] + 1];
        for (int a = 0; a < na; ++a) mpos[a + 1] += mpos[a];
        {
            std::vector<int> cur(mpos.begin(), mpos.end() - 1);
            for (int i = 0; i < F.n_nodes; ++i) mem[cur[agg[i]]++] = i;
        }
        // near-null-space rows of level 0: rigid-body modes about the centroid
        if (fine) {
            for (int a = 0; a < na; ++a) {
                double cx = 0.0, cy = 0.0;
                const int m0 = mpos[a], m1 = mpos[a + 1];
                for (int q = m0; q < m1; ++q) {
                    cx += xy[2 * mem[q]];
                    cy += xy[2 * mem[q] + 1];
                }
                cx /= (m1 - m0);
                cy /= (m1 - m0);
                for (int q = m0; q < m1; ++q) {
                    const int i = mem[q];
                    double* B = &F.nullspace[6 * (size_t)i];
                    const double dx = xy[2 * i] - cx, dy = xy[2 * i + 1] - cy;
                    if (mask[2 * i]) { B[0] = 1.0; B[1] = 0.0; B[2] = -dy; }
                    if (mask[2 * i + 1]) { B[3] = 0.0; B[4] = 1.0; B[5] = dx; }
                }
            }
        }
        // tentative prolongator and the next level's near-null space (R factors)
        F.T.assign((size_t)F.n_nodes * fb * 3, 0.0);
        Level C;
        C.n_nodes = na;
        C.fb = 3;
        C.part_pos = cpart;
        C.nullspace.assign(9 * (size_t)na, 0.0);
        for (int a = 0; a < na; ++a) {
            const int m0 = mpos[a], m1 = mpos[a + 1], rows = (m1 - m0) * fb;
            std::vector<double> B((size_t)rows * 3);
            for (int q = m0; q < m1; ++q)
                std::memcpy(&B[(size_t)(q - m0) * fb * 3], &F.nullspace[(size_t)mem[q] * fb * 3], sizeof(double) * fb * 3);
            double R[9];
            mgs(B, rows, R);
            for (int q = m0; q < m1; ++q)
                std::memcpy(&F.T[(size_t)mem[q] * fb * 3], &B[(size_t)(q - m0) * fb * 3], sizeof(double) * fb * 3);
            std::memcpy(&C.nullspace[9 * (size_t)a], R, sizeof R);
        }
        // coarse graph: aggregates reached from the members' rows, first occurrence
        C.adj_pos.assign(na + 1, 0);
        std::vector<std::vector<int>> nb(na);
        for (int a = 0; a < na; ++a)
            for (int q = mpos[a]; q < mpos[a + 1]; ++q) {
                const int i = mem[q];
                for (int r = F.adj_pos[i]; r < F.adj_pos[i + 1]; ++r) {
                    const int b = agg[F.adj[r]];
                    if (b != a && std::find(nb[a].begin(), nb[a].end(), b) == nb[a].end()) nb[a].push_back(b);
                }
            }
        for (int a = 0; a < na; ++a) C.adj_pos[a + 1] = C.adj_pos[a] + (int)nb[a].size();
        C.adj.reserve(C.adj_pos[na]);
        for (int a = 0; a < na; ++a) C.adj.insert(C.adj.end(), nb[a].begin(), nb[a].end());
        // Galerkin map: coarse block (a, slot) <- fine blocks (i in a, slot k), in
        // fine-row order
        std::vector<int> cbp(na + 1, 0);
        for (int a = 0; a < na; ++a) cbp[a + 1] = cbp[a] + 1 + (int)nb[a].size();
        std::vector<std::vector<int>> src(cbp[na]);
        for (int i = 0; i < F.n_nodes; ++i) {
            const int a = agg[i];
            for (int k = 0; k <= F.adj_pos[i + 1] - F.adj_pos[i]; ++k) {
                const int j = k == 0 ? i : F.adj[F.adj_pos[i] + k - 1];
                const int b = agg[j];
                int s = 0;
                if (b != a) s = 1 + (int)(std::find(nb[a].begin(), nb[a].end(), b) - nb[a].begin());
                src[cbp[a] + s].push_back(F.block_pos[i] + k);
            }
        }
        F.gal_pos.assign(cbp[na] + 1, 0);
        for (int b = 0; b < cbp[na]; ++b) F.gal_pos[b + 1] = F.gal_pos[b] + (int)src[b].size();
        F.gal_src.reserve(F.gal_pos[cbp[na]]);
        for (auto& v : src) F.gal_src.insert(F.gal_src.end(), v.begin(), v.end());
        h.levels.push_back(std::move(C));
    }
    return h;
}

DeviceMaps device_maps(const Hierarchy& h, int l, const int* slice_ptr) {
    const Level& F = h.levels.at(l);
    const int n = F.n_nodes, nb = F.block_pos[n];
    DeviceMaps d;
    if (l > 0) {
        d.rp = F.block_pos;
        d.ci.resize(nb);
        for (int i = 0; i < n; ++i) {
            int q = F.block_pos[i];
            d.ci[q++] = i;
            for (int r = F.adj_pos[i]; r < F.adj_pos[i + 1]; ++r) d.ci[q++] = F.adj[r];
        }
    }
    if (F.agg.empty()) return d;  // the coarsest level
    const int nn = F.n_aggs;
    d.mem_pos.assign(nn + 1, 0);
    d.mem.resize(n);
    for (int i = 0; i < n; ++i) ++d.mem_pos[F.agg[i] + 1];
    for (int a = 0; a < nn; ++a) d.mem_pos[a + 1] += d.mem_pos[a];
    {
        std::vector<int> cur(d.mem_pos.begin(), d.mem_pos.end() - 1);
        for (int i = 0; i < n; ++i) d.mem[cur[F.agg[i]]++] = i;
    }
    std::vector<int> row_of(nb), col_of(nb), k_of(nb);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k <= F.adj_pos[i + 1] - F.adj_pos[i]; ++k) {
            const int b = F.block_pos[i] + k;
            row_of[b] = i;
            col_of[b] = k == 0 ? i : F.adj[F.adj_pos[i] + k - 1];
            k_of[b] = k;
        }
    if (l == 0 && !slice_ptr) throw std::invalid_argument("amg: level 0 needs the sliced layout");
    d.gal_pos = F.gal_pos;
    d.gal.resize(4 * F.gal_src.size());
    for (size_t q = 0; q < F.gal_src.size(); ++q) {
        const int b = F.gal_src[q], i = row_of[b];
        d.gal[4 * q] = l == 0 ? slice_ptr[i >> 5] + 32 * k_of[b] + (i & 31) : b;
        d.gal[4 * q + 1] = i;
        d.gal[4 * q + 2] = col_of[b];
        d.gal[4 * q + 3] = 0;
    }
    return d;
}

void galerkin(const Hierarchy& h, int l, const double* fine, double* coarse) {
    const Level& F = h.levels.at(l);
    const Level& C = h.levels.at(l + 1);
    const int fb = F.fb;
    // the fine row and column node of every fine block
    std::vector<int> row_of(F.block_pos[F.n_nodes]), col_of(F.block_pos[F.n_nodes]);
    for (int i = 0; i < F.n_nodes; ++i)
        for (int k = 0; k <= F.adj_pos[i + 1] - F.adj_pos[i]; ++k) {
            row_of[F.block_pos[i] + k] = i;
            col_of[F.block_pos[i] + k] = k == 0 ? i : F.adj[F.adj_pos[i] + k - 1];
        }
    const int ncb = C.n_nodes + C.adj_pos[C.n_nodes];
    for (int b = 0; b < ncb; ++b) {
        double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int q = F.gal_pos[b]; q < F.gal_pos[b + 1]; ++q) {
            const int fbk = F.gal_src[q];
            const double* K = fine + (size_t)fbk * fb * fb;
            const double* Ti = &F.T[(size_t)row_of[fbk] * fb * 3];
            const double* Tj = &F.T[(size_t)col_of[fbk] * fb * 3];
            // acc += Ti^T K Tj
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) {
                    double s = 0.0;
                    for (int x = 0; x < fb; ++x)
                        for (int y = 0; y < fb; ++y) s += Ti[x * 3 + r] * K[x * fb + y] * Tj[y * 3 + c];
                    acc[3 * r + c] += s;
                }
        }
        std::memcpy(coarse + 9 * (size_t)b, acc, sizeof acc);
    }
}

}  // namespace amg
}  // namespace cp
