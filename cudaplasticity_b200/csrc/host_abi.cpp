// extern "C" wrappers of the host-side drop-in classes (include/cuplast_host.h).
#include <algorithm>
#include <exception>
#include <new>
#include <stdexcept>
#include <vector>

#include "../../include/cuplast/LoadConditions.hpp"
#include "../../include/cuplast_host.h"
#include "amg.h"

struct cpx_mesh {
    cuplast::Mesh m;
};
struct cpx_loads {
    cuplast::LoadConditions l;
};
struct cpx_amg {
    cp::amg::Hierarchy h;
};

namespace {
template <typename F>
int guard(F&& f) {
    try {
        f();
        return CP_OK;
    } catch (const std::bad_alloc&) {
        return CP_ERR_NOMEM;
    } catch (const std::out_of_range&) {
        return CP_ERR_INVALID;
    } catch (const std::invalid_argument&) {
        return CP_ERR_UNSUPPORTED;
    } catch (...) {
        return CP_ERR_INVALID;
    }
}
}  // namespace

extern "C" {

CP_API int cpx_mesh_create(cpx_mesh** out) {
    if (!out) return CP_ERR_INVALID;
    *out = new (std::nothrow) cpx_mesh();
    return *out ? CP_OK : CP_ERR_NOMEM;
}
CP_API int cpx_mesh_destroy(cpx_mesh* m) {
    delete m;
    return CP_OK;
}
CP_API int cpx_mesh_gen_rect(cpx_mesh* m, double x1, double x2, double y1, double y2, int n1, int n2, int order) {
    if (!m || n1 <= 0 || n2 <= 0 || (order != 1 && order != 2)) return CP_ERR_INVALID;
    return guard([&] { m->m.genRectangle(x1, x2, y1, y2, n1, n2, order); });
}
CP_API int cpx_mesh_gen_rect_with_hole(cpx_mesh* m, double x1, double x2, double y1, double y2, double r, int n1,
                                       int n2, int rad_n, int order) {
    if (!m || n1 <= 0 || n2 <= 0 || !(r > 0) || (order != 1 && order != 2)) return CP_ERR_INVALID;
    return guard([&] { m->m.genRectWithHole(x1, x2, y1, y2, r, n1, n2, order, rad_n); });
}
CP_API int cpx_mesh_gen_ring(cpx_mesh* m, double a, double b, int n_phi, int n_r, int order) {
    if (!m || n_phi < 3 || n_r <= 0 || !(b > a) || !(a > 0) || (order != 1 && order != 2)) return CP_ERR_INVALID;
    return guard([&] { m->m.genRing(a, b, n_phi, n_r, order); });
}
CP_API int cpx_mesh_load_inp(cpx_mesh* m, const char* path) {
    if (!m || !path) return CP_ERR_INVALID;
    return guard([&] { m->m.loadFromFile(path); });
}
CP_API int cpx_mesh_renum_by_direction(cpx_mesh* m, double dx, double dy) {
    if (!m) return CP_ERR_INVALID;
    return guard([&] { m->m.renumByDirection(cuplast::vec2(dx, dy)); });
}
CP_API int cpx_mesh_smooth_ring(cpx_mesh* m, int border_n) {
    if (!m || border_n < 3 || m->m.nodeCount % border_n) return CP_ERR_INVALID;
    return guard([&] { m->m.smoothRing(border_n); });
}
CP_API int cpx_mesh_quality(const cpx_mesh* m, double* aspect, double* skew_sin, double* avr_size) {
    if (!m) return CP_ERR_INVALID;
    return guard([&] {
        for (int e = 0; e < m->m.count4; ++e) {
            if (aspect) aspect[e] = m->m.aspectRatio(e);
            if (skew_sin) skew_sin[e] = m->m.skewAngleSin(e);
        }
        if (avr_size) *avr_size = m->m.avrElemSize();
    });
}
CP_API int cpx_mesh_split_t3(cpx_mesh* m) {
    if (!m) return CP_ERR_INVALID;
    return guard([&] { m->m.splitToTriangles(); });
}
CP_API int cpx_mesh_set(cpx_mesh* m, int nodes, const double* xy, int c3, const int* e3, int c4, const int* e4,
                        int nb, const int* bl, const int* bn, int c8, const int* e8) {
    if (!m || nodes <= 0 || !xy || c3 < 0 || c4 < 0 || nb < 0 || c8 < 0 || (c8 && !e8)) return CP_ERR_INVALID;
    return guard([&] {
        std::vector<std::vector<int>> borders(nb);
        int off = 0;
        for (int b = 0; b < nb; ++b) {
            borders[b].assign(bn + off, bn + off + bl[b]);
            off += bl[b];
        }
        m->m.assign(nodes, xy, c3, e3, c4, e4, borders, c8, e8);
    });
}
CP_API int cpx_mesh_counts(const cpx_mesh* m, int* nodes, int* c3, int* c4, int* nb, int* bt, int* c8) {
    if (!m) return CP_ERR_INVALID;
    if (c8) *c8 = m->m.count8;
    if (nodes) *nodes = m->m.nodeCount;
    if (c3) *c3 = m->m.count3;
    if (c4) *c4 = m->m.count4;
    if (nb) *nb = m->m.bordersCount;
    if (bt) {
        int t = 0;
        for (int b = 0; b < m->m.bordersCount; ++b) t += m->m.borderLength[b];
        *bt = t;
    }
    return CP_OK;
}
CP_API int cpx_mesh_get(const cpx_mesh* m, double* xy, int* e3, int* e4, int* bl, int* bn, int* e8) {
    if (!m) return CP_ERR_INVALID;
    const cuplast::Mesh& M = m->m;
    if (e8)
        for (int i = 0; i < 8 * M.count8; ++i) e8[i] = M.elem8[i];
    if (xy)
        for (int i = 0; i < M.nodeCount; ++i) {
            xy[2 * i] = M.node[i].x;
            xy[2 * i + 1] = M.node[i].y;
        }
    if (e3)
        for (int i = 0; i < 3 * M.count3; ++i) e3[i] = M.elem3[i];
    if (e4)
        for (int i = 0; i < 4 * M.count4; ++i) e4[i] = M.elem4[i];
    int off = 0;
    for (int b = 0; b < M.bordersCount; ++b) {
        if (bl) bl[b] = M.borderLength[b];
        if (bn)
            for (int j = 0; j < M.borderLength[b]; ++j) bn[off + j] = M.borders[b][j];
        off += M.borderLength[b];
    }
    return CP_OK;
}
CP_API int cpx_mesh_max_index_diff(const cpx_mesh* m, int* out) {
    if (!m || !out) return CP_ERR_INVALID;
    *out = m->m.findMaxIndexDiff();
    return CP_OK;
}

CP_API int cpx_loads_create(cpx_loads** out) {
    if (!out) return CP_ERR_INVALID;
    *out = new (std::nothrow) cpx_loads();
    return *out ? CP_OK : CP_ERR_NOMEM;
}
CP_API int cpx_loads_destroy(cpx_loads* l) {
    delete l;
    return CP_OK;
}
#define CPX_L(body)                  \
    if (!l) return CP_ERR_INVALID;   \
    return guard([&] { body; });
CP_API int cpx_loads_set_force(cpx_loads* l, int b, double fx, double fy, int normal) {
    CPX_L(l->l.setForce(b, cuplast::vec2(fx, fy), normal != 0))
}
CP_API int cpx_loads_set_displacement(cpx_loads* l, int b, double ux, double uy, int mx, int my) {
    CPX_L(l->l.setDisplacement(b, cuplast::vec2(ux, uy), mx != 0, my != 0))
}
CP_API int cpx_loads_fix_border(cpx_loads* l, int b) { CPX_L(l->l.fixBorder(b)) }
CP_API int cpx_loads_fix_border_vert(cpx_loads* l, int b) { CPX_L(l->l.fixBorderVert(b)) }
CP_API int cpx_loads_fix_border_hor(cpx_loads* l, int b) { CPX_L(l->l.fixBorderHor(b)) }
CP_API int cpx_loads_fix_vert_axis(cpx_loads* l, double x) { CPX_L(l->l.fixVertAxis(x)) }
CP_API int cpx_loads_fix_hor_axis(cpx_loads* l, double y) { CPX_L(l->l.fixHorAxis(y)) }
CP_API int cpx_loads_fix_point(cpx_loads* l, double x, double y) { CPX_L(l->l.fixPoint(cuplast::vec2(x, y))) }
CP_API int cpx_loads_set_displ_point(cpx_loads* l, double x, double y, double ux, double uy) {
    CPX_L(l->l.setDisplPoint(cuplast::vec2(x, y), cuplast::vec2(ux, uy)))
}
CP_API int cpx_loads_set_force_point(cpx_loads* l, double x, double y, double fx, double fy) {
    CPX_L(l->l.setForcePoint(cuplast::vec2(x, y), cuplast::vec2(fx, fy)))
}
CP_API int cpx_loads_set_gravity(cpx_loads* l, double g, double dx, double dy) {
    CPX_L(l->l.setGravity(g, cuplast::vec2(dx, dy)))
}
CP_API int cpx_loads_set_rotation(cpx_loads* l, double w, double ax, double ay) {
    CPX_L(l->l.setRotation(w, cuplast::vec2(ax, ay)))
}
CP_API int cpx_loads_fix_dof(cpx_loads* l, int dof) { CPX_L(l->l.fixDof(dof)) }
#undef CPX_L

CP_API int cpx_loads_build(const cpx_mesh* m, const cpx_loads* l, double h, double rho, double* rp,
                           unsigned char* mask, double* uv) {
    if (!m || !l || !rp || !mask || !uv) return CP_ERR_INVALID;
    return guard([&] {
        std::vector<double> r, u;
        std::vector<unsigned char> k;
        cuplast::buildConditions(m->m, l->l, h, rho, r, k, u);
        std::copy(r.begin(), r.end(), rp);
        std::copy(k.begin(), k.end(), mask);
        std::copy(u.begin(), u.end(), uv);
    });
}

CP_API int cpx_amg_build(int node_count, const int* adj_pos, const int* adj, const double* xy,
                         const unsigned char* mask, int min_coarse_dofs, int part_nodes, cpx_amg** out) {
    if (!out || node_count <= 0 || !adj_pos || !adj || !xy || !mask || min_coarse_dofs < 0 || part_nodes < 0)
        return CP_ERR_INVALID;
    *out = nullptr;
    for (int n = 0; n < node_count; ++n)
        if (adj_pos[n + 1] < adj_pos[n]) return CP_ERR_INVALID;
    for (int q = 0; q < adj_pos[node_count]; ++q)
        if (adj[q] < 0 || adj[q] >= node_count) return CP_ERR_INVALID;
    return guard([&] {
        auto* p = new cpx_amg();
        try {
            p->h = cp::amg::build(node_count, adj_pos, adj, xy, mask, min_coarse_dofs, part_nodes);
        } catch (...) {
            delete p;
            throw;
        }
        *out = p;
    });
}
CP_API int cpx_amg_destroy(cpx_amg* h) {
    delete h;
    return CP_OK;
}
CP_API int cpx_amg_levels(const cpx_amg* h, int* n_levels) {
    if (!h || !n_levels) return CP_ERR_INVALID;
    *n_levels = (int)h->h.levels.size();
    return CP_OK;
}
CP_API int cpx_amg_level_sizes(const cpx_amg* h, int level, int* node_count, int* dofs_per_node, int* n_blocks,
                               int* n_aggregates) {
    if (!h || level < 0 || level >= (int)h->h.levels.size()) return CP_ERR_INVALID;
    const cp::amg::Level& L = h->h.levels[level];
    if (node_count) *node_count = L.n_nodes;
    if (dofs_per_node) *dofs_per_node = L.fb;
    if (n_blocks) *n_blocks = L.n_nodes + L.adj_pos[L.n_nodes];
    if (n_aggregates) *n_aggregates = L.n_aggs;
    return CP_OK;
}
CP_API int cpx_amg_level_parts(const cpx_amg* h, int level, int* n_parts, int* part_pos) {
    if (!h || level < 0 || level >= (int)h->h.levels.size()) return CP_ERR_INVALID;
    const cp::amg::Level& L = h->h.levels[level];
    if (n_parts) *n_parts = (int)L.part_pos.size() - 1;
    if (part_pos) std::copy(L.part_pos.begin(), L.part_pos.end(), part_pos);
    return CP_OK;
}
CP_API int cpx_amg_level_get(const cpx_amg* h, int level, int* adj_pos, int* adj, int* agg, double* T) {
    if (!h || level < 0 || level >= (int)h->h.levels.size()) return CP_ERR_INVALID;
    const cp::amg::Level& L = h->h.levels[level];
    if (adj_pos) std::copy(L.adj_pos.begin(), L.adj_pos.end(), adj_pos);
    if (adj) std::copy(L.adj.begin(), L.adj.end(), adj);
    if (agg) std::copy(L.agg.begin(), L.agg.end(), agg);
    if (T) std::copy(L.T.begin(), L.T.end(), T);
    return CP_OK;
}
CP_API int cpx_amg_device_maps(const cpx_amg* h, int level, const int* slice_ptr, int* counts, int* rp, int* ci,
                               int* mem_pos, int* mem, int* gal_pos, int* gal) {
    if (!h || !counts || level < 0 || level >= (int)h->h.levels.size() || (level == 0 && !slice_ptr))
        return CP_ERR_INVALID;
    return guard([&] {
        const cp::amg::DeviceMaps d = cp::amg::device_maps(h->h, level, slice_ptr);
        const std::vector<int>* v[6] = {&d.rp, &d.ci, &d.mem_pos, &d.mem, &d.gal_pos, &d.gal};
        int* out[6] = {rp, ci, mem_pos, mem, gal_pos, gal};
        for (int k = 0; k < 6; ++k) {
            counts[k] = (int)v[k]->size();
            if (out[k]) std::copy(v[k]->begin(), v[k]->end(), out[k]);
        }
    });
}
CP_API int cpx_amg_galerkin(const cpx_amg* h, int level, const double* fine, double* coarse) {
    if (!h || !fine || !coarse || level < 0 || level + 1 >= (int)h->h.levels.size()) return CP_ERR_INVALID;
    return guard([&] { cp::amg::galerkin(h->h, level, fine, coarse); });
}

}  // extern "C"
