/*
 * cuplast_oracle.c -- CPU restatement of CudaPlasticity's 2D elasto-plastic
 * hot path. TEST INFRASTRUCTURE ONLY: it is the checker of the CUDA product,
 * never part of it. Each function names the reference code it restates
 * (paths relative to the reference project root).
 *
 * Scope: T3 (extension; the reference only declares it), Q4 and Q8 elements,
 * plane stress/strain, the reference's CSR ordering, masked unpreconditioned
 * CG, the secant (variable elastic parameters) update with the reference's
 * linear/power diagrams plus the injected Hollomon and piecewise-linear
 * diagrams, the plastic-strain post-processing and the strain energy.
 *
 * Deliberate differences from the reference, all below the parity tolerance:
 *  - assembly adds element matrices straight into the CSR values in element
 *    order (the reference adds them into a band matrix with omp atomics and
 *    gathers it into CSR, src/PlasticitySolver.cu:786-810); with one thread the
 *    summation order, and so every value, is the same;
 *  - CG returns the last iterate in the caller's buffer (the reference's
 *    pointer swap can leave x_{k-1} there, src/ConjGradSolver.h:53,69,100) and
 *    skips the loop when the initial residual is exactly zero (the reference
 *    would divide 0/0);
 *  - body forces are evaluated at the element's node (the reference indexes the
 *    node array with the DOF index, src/PlasticitySolver.cu:937-940, which only
 *    gives the same value for constant fields such as gravity);
 *  - the Q8 Gauss rule uses sqrt(0.6), 5/9 and 8/9 to full precision (the
 *    reference writes them with 15 decimals, src/PlasticitySolver.cu:70,190),
 *    a difference of about 1e-15 relative; the shape-function derivatives are
 *    the standard serendipity ones in factored form rather than the
 *    reference's expanded polynomials (same values up to rounding).
 */
#include "cuplast_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#include "cpbin.h"

/* ------------------------------------------------------------------ job -- */

enum { DG_NONE, DG_LINEAR, DG_POWER, DG_HOLLOMON, DG_PIECEWISE };

typedef struct {
    int kind;
    double E, sigmaT, K_T, A, m;   /* linear / power (src/Material.cu:3-23) */
    double sy, eps0, n;            /* Hollomon, inverted by Newton */
    int npw;
    double pw_e[16], pw_s[16];     /* piecewise linear breakpoints */
} diagram_t;

#define MAXB 64
#define MAXL 256

typedef struct {
    char mode[16];
    char mesh_path[1024];
    double E, nu, h, rho;
    int have_material;
    diagram_t dg;
    int plane_strain;
    double cg_eps, outer_eps;
    int max_outer, levels;
    int dump_k, dump_csr;
    /* loads (src/LoadConditions.cuh) */
    int force_set[MAXB];
    double force_v[MAXB][2];
    int force_norm[MAXB];
    int displ_set[MAXB];
    double displ_v[MAXB][2];
    int displ_midx[MAXB], displ_midy[MAXB];
    int fixb_set[MAXB], fixb_vert[MAXB];
    int n_axis;
    int axis_vert[MAXL];
    double axis_coord[MAXL];
    int n_fpt;
    double fpt[MAXL][4];
    int n_dpt;
    double dpt[MAXL][4];
    int grav_set;
    double grav[2];
    int n_fixdof;
    int fixdof[4096];
} job_t;

typedef struct {
    int n_nodes;
    double* xy;
    int c3, c4, c8;
    int* e3;
    int* e4;
    int* e8;
    unsigned char* sec;   /* second-order (mid-side) nodes: Mesh::secOrdNodes */
    int n_borders;
    int* border_len;
    int** borders;
} mesh_t;

static int parse_job(const char* path, job_t* j) {
    FILE* f = fopen(path, "r");
    char line[8192];
    if (!f) return -1;
    memset(j, 0, sizeof *j);
    strcpy(j->mode, "solve");
    j->nu = 0.3;
    j->h = 1.0;
    j->rho = 1.0;
    j->cg_eps = 1e-7;
    j->outer_eps = 1e-5;
    j->max_outer = 50;
    j->levels = 1;
    while (fgets(line, sizeof line, f)) {
        char key[64] = {0};
        int off = 0;
        if (sscanf(line, "%63s%n", key, &off) != 1 || key[0] == '#') continue;
        const char* rest = line + off;
        if (!strcmp(key, "mode")) sscanf(rest, "%15s", j->mode);
        else if (!strcmp(key, "mesh")) {
            char kind[32];
            sscanf(rest, "%31s %1023s", kind, j->mesh_path);
            if (strcmp(kind, "file")) { fclose(f); return -2; }
        } else if (!strcmp(key, "material")) {
            sscanf(rest, "%lf %lf %lf", &j->E, &j->nu, &j->h);
            j->have_material = 1;
        } else if (!strcmp(key, "diagram")) {
            char kind[32];
            int o2 = 0;
            sscanf(rest, "%31s%n", kind, &o2);
            const char* r2 = rest + o2;
            diagram_t* d = &j->dg;
            if (!strcmp(kind, "linear")) { d->kind = DG_LINEAR; sscanf(r2, "%lf %lf %lf", &d->E, &d->sigmaT, &d->K_T); }
            else if (!strcmp(kind, "power")) { d->kind = DG_POWER; sscanf(r2, "%lf %lf %lf %lf", &d->E, &d->sigmaT, &d->A, &d->m); }
            else if (!strcmp(kind, "hollomon")) {
                d->kind = DG_HOLLOMON;
                sscanf(r2, "%lf %lf %lf %lf", &d->E, &d->sy, &d->eps0, &d->n);
                d->sigmaT = d->sy;
            } else if (!strcmp(kind, "piecewise")) {
                int o3 = 0, i;
                d->kind = DG_PIECEWISE;
                sscanf(r2, "%lf %d%n", &d->E, &d->npw, &o3);
                r2 += o3;
                for (i = 0; i < d->npw && i < 16; ++i) {
                    int o4 = 0;
                    sscanf(r2, "%lf %lf%n", &d->pw_e[i], &d->pw_s[i], &o4);
                    r2 += o4;
                }
                d->sigmaT = d->pw_s[0];
            }
        } else if (!strcmp(key, "plane")) { char w[16]; sscanf(rest, "%15s", w); j->plane_strain = !strcmp(w, "strain"); }
        else if (!strcmp(key, "cg_eps")) sscanf(rest, "%lf", &j->cg_eps);
        else if (!strcmp(key, "outer_eps")) sscanf(rest, "%lf", &j->outer_eps);
        else if (!strcmp(key, "max_outer")) sscanf(rest, "%d", &j->max_outer);
        else if (!strcmp(key, "levels")) sscanf(rest, "%d", &j->levels);
        else if (!strcmp(key, "dump_k")) sscanf(rest, "%d", &j->dump_k);
        else if (!strcmp(key, "dump_csr")) sscanf(rest, "%d", &j->dump_csr);
        else if (!strcmp(key, "fixdof")) { if (j->n_fixdof < 4096) sscanf(rest, "%d", &j->fixdof[j->n_fixdof++]); }
        else if (!strcmp(key, "force")) {
            int b, nrm; double fx, fy;
            sscanf(rest, "%d %lf %lf %d", &b, &fx, &fy, &nrm);
            j->force_set[b] = 1; j->force_v[b][0] = fx; j->force_v[b][1] = fy; j->force_norm[b] = nrm;
        } else if (!strcmp(key, "displ")) {
            int b, mx, my; double ux, uy;
            sscanf(rest, "%d %lf %lf %d %d", &b, &ux, &uy, &mx, &my);
            j->displ_set[b] = 1; j->displ_v[b][0] = ux; j->displ_v[b][1] = uy; j->displ_midx[b] = mx; j->displ_midy[b] = my;
        } else if (!strcmp(key, "fixborderhor")) { int b; sscanf(rest, "%d", &b); j->fixb_set[b] = 1; j->fixb_vert[b] = 0; }
        else if (!strcmp(key, "fixbordervert")) { int b; sscanf(rest, "%d", &b); j->fixb_set[b] = 1; j->fixb_vert[b] = 1; }
        else if (!strcmp(key, "fixvertaxis")) { j->axis_vert[j->n_axis] = 1; sscanf(rest, "%lf", &j->axis_coord[j->n_axis++]); }
        else if (!strcmp(key, "fixhoraxis")) { j->axis_vert[j->n_axis] = 0; sscanf(rest, "%lf", &j->axis_coord[j->n_axis++]); }
        else if (!strcmp(key, "fixpoint")) { double* p = j->dpt[j->n_dpt++]; sscanf(rest, "%lf %lf", &p[0], &p[1]); p[2] = p[3] = 0.0; }
        else if (!strcmp(key, "displpoint")) { double* p = j->dpt[j->n_dpt++]; sscanf(rest, "%lf %lf %lf %lf", &p[0], &p[1], &p[2], &p[3]); }
        else if (!strcmp(key, "forcepoint")) { double* p = j->fpt[j->n_fpt++]; sscanf(rest, "%lf %lf %lf %lf", &p[0], &p[1], &p[2], &p[3]); }
        else if (!strcmp(key, "gravity")) {
            double g, dx, dy, nn;
            sscanf(rest, "%lf %lf %lf", &g, &dx, &dy);
            nn = sqrt(dx * dx + dy * dy);
            j->grav_set = 1; j->grav[0] = g * (dx * (1.0 / nn)); j->grav[1] = g * (dy * (1.0 / nn));
        } else { fclose(f); return -3; }
    }
    fclose(f);
    if (!j->have_material) j->E = j->dg.E;
    return 0;
}

static int load_mesh(const char* path, mesh_t* m) {
    cpbin_file f;
    const cpbin_rec *xy, *e3, *e4, *e8, *bl, *bn;
    int b, off = 0, e, i;
    memset(m, 0, sizeof *m);
    if (cpbin_read(path, &f) != 0) return -1;
    xy = cpbin_get(&f, "node_xy");
    e3 = cpbin_get(&f, "elem3");
    e4 = cpbin_get(&f, "elem4");
    e8 = cpbin_get(&f, "elem8");
    bl = cpbin_get(&f, "border_len");
    bn = cpbin_get(&f, "border_nodes");
    if (!xy) { cpbin_free(&f); return -2; }
    m->n_nodes = (int)(xy->count / 2);
    m->xy = (double*)malloc(sizeof(double) * 2 * (size_t)m->n_nodes);
    memcpy(m->xy, xy->data, sizeof(double) * 2 * (size_t)m->n_nodes);
    m->c3 = e3 ? (int)(e3->count / 3) : 0;
    m->c4 = e4 ? (int)(e4->count / 4) : 0;
    m->e3 = (int*)malloc(sizeof(int) * (3 * (size_t)m->c3 + 1));
    m->e4 = (int*)malloc(sizeof(int) * (4 * (size_t)m->c4 + 1));
    if (m->c3) memcpy(m->e3, e3->data, sizeof(int) * 3 * (size_t)m->c3);
    if (m->c4) memcpy(m->e4, e4->data, sizeof(int) * 4 * (size_t)m->c4);
    m->c8 = e8 ? (int)(e8->count / 8) : 0;
    m->e8 = (int*)malloc(sizeof(int) * (8 * (size_t)m->c8 + 1));
    if (m->c8) memcpy(m->e8, e8->data, sizeof(int) * 8 * (size_t)m->c8);
    /* the mid-side nodes of 8-node elements are the second-order nodes */
    m->sec = (unsigned char*)calloc((size_t)m->n_nodes + 1, 1);
    for (e = 0; e < m->c8; ++e)
        for (i = 4; i < 8; ++i) m->sec[m->e8[8 * e + i]] = 1;
    m->n_borders = bl ? (int)bl->count : 0;
    m->border_len = (int*)malloc(sizeof(int) * (size_t)(m->n_borders + 1));
    m->borders = (int**)malloc(sizeof(int*) * (size_t)(m->n_borders + 1));
    for (b = 0; b < m->n_borders; ++b) {
        int len = ((int*)bl->data)[b];
        m->border_len[b] = len;
        m->borders[b] = (int*)malloc(sizeof(int) * (size_t)len);
        memcpy(m->borders[b], (int*)bn->data + off, sizeof(int) * (size_t)len);
        off += len;
    }
    cpbin_free(&f);
    return 0;
}

static void free_mesh(mesh_t* m) {
    int b;
    for (b = 0; b < m->n_borders; ++b) free(m->borders[b]);
    free(m->borders);
    free(m->border_len);
    free(m->xy);
    free(m->e3);
    free(m->e4);
    free(m->e8);
    free(m->sec);
}

/* ------------------------------------------------------------- diagrams -- */

/* src/Material.cu:14-23 (linear, power) and the injected diagrams. */
static double diagram_f(const diagram_t* d, double eps) {
    double E = d->E;
    switch (d->kind) {
    case DG_LINEAR: {
        double epsT = d->sigmaT / E;
        return eps < epsT ? eps * E : d->sigmaT + (eps - epsT) * d->K_T;
    }
    case DG_POWER: {
        double epsT = d->sigmaT / E, A = d->A, m = d->m;
        return eps < epsT ? eps * E
                          : d->sigmaT + A * pow(eps - epsT + pow(E / (A * m), 1. / (m - 1.)), m) -
                                A * pow(E / (A * m), m / (m - 1.));
    }
    case DG_HOLLOMON: {
        /* sigma = sy (1 + eps_p/eps0)^n with eps = sigma/E + eps_p, i.e.
         * eps = s/E + eps0((s/sy)^(1/n) - 1); Newton from s = sy. */
        double sy = d->sy, e0 = d->eps0, n = d->n, s = sy;
        int it;
        if (eps < sy / E) return eps * E;
        for (it = 0; it < 200; ++it) {
            double t = pow(s / sy, 1.0 / n);
            double g = s / E + e0 * (t - 1.0) - eps;
            double dg = 1.0 / E + e0 * t / (n * s);
            double ds = g / dg;
            s -= ds;
            if (fabs(ds) <= 1e-15 * s) break;
        }
        return s;
    }
    case DG_PIECEWISE: {
        int k = 0;
        double slope;
        if (eps < d->pw_e[0]) return eps * E;
        while (k + 1 < d->npw - 1 && eps >= d->pw_e[k + 1]) ++k;
        slope = (d->pw_s[k + 1] - d->pw_s[k]) / (d->pw_e[k + 1] - d->pw_e[k]);
        return d->pw_s[k] + (eps - d->pw_e[k]) * slope;
    }
    default:
        return eps * E;
    }
}

/* ---------------------------------------------------------------- CSR ---- */

/* SparseSLAE(Mesh&, dim=2), src/SparseSLAE.h:60-196: per node the distinct
 * other nodes of its elements in first-occurrence order over the traversal
 * elem3, then elem4, then elem8 (element order, local i, local j != i). */
int orc_csr_build(int n, int c3, const int* e3, int c4, const int* e4, int c8, const int* e8,
                  int* rows, int* cols, int* adj_pos, int* adj, long long* nnz, long long* nadj) {
    int* cnt = (int*)calloc((size_t)n + 1, sizeof(int));
    int* cap_pos = (int*)calloc((size_t)n + 1, sizeof(int));
    int* links;
    int* ucnt;
    long long total = 0, tot_adj = 0;
    int e, i, jj, node;
    for (i = 0; i < 3 * c3; ++i) cnt[e3[i]] += 2;
    for (i = 0; i < 4 * c4; ++i) cnt[e4[i]] += 3;
    for (i = 0; i < 8 * c8; ++i) cnt[e8[i]] += 7;
    for (node = 0; node < n; ++node) { cap_pos[node] = (int)total; total += cnt[node]; }
    cap_pos[n] = (int)total;
    links = (int*)malloc(sizeof(int) * (size_t)(total + 1));
    ucnt = (int*)calloc((size_t)n + 1, sizeof(int));
#define ADD_LINK(nd, lk)                                                     \
    do {                                                                     \
        int _nd = (nd), _lk = (lk), _q, _dup = 0;                            \
        int* _L = links + cap_pos[_nd];                                      \
        for (_q = 0; _q < ucnt[_nd]; ++_q)                                   \
            if (_L[_q] == _lk) { _dup = 1; break; }                          \
        if (!_dup) _L[ucnt[_nd]++] = _lk;                                    \
    } while (0)
    for (e = 0; e < c3; ++e)
        for (i = 0; i < 3; ++i)
            for (jj = 0; jj < 3; ++jj)
                if (i != jj) ADD_LINK(e3[3 * e + i], e3[3 * e + jj]);
    for (e = 0; e < c4; ++e)
        for (i = 0; i < 4; ++i)
            for (jj = 0; jj < 4; ++jj)
                if (i != jj) ADD_LINK(e4[4 * e + i], e4[4 * e + jj]);
    for (e = 0; e < c8; ++e)
        for (i = 0; i < 8; ++i)
            for (jj = 0; jj < 8; ++jj)
                if (i != jj) ADD_LINK(e8[8 * e + i], e8[8 * e + jj]);
#undef ADD_LINK
    for (node = 0; node < n; ++node) tot_adj += ucnt[node];
    *nadj = tot_adj;
    *nnz = 4 * (tot_adj + n);
    if (rows) {
        long long a = 0;
        adj_pos[0] = 0;
        for (node = 0; node < n; ++node) {
            memcpy(adj + a, links + cap_pos[node], sizeof(int) * (size_t)ucnt[node]);
            a += ucnt[node];
            adj_pos[node + 1] = (int)a;
        }
        rows[0] = 0;
        for (node = 0; node < n; ++node) {
            int begin = adj_pos[node], size = adj_pos[node + 1] - begin, r, k;
            for (r = 0; r < 2; ++r)
                rows[2 * node + r + 1] = begin * 4 + (r + 1) * size * 2 + (2 * node + r + 1) * 2;
            for (r = 0; r < 2; ++r) {
                int base = rows[2 * node + r];
                cols[base] = 2 * node;
                cols[base + 1] = 2 * node + 1;
                for (k = 0; k < size; ++k) {
                    cols[base + 2 * (k + 1)] = 2 * adj[begin + k];
                    cols[base + 2 * (k + 1) + 1] = 2 * adj[begin + k] + 1;
                }
            }
        }
    }
    free(cnt);
    free(cap_pos);
    free(links);
    free(ucnt);
    return 0;
}

static int block_slot(const int* rows, const int* adj_pos, const int* adj, int ni, int nj) {
    int k;
    if (ni == nj) return rows[2 * ni];
    for (k = adj_pos[ni]; k < adj_pos[ni + 1]; ++k)
        if (adj[k] == nj) return rows[2 * ni] + 2 * (k - adj_pos[ni] + 1);
    return -1;
}

int orc_slot_map(int n, int c3, const int* e3, int c4, const int* e4, int c8, const int* e8,
                 const int* rows, const int* adj_pos, const int* adj, int* slots) {
    int e, i, j;
    (void)n;
    for (e = 0; e < c3; ++e)
        for (i = 0; i < 3; ++i)
            for (j = 0; j < 3; ++j)
                slots[9 * e + 3 * i + j] = block_slot(rows, adj_pos, adj, e3[3 * e + i], e3[3 * e + j]);
    for (e = 0; e < c4; ++e)
        for (i = 0; i < 4; ++i)
            for (j = 0; j < 4; ++j)
                slots[9 * c3 + 16 * e + 4 * i + j] = block_slot(rows, adj_pos, adj, e4[4 * e + i], e4[4 * e + j]);
    for (e = 0; e < c8; ++e)
        for (i = 0; i < 8; ++i)
            for (j = 0; j < 8; ++j)
                slots[9 * c3 + 16 * c4 + 64 * e + 8 * i + j] =
                    block_slot(rows, adj_pos, adj, e8[8 * e + i], e8[8 * e + j]);
    return 0;
}

/* ------------------------------------------------------------ elements --- */

/* calcB4, src/PlasticitySolver.cu:26-64: 2x2 Gauss, B[k] = [dN/dx; dN/dy]. */
static void calc_b4(const double* xy, const int* el, double B[4][2][4], double detJ[4]) {
    static const double gp[2] = {-0.577350269189626, 0.577350269189626};
    double x1 = xy[2 * el[0]], y1 = xy[2 * el[0] + 1], x2 = xy[2 * el[1]], y2 = xy[2 * el[1] + 1];
    double x3 = xy[2 * el[2]], y3 = xy[2 * el[2] + 1], x4 = xy[2 * el[3]], y4 = xy[2 * el[3] + 1];
    int i, j;
    for (i = 0; i < 2; ++i)
        for (j = 0; j < 2; ++j) {
            int k = i * 2 + j;
            double r = gp[i], s = gp[j], J[4], iJ[4], inv;
            J[0] = 0.25 * ((1. + s) * x1 - (1. + s) * x2 - (1. - s) * x3 + (1. - s) * x4);
            J[2] = 0.25 * ((1. + r) * x1 + (1. - r) * x2 - (1. - r) * x3 - (1. + r) * x4);
            J[1] = 0.25 * ((1. + s) * y1 - (1. + s) * y2 - (1. - s) * y3 + (1. - s) * y4);
            J[3] = 0.25 * ((1. + r) * y1 + (1. - r) * y2 - (1. - r) * y3 - (1. + r) * y4);
            detJ[k] = J[0] * J[3] - J[1] * J[2];
            inv = 1. / detJ[k];
            iJ[0] = J[3] * inv;
            iJ[1] = -J[1] * inv;
            iJ[2] = -J[2] * inv;
            iJ[3] = J[0] * inv;
            B[k][0][0] = 0.25 * ((1. + s) * iJ[0] + (1. + r) * iJ[1]);
            B[k][1][0] = 0.25 * ((1. + s) * iJ[2] + (1. + r) * iJ[3]);
            B[k][0][1] = 0.25 * ((-1. - s) * iJ[0] + (1. - r) * iJ[1]);
            B[k][1][1] = 0.25 * ((-1. - s) * iJ[2] + (1. - r) * iJ[3]);
            B[k][0][2] = 0.25 * ((-1. + s) * iJ[0] - (1. - r) * iJ[1]);
            B[k][1][2] = 0.25 * ((-1. + s) * iJ[2] - (1. - r) * iJ[3]);
            B[k][0][3] = 0.25 * ((1. - s) * iJ[0] - (1. + r) * iJ[1]);
            B[k][1][3] = 0.25 * ((1. - s) * iJ[2] - (1. + r) * iJ[3]);
        }
}

/* CST triangle (extension: the reference only declares calcB3/formKe3,
 * src/PlasticitySolver.cu:21-23,153-154). B = [dN/dx; dN/dy], area signed
 * like the reference's detJ. */
static void calc_b3(const double* xy, const int* el, double B[2][3], double* area) {
    double x1 = xy[2 * el[0]], y1 = xy[2 * el[0] + 1], x2 = xy[2 * el[1]], y2 = xy[2 * el[1] + 1];
    double x3 = xy[2 * el[2]], y3 = xy[2 * el[2] + 1];
    double twoA = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1), inv = 1.0 / twoA;
    B[0][0] = (y2 - y3) * inv; B[0][1] = (y3 - y1) * inv; B[0][2] = (y1 - y2) * inv;
    B[1][0] = (x3 - x2) * inv; B[1][1] = (x1 - x3) * inv; B[1][2] = (x2 - x1) * inv;
    *area = 0.5 * twoA;
}

/* calcB8, src/PlasticitySolver.cu:67-134: 3x3 Gauss, point k = 3 i + j at
 * (r_i, s_j). Local nodes: corners (1,1), (-1,1), (-1,-1), (1,-1), then the
 * mid-sides of the edges s = 1, r = -1, s = -1, r = 1. Serendipity shape
 * functions: corners N = (1 + r ri)(1 + s si)(r ri + s si - 1)/4, mid-sides
 * N = (1 - r^2)(1 + s si)/2 or (1 + r ri)(1 - s^2)/2. */
static const double q8_ri[8] = {1., -1., -1., 1., 0., -1., 0., 1.};
static const double q8_si[8] = {1., 1., -1., -1., 1., 0., -1., 0.};
static double q8_gp[3], q8_gw[3];

static void q8_rule(void) {
    q8_gp[0] = -sqrt(0.6); q8_gp[1] = 0.0; q8_gp[2] = sqrt(0.6);
    q8_gw[0] = 5.0 / 9.0; q8_gw[1] = 8.0 / 9.0; q8_gw[2] = 5.0 / 9.0;
}

static void q8_dshape(double r, double s, double dr[8], double ds[8]) {
    int k;
    for (k = 0; k < 8; ++k) {
        double ri = q8_ri[k], si = q8_si[k];
        if (k < 4) {
            dr[k] = 0.25 * ri * (1. + s * si) * (2. * r * ri + s * si);
            ds[k] = 0.25 * si * (1. + r * ri) * (r * ri + 2. * s * si);
        } else if (ri == 0.) {
            dr[k] = -r * (1. + s * si);
            ds[k] = 0.5 * si * (1. - r * r);
        } else {
            dr[k] = 0.5 * ri * (1. - s * s);
            ds[k] = -s * (1. + r * ri);
        }
    }
}

static void calc_b8(const double* xy, const int* el, double B[9][2][8], double detJ[9]) {
    int i, j, k;
    for (i = 0; i < 3; ++i)
        for (j = 0; j < 3; ++j) {
            int q = 3 * i + j;
            double dr[8], ds[8], xr = 0., yr = 0., xs = 0., ys = 0., inv, rx, sx, ry, sy;
            q8_dshape(q8_gp[i], q8_gp[j], dr, ds);
            for (k = 0; k < 8; ++k) {
                double x = xy[2 * el[k]], y = xy[2 * el[k] + 1];
                xr += dr[k] * x; yr += dr[k] * y;
                xs += ds[k] * x; ys += ds[k] * y;
            }
            detJ[q] = xr * ys - yr * xs;
            inv = 1. / detJ[q];
            rx = ys * inv; sx = -yr * inv; ry = -xs * inv; sy = xr * inv;
            for (k = 0; k < 8; ++k) {
                B[q][0][k] = dr[k] * rx + ds[k] * sx;
                B[q][1][k] = dr[k] * ry + ds[k] * sy;
            }
        }
}

/* formC_plainStress / formC_plainStrain, src/PlasticitySolver.cu:226-242. */
static void form_c(int strain, double E, double nu, double C[9]) {
    int i;
    double coef;
    for (i = 0; i < 9; ++i) C[i] = 0.0;
    if (!strain) {
        C[0] = C[4] = 1.; C[1] = C[3] = nu; C[8] = (1.0 - nu) * 0.5;
        coef = E / (1.0 - nu * nu);
    } else {
        C[0] = C[4] = 1.; C[1] = C[3] = nu / (1. - nu); C[8] = (1. - 2. * nu) * 0.5 / (1. - nu);
        coef = E * (1. - nu) / ((1. + nu) * (1 - 2. * nu));
    }
    for (i = 0; i < 9; ++i) C[i] *= coef;
}

#define SYM(i, j) ((i) * ((i) + 1) / 2 + (j))

/* formKe4, src/PlasticitySolver.cu:157-186 (packed lower triangle, DOF order
 * u1 v1 u2 v2 ...); the generic body also serves the CST with one point. */
static void form_ke(int nen, int npts, const double* Bp /* [npts][2][nen] */, const double* w,
                    const double C[9], double h, double* Ke) {
    int k, i, j, q;
    int nd = 2 * nen;
    for (i = 0; i < nd * (nd + 1) / 2; ++i) Ke[i] = 0.0;
    for (k = 0; k < npts; ++k) {
        const double* B0 = Bp + (size_t)k * 2 * nen;
        const double* B1 = B0 + nen;
        double dJ = w[k], BC[2][3];
        for (i = 0; i < nen; ++i) {
            int i2 = i * 2;
            for (q = 0; q < 3; ++q) {
                BC[0][q] = (B0[i] * C[0 * 3 + q] + B1[i] * C[2 * 3 + q]) * dJ;
                BC[1][q] = (B1[i] * C[1 * 3 + q] + B0[i] * C[2 * 3 + q]) * dJ;
            }
            Ke[SYM(i2, i2)] += BC[0][0] * B0[i] + BC[0][2] * B1[i];
            Ke[SYM(i2 + 1, i2)] += BC[1][0] * B0[i] + BC[1][2] * B1[i];
            Ke[SYM(i2 + 1, i2 + 1)] += BC[1][1] * B1[i] + BC[1][2] * B0[i];
            for (j = 0; j < i; ++j) {
                int j2 = j * 2;
                Ke[SYM(i2, j2)] += BC[0][0] * B0[j] + BC[0][2] * B1[j];
                Ke[SYM(i2, j2 + 1)] += BC[0][1] * B1[j] + BC[0][2] * B0[j];
                Ke[SYM(i2 + 1, j2)] += BC[1][0] * B0[j] + BC[1][2] * B1[j];
                Ke[SYM(i2 + 1, j2 + 1)] += BC[1][1] * B1[j] + BC[1][2] * B0[j];
            }
        }
    }
    for (i = 0; i < nd * (nd + 1) / 2; ++i) Ke[i] *= h;
}

/* ------------------------------------------------------------- problem --- */

typedef struct {
    mesh_t mesh;
    job_t job;
    int N, E;               /* DOF count, element count */
    int* rows; int* cols; int* adj_pos; int* adj;
    long long nnz, nadj;
    int* slots;
    double* data;
    double* B4; double* detJ4;     /* [c4][4][2][4], [c4][4] */
    double* B3; double* area3;     /* [c3][2][3], [c3] */
    double* B8; double* wJ8;       /* [c8][9][2][8], [c8][9] Gauss weight x detJ */
    double *rp, *uv;
    unsigned char* mask;
    double *exx, *eyy, *gam, *epsI, *sxx, *syy, *tau, *sigI, *tabS, *psi, *Ec, *nuc;
    double *exx_p, *eyy_p, *gam_p, *epsI_p;
    double* Cst;            /* [E][9] C used by the last assembly */
} prob_t;

static double* dalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

/* calcBs, src/PlasticitySolver.cu:1225-1235 */
static void calc_bs(prob_t* p) {
    int e;
    const mesh_t* m = &p->mesh;
#pragma omp parallel for
    for (e = 0; e < m->c4; ++e)
        calc_b4(m->xy, m->e4 + 4 * e, (double(*)[2][4])(p->B4 + 32 * (size_t)e), p->detJ4 + 4 * (size_t)e);
#pragma omp parallel for
    for (e = 0; e < m->c3; ++e)
        calc_b3(m->xy, m->e3 + 3 * e, (double(*)[3])(p->B3 + 6 * (size_t)e), p->area3 + e);
#pragma omp parallel for
    for (e = 0; e < m->c8; ++e) {
        double* wJ = p->wJ8 + 9 * (size_t)e;
        int q;
        calc_b8(m->xy, m->e8 + 8 * e, (double(*)[2][8])(p->B8 + 144 * (size_t)e), wJ);
        /* formKe8 (src/PlasticitySolver.cu:189-224) weights each point by
         * w_i w_j detJ */
        for (q = 0; q < 9; ++q) wJ[q] *= q8_gw[q / 3] * q8_gw[q % 3];
    }
}

/* fillGlobalStiffness + distribKe4/distribKe8, src/PlasticitySolver.cu:711-810:
 * Ke of every element added into CSR values through the slot map. */
static void assemble(prob_t* p) {
    const mesh_t* m = &p->mesh;
    int e, i, j;
    memset(p->data, 0, sizeof(double) * (size_t)p->nnz);
    for (e = 0; e < p->E; ++e) {
        int kind = e < m->c3 ? 3 : e < m->c3 + m->c4 ? 4 : 8, nen = kind;
        int le = kind == 3 ? e : kind == 4 ? e - m->c3 : e - m->c3 - m->c4;
        const int* el = kind == 3 ? m->e3 + 3 * le : kind == 4 ? m->e4 + 4 * le : m->e8 + 8 * le;
        const int* sl = kind == 3 ? p->slots + 9 * le
                      : kind == 4 ? p->slots + 9 * (size_t)m->c3 + 16 * (size_t)le
                                  : p->slots + 9 * (size_t)m->c3 + 16 * (size_t)m->c4 + 64 * (size_t)le;
        double C[9], Ke[136];
        form_c(p->job.plane_strain, p->Ec[e], p->nuc[e], C);
        memcpy(p->Cst + 9 * (size_t)e, C, sizeof C);
        if (kind == 3) form_ke(3, 1, p->B3 + 6 * (size_t)le, p->area3 + le, C, p->job.h, Ke);
        else if (kind == 4) form_ke(4, 4, p->B4 + 32 * (size_t)le, p->detJ4 + 4 * (size_t)le, C, p->job.h, Ke);
        else form_ke(8, 9, p->B8 + 144 * (size_t)le, p->wJ8 + 9 * (size_t)le, C, p->job.h, Ke);
        for (i = 0; i < nen; ++i) {
            int ni = el[i], Li = p->rows[2 * ni + 1] - p->rows[2 * ni];
            for (j = 0; j < nen; ++j) {
                int s = sl[i * nen + j];
                int a = 2 * i, b = 2 * j;
                /* K(2ni+r, 2nj+c) = Ke(a+r, b+c), read from the packed lower triangle
                 * exactly as distribKe4 does (the upper part mirrors the lower). */
                double k00, k01, k10, k11;
                if (i == j) {
                    k00 = Ke[SYM(a, a)]; k10 = Ke[SYM(a + 1, a)]; k01 = k10; k11 = Ke[SYM(a + 1, a + 1)];
                } else if (i > j) {
                    k00 = Ke[SYM(a, b)]; k01 = Ke[SYM(a, b + 1)]; k10 = Ke[SYM(a + 1, b)]; k11 = Ke[SYM(a + 1, b + 1)];
                } else {
                    k00 = Ke[SYM(b, a)]; k01 = Ke[SYM(b + 1, a)]; k10 = Ke[SYM(b, a + 1)]; k11 = Ke[SYM(b + 1, a + 1)];
                }
                p->data[s] += k00;
                p->data[s + 1] += k01;
                p->data[s + Li] += k10;
                p->data[s + Li + 1] += k11;
            }
        }
    }
}

static int find_node(const mesh_t* m, double x, double y) {
    int i;
    for (i = 0; i < m->n_nodes; ++i) {
        double dx = m->xy[2 * i] - x, dy = m->xy[2 * i + 1] - y;
        if (sqrt(dx * dx + dy * dy) < 1e-14) return i;
    }
    return -1;
}

/* The quadratic-edge branch of initConditions, src/PlasticitySolver.cu:822-865:
 * a border traction over corner a, mid-side c, corner d gives the consistent
 * nodal forces f_a L1/3, f_c (4/3)(L1 + L2)/2, f_d L2/3 (L1 = |ac|, L2 = |cd|),
 * times h. A normal/tangential traction turns with each half edge; the
 * mid-side node takes the mean of the two frames. */
static void quad_edge_force(prob_t* p, int b, int na, int nc, int nd) {
    const mesh_t* m = &p->mesh;
    const job_t* j = &p->job;
    double xa = m->xy[2 * na], ya = m->xy[2 * na + 1], xc = m->xy[2 * nc], yc = m->xy[2 * nc + 1];
    double xd = m->xy[2 * nd], yd = m->xy[2 * nd + 1];
    double hx1 = 0.5 * (xa - xc), hy1 = 0.5 * (ya - yc), hx2 = 0.5 * (xc - xd), hy2 = 0.5 * (yc - yd);
    double dl1 = sqrt(hx1 * hx1 + hy1 * hy1), dl2 = sqrt(hx2 * hx2 + hy2 * hy2);
    double fx = j->force_v[b][0], fy = j->force_v[b][1];
    double f1x = fx, f1y = fy, f2x = fx, f2y = fy, f3x = fx, f3y = fy, R[6];
    int a;
    if (j->force_norm[b]) {
        double t1x = xc - xa, t1y = yc - ya, t2x = xd - xc, t2y = yd - yc, tn, n1x, n1y, n2x, n2y, nn;
        tn = sqrt(t1x * t1x + t1y * t1y); t1x = t1x * (1. / tn); t1y = t1y * (1. / tn);
        n1x = t1y; n1y = -t1x; nn = sqrt(n1x * n1x + n1y * n1y); n1x = n1x * (1. / nn); n1y = n1y * (1. / nn);
        tn = sqrt(t2x * t2x + t2y * t2y); t2x = t2x * (1. / tn); t2y = t2y * (1. / tn);
        n2x = t2y; n2y = -t2x; nn = sqrt(n2x * n2x + n2y * n2y); n2x = n2x * (1. / nn); n2y = n2y * (1. / nn);
        f1x = n1x * fx + t1x * fy; f1y = n1y * fx + t1y * fy;
        f2x = 0.5 * ((n1x + n2x) * fx + (t1x + t2x) * fy);
        f2y = 0.5 * ((n1y + n2y) * fx + (t1y + t2y) * fy);
        f3x = n2x * fx + t2x * fy; f3y = n2y * fx + t2y * fy;
    }
    R[0] = f1x / 3.; R[1] = f1y / 3.;
    R[2] = f2x * 4. / 3.; R[3] = f2y * 4. / 3.;
    R[4] = f3x / 3.; R[5] = f3y / 3.;
    for (a = 0; a < 2; ++a) {
        R[a] *= j->h * dl1 * 2.;
        R[2 + a] *= j->h * (dl1 + dl2);
        R[4 + a] *= j->h * dl2 * 2.;
    }
    p->rp[2 * na] += R[0]; p->rp[2 * na + 1] += R[1];
    p->rp[2 * nc] += R[2]; p->rp[2 * nc + 1] += R[3];
    p->rp[2 * nd] += R[4]; p->rp[2 * nd + 1] += R[5];
}

/* Mesh::elemSpace8 (src/Mesh.cuh:269-278): area of the polygon through the
 * corners and mid-side nodes. */
static double elem_space8(const mesh_t* m, const int* el) {
    double s1 = 0., s2 = 0.;
    int i;
    for (i = 0; i < 3; ++i) {
        s1 += m->xy[2 * el[i]] * m->xy[2 * el[i + 4] + 1] + m->xy[2 * el[i + 4]] * m->xy[2 * el[i + 1] + 1];
        s2 += m->xy[2 * el[i] + 1] * m->xy[2 * el[i + 4]] + m->xy[2 * el[i + 4] + 1] * m->xy[2 * el[i + 1]];
    }
    s1 += m->xy[2 * el[3]] * m->xy[2 * el[7] + 1] + m->xy[2 * el[7]] * m->xy[2 * el[0] + 1];
    s2 += m->xy[2 * el[3] + 1] * m->xy[2 * el[7]] + m->xy[2 * el[7] + 1] * m->xy[2 * el[0]];
    return fabs(s1 - s2) * 0.5;
}

/* initConditions(SparseSLAE&), src/PlasticitySolver.cu:812-1005, for
 * constant-valued loads (linear and quadratic border segments). */
static void init_conditions(prob_t* p) {
    const mesh_t* m = &p->mesh;
    const job_t* j = &p->job;
    int b, i, a;
    for (i = 0; i < p->N; ++i) { p->rp[i] = 0.0; p->mask[i] = 1; p->uv[i] = 0.0; }
    for (b = 0; b < MAXB && b < m->n_borders; ++b) {
        const int* bd;
        if (!j->force_set[b]) continue;
        bd = m->borders[b];
        for (i = 1; i < m->border_len[b]; ++i) {
            double x1, y1, x2, y2, hd1, hd2;
            if (m->sec[bd[i]] && i + 1 < m->border_len[b]) {
                quad_edge_force(p, b, bd[i - 1], bd[i], bd[i + 1]);
                ++i;
                continue;
            }
            x1 = m->xy[2 * bd[i - 1]]; y1 = m->xy[2 * bd[i - 1] + 1];
            x2 = m->xy[2 * bd[i]]; y2 = m->xy[2 * bd[i] + 1];
            hd1 = 0.5 * (x1 - x2); hd2 = 0.5 * (y1 - y2);
            double dl = sqrt(hd1 * hd1 + hd2 * hd2);
            double f1x = j->force_v[b][0], f1y = j->force_v[b][1], f2x = f1x, f2y = f1y;
            double R[4];
            if (j->force_norm[b]) {
                double tx = x2 - x1, ty = y2 - y1, tn = sqrt(tx * tx + ty * ty), nx, ny, nn;
                tx = tx * (1. / tn); ty = ty * (1. / tn);
                nx = ty; ny = -tx;
                nn = sqrt(nx * nx + ny * ny);
                nx = nx * (1. / nn); ny = ny * (1. / nn);
                f1x = nx * j->force_v[b][0] + tx * j->force_v[b][1];
                f1y = ny * j->force_v[b][0] + ty * j->force_v[b][1];
                f2x = f1x; f2y = f1y;
            }
            R[0] = f1x; R[1] = f1y; R[2] = f2x; R[3] = f2y;
            for (a = 0; a < 4; ++a) R[a] *= j->h * dl;
            p->rp[2 * bd[i - 1]] += R[0];
            p->rp[2 * bd[i - 1] + 1] += R[1];
            p->rp[2 * bd[i]] += R[2];
            p->rp[2 * bd[i] + 1] += R[3];
        }
    }
    if (j->grav_set) {
        int e;
        for (e = 0; e < m->c4; ++e) {
            const int* el = m->e4 + 4 * e;
            double s1 = 0, s2 = 0, area, coef;
            for (i = 1; i < 4; ++i) {
                s1 += m->xy[2 * el[i - 1]] * m->xy[2 * el[i] + 1];
                s2 += m->xy[2 * el[i - 1] + 1] * m->xy[2 * el[i]];
            }
            s1 += m->xy[2 * el[3]] * m->xy[2 * el[0] + 1];
            s2 += m->xy[2 * el[3] + 1] * m->xy[2 * el[0]];
            area = fabs(s1 - s2) * 0.5;
            coef = 0.25 * p->job.rho * j->h * area;
            for (i = 0; i < 4; ++i) {
                p->rp[2 * el[i]] += coef * j->grav[0];
                p->rp[2 * el[i] + 1] += coef * j->grav[1];
            }
        }
        /* 8-node elements, src/PlasticitySolver.cu:911-929: -1/12 of the
         * element's load to each corner, 1/3 to each mid-side node */
        for (e = 0; e < m->c8; ++e) {
            const int* el = m->e8 + 8 * e;
            double space = elem_space8(m, el);
            double coef1 = -p->job.rho * j->h * space / 12., coef2 = p->job.rho * j->h * space / 3.;
            for (i = 0; i < 8; ++i) {
                double c = i < 4 ? coef1 : coef2;
                p->rp[2 * el[i]] += c * j->grav[0];
                p->rp[2 * el[i] + 1] += c * j->grav[1];
            }
        }
    }
    for (b = 0; b < MAXB && b < m->n_borders; ++b) {
        const int* bd;
        int len, end, mid;
        if (!j->displ_set[b]) continue;
        bd = m->borders[b];
        len = m->border_len[b];
        end = len - (bd[0] == bd[len - 1] ? 1 : 0);
        mid = bd[len / 2];
        if (j->displ_midx[b]) { p->mask[2 * mid] = 0; p->uv[2 * mid] = j->displ_v[b][0]; }
        else for (i = 0; i < end; ++i) { p->mask[2 * bd[i]] = 0; p->uv[2 * bd[i]] = j->displ_v[b][0]; }
        if (j->displ_midy[b]) { p->mask[2 * mid + 1] = 0; p->uv[2 * mid + 1] = j->displ_v[b][1]; }
        else for (i = 0; i < end; ++i) { p->mask[2 * bd[i] + 1] = 0; p->uv[2 * bd[i] + 1] = j->displ_v[b][1]; }
    }
    for (a = 0; a < j->n_axis; ++a)
        for (i = 0; i < m->n_nodes; ++i) {
            if (j->axis_vert[a]) { if (fabs(m->xy[2 * i] - j->axis_coord[a]) < 1e-14) p->mask[2 * i] = 0; }
            else if (fabs(m->xy[2 * i + 1] - j->axis_coord[a]) < 1e-14) p->mask[2 * i + 1] = 0;
        }
    for (b = 0; b < MAXB && b < m->n_borders; ++b) {
        const int* bd;
        int len, end;
        if (!j->fixb_set[b]) continue;
        bd = m->borders[b];
        len = m->border_len[b];
        end = len - (bd[0] == bd[len - 1] ? 1 : 0);
        for (i = 0; i < end; ++i) p->mask[2 * bd[i] + (j->fixb_vert[b] ? 0 : 1)] = 0;
    }
    for (a = 0; a < j->n_fpt; ++a) {
        int nd = find_node(m, j->fpt[a][0], j->fpt[a][1]);
        if (nd >= 0) { p->rp[2 * nd] += j->fpt[a][2]; p->rp[2 * nd + 1] += j->fpt[a][3]; }
    }
    for (a = 0; a < j->n_dpt; ++a) {
        int nd = find_node(m, j->dpt[a][0], j->dpt[a][1]);
        if (nd >= 0) {
            p->uv[2 * nd] = j->dpt[a][2]; p->uv[2 * nd + 1] = j->dpt[a][3];
            p->mask[2 * nd] = 0; p->mask[2 * nd + 1] = 0;
        }
    }
    for (a = 0; a < j->n_fixdof; ++a) p->mask[j->fixdof[a]] = 0;
}

/* ConjGradSolver::solve, src/ConjGradSolver.h:25-41 (normB) and :52-101. */
static long long cg_solve(prob_t* p, double* x, const double* b, double eps) {
    int N = p->N, i;
    double *r = dalloc((size_t)N), *z = dalloc((size_t)N), *Az = dalloc((size_t)N);
    double normB = 0.0, rr = 0.0;
    long long it = 0;
    for (i = 0; i < N; ++i) normB += b[i] * b[i];
    normB = 1.0 / normB;
#pragma omp parallel for reduction(+ : rr)
    for (i = 0; i < N; ++i) {
        double s = 0.0, rk;
        int q;
        for (q = p->rows[i]; q < p->rows[i + 1]; ++q) s += p->data[q] * x[p->cols[q]];
        rk = p->mask[i] * (b[i] - s);
        z[i] = r[i] = rk;
        rr += rk * rk;
    }
    if (rr > 0.0) {
        double rnext;
        do {
            double Azz = 0.0, alpha, beta;
            rnext = 0.0;
#pragma omp parallel for reduction(+ : Azz)
            for (i = 0; i < N; ++i) {
                double s = 0.0;
                int q;
                for (q = p->rows[i]; q < p->rows[i + 1]; ++q) s += p->data[q] * z[p->cols[q]];
                Az[i] = s;
                Azz += s * z[i];
            }
            alpha = rr / Azz;
#pragma omp parallel for reduction(+ : rnext)
            for (i = 0; i < N; ++i) {
                double rk;
                x[i] = x[i] + alpha * z[i];
                rk = r[i] - p->mask[i] * alpha * Az[i];
                r[i] = rk;
                rnext += rk * rk;
            }
            beta = rnext / rr;
#pragma omp parallel for
            for (i = 0; i < N; ++i) z[i] = r[i] + beta * z[i];
            rr = rnext;
            ++it;
            if (!(rnext == rnext) || it > 10000000) break;
        } while (rnext * normB > eps * eps);
    }
    free(r);
    free(z);
    free(Az);
    return it;
}

/* updateParameters, src/PlasticitySolver.cu:1249-1335 (Q4 and Q8) plus the CST. */
static void update_parameters(prob_t* p) {
    const mesh_t* m = &p->mesh;
    const double E0 = p->job.E, nu0 = p->job.nu;
    int e;
#pragma omp parallel for
    for (e = 0; e < p->E; ++e) {
        const double* C = p->Cst + 9 * (size_t)e;
        if (e < m->c3) {
            const int* el = m->e3 + 3 * e;
            const double* B = p->B3 + 6 * (size_t)e;
            double u1 = p->uv[2 * el[0]], v1 = p->uv[2 * el[0] + 1], u2 = p->uv[2 * el[1]], v2 = p->uv[2 * el[1] + 1];
            double u3 = p->uv[2 * el[2]], v3 = p->uv[2 * el[2] + 1];
            p->exx[e] = u1 * B[0] + u2 * B[1] + u3 * B[2];
            p->eyy[e] = v1 * B[3] + v2 * B[4] + v3 * B[5];
            p->gam[e] = u1 * B[3] + u2 * B[4] + u3 * B[5] + v1 * B[0] + v2 * B[1] + v3 * B[2];
        } else if (e >= m->c3 + m->c4) {
            /* src/PlasticitySolver.cu:1280-1305: Gauss-weighted mean over the
             * reference square, (1/4) sum_ij w_i w_j eps(r_i, s_j) */
            int le = e - m->c3 - m->c4, a, q;
            const int* el = m->e8 + 8 * le;
            double u[8], v[8], ex = 0., ey = 0., g = 0.;
            for (a = 0; a < 8; ++a) { u[a] = p->uv[2 * el[a]]; v[a] = p->uv[2 * el[a] + 1]; }
            for (q = 0; q < 9; ++q) {
                const double* B = p->B8 + 144 * (size_t)le + 16 * q; /* B(r,c) = B[r*8+c] */
                double exl = 0., eyl = 0., gl = 0., w = q8_gw[q / 3] * q8_gw[q % 3];
                for (a = 0; a < 8; ++a) {
                    exl += u[a] * B[a];
                    eyl += v[a] * B[8 + a];
                    gl += u[a] * B[8 + a] + v[a] * B[a];
                }
                ex += exl * w; ey += eyl * w; g += gl * w;
            }
            p->exx[e] = ex * 0.25;
            p->eyy[e] = ey * 0.25;
            p->gam[e] = g * 0.25;
        } else {
            int le = e - m->c3, k;
            const int* el = m->e4 + 4 * le;
            double u1 = p->uv[2 * el[0]], v1 = p->uv[2 * el[0] + 1], u2 = p->uv[2 * el[1]], v2 = p->uv[2 * el[1] + 1];
            double u3 = p->uv[2 * el[2]], v3 = p->uv[2 * el[2] + 1], u4 = p->uv[2 * el[3]], v4 = p->uv[2 * el[3] + 1];
            double ex = 0., ey = 0., g = 0.;
            for (k = 0; k < 4; ++k) {
                const double* B = p->B4 + 32 * (size_t)le + 8 * k; /* B(r,c) = B[r*4+c] */
                ex += u1 * B[0] + u2 * B[1] + u3 * B[2] + u4 * B[3];
                ey += v1 * B[4] + v2 * B[5] + v3 * B[6] + v4 * B[7];
                g += u1 * B[4] + u2 * B[5] + u3 * B[6] + u4 * B[7] + v1 * B[0] + v2 * B[1] + v3 * B[2] + v4 * B[3];
            }
            p->exx[e] = ex * 0.25;
            p->eyy[e] = ey * 0.25;
            p->gam[e] = g * 0.25;
        }
        {
            double sx = C[0] * p->exx[e] + C[1] * p->eyy[e];
            double sy = C[1] * p->exx[e] + C[4] * p->eyy[e];
            double t = C[8] * p->gam[e];
            double sI, eI, tab, ps;
            p->sxx[e] = sx; p->syy[e] = sy; p->tau[e] = t;
            sI = sqrt(0.5 * (sx * sx + sy * sy + (sx - sy) * (sx - sy) + 6. * (t * t)));
            eI = sI / p->Ec[e];
            tab = diagram_f(&p->job.dg, eI);
            ps = E0 * eI / tab;
            p->sigI[e] = sI; p->epsI[e] = eI; p->tabS[e] = tab; p->psi[e] = ps;
            p->Ec[e] = E0 / ps;
            p->nuc[e] = 0.5 * (1. - (1. - 2. * nu0) / ps);
        }
    }
}

/* exitCondition, src/PlasticitySolver.cuh:154-163 */
static double exit_condition(const prob_t* p) {
    double norm = 0.0, den = 0.0;
    int e;
    for (e = 0; e < p->E; ++e) {
        double d = p->sigI[e] - p->tabS[e];
        norm += d * d;
        den += p->tabS[e] * p->tabS[e];
    }
    return sqrt(norm / den);
}

/* calcPlastDeform, src/PlasticitySolver.cu:1356-1368 */
static void plast_deform(prob_t* p) {
    double E0 = p->job.E, nu0 = p->job.nu, G = E0 * 0.5 / (1. + nu0);
    int e;
    for (e = 0; e < p->E; ++e) {
        double Gc = p->Ec[e] * 0.5 / (1. + p->nuc[e]);
        p->exx_p[e] = (1. / p->Ec[e] - 1. / E0) * p->sxx[e];
        p->eyy_p[e] = (1. / p->Ec[e] - 1. / E0) * p->syy[e];
        p->gam_p[e] = (1. / Gc - 1. / G) * p->tau[e];
        p->epsI_p[e] = sqrt(2.) / 3. * sqrt((p->exx_p[e] - p->eyy_p[e]) * (p->exx_p[e] - p->eyy_p[e]) +
                                            6. * (p->gam_p[e] * p->gam_p[e]));
        p->psi[e] = E0 / p->Ec[e];
    }
}

/* deformEnergy, src/PlasticitySolver.cuh:415-445. Q4 and CST elements on the
 * plastic branch integrate the diagram; Q8 elements always take the secant
 * energy eps_i sig_i / 2 (the reference's Q8 loop has no plastic branch). */
static double deform_energy(const prob_t* p) {
    const mesh_t* m = &p->mesh;
    const diagram_t* d = &p->job.dg;
    double energy = 0.0, sT = d->sigmaT, E0 = p->job.E;
    int e, i, k;
    for (e = 0; e < p->E; ++e) {
        double area, vol;
        if (e >= m->c3 + m->c4) {
            energy += p->epsI[e] * p->sigI[e] * 0.5 * (p->job.h * elem_space8(m, m->e8 + 8 * (e - m->c3 - m->c4)));
            continue;
        }
        if (e < m->c3) area = fabs(p->area3[e]);
        else {
            const int* el = m->e4 + 4 * (e - m->c3);
            double s1 = 0., s2 = 0.;
            for (i = 1; i < 4; ++i) {
                s1 += m->xy[2 * el[i - 1]] * m->xy[2 * el[i] + 1];
                s2 += m->xy[2 * el[i - 1] + 1] * m->xy[2 * el[i]];
            }
            s1 += m->xy[2 * el[3]] * m->xy[2 * el[0] + 1];
            s2 += m->xy[2 * el[3] + 1] * m->xy[2 * el[0]];
            area = fabs(s1 - s2) * 0.5;
        }
        vol = p->job.h * area;
        if (d->kind != DG_NONE && p->sigI[e] > sT) {
            double ET = sT / E0, heps = (p->epsI[e] - ET) * 0.01;
            energy += sT * ET * 0.5 * vol;
            for (k = 0; k < 100; ++k)
                energy += heps * 0.5 * (diagram_f(d, ET + heps * k) + diagram_f(d, ET + heps * (k + 1))) * vol;
        } else
            energy += p->epsI[e] * p->sigI[e] * 0.5 * vol;
    }
    return energy;
}

/* ------------------------------------------------------------ driver ----- */

int orc_run_job(const char* job_path, const char* out_path) {
    prob_t P;
    prob_t* p = &P;
    FILE* out;
    int e, i, lev, N;
    long long cg_total = 0;
    int* outer_lv;
    int* cg_lv;
    double* err_lv;
    double t0, rpfull_norm = 0.0;
    double *rp_full, *uv_full;
    memset(p, 0, sizeof *p);
    if (parse_job(job_path, &p->job) != 0) return 1;
    if (load_mesh(p->job.mesh_path, &p->mesh) != 0) return 2;
    if (p->job.dg.kind == DG_NONE) { p->job.dg.kind = DG_LINEAR; p->job.dg.E = p->job.E; p->job.dg.sigmaT = 1e300; p->job.dg.K_T = p->job.E; }
    p->job.dg.E = p->job.E;
    N = p->N = 2 * p->mesh.n_nodes;
    p->E = p->mesh.c3 + p->mesh.c4 + p->mesh.c8;
    q8_rule();
    out = cpbin_open_write(out_path);
    if (!out) return 3;

    orc_csr_build(p->mesh.n_nodes, p->mesh.c3, p->mesh.e3, p->mesh.c4, p->mesh.e4, p->mesh.c8, p->mesh.e8, NULL, NULL,
                  NULL, NULL, &p->nnz, &p->nadj);
    p->rows = (int*)malloc(sizeof(int) * (size_t)(N + 1));
    p->cols = (int*)malloc(sizeof(int) * (size_t)p->nnz);
    p->adj_pos = (int*)malloc(sizeof(int) * (size_t)(p->mesh.n_nodes + 1));
    p->adj = (int*)malloc(sizeof(int) * (size_t)(p->nadj + 1));
    orc_csr_build(p->mesh.n_nodes, p->mesh.c3, p->mesh.e3, p->mesh.c4, p->mesh.e4, p->mesh.c8, p->mesh.e8, p->rows,
                  p->cols, p->adj_pos, p->adj, &p->nnz, &p->nadj);
    if (!strcmp(p->job.mode, "csr") || p->job.dump_csr) {
        size_t ns = 9 * (size_t)p->mesh.c3 + 16 * (size_t)p->mesh.c4 + 64 * (size_t)p->mesh.c8;
        int* sl = (int*)malloc(sizeof(int) * (ns + 1));
        orc_slot_map(p->mesh.n_nodes, p->mesh.c3, p->mesh.e3, p->mesh.c4, p->mesh.e4, p->mesh.c8, p->mesh.e8, p->rows,
                     p->adj_pos, p->adj, sl);
        cpbin_put(out, "rows", 'i', N + 1, p->rows);
        cpbin_put(out, "cols", 'i', p->nnz, p->cols);
        cpbin_put(out, "adj_pos", 'i', p->mesh.n_nodes + 1, p->adj_pos);
        cpbin_put(out, "adj", 'i', p->nadj, p->adj);
        cpbin_put(out, "slots", 'i', (int64_t)ns, sl);
        free(sl);
        if (!strcmp(p->job.mode, "csr")) goto done;
    }
    p->slots = (int*)malloc(sizeof(int) * (9 * (size_t)p->mesh.c3 + 16 * (size_t)p->mesh.c4 + 64 * (size_t)p->mesh.c8 + 1));
    orc_slot_map(p->mesh.n_nodes, p->mesh.c3, p->mesh.e3, p->mesh.c4, p->mesh.e4, p->mesh.c8, p->mesh.e8, p->rows,
                 p->adj_pos, p->adj, p->slots);
    p->data = dalloc((size_t)p->nnz);
    p->B4 = dalloc(32 * (size_t)p->mesh.c4);
    p->detJ4 = dalloc(4 * (size_t)p->mesh.c4);
    p->B3 = dalloc(6 * (size_t)p->mesh.c3);
    p->area3 = dalloc((size_t)p->mesh.c3);
    p->B8 = dalloc(144 * (size_t)p->mesh.c8);
    p->wJ8 = dalloc(9 * (size_t)p->mesh.c8);
    p->rp = dalloc((size_t)N); p->uv = dalloc((size_t)N);
    p->mask = (unsigned char*)calloc((size_t)N, 1);
    p->exx = dalloc(p->E); p->eyy = dalloc(p->E); p->gam = dalloc(p->E); p->epsI = dalloc(p->E);
    p->sxx = dalloc(p->E); p->syy = dalloc(p->E); p->tau = dalloc(p->E); p->sigI = dalloc(p->E);
    p->tabS = dalloc(p->E); p->psi = dalloc(p->E); p->Ec = dalloc(p->E); p->nuc = dalloc(p->E);
    p->exx_p = dalloc(p->E); p->eyy_p = dalloc(p->E); p->gam_p = dalloc(p->E); p->epsI_p = dalloc(p->E);
    p->Cst = dalloc(9 * (size_t)p->E);
    for (e = 0; e < p->E; ++e) { p->psi[e] = 1.0; p->Ec[e] = p->job.E; p->nuc[e] = p->job.nu; }

    t0 = omp_get_wtime();
    calc_bs(p);
    init_conditions(p);
    cpbin_put(out, "rp", 'd', N, p->rp);
    cpbin_put(out, "mask", 'b', N, p->mask);
    rp_full = dalloc((size_t)N);
    uv_full = dalloc((size_t)N);
    memcpy(rp_full, p->rp, sizeof(double) * (size_t)N);
    memcpy(uv_full, p->uv, sizeof(double) * (size_t)N);
    for (i = 0; i < N; ++i) rpfull_norm += rp_full[i] * rp_full[i];
    outer_lv = (int*)calloc((size_t)p->job.levels + 1, sizeof(int));
    cg_lv = (int*)calloc((size_t)p->job.levels + 1, sizeof(int));
    err_lv = dalloc((size_t)p->job.levels + 1);
    {
        int elastic = !strcmp(p->job.mode, "elastic");
        double cg_eps = p->job.cg_eps, outer_eps = p->job.outer_eps;
        int max_outer = p->job.max_outer;
        if (!strcmp(p->job.mode, "solve")) { cg_eps = 1e-7; outer_eps = 1e-5; max_outer = 50; }
        for (lev = 1; lev <= p->job.levels; ++lev) {
            double lam = (double)lev / p->job.levels, relErr = 0.0;
            int iter = 0;
            long long cg_lev = 0;
            for (i = 0; i < N; ++i) p->rp[i] = lam * rp_full[i];
            for (i = 0; i < N; ++i) if (!p->mask[i]) p->uv[i] = lam * uv_full[i];
            do {
                assemble(p);
                if (p->job.dump_k && lev == 1 && iter == 0) cpbin_put(out, "k_data", 'd', p->nnz, p->data);
                cg_lev += cg_solve(p, p->uv, p->rp, cg_eps);
                update_parameters(p);
                relErr = exit_condition(p);
                ++iter;
                if (elastic) break;
            } while (relErr > outer_eps && iter < max_outer);
            outer_lv[lev - 1] = iter;
            cg_lv[lev - 1] = (int)cg_lev;
            err_lv[lev - 1] = relErr;
            cg_total += cg_lev;
        }
    }
    plast_deform(p);
    {
        double wall = omp_get_wtime() - t0;
        cpbin_put(out, "uv", 'd', N, p->uv);
        cpbin_put(out, "exx", 'd', p->E, p->exx);
        cpbin_put(out, "eyy", 'd', p->E, p->eyy);
        cpbin_put(out, "gamma", 'd', p->E, p->gam);
        cpbin_put(out, "eps_i", 'd', p->E, p->epsI);
        cpbin_put(out, "sxx", 'd', p->E, p->sxx);
        cpbin_put(out, "syy", 'd', p->E, p->syy);
        cpbin_put(out, "tau", 'd', p->E, p->tau);
        cpbin_put(out, "sig_i", 'd', p->E, p->sigI);
        cpbin_put(out, "table_s", 'd', p->E, p->tabS);
        cpbin_put(out, "psi", 'd', p->E, p->psi);
        cpbin_put(out, "E_c", 'd', p->E, p->Ec);
        cpbin_put(out, "nu_c", 'd', p->E, p->nuc);
        cpbin_put(out, "exx_p", 'd', p->E, p->exx_p);
        cpbin_put(out, "eyy_p", 'd', p->E, p->eyy_p);
        cpbin_put(out, "gamma_p", 'd', p->E, p->gam_p);
        cpbin_put(out, "eps_p_i", 'd', p->E, p->epsI_p);
        cpbin_put(out, "outer_per_level", 'i', p->job.levels, outer_lv);
        cpbin_put(out, "cg_per_level", 'i', p->job.levels, cg_lv);
        cpbin_put(out, "err_per_level", 'd', p->job.levels, err_lv);
        cpbin_put_d(out, "wall_seconds", wall);
        cpbin_put_d(out, "energy", deform_energy(p));
        cpbin_put_d(out, "cg_total", (double)cg_total);
        cpbin_put_i(out, "threads", omp_get_max_threads());
    }
    free(rp_full); free(uv_full); free(outer_lv); free(cg_lv); free(err_lv);
    free(p->slots); free(p->data); free(p->B4); free(p->detJ4); free(p->B3); free(p->area3);
    free(p->B8); free(p->wJ8);
    free(p->rp); free(p->uv); free(p->mask);
    free(p->exx); free(p->eyy); free(p->gam); free(p->epsI); free(p->sxx); free(p->syy); free(p->tau);
    free(p->sigI); free(p->tabS); free(p->psi); free(p->Ec); free(p->nuc);
    free(p->exx_p); free(p->eyy_p); free(p->gam_p); free(p->epsI_p); free(p->Cst);
done:
    fclose(out);
    free(p->rows); free(p->cols); free(p->adj_pos); free(p->adj);
    free_mesh(&p->mesh);
    return 0;
}
