/*
 * ref_harness.cu -- drives the UNMODIFIED reference implementation (its CPU
 * path) so that the oracle restatement and the golden fixtures can be pinned
 * to it. TEST INFRASTRUCTURE ONLY: built by oracle/Makefile from the reference
 * sources where they lie, into oracle/_ref/cpref; never linked into the product.
 *
 * The reference has no API below its PlasticitySolver class, so this driver
 * reaches its private phases (calcBs, initConditions, fillGlobalStiffness,
 * ConjGradSolver::solve, updateParameters, exitCondition, calcPlastDeform) by
 * re-declaring access after the standard headers are in. That lets a job run
 * with tight tolerances, per-increment load levels and injected hardening
 * diagrams, exactly as the solve loop of PlasticitySolver::solveCPU
 * (src/PlasticitySolver.cu:325-366) would, but with the caller's epsilons.
 *
 * Usage: cpref <job.txt> <out.bin>
 * Job lines (one per line, '#' comments):
 *   mode mesh|csr|loads|solve|phases|elastic   (loads: initConditions only)
 *   mesh hole x1 x2 y1 y2 R N1 N2 order      (Mesh::genRectWithHole, src/Mesh.cu:112)
 *   mesh ring a b Nphi Nr order              (Mesh::genRing, src/Mesh.cu:249)
 *   mesh rect x1 x2 y1 y2 N1 N2 order        (Mesh::genRectangle, src/Mesh.cu:17)
 *   mesh file path.bin                       (arrays written by the test helpers)
 *   renum dx dy | smooth_ring borderN        (Mesh::renumByDirection / smoothRing after the mesh is made)
 *   mesh inp path.inp                        (Mesh::loadFromFile, src/Mesh.cu:725)
 *   material E nu h
 *   diagram linear E sigmaT K_T              (Material::setLinearPlast)
 *   diagram power E sigmaT A m               (Material::setPowerPlast)
 *   diagram hollomon E sigmaY eps0 n         (injected: sigma = sY (1 + eps_p/eps0)^n)
 *   diagram piecewise E n e1 s1 ... en sn    (injected: elastic to (e1,s1), then linear)
 *   plane stress|strain
 *   force B fx fy normal | fixborderhor B | fixbordervert B | fixvertaxis x
 *   fixhoraxis y | fixpoint x y | displ B ux uy midx midy | forcepoint x y fx fy
 *   displpoint x y ux uy | gravity g dx dy | fixdof d (extra Dirichlet DOF, value 0)
 *   cg_eps e | outer_eps e | max_outer n | levels k (load factors k/n for k=1..n)
 *   dump_k 1 | dump_csr 1
 *   prefix_outer n                           (phases / phases_csr: stop after n outer iterations in all)
 *
 * mode phases_csr is mode phases with one change, for meshes whose band
 * matrix does not fit in host memory (the reference's fillGlobalStiffness
 * assembles into a StripSLAE of N x (2W + 1) doubles, W about 4 n_r on the
 * ring-numbered O-grid: about 138 GB for the 1024 x 1024 plate): each
 * element's C and Ke come from the reference's own formC / formKe4, and Ke
 * is added straight into the CSR values through a table of CSR positions
 * built once from the reference's SparseSLAE. Everything else (calcBs,
 * initConditions, ConjGradSolver::solve, updateParameters, exitCondition)
 * is the reference's. 4-node elements only.
 */
#include <unistd.h>
#include <csetjmp>
#include <csignal>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <sstream>
#include <fstream>
#include <iostream>
#include <functional>
#include <map>
#include <list>
#include <filesystem>
#include <omp.h>
#include <cuda_runtime.h>
#include <nvfunctional>

#define private public
#define protected public
#ifdef CPREF_SOLVER_SOURCE
/* the phases_csr build (cpref_csr): the solver's source in this unit, so
 * that its file-local element routines (formKe4) can be called; linked
 * without the separately compiled PlasticitySolver object */
#include "PlasticitySolver.cu"
#else
#include "PlasticitySolver.cuh"
#endif
#include "ConjGradSolver.h"
#undef private
#undef protected

#include "cpbin.h"

/* ---- injected diagrams (parameters live in globals: Material::host_f is a
 *      plain 6-argument function pointer, src/Material.cuh:17-18) ---------- */
static double g_hol_sy, g_hol_eps0, g_hol_n;
static int g_pw_n;
static double g_pw_e[16], g_pw_s[16];

static double hollomonDiagram(double eps, double E, double, double, double, double) {
    double sy = g_hol_sy, e0 = g_hol_eps0, n = g_hol_n;
    if (eps < sy / E) return eps * E;
    /* Newton on g(s) = s/E + e0((s/sy)^(1/n) - 1) - eps, from s = sy. */
    double s = sy;
    for (int it = 0; it < 200; ++it) {
        double t = pow(s / sy, 1.0 / n);
        double g = s / E + e0 * (t - 1.0) - eps;
        double dg = 1.0 / E + e0 * t / (n * s);
        double ds = g / dg;
        s -= ds;
        if (fabs(ds) <= 1e-15 * s) break;
    }
    return s;
}

static double piecewiseDiagram(double eps, double E, double, double, double, double) {
    if (eps < g_pw_e[0]) return eps * E;
    int k = 0;
    while (k + 1 < g_pw_n - 1 && eps >= g_pw_e[k + 1]) ++k;
    /* segment k runs from point k to point k+1; the last one extends */
    double slope = (g_pw_s[k + 1] - g_pw_s[k]) / (g_pw_e[k + 1] - g_pw_e[k]);
    return g_pw_s[k] + (eps - g_pw_e[k]) * slope;
}

struct Job {
    std::string mode = "solve";
    std::vector<std::string> meshSpec;
    std::vector<std::vector<std::string>> meshOps;  // renum dx dy | smooth_ring borderN, in order
    double E = 0, nu = 0.3, h = 1.0;
    bool haveMaterialLine = false;
    std::vector<std::string> diagram;
    bool planeStrain = false;
    double cgEps = 1e-7, outerEps = 1e-5;
    int maxOuter = 50, levels = 1;
    bool dumpK = false, dumpCsr = false;
    std::vector<int> fixDofs;
    std::vector<std::vector<std::string>> loads;
    long long prefixOuter = 0;
};

static std::vector<std::string> split(const std::string& s) {
    std::istringstream ss(s);
    std::vector<std::string> out;
    std::string w;
    while (ss >> w) out.push_back(w);
    return out;
}

static Job parseJob(const char* path) {
    Job j;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        auto w = split(line);
        if (w.empty() || w[0][0] == '#') continue;
        const std::string& k = w[0];
        if (k == "mode") j.mode = w[1];
        else if (k == "mesh") j.meshSpec.assign(w.begin() + 1, w.end());
        else if (k == "renum" || k == "smooth_ring") j.meshOps.push_back(w);
        else if (k == "material") { j.E = atof(w[1].c_str()); j.nu = atof(w[2].c_str()); j.h = atof(w[3].c_str()); j.haveMaterialLine = true; }
        else if (k == "diagram") j.diagram.assign(w.begin() + 1, w.end());
        else if (k == "plane") j.planeStrain = (w[1] == "strain");
        else if (k == "cg_eps") j.cgEps = atof(w[1].c_str());
        else if (k == "outer_eps") j.outerEps = atof(w[1].c_str());
        else if (k == "max_outer") j.maxOuter = atoi(w[1].c_str());
        else if (k == "levels") j.levels = atoi(w[1].c_str());
        else if (k == "dump_k") j.dumpK = atoi(w[1].c_str()) != 0;
        else if (k == "dump_csr") j.dumpCsr = atoi(w[1].c_str()) != 0;
        else if (k == "fixdof") j.fixDofs.push_back(atoi(w[1].c_str()));
        else if (k == "prefix_outer") j.prefixOuter = atoll(w[1].c_str());
        else j.loads.push_back(w);
    }
    return j;
}

static sigjmp_buf g_trap;
static void on_trap(int) { siglongjmp(g_trap, 1); }

static void buildMesh(const Job& j, Mesh& mesh) {
    const auto& s = j.meshSpec;
    auto d = [&](int i) { return atof(s[i].c_str()); };
    auto n = [&](int i) { return (size_t)atol(s[i].c_str()); };
    if (s[0] == "hole") mesh.genRectWithHole(d(1), d(2), d(3), d(4), d(5), n(6), n(7), (int)n(8));
    else if (s[0] == "ring") mesh.genRing(d(1), d(2), n(3), n(4), (int)n(5));
    else if (s[0] == "rect") mesh.genRectangle(d(1), d(2), d(3), d(4), n(5), n(6), (int)n(7));
    else if (s[0] == "inp") {
        // the reference looks the file up relative to the working directory
        std::string path = s[1], dir = ".", name = path;
        const size_t cut = path.rfind('/');
        if (cut != std::string::npos) { dir = path.substr(0, cut); name = path.substr(cut + 1); }
        if (chdir(dir.c_str()) != 0) { fprintf(stderr, "cannot enter %s\n", dir.c_str()); exit(2); }
        mesh.useCuda = false;
        // loadFromFile is declared bool but ends without a return (undefined
        // behaviour). Built at -O0 (the cpref_inp binary) the compiler puts a
        // trap instruction exactly there, after the whole load: catch it and
        // come back with the loaded mesh.
        struct sigaction sa = {}, old = {};
        sa.sa_handler = on_trap;
        sigemptyset(&sa.sa_mask);
        sigaction(SIGILL, &sa, &old);
        try {
            if (sigsetjmp(g_trap, 1) == 0) mesh.loadFromFile(name);
        } catch (const char* e) {
            fprintf(stderr, "loadFromFile: %s\n", e);
            exit(3);
        }
        sigaction(SIGILL, &old, nullptr);
    }
    else if (s[0] == "file") {
        cpbin_file f;
        if (cpbin_read(s[1].c_str(), &f) != 0) { fprintf(stderr, "cannot read mesh file\n"); exit(2); }
        const cpbin_rec* xy = cpbin_get(&f, "node_xy");
        const cpbin_rec* e3 = cpbin_get(&f, "elem3");
        const cpbin_rec* e4 = cpbin_get(&f, "elem4");
        const cpbin_rec* e8 = cpbin_get(&f, "elem8");
        const cpbin_rec* bl = cpbin_get(&f, "border_len");
        const cpbin_rec* bn = cpbin_get(&f, "border_nodes");
        mesh.nodeCount = (int)(xy->count / 2);
        mesh.node = new vec2[mesh.nodeCount];
        mesh.secOrdNodes = new bool[mesh.nodeCount];
        for (int i = 0; i < mesh.nodeCount; ++i) {
            mesh.node[i].x = ((double*)xy->data)[2 * i];
            mesh.node[i].y = ((double*)xy->data)[2 * i + 1];
            mesh.secOrdNodes[i] = false;
        }
        mesh.count3 = e3 ? (int)(e3->count / 3) : 0;
        mesh.count4 = e4 ? (int)(e4->count / 4) : 0;
        mesh.count8 = e8 ? (int)(e8->count / 8) : 0;
        mesh.elem3 = new int[3 * mesh.count3 + 1];
        mesh.elem4 = new int[4 * mesh.count4 + 1];
        mesh.elem8 = new int[8 * mesh.count8 + 1];
        if (mesh.count3) memcpy(mesh.elem3, e3->data, e3->count * 4);
        if (mesh.count4) memcpy(mesh.elem4, e4->data, e4->count * 4);
        if (mesh.count8) memcpy(mesh.elem8, e8->data, e8->count * 4);
        for (int e = 0; e < mesh.count8; ++e)
            for (int i = 4; i < 8; ++i) mesh.secOrdNodes[mesh.elem8[8 * e + i]] = true;
        mesh.bordersCount = bl ? (int)bl->count : 0;
        mesh.borderLength = new int[mesh.bordersCount + 1];
        mesh.borders = new int*[mesh.bordersCount + 1];
        int off = 0;
        for (int b = 0; b < mesh.bordersCount; ++b) {
            int len = ((int*)bl->data)[b];
            mesh.borderLength[b] = len;
            mesh.borders[b] = new int[len];
            memcpy(mesh.borders[b], (int*)bn->data + off, len * 4);
            off += len;
        }
        mesh.fillPos();
        mesh.ramSaved = true;
        mesh.analysed = false;
        cpbin_free(&f);
    }
    mesh.useCuda = false;
    mesh.ramSaved = true;
}

static void setupMaterial(const Job& j, Material& m) {
    const auto& d = j.diagram;
    auto v = [&](int i) { return atof(d[i].c_str()); };
    if (d.empty()) { m.setLinearPlast(j.E, 1e300, j.E); }
    else if (d[0] == "linear") m.setLinearPlast(v(1), v(2), v(3));
    else if (d[0] == "power") m.setPowerPlast(v(1), v(2), v(3), v(4));
    else if (d[0] == "hollomon") {
        m.setLinearPlast(v(1), v(2), 0.0);
        g_hol_sy = v(2); g_hol_eps0 = v(3); g_hol_n = v(4);
        m.host_f = hollomonDiagram;
    } else if (d[0] == "piecewise") {
        m.setLinearPlast(v(1), 0.0, 0.0);
        g_pw_n = atoi(d[2].c_str());
        for (int i = 0; i < g_pw_n; ++i) { g_pw_e[i] = v(3 + 2 * i); g_pw_s[i] = v(4 + 2 * i); }
        m.sigmaT = g_pw_s[0];
        m.host_f = piecewiseDiagram;
    }
    if (j.haveMaterialLine) { m.E = j.E; }
    m.nu = j.nu;
    m.h = j.h;
}

static void setupLoads(const Job& j, LoadConditions& lc) {
    for (const auto& w : j.loads) {
        auto v = [&](int i) { return atof(w[i].c_str()); };
        const std::string& k = w[0];
        if (k == "force") lc.setForce(atoi(w[1].c_str()), vec2(v(2), v(3)), atoi(w[4].c_str()) != 0);
        else if (k == "fixborderhor") lc.fixBorderHor(atoi(w[1].c_str()));
        else if (k == "fixbordervert") lc.fixBorderVert(atoi(w[1].c_str()));
        else if (k == "fixvertaxis") lc.fixVertAxis(v(1));
        else if (k == "fixhoraxis") lc.fixHorAxis(v(1));
        else if (k == "fixpoint") lc.fixPoint(vec2(v(1), v(2)));
        else if (k == "displ") lc.setDisplacement(atoi(w[1].c_str()), vec2(v(2), v(3)), atoi(w[4].c_str()) != 0, atoi(w[5].c_str()) != 0);
        else if (k == "forcepoint") lc.setForcePoint(vec2(v(1), v(2)), vec2(v(3), v(4)));
        else if (k == "displpoint") lc.setDisplPoint(vec2(v(1), v(2)), vec2(v(3), v(4)));
        else if (k == "gravity") lc.setGravity(v(1), vec2(v(2), v(3)));
        else { fprintf(stderr, "unknown job line %s\n", k.c_str()); exit(2); }
    }
}

static void dumpMesh(FILE* f, Mesh& mesh) {
    std::vector<double> xy(2 * mesh.nodeCount);
    for (int i = 0; i < mesh.nodeCount; ++i) { xy[2 * i] = mesh.node[i].x; xy[2 * i + 1] = mesh.node[i].y; }
    cpbin_put(f, "node_xy", 'd', xy.size(), xy.data());
    cpbin_put(f, "elem3", 'i', 3 * mesh.count3, mesh.elem3);
    cpbin_put(f, "elem4", 'i', 4 * mesh.count4, mesh.elem4);
    cpbin_put(f, "elem8", 'i', 8 * mesh.count8, mesh.elem8);
    std::vector<int> bl(mesh.bordersCount), bn;
    for (int b = 0; b < mesh.bordersCount; ++b) {
        bl[b] = mesh.borderLength[b];
        for (int i = 0; i < bl[b]; ++i) bn.push_back(mesh.borders[b][i]);
    }
    cpbin_put(f, "border_len", 'i', bl.size(), bl.data());
    cpbin_put(f, "border_nodes", 'i', bn.size(), bn.data());
    std::vector<unsigned char> so(mesh.nodeCount);
    for (int i = 0; i < mesh.nodeCount; ++i) so[i] = mesh.secOrdNodes[i] ? 1 : 0;
    cpbin_put(f, "sec_ord", 'b', so.size(), so.data());
    cpbin_put_i(f, "max_index_diff", mesh.findMaxIndexDiff());
    std::vector<double> aspect(mesh.count4), skew(mesh.count4);
    for (int e = 0; e < mesh.count4; ++e) { aspect[e] = mesh.aspectRatio(e); skew[e] = mesh.skewAngleSin(e); }
    cpbin_put(f, "aspect", 'd', aspect.size(), aspect.data());
    cpbin_put(f, "skew_sin", 'd', skew.size(), skew.data());
    cpbin_put_d(f, "avr_elem_size", mesh.avrElemSize());
}

static void dumpCsr(FILE* f, SparseSLAE& sp, int nodeCount) {
    cpbin_put(f, "rows", 'i', sp.N + 1, sp.rows);
    cpbin_put(f, "cols", 'i', sp.rows[sp.N], sp.cols);
    cpbin_put(f, "adj_pos", 'i', nodeCount + 1, sp.adjPos);
    cpbin_put(f, "adj", 'i', sp.adjPos[nodeCount], sp.adj);
}

static void dumpState(FILE* f, PlasticitySolver& ps, int E, int N) {
    cpbin_put(f, "uv", 'd', N, ps.uv.data());
    cpbin_put(f, "exx", 'd', E, ps.exx);
    cpbin_put(f, "eyy", 'd', E, ps.eyy);
    cpbin_put(f, "gamma", 'd', E, ps.gamma);
    cpbin_put(f, "eps_i", 'd', E, ps.intensityE);
    cpbin_put(f, "sxx", 'd', E, ps.sxx);
    cpbin_put(f, "syy", 'd', E, ps.syy);
    cpbin_put(f, "tau", 'd', E, ps.tau);
    cpbin_put(f, "sig_i", 'd', E, ps.intensityS);
    cpbin_put(f, "table_s", 'd', E, ps.tableS);
    cpbin_put(f, "psi", 'd', E, ps.psi);
    cpbin_put(f, "E_c", 'd', E, ps.E_c);
    cpbin_put(f, "nu_c", 'd', E, ps.nu_c);
    cpbin_put(f, "exx_p", 'd', E, ps.exx_p);
    cpbin_put(f, "eyy_p", 'd', E, ps.eyy_p);
    cpbin_put(f, "gamma_p", 'd', E, ps.gamma_p);
    cpbin_put(f, "eps_p_i", 'd', E, ps.intE_p);
}

#ifdef CPREF_SOLVER_SOURCE
/* CSR position of every (local row, local column) DOF pair of every 4-node
 * element: 64 per element, row-major over the element's 8 DOFs. */
static std::vector<int> csrSlots4(const Mesh& mesh, const SparseSLAE& sp) {
    std::vector<int> slots((size_t)mesh.count4 * 64);
#pragma omp parallel for
    for (long long e = 0; e < (long long)mesh.count4; ++e) {
        for (int a = 0; a < 8; ++a) {
            const int gi = 2 * mesh.elem4[4 * e + a / 2] + a % 2;
            for (int b = 0; b < 8; ++b) {
                const int gj = 2 * mesh.elem4[4 * e + b / 2] + b % 2;
                int pos = -1;
                for (int q = sp.rows[gi]; q < sp.rows[gi + 1]; ++q)
                    if (sp.cols[q] == gj) { pos = q; break; }
                slots[(size_t)e * 64 + 8 * a + b] = pos;
            }
        }
    }
    return slots;
}

/* fillGlobalStiffness with the band matrix replaced by the CSR slot table
 * (see the file comment); the per-element arithmetic is the reference's. */
static void fillCsrDirect(PlasticitySolver& ps, SparseSLAE& spK, const std::vector<int>& slots) {
    const Mesh& mesh = ps.mesh;
    const int nnz = spK.rows[2 * mesh.nodeCount];
    std::memset(spK.data, 0, sizeof(double) * (size_t)nnz);
#pragma omp parallel for
    for (int e = mesh.elemPos[0]; e < mesh.elemPos[1]; ++e) {
        StaticMatrix<3, 3, double> Ce;
        (*ps.formC)(Ce, ps.E_c[e], ps.nu_c[e]);
        std::memcpy(ps.C + e, &Ce, sizeof(Ce));
        SymMatrix<8, double> Ke;
        formKe4(Ke, e, ps.B4, ps.detJ4, Ce, ps.m.h);
        const int le = e - mesh.elemPos[0];
        for (int a = 0; a < 8; ++a)
            for (int b = 0; b < 8; ++b) {
                const double v = a >= b ? Ke(a, b) : Ke(b, a);
#pragma omp atomic
                spK.data[slots[(size_t)le * 64 + 8 * a + b]] += v;
            }
    }
}
#endif

int main(int argc, char** argv) {
    if (argc != 3) { fprintf(stderr, "usage: cpref job.txt out.bin\n"); return 2; }
    Job j = parseJob(argv[1]);
    std::cout.setstate(std::ios_base::failbit); /* silence the reference's progress prints */

    Mesh mesh;
    buildMesh(j, mesh);
    for (const auto& op : j.meshOps) {
        if (op[0] == "renum") mesh.renumByDirection(vec2(atof(op[1].c_str()), atof(op[2].c_str())));
        else mesh.smoothRing(atoi(op[1].c_str()));
    }
    FILE* out = cpbin_open_write(argv[2]);
    if (!out) return 3;

    if (j.mode == "mesh") { dumpMesh(out, mesh); fclose(out); return 0; }
    if (j.mode == "csr") {
        SparseSLAE sp(mesh, 2);
        dumpCsr(out, sp, mesh.nodeCount);
        fclose(out);
        return 0;
    }

    Material m;
    setupMaterial(j, m);
    LoadConditions lc;
    setupLoads(j, lc);
    PlasticitySolver ps(m, mesh, lc);
    if (j.planeStrain) ps.setPlainCondition(strain);
    ps.iterOutput = false;
    const int E = ps.mesh.elemCount(), N = 2 * ps.mesh.nodeCount;

    if (j.mode == "solve") {
        /* The reference's own public entry point, untouched: its CPU path with
         * CG eps 1e-7 and outer 1e-5 (src/PlasticitySolver.cu:325-366). */
        double t0 = omp_get_wtime();
        double t = ps.solve();
        double wall = omp_get_wtime() - t0;
        dumpState(out, ps, E, N);
        cpbin_put_d(out, "solve_seconds", t);
        cpbin_put_d(out, "wall_seconds", wall);
        cpbin_put_d(out, "exit_error", ps.exitCondition());
        cpbin_put_d(out, "energy", ps.deformEnergy());
        cpbin_put_i(out, "threads", omp_get_max_threads());
        fclose(out);
        return 0;
    }

    /* Phase driver: the body of solveCPU with caller tolerances. */
    const bool csrDirect = (j.mode == "phases_csr");
#ifndef CPREF_SOLVER_SOURCE
    if (csrDirect) { fprintf(stderr, "phases_csr: use the cpref_csr build\n"); return 4; }
#endif
    if (csrDirect && (ps.mesh.count3 || ps.mesh.count8)) { fprintf(stderr, "phases_csr: 4-node meshes only\n"); return 4; }
    double t0 = omp_get_wtime();
    StripSLAE K(csrDirect ? 1 : N, csrDirect ? 1 : 2 * ps.mesh.findMaxIndexDiff() + 1);
    K.factN = csrDirect ? 1 : N;
    ps.calcBs();
    SparseSLAE spK(ps.mesh, 2);
#ifdef CPREF_SOLVER_SOURCE
    std::vector<int> slots;
    if (csrDirect) slots = csrSlots4(ps.mesh, spK);
#endif
    ps.initConditions(spK);
    for (int d : j.fixDofs) ps.kinMask[d] = false;
    std::vector<double> rpFull(spK.rp, spK.rp + N), uvFull(ps.uv.begin(), ps.uv.begin() + N);
    std::vector<unsigned char> mask(N);
    for (int i = 0; i < N; ++i) mask[i] = ps.kinMask[i] ? 1 : 0;
    if (j.dumpCsr) dumpCsr(out, spK, ps.mesh.nodeCount);
    cpbin_put(out, "rp", 'd', N, rpFull.data());
    cpbin_put(out, "mask", 'b', N, mask.data());
    if (j.mode == "loads") {
        cpbin_put(out, "uv", 'd', N, uvFull.data());
        fclose(out);
        return 0;
    }

    std::vector<int> outerPerLevel, cgPerLevel;
    std::vector<double> errPerLevel;
    long long cgTotal = 0, outerTotal = 0;
    double tAsm = 0, tCg = 0, tUpd = 0;
    const double tSetup = omp_get_wtime() - t0;
    bool elastic = (j.mode == "elastic");
    bool stopped = false;
    for (int lev = 1; lev <= j.levels; ++lev) {
        double lam = (double)lev / j.levels;
        for (int i = 0; i < N; ++i) spK.rp[i] = lam * rpFull[i];
        for (int i = 0; i < N; ++i) if (!ps.kinMask[i]) ps.uv[i] = lam * uvFull[i];
        ConjGradSolver cjs(spK);
        int iter = 0;
        long long cgLevel = 0;
        double relErr = 0.;
        do {
            double ta = omp_get_wtime();
#ifdef CPREF_SOLVER_SOURCE
            if (csrDirect) fillCsrDirect(ps, spK, slots);
            else
#endif
            ps.fillGlobalStiffness(K, spK);
            double tb = omp_get_wtime();
            if (j.dumpK && lev == 1 && iter == 0) cpbin_put(out, "k_data", 'd', spK.rows[N], spK.data);
            size_t inner = 0;
            cjs.solve(ps.uv.data(), ps.kinMask, inner, j.cgEps);
            double tc = omp_get_wtime();
            cgLevel += (long long)inner;
            ps.updateParameters(iter);
            relErr = ps.exitCondition();
            double td = omp_get_wtime();
            tAsm += tb - ta;
            tCg += tc - tb;
            tUpd += td - tc;
            ++iter;
            ++outerTotal;
            if (j.prefixOuter && outerTotal >= j.prefixOuter) { stopped = true; break; }
            if (elastic) break;
        } while (relErr > j.outerEps && iter < j.maxOuter);
        outerPerLevel.push_back(iter);
        cgPerLevel.push_back((int)cgLevel);
        errPerLevel.push_back(relErr);
        cgTotal += cgLevel;
        if (stopped) break;
    }
    ps.calcPlastDeform();
    double wall = omp_get_wtime() - t0;
    dumpState(out, ps, E, N);
    cpbin_put(out, "outer_per_level", 'i', outerPerLevel.size(), outerPerLevel.data());
    cpbin_put(out, "cg_per_level", 'i', cgPerLevel.size(), cgPerLevel.data());
    cpbin_put(out, "err_per_level", 'd', errPerLevel.size(), errPerLevel.data());
    cpbin_put_d(out, "wall_seconds", wall);
    cpbin_put_d(out, "setup_seconds", tSetup);
    cpbin_put_d(out, "assembly_seconds", tAsm);
    cpbin_put_d(out, "cg_seconds", tCg);
    cpbin_put_d(out, "update_seconds", tUpd);
    cpbin_put_d(out, "energy", ps.deformEnergy());
    cpbin_put_i(out, "threads", omp_get_max_threads());
    fclose(out);
    return 0;
}
