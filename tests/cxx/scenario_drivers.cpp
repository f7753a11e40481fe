// Scenario drivers written against the drop-in C++ API (include/cuplast/*.hpp)
// the way a user of the reference writes them: each function restates one
// scenario of the reference's src/Main.cpp with the same mesh, material and
// loads, only with `#include "cuplast/PlasticitySolver.hpp"` and namespace
// cuplast in place of the reference's headers. tests/test_cxx_api.py builds
// this file with g++ against libcuplast.so and checks the outputs against the
// reference's shipped results.
//
//   scenario_drivers solverTest <out.vtk>
//   scenario_drivers plasticityTest <out.vtk>
//   scenario_drivers energyConvTest <order> <power|linear|elastic>   (prints the energy)
//   scenario_drivers kirschTest <segments> <out.vtk>                  (prints the error norms)
//   scenario_drivers meshVtk <out.vtk>                                (mesh tooling only: no device)
//   scenario_drivers noDevice                                         (expects a clean error)
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <stdexcept>
#include <string>

#include "cuplast/PlasticitySolver.hpp"

using namespace cuplast;

namespace {

const double E_304L = 193e9;
const double s_T_304L = 170e6;
const double nu_304L = 0.29;

// solverTest, src/Main.cpp:14-38: elastic 4x4 patch, one edge pulled.
int solverTest(const char* out) {
    Mesh mesh;
    mesh.genRectangle(-1., 1., -1., 1., 4, 4);
    LoadConditions lc;
    lc.setDisplacement(2, vec2(0, 0.), false, true);
    lc.setForce(0, vec2(1, 0));
    Material m;
    m.setLinearPlast(E_304L * 1e-6, s_T_304L, E_304L * 1e-6);
    m.E = E_304L * 1e-6;
    m.nu = nu_304L * 1e-6;
    m.h = 1.;
    PlasticitySolver ps(m, mesh, lc);
    ps.iterOutput = false;
    ps.solveElast();
    ps.saveAsVtk(out);
    return 0;
}

// plasticityTest, src/Main.cpp:252-296: the plate with a hole under tension,
// power-law hardening, reference tolerances.
int plasticityTest(const char* out) {
    Mesh mesh;
    mesh.genRectWithHole(-3., 3., -2., 2., 0.5, 48, 32, 1);
    double S = 170;
    LoadConditions lc;
    lc.setForce(1, vec2(S, 0.));
    lc.setForce(3, vec2(-S, 0.));
    lc.fixVertAxis(0.);
    lc.fixHorAxis(0.);
    Material m;
    m.h = 1.;
    m.setPowerPlast(E_304L * 1e-6, s_T_304L * 1e-6, E_304L * 0.01 * 1e-6, 0.015);
    m.nu = nu_304L;
    PlasticitySolver ps(m, mesh, lc);
    ps.iterOutput = false;
    ps.solve();
    ps.saveAsVtk(out);
    return 0;
}

// energyConvTest, src/Main.cpp:110-175, one mesh of its sequence (the
// 2880-element plate) at element order 1 or 2; prints the strain energy.
int energyConvTest(int order, const std::string& kind) {
    LoadConditions lc;
    double S = kind == "elastic" ? 1e6 : 170e6;
    lc.setForce(1, vec2(S, 0));
    lc.setForce(3, vec2(-S, 0));
    lc.fixVertAxis(0.);
    lc.fixHorAxis(0.);
    Material m;
    if (kind == "linear")
        m.setLinearPlast(E_304L, s_T_304L, E_304L * 0.1);
    else
        m.setPowerPlast(E_304L, s_T_304L, E_304L * 0.01, 0.015);
    m.nu = nu_304L;
    m.h = 1.;
    Mesh mesh;
    mesh.genRectWithHole(-3., 3., -2., 2., 0.5, 36, 24, order);
    PlasticitySolver ps(m, mesh, lc);
    ps.iterOutput = false;
    ps.solve();
    std::printf("elements %d energy %.17g\n", mesh.elemCount(), ps.deformEnergy());
    return 0;
}

// kirschConvTest, src/Main.cpp:178-227, one mesh of its sequence: the
// elastic plate with a hole against Kirsch's analytic stresses, through
// polarSigmaError (and sigmaError with zero reference stresses, which gives
// the scaled largest stress of each component). The linear solve is tightened
// (cgTol, an extension member) so that the norms are those of the exact
// discrete solution. Writes the polar-coordinate VTK.
int kirschTest(int segments, const char* out) {
    Material m;
    m.E = E_304L;
    m.nu = nu_304L;
    m.h = 1.;
    const double a = 0.5, S = 1e6;
    LoadConditions lc;
    lc.setForce(1, vec2(S, 0));
    lc.setForce(3, vec2(-S, 0));
    lc.fixVertAxis(0.);
    lc.fixHorAxis(0.);
    auto s_r = [&](vec2 r) {
        return 0.5 * S * (1. - a * a / (r.x * r.x)) +
               0.5 * S * (1. + 3. * std::pow(a, 4.) / std::pow(r.x, 4.) - 4. * a * a / (r.x * r.x)) * std::cos(2. * r.y);
    };
    auto s_phi = [&](vec2 r) {
        return 0.5 * S * (1. + a * a / (r.x * r.x)) - 0.5 * S * (1. + 3. * std::pow(a, 4.) / std::pow(r.x, 4.)) * std::cos(2. * r.y);
    };
    auto tau = [&](vec2 r) {
        return -0.5 * S * (1. - 3. * std::pow(a, 4.) / std::pow(r.x, 4.) + 2. * a * a / (r.x * r.x)) * std::sin(2. * r.y);
    };
    Mesh mesh;
    mesh.genRectWithHole(-3., 3., -2., 2., a, segments, segments);
    PlasticitySolver ps(m, mesh, lc);
    ps.iterOutput = false;
    ps.cgTol = 1e-13;
    ps.solveElast();
    auto zero = [](vec2) { return 0.0; };
    std::printf("polar %.17g cartesian_zero %.17g\n", ps.polarSigmaError(s_r, s_phi, tau, 2.),
                ps.sigmaError(zero, zero, zero));
    ps.polarCoord = true;
    ps.saveAsVtk(out);
    return 0;
}

// The mesh tooling as src/Main.cpp:229-246 (meshTransferTest) uses it: the
// analysis, a copy, the mesh VTK. Host only.
int meshVtk(const char* out) {
    Mesh mesh;
    mesh.genRectWithHole(-3., 3., -2., 2., 0.5, 12, 8);
    mesh.renumByDirection();
    mesh.printAnalysis();
    Mesh copy(mesh);
    copy.meshToRAM();
    copy.saveAsVtk(out);
    std::printf("avr %.17g max_index_diff %d\n", copy.avrElemSize(), copy.findMaxIndexDiff());
    return 0;
}

// Without a device the drop-in classes report the library's status as a
// std::runtime_error (the reference has no error reporting at all).
int noDevice() {
    Mesh mesh;
    mesh.genRectangle(0., 1., 0., 1., 2, 2);
    LoadConditions lc;
    lc.setForce(0, vec2(1, 0));
    lc.fixBorder(2);
    Material m;
    m.setLinearPlast(1000., 10., 100.);
    try {
        PlasticitySolver ps(m, mesh, lc);
        ps.iterOutput = false;
        ps.solve();
    } catch (const std::runtime_error& e) {
        std::printf("error: %s\n", e.what());
        return 0;
    }
    std::printf("solved without a device\n");
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    const std::string what = argc > 1 ? argv[1] : "";
    try {
        if (what == "solverTest" && argc > 2) return solverTest(argv[2]);
        if (what == "plasticityTest" && argc > 2) return plasticityTest(argv[2]);
        if (what == "energyConvTest" && argc > 3) return energyConvTest(std::atoi(argv[2]), argv[3]);
        if (what == "kirschTest" && argc > 3) return kirschTest(std::atoi(argv[2]), argv[3]);
        if (what == "meshVtk" && argc > 2) return meshVtk(argv[2]);
        if (what == "noDevice") return noDevice();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s: %s\n", what.c_str(), e.what());
        return 2;
    }
    std::fprintf(stderr, "usage: scenario_drivers solverTest|plasticityTest <out.vtk> | energyConvTest <order> "
                         "<power|linear|elastic> | kirschTest <segments> <out.vtk> | meshVtk <out.vtk> | noDevice\n");
    return 64;
}
