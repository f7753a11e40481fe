// PlasticitySolver of the drop-in API (the reference's class, src/PlasticitySolver.cuh:23-543),
// running every phase on the GPU through the C ABI of include/cuplast.h.
#pragma once

#include <functional>
#include <string>
#include <vector>

#include "../cuplast.h"
#include "LoadConditions.hpp"
#include "Material.hpp"
#include "Mesh.hpp"

namespace cuplast {

enum plainCondition { stress, strain };

class CUPLAST_CXX_API PlasticitySolver {
public:
    // public flags of the reference (src/PlasticitySolver.cuh:207-211)
    bool polarCoord = false;
    bool iterOutput = true;
    // the reference's two phases (solveCUDA_FD, src/PlasticitySolver.cu:631-708): reduced precision to
    // relErr 1e-4 (here FP32 matrix and inner CG inside FP64 defect correction), then FP64
    bool floatBoost = false;

    // Extensions: the reference hard-codes CG 1e-7, outer 1e-5 and (CPU) 50 iterations.
    double cgTol = 1e-7;
    double outerTol = 1e-5;
    int maxOuter = 50;
    int levels = 1;          // load increments, each a deformation-theory solve warm-started from the last
    bool aitken = false;     // Aitken-relaxed secant iteration (same fixed point)
    bool adaptiveCg = false; // loose linear solves while the secant iteration is far from converged
    int adaptiveRule = 1;    // adaptiveCg: 1 tight within 10x of outerTol; 2 looser until outerTol (cp_solve_opts)
    bool predict = false;    // levels from the third on start from the extrapolation of the last two
    int precond = 0;         // linear solver (cp_solve_opts): 0 CG as the reference, 1 2x2 block-Jacobi PCG,
                             // 2 aggregation-multigrid PCG (FP64; not with floatBoost)
    double innerTol = 1e-4;  // floatBoost's first phase: FP32 inner solves' relative tolerance
    int recycle = 0;         // 0..6: FP64 linear solves start from the projection onto the level's last
                             // `recycle` solution increments (cp_solve_opts.recycle; same fixed point)
    int device = 0;

    PlasticitySolver(const Material& material, Mesh& mesh, const LoadConditions& loadConditions);
    PlasticitySolver(const PlasticitySolver&) = delete;
    PlasticitySolver& operator=(const PlasticitySolver&) = delete;
    ~PlasticitySolver();

    void setPlainCondition(plainCondition pc);

    // Both return seconds of device time, like the reference returns wall time.
    double solve();
    double solveElast();
    // The reference's explicit device paths (src/PlasticitySolver.cuh:379-407):
    // FP64, floatBoost's two phases, and the elastic solve. There is no CPU
    // path (solveCPU / solveElastCPU): the library has no CPU fallback.
    double solveCUDA();
    double solveCUDA_FD();
    double solveElastCUDA();

    double deformEnergy();                               // src/PlasticitySolver.cuh:415-445
    void saveDisplsToFile(const std::string& fileName);  // src/PlasticitySolver.cuh:448-458
    void saveAsVtk(const std::string& fileName);         // src/PlasticitySolver.cu:1784-1945
    double getSxx0() const;
    double getExx0() const;

    // Largest element-centre deviation from analytic stresses, each component
    // scaled by the mean of that component over the area (4-node elements;
    // src/PlasticitySolver.cuh:464-494).
    double sigmaError(std::function<double(vec2)> s_x, std::function<double(vec2)> s_y,
                      std::function<double(vec2)> s_xy) const;
    // The same in polar components about the origin, for element centres
    // within maxR; the analytic functions take (r, phi) as a vec2 (the Kirsch
    // problem; src/PlasticitySolver.cuh:496-540).
    double polarSigmaError(std::function<double(vec2)> s_r, std::function<double(vec2)> s_phi,
                           std::function<double(vec2)> s_rphi, double maxR) const;

    // Host copy of a field ("uv", "exx", ... as in cp_get_field).
    std::vector<double> field(const std::string& name) const;
    const cp_solve_report& lastReport() const { return report_; }

private:
    Material m_;
    Mesh mesh_;
    LoadConditions cond_;
    plainCondition pc_ = stress;
    bool plastSolved_ = false;
    cp_context* ctx_ = nullptr;
    cp_instance* inst_ = nullptr;
    cp_solve_report report_{};
    void ensureInstance();
    void check(int status) const;
    double run(bool elastic);
};

// SparseSLAE(Mesh&, dim) of the reference (src/SparseSLAE.h:60-196): the
// CSR structure in the reference's ordering, built on the GPU and copied back.
class CUPLAST_CXX_API SparseSLAE {
public:
    int N = 0;
    int dim = 2;
    double* rp = nullptr;
    double* data = nullptr;
    int* rows = nullptr;
    int* cols = nullptr;
    int* adj = nullptr;
    int* adjPos = nullptr;

    explicit SparseSLAE(Mesh& mesh, int dim = 2, int device = 0);
    SparseSLAE(const SparseSLAE&) = delete;
    SparseSLAE& operator=(const SparseSLAE&) = delete;
    ~SparseSLAE();
};

}  // namespace cuplast
