// Loads and boundary conditions of the drop-in API (the reference's class
// LoadConditions, src/LoadConditions.cuh:47-180), with std::function in place
// of nvstd::function: they are evaluated on the host when the right-hand side
// and the Dirichlet mask are built.
#pragma once

#include <functional>
#include <list>
#include <map>
#include <vector>

#include "Mesh.hpp"
#include "vec2.hpp"

namespace cuplast {

struct ForceCondition {
    std::function<vec2(vec2)> forceFunc;
    vec2 value;
    bool normOrient = false;  // x: normal component, y: tangential component
};

struct DisplacementCondition {
    std::function<vec2(vec2)> displFunc;
    bool fixMidX = false;
    bool fixMidY = false;
};

struct FixedAxis {
    bool vertical = true;
    double coord = 0.;
};

struct FixedBorder {
    bool vertical = true;
};

struct PointCondition {
    vec2 point;
    vec2 value;
};

class CUPLAST_CXX_API LoadConditions {
public:
    bool Rset = false;
    std::function<vec2(vec2)> R = [](vec2) { return vec2(0., 0.); };
    std::map<int, DisplacementCondition> displCond;
    std::map<int, ForceCondition> forceCond;
    std::map<int, FixedBorder> fixedBorder;
    std::list<FixedAxis> fixedAxis;
    std::list<PointCondition> forcePoint;
    std::list<PointCondition> displPoint;
    std::vector<int> fixedDofs;  // extension: extra Dirichlet DOFs (value 0)

    void setDisplacement(size_t borderId, vec2 u, bool fixOnlyMiddleX = false, bool fixOnlyMiddleY = false);
    void setDisplacement(size_t borderId, std::function<vec2(vec2)> displFunc);
    void setForce(size_t borderId, vec2 f, bool normalOriented = false);
    void setForce(size_t borderId, std::function<vec2(vec2)> forceFunc, bool normalOriented = false);
    void fixVertAxis(double x);
    void fixHorAxis(double y);
    void fixBorder(size_t borderId);
    void fixBorderVert(size_t borderId);
    void fixBorderHor(size_t borderId);
    void fixPoint(vec2 point);
    void setDisplPoint(vec2 point, vec2 displ);
    void setForcePoint(vec2 point, vec2 force);
    void setGravity(double g = 9.81, vec2 direction = vec2(0., -1.));
    void setRotation(double omega, vec2 rotationAxis = vec2(0., 0.));
    void setVolumeForce(std::function<vec2(vec2)> R);
    void fixDof(int dof) { fixedDofs.push_back(dof); }
};

// initConditions (src/PlasticitySolver.cu:812-1005): consistent nodal forces
// of border tractions and body forces, the Dirichlet mask (1 = free) and the
// prescribed displacements, for linear (T3/Q4) borders. Host-side set-up,
// done once per solve like in the reference.
CUPLAST_CXX_API void buildConditions(const Mesh& mesh, const LoadConditions& cond, double h, double rho, std::vector<double>& rp,
                     std::vector<unsigned char>& mask, std::vector<double>& uv);

}  // namespace cuplast
