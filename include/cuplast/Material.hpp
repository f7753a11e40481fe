// Material and hardening diagram of the drop-in API (the reference's class
// Material, src/Material.cuh:9-40 and src/Material.cu:1-43). The diagram is a
// tagged description instead of host/device function pointers, so the same
// object drives the CUDA kernels (compile-time dispatch there).
#pragma once

#include <utility>
#include <vector>

#include "../cuplast.h"
#include "vec2.hpp"

namespace cuplast {

class CUPLAST_CXX_API Material {
public:
    double E = 0.;      // elastic modulus
    double nu = 0.3;    // Poisson ratio
    double h = 1.;      // thickness
    double rho = 1.;    // density (body forces)
    double sigmaT = 0.; // yield stress

    // sigma = E eps below sigmaT / E, then sigmaT + (eps - sigmaT/E) K_T (src/Material.cu:14-17)
    void setLinearPlast(double E, double sigmaT, double K_T);
    // sigmaT + A (eps - epsT + (E/(A m))^(1/(m-1)))^m - A (E/(A m))^(m/(m-1)) (src/Material.cu:19-23)
    void setPowerPlast(double E, double sigmaT, double A, double m);
    // Extension: sigma = sy (1 + eps_p / eps0)^n in terms of the total strain
    // eps = sigma / E + eps_p (inverted by Newton).
    void setHollomonPlast(double E, double sigmaY, double eps0, double n);
    // Extension: elastic up to points[0], then linear between the points
    // (strain, stress); the last segment extends.
    void setPiecewisePlast(double E, const std::vector<std::pair<double, double>>& points);

    // sigma = f(eps_i) on the host (Material::f, src/Material.cuh:33-35)
    double f(double eps) const;

    cp_material toC(int plane) const;

private:
    int diagram_ = CP_DIAGRAM_ELASTIC;
    double K_T_ = 0., A_ = 0., m_ = 0., eps0_ = 0., n_ = 0.;
    std::vector<std::pair<double, double>> points_;
};

}  // namespace cuplast
