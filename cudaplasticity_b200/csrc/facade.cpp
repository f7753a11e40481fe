// Drop-in C++ classes (Material, LoadConditions, PlasticitySolver, SparseSLAE)
// written on top of the C ABI of include/cuplast.h.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cuplast/PlasticitySolver.hpp"

namespace cuplast {

// ------------------------------------------------------------- Material --

void Material::setLinearPlast(double E_, double sigmaT_, double K_T) {
    E = E_;
    sigmaT = sigmaT_;
    K_T_ = K_T;
    diagram_ = CP_DIAGRAM_LINEAR;
}

void Material::setPowerPlast(double E_, double sigmaT_, double A, double m) {
    E = E_;
    sigmaT = sigmaT_;
    A_ = A;
    m_ = m;
    diagram_ = CP_DIAGRAM_POWER;
}

void Material::setHollomonPlast(double E_, double sigmaY, double eps0, double n) {
    E = E_;
    sigmaT = sigmaY;
    eps0_ = eps0;
    n_ = n;
    diagram_ = CP_DIAGRAM_HOLLOMON;
}

void Material::setPiecewisePlast(double E_, const std::vector<std::pair<double, double>>& points) {
    if (points.size() < 2 || points.size() > CP_MAX_PW) throw std::invalid_argument("piecewise diagram: 2..16 points");
    E = E_;
    points_ = points;
    sigmaT = points.front().second;
    diagram_ = CP_DIAGRAM_PIECEWISE;
}

double Material::f(double eps) const {
    switch (diagram_) {
    case CP_DIAGRAM_LINEAR: {
        double epsT = sigmaT / E;
        return eps < epsT ? eps * E : sigmaT + (eps - epsT) * K_T_;
    }
    case CP_DIAGRAM_POWER: {
        double epsT = sigmaT / E;
        return eps < epsT ? eps * E
                          : sigmaT + A_ * std::pow(eps - epsT + std::pow(E / (A_ * m_), 1. / (m_ - 1.)), m_) -
                                A_ * std::pow(E / (A_ * m_), m_ / (m_ - 1.));
    }
    case CP_DIAGRAM_HOLLOMON: {
        double sy = sigmaT, s = sy;
        if (eps < sy / E) return eps * E;
        for (int it = 0; it < 200; ++it) {
            double t = std::pow(s / sy, 1.0 / n_);
            double g = s / E + eps0_ * (t - 1.0) - eps;
            double dg = 1.0 / E + eps0_ * t / (n_ * s);
            double ds = g / dg;
            s -= ds;
            if (std::fabs(ds) <= 1e-15 * s) break;
        }
        return s;
    }
    case CP_DIAGRAM_PIECEWISE: {
        if (eps < points_[0].first) return eps * E;
        size_t k = 0;
        while (k + 1 < points_.size() - 1 && eps >= points_[k + 1].first) ++k;
        double slope = (points_[k + 1].second - points_[k].second) / (points_[k + 1].first - points_[k].first);
        return points_[k].second + (eps - points_[k].first) * slope;
    }
    default:
        return eps * E;
    }
}

cp_material Material::toC(int plane) const {
    cp_material c{};
    c.E = E;
    c.nu = nu;
    c.h = h;
    c.rho = rho;
    c.plane = plane;
    c.diagram = diagram_;
    c.sigma_t = sigmaT;
    c.k_t = K_T_;
    c.a = A_;
    c.m = m_;
    c.eps0 = eps0_;
    c.n = n_;
    c.n_points = (int)points_.size();
    for (size_t i = 0; i < points_.size(); ++i) {
        c.pw_eps[i] = points_[i].first;
        c.pw_sig[i] = points_[i].second;
    }
    return c;
}

// ------------------------------------------------------- LoadConditions --

void LoadConditions::setDisplacement(size_t id, vec2 u, bool mx, bool my) {
    auto& d = displCond[(int)id];
    d.displFunc = [=](vec2) { return u; };
    d.fixMidX = mx;
    d.fixMidY = my;
}
void LoadConditions::setDisplacement(size_t id, std::function<vec2(vec2)> fn) {
    auto& d = displCond[(int)id];
    d.displFunc = fn;
    d.fixMidX = d.fixMidY = false;
}
void LoadConditions::setForce(size_t id, vec2 f, bool normal) {
    auto& c = forceCond[(int)id];
    c.forceFunc = [=](vec2) { return f; };
    c.value = f;
    c.normOrient = normal;
}
void LoadConditions::setForce(size_t id, std::function<vec2(vec2)> fn, bool normal) {
    auto& c = forceCond[(int)id];
    c.forceFunc = fn;
    c.normOrient = normal;
}
void LoadConditions::fixVertAxis(double x) { fixedAxis.push_back(FixedAxis{true, x}); }
void LoadConditions::fixHorAxis(double y) { fixedAxis.push_back(FixedAxis{false, y}); }
void LoadConditions::fixBorder(size_t id) {
    auto& d = displCond[(int)id];
    d.displFunc = [](vec2) { return vec2(0., 0.); };
    d.fixMidX = d.fixMidY = false;
}
void LoadConditions::fixBorderVert(size_t id) { fixedBorder[(int)id].vertical = true; }
void LoadConditions::fixBorderHor(size_t id) { fixedBorder[(int)id].vertical = false; }
void LoadConditions::fixPoint(vec2 p) { displPoint.push_back(PointCondition{p, vec2(0., 0.)}); }
void LoadConditions::setDisplPoint(vec2 p, vec2 d) { displPoint.push_back(PointCondition{p, d}); }
void LoadConditions::setForcePoint(vec2 p, vec2 f) { forcePoint.push_back(PointCondition{p, f}); }
void LoadConditions::setGravity(double g, vec2 dir) {
    vec2 force = dir.normalize() * g;
    R = [=](vec2) { return force; };
    Rset = true;
}
void LoadConditions::setRotation(double omega, vec2 axis) {
    double w2 = omega * omega;
    R = [=](vec2 r) { return (r - axis) * w2; };
    Rset = true;
}
void LoadConditions::setVolumeForce(std::function<vec2(vec2)> fn) {
    R = fn;
    Rset = true;
}

void buildConditions(const Mesh& mesh, const LoadConditions& cond, double h, double rho, std::vector<double>& rp,
                     std::vector<unsigned char>& mask, std::vector<double>& uv) {
    const int N = 2 * mesh.nodeCount;
    rp.assign(N, 0.0);
    mask.assign(N, 1);
    uv.assign(N, 0.0);
    for (const auto& [id, force] : cond.forceCond) {
        if (id < 0 || id >= mesh.bordersCount) throw std::out_of_range("force on a border that does not exist");
        const int* border = mesh.borders[id];
        for (int i = 1; i < mesh.borderLength[id]; ++i) {
            if (mesh.secOrdNodes[border[i]]) {
                // quadratic edge (corner, mid-side, corner): consistent nodal
                // loads 1/3, 4/3, 1/3 of the half-lengths' weights
                // (src/PlasticitySolver.cu:823-866)
                ++i;
                if (i >= mesh.borderLength[id]) throw std::out_of_range("border ends on a mid-side node");
                vec2 n1 = mesh.node[border[i - 2]], n2 = mesh.node[border[i - 1]], n3 = mesh.node[border[i]];
                double hx1 = 0.5 * (n1.x - n2.x), hy1 = 0.5 * (n1.y - n2.y);
                double hx2 = 0.5 * (n2.x - n3.x), hy2 = 0.5 * (n2.y - n3.y);
                double dl1 = std::sqrt(hx1 * hx1 + hy1 * hy1), dl2 = std::sqrt(hx2 * hx2 + hy2 * hy2);
                vec2 f1 = force.forceFunc(n1), f2 = force.forceFunc(n2), f3 = force.forceFunc(n3);
                if (force.normOrient) {
                    vec2 t1 = (n2 - n1).normalize();
                    vec2 m1 = vec2(t1.y, -t1.x).normalize();
                    vec2 t2 = (n3 - n2).normalize();
                    vec2 m2 = vec2(t2.y, -t2.x).normalize();
                    f1 = m1 * f1.x + t1 * f1.y;
                    f2 = 0.5 * ((m1 + m2) * f2.x + (t1 + t2) * f2.y);
                    f3 = m2 * f3.x + t2 * f3.y;
                }
                double R[6] = {f1.x / 3., f1.y / 3., f2.x * 4. / 3., f2.y * 4. / 3., f3.x / 3., f3.y / 3.};
                R[0] *= h * dl1 * 2.;
                R[1] *= h * dl1 * 2.;
                R[2] *= h * (dl1 + dl2);
                R[3] *= h * (dl1 + dl2);
                R[4] *= h * dl2 * 2.;
                R[5] *= h * dl2 * 2.;
                const int gi = 2 * border[i - 2], gj = 2 * border[i - 1], gk = 2 * border[i];
                rp[gi] += R[0];
                rp[gi + 1] += R[1];
                rp[gj] += R[2];
                rp[gj + 1] += R[3];
                rp[gk] += R[4];
                rp[gk + 1] += R[5];
                continue;
            }
            vec2 n1 = mesh.node[border[i - 1]], n2 = mesh.node[border[i]];
            double hd1 = 0.5 * (n1.x - n2.x), hd2 = 0.5 * (n1.y - n2.y);
            double dl = std::sqrt(hd1 * hd1 + hd2 * hd2);
            vec2 f1 = force.forceFunc(n1), f2 = force.forceFunc(n2);
            if (force.normOrient) {
                vec2 tang = (n2 - n1).normalize();
                vec2 nrm = vec2(tang.y, -tang.x).normalize();
                f1 = nrm * f1.x + tang * f1.y;
                f2 = nrm * f2.x + tang * f2.y;
            }
            double R[4] = {f1.x, f1.y, f2.x, f2.y};
            for (int j = 0; j < 4; ++j) R[j] *= h * dl;
            int gi = 2 * border[i - 1], gj = 2 * border[i];
            rp[gi] += R[0];
            rp[gi + 1] += R[1];
            rp[gj] += R[2];
            rp[gj + 1] += R[3];
        }
    }
    if (cond.Rset) {
        // body forces: a quarter (quad) / a third (triangle) of the element's
        // load to each node (src/PlasticitySolver.cu:926-945), evaluated at the node
        for (int e = 0; e < mesh.count4; ++e) {
            double coef = 0.25 * rho * h * mesh.elemSpace4(e);
            for (int i = 4 * e; i < 4 * (e + 1); ++i) {
                int nd = mesh.elem4[i];
                vec2 R = cond.R(mesh.node[nd]);
                rp[2 * nd] += coef * R.x;
                rp[2 * nd + 1] += coef * R.y;
            }
        }
        // 8-node elements: -1/12 of the load to each corner, 1/3 to each
        // mid-side node (src/PlasticitySolver.cu:911-927)
        for (int e = 0; e < mesh.count8; ++e) {
            double space = mesh.elemSpace8(e);
            double c1 = -rho * h * space / 12., c2 = rho * h * space / 3.;
            for (int i = 8 * e; i < 8 * (e + 1); ++i) {
                int nd = mesh.elem8[i];
                vec2 R = cond.R(mesh.node[nd]);
                const double c = i < 8 * e + 4 ? c1 : c2;
                rp[2 * nd] += c * R.x;
                rp[2 * nd + 1] += c * R.y;
            }
        }
        for (int e = 0; e < mesh.count3; ++e) {
            double coef = rho * h * mesh.elemSpace3(e) / 3.;
            for (int i = 3 * e; i < 3 * (e + 1); ++i) {
                int nd = mesh.elem3[i];
                vec2 R = cond.R(mesh.node[nd]);
                rp[2 * nd] += coef * R.x;
                rp[2 * nd + 1] += coef * R.y;
            }
        }
    }
    for (const auto& [id, displ] : cond.displCond) {
        if (id < 0 || id >= mesh.bordersCount) throw std::out_of_range("displacement on a border that does not exist");
        const int* border = mesh.borders[id];
        const int len = mesh.borderLength[id];
        const int end = len - (border[0] == border[len - 1] ? 1 : 0);
        const int mid = border[len / 2];
        if (displ.fixMidX) {
            mask[2 * mid] = 0;
            uv[2 * mid] = displ.displFunc(mesh.node[mid]).x;
        } else
            for (int i = 0; i < end; ++i) {
                mask[2 * border[i]] = 0;
                uv[2 * border[i]] = displ.displFunc(mesh.node[border[i]]).x;
            }
        if (displ.fixMidY) {
            mask[2 * mid + 1] = 0;
            uv[2 * mid + 1] = displ.displFunc(mesh.node[mid]).y;
        } else
            for (int i = 0; i < end; ++i) {
                mask[2 * border[i] + 1] = 0;
                uv[2 * border[i] + 1] = displ.displFunc(mesh.node[border[i]]).y;
            }
    }
    for (const auto& ax : cond.fixedAxis) {
        for (int i = 0; i < mesh.nodeCount; ++i) {
            if (ax.vertical) {
                if (std::fabs(mesh.node[i].x - ax.coord) < 1e-14) mask[2 * i] = 0;
            } else if (std::fabs(mesh.node[i].y - ax.coord) < 1e-14)
                mask[2 * i + 1] = 0;
        }
    }
    for (const auto& [id, fb] : cond.fixedBorder) {
        if (id < 0 || id >= mesh.bordersCount) throw std::out_of_range("fixed border that does not exist");
        const int* border = mesh.borders[id];
        const int len = mesh.borderLength[id];
        const int end = len - (border[0] == border[len - 1] ? 1 : 0);
        for (int i = 0; i < end; ++i) mask[2 * border[i] + (fb.vertical ? 0 : 1)] = 0;
    }
    for (const auto& fp : cond.forcePoint)
        for (int i = 0; i < mesh.nodeCount; ++i)
            if ((mesh.node[i] - fp.point).norm() < 1e-14) {
                rp[2 * i] += fp.value.x;
                rp[2 * i + 1] += fp.value.y;
                break;
            }
    for (const auto& dp : cond.displPoint)
        for (int i = 0; i < mesh.nodeCount; ++i)
            if ((mesh.node[i] - dp.point).norm() < 1e-14) {
                uv[2 * i] = dp.value.x;
                uv[2 * i + 1] = dp.value.y;
                mask[2 * i] = mask[2 * i + 1] = 0;
                break;
            }
    for (int d : cond.fixedDofs) {
        if (d < 0 || d >= N) throw std::out_of_range("fixed DOF out of range");
        mask[d] = 0;
    }
}

// ----------------------------------------------------- PlasticitySolver --

PlasticitySolver::PlasticitySolver(const Material& material, Mesh& mesh, const LoadConditions& lc)
    : m_(material), mesh_(mesh), cond_(lc) {}

PlasticitySolver::~PlasticitySolver() {
    if (inst_) cp_instance_destroy(inst_);
    if (ctx_) cp_context_destroy(ctx_);
}

void PlasticitySolver::setPlainCondition(plainCondition pc) {
    pc_ = pc;
    if (inst_) {  // the plane condition is part of the instance's material
        cp_instance_destroy(inst_);
        inst_ = nullptr;
    }
}

void PlasticitySolver::check(int status) const {
    if (status == CP_OK) return;
    std::string msg = std::string("cuplast: ") + cp_status_string(status);
    if (ctx_ && *cp_context_last_error(ctx_)) msg += std::string(": ") + cp_context_last_error(ctx_);
    throw std::runtime_error(msg);
}

void PlasticitySolver::ensureInstance() {
    if (!ctx_) check(cp_context_create(device, &ctx_));
    if (inst_) return;
    cp_mesh_view v{};
    std::vector<double> xy(2 * (size_t)mesh_.nodeCount);
    for (int i = 0; i < mesh_.nodeCount; ++i) {
        xy[2 * i] = mesh_.node[i].x;
        xy[2 * i + 1] = mesh_.node[i].y;
    }
    v.node_count = mesh_.nodeCount;
    v.node_xy = xy.data();
    v.count3 = mesh_.count3;
    v.elem3 = mesh_.elem3;
    v.count4 = mesh_.count4;
    v.elem4 = mesh_.elem4;
    v.count8 = mesh_.count8;
    v.elem8 = mesh_.elem8;
    cp_material mc = m_.toC(pc_ == stress ? CP_PLANE_STRESS : CP_PLANE_STRAIN);
    check(cp_instance_create(ctx_, &v, &mc, &inst_));
    std::vector<double> rp, uv;
    std::vector<unsigned char> mask;
    buildConditions(mesh_, cond_, m_.h, m_.rho, rp, mask, uv);
    check(cp_instance_set_loads(inst_, rp.data(), mask.data(), uv.data()));
}

double PlasticitySolver::run(bool elastic) {
    ensureInstance();
    check(cp_instance_reset_state(inst_));
    cp_solve_opts o;
    cp_solve_opts_default(&o);
    o.precision = floatBoost && !elastic ? CP_PREC_FLOAT_BOOST : CP_PREC_FP64;
    o.cg_tol = cgTol;
    o.outer_tol = outerTol;
    o.max_outer = elastic ? 1 : maxOuter;
    o.levels = elastic ? 1 : levels;
    o.aitken = aitken ? 1 : 0;
    o.adaptive_cg = adaptiveCg ? (adaptiveRule == 2 ? 2 : 1) : 0;
    o.predict = predict ? 1 : 0;
    o.precond = precond;
    o.inner_tol = innerTol;
    o.recycle = recycle;
    if (elastic) o.outer_tol = 1e300;  // one linear solve + stress update (solveElast)
    int st = cp_solve(inst_, &o, &report_);
    if (st != CP_OK && st != CP_ERR_NOT_CONVERGED) check(st);
    if (iterOutput)
        std::cout << "Iterations: " << report_.outer_iters << ", CG iterations: " << report_.cg_iters
                  << ", exit error: " << report_.rel_err << ", time: " << report_.seconds << " s" << std::endl;
    plastSolved_ = !elastic;
    return report_.seconds;
}

double PlasticitySolver::solve() { return run(false); }
double PlasticitySolver::solveElast() { return run(true); }
double PlasticitySolver::solveElastCUDA() { return run(true); }

namespace {
// Sets a flag for one call and puts the caller's value back, also when the
// call throws.
struct FlagFor {
    bool& flag;
    bool saved;
    FlagFor(bool& f, bool v) : flag(f), saved(f) { flag = v; }
    ~FlagFor() { flag = saved; }
};
}  // namespace

double PlasticitySolver::solveCUDA() {
    FlagFor f(floatBoost, false);
    return run(false);
}

double PlasticitySolver::solveCUDA_FD() {
    FlagFor f(floatBoost, true);
    return run(false);
}

std::vector<double> PlasticitySolver::field(const std::string& name) const {
    if (!inst_) throw std::logic_error("solve() first");
    int nodes = 0, elems = 0;
    cp_instance_sizes(inst_, &nodes, &elems, nullptr, nullptr);
    std::vector<double> out(name == "uv" || name == "rp" ? 2 * (size_t)nodes : (size_t)elems);
    check(cp_get_field(inst_, name.c_str(), out.data()));
    return out;
}

double PlasticitySolver::getSxx0() const { return field("sxx")[0]; }
double PlasticitySolver::getExx0() const { return field("exx")[0]; }

namespace {

// Centre of 4-node element e: the mean of its corners, as the reference's
// polar transforms and error norms take it (src/PlasticitySolver.cuh:169-200).
vec2 centre4(const Mesh& m, int e) {
    vec2 ec;
    for (int i = e * 4; i < (e + 1) * 4; ++i) ec += m.node[m.elem4[i]];
    ec /= 4;
    return ec;
}

// A symmetric tensor (xx, yy, xy) in polar components about the origin at
// point ec: _rr, _phiphi, _rphi of src/PlasticitySolver.cuh:169-200.
struct Polar {
    double rr, pp, rp;
};
Polar to_polar(vec2 ec, double x, double y, double xy) {
    const double r = ec.norm();
    const double c = ec.x / r, s = ec.y / r;
    return {c * c * x + s * s * y + 2. * c * s * xy, s * s * x + c * c * y - 2. * c * s * xy,
            c * s * (-x + y) + xy * (c * c - s * s)};
}

}  // namespace

double PlasticitySolver::sigmaError(std::function<double(vec2)> s_x, std::function<double(vec2)> s_y,
                                    std::function<double(vec2)> s_xy) const {
    const std::vector<double> sxx = field("sxx"), syy = field("syy"), tau = field("tau");
    double avrSxx = 0., avrSyy = 0., avrSxy = 0., vol = 0., maxSxx = 0., maxSyy = 0., maxSxy = 0.;
    for (int e = 0; e < mesh_.count4; ++e) {
        const int i = mesh_.count3 + e;
        const double loc = mesh_.elemSpace4(e);
        avrSxx += sxx[i] * loc;
        avrSyy += syy[i] * loc;
        avrSxy += tau[i] * loc;
        vol += loc;
        const vec2 ec = centre4(mesh_, e);
        maxSxx = std::fmax(maxSxx, std::fabs(s_x(ec) - sxx[i]));
        maxSyy = std::fmax(maxSyy, std::fabs(s_y(ec) - syy[i]));
        maxSxy = std::fmax(maxSxy, std::fabs(s_xy(ec) - tau[i]));
    }
    maxSxx *= vol / avrSxx;
    maxSyy *= vol / avrSyy;
    maxSxy *= vol / avrSxy;
    return std::fmax(std::fmax(maxSxx, maxSyy), maxSxy);
}

double PlasticitySolver::polarSigmaError(std::function<double(vec2)> s_r, std::function<double(vec2)> s_phi,
                                         std::function<double(vec2)> s_rphi, double maxR) const {
    const std::vector<double> sxx = field("sxx"), syy = field("syy"), tau = field("tau");
    const double pi = 3.141592653589793;
    double avrSrr = 0., avrSpp = 0., avrSrp = 0., vol = 0., maxSrr = 0., maxSpp = 0., maxSrp = 0.;
    for (int e = 0; e < mesh_.count4; ++e) {
        const int i = mesh_.count3 + e;
        const vec2 ec = centre4(mesh_, e);
        const vec2 r(std::sqrt(ec.x * ec.x + ec.y * ec.y), std::atan(ec.y / ec.x) + (ec.x < 0. ? pi : 0.));
        if (r.x > maxR) continue;
        const Polar p = to_polar(ec, sxx[i], syy[i], tau[i]);
        const double loc = mesh_.elemSpace4(e);
        avrSrr += std::fabs(p.rr) * loc;
        avrSpp += std::fabs(p.pp) * loc;
        avrSrp += std::fabs(p.rp) * loc;
        vol += loc;
        maxSrr = std::fmax(maxSrr, std::fabs(s_r(r) - p.rr));
        maxSpp = std::fmax(maxSpp, std::fabs(s_phi(r) - p.pp));
        maxSrp = std::fmax(maxSrp, std::fabs(s_rphi(r) - p.rp));
    }
    maxSrr *= vol / avrSrr;
    maxSpp *= vol / avrSpp;
    maxSrp *= vol / avrSrp;
    if (iterOutput) std::cout << maxSrr << " " << maxSpp << " " << maxSrp << "\n";
    return std::fmax(std::fmax(maxSrr, maxSpp), maxSrp);
}

// deformEnergy (src/PlasticitySolver.cuh:415-445): elements on the plastic
// branch integrate the diagram, except 8-node ones, for which the reference
// always takes the secant energy eps_i sig_i / 2.
double PlasticitySolver::deformEnergy() {
    std::vector<double> sI = field("sig_i"), eI = field("eps_i");
    double energy = 0.;
    const int q8 = mesh_.count3 + mesh_.count4;
    for (int e = 0; e < mesh_.elemCount(); ++e) {
        if (e >= q8) {
            energy += eI[e] * sI[e] * 0.5 * (m_.h * mesh_.elemSpace8(e - q8));
            continue;
        }
        double vol = m_.h * (e < mesh_.count3 ? mesh_.elemSpace3(e) : mesh_.elemSpace4(e - mesh_.count3));
        if (sI[e] > m_.sigmaT) {
            double ET = m_.sigmaT / m_.E;
            energy += m_.sigmaT * ET * 0.5 * vol;
            double heps = (eI[e] - ET) * 0.01;
            for (int j = 0; j < 100; ++j) energy += heps * 0.5 * (m_.f(ET + heps * j) + m_.f(ET + heps * (j + 1))) * vol;
        } else
            energy += eI[e] * sI[e] * 0.5 * vol;
    }
    return energy;
}

void PlasticitySolver::saveDisplsToFile(const std::string& fileName) {
    std::vector<double> uv = field("uv");
    std::ofstream f(fileName);
    for (int i = 0; i < mesh_.nodeCount; ++i)
        f << mesh_.node[i].x << " " << mesh_.node[i].y << " " << uv[2 * i] << " " << uv[2 * i + 1] << "\n";
}

void PlasticitySolver::saveAsVtk(const std::string& fileName) {
    std::ofstream f(fileName);
    const int ne = mesh_.elemCount();
    f << "# vtk DataFile Version 2.0\nSolution\nASCII\nDATASET POLYDATA\n";
    f << "POINTS " << mesh_.nodeCount << " float\n";
    for (int i = 0; i < mesh_.nodeCount; ++i) f << mesh_.node[i].x << " " << mesh_.node[i].y << " " << 0 << "\n";
    f << "POLYGONS " << ne << " " << 4 * mesh_.count3 + 5 * mesh_.count4 + 9 * mesh_.count8;
    for (int i = 0; i < mesh_.count3; ++i) {
        f << "\n3 ";
        for (int j = 3 * i; j < 3 * (i + 1); ++j) f << mesh_.elem3[j] << " ";
    }
    for (int i = 0; i < mesh_.count4; ++i) {
        f << "\n4 ";
        for (int j = 4 * i; j < 4 * (i + 1); ++j) f << mesh_.elem4[j] << " ";
    }
    // an 8-node element as the polygon corner, mid-side, corner, ...
    for (int i = 0; i < mesh_.count8; ++i) {
        f << "\n8 ";
        for (int j = 8 * i; j < 8 * i + 4; ++j) f << mesh_.elem8[j] << " " << mesh_.elem8[j + 4] << " ";
    }
    f << "\nCELL_DATA " << ne << "\nSCALARS ElementID int 1\nLOOKUP_TABLE default\n";
    for (int i = 0; i < ne; ++i) f << i << "\n";
    f.precision(16);
    // (name, values): Cartesian components of every element, or with
    // polarCoord the polar components of the 4-node elements about the
    // origin. As in the reference (src/PlasticitySolver.cu:1820-1925) the
    // polar strains are taken from the tensor shear gamma / 2 and written
    // under the Gamma_ names.
    std::vector<std::pair<std::string, std::vector<double>>> fields;
    auto group = [&](const char* nx, const char* ny, const char* nxy, const char* fx, const char* fy,
                     const char* fxy, double shear) {
        const std::vector<double> x = field(fx), y = field(fy), xy = field(fxy);
        if (!polarCoord) {
            fields.emplace_back(nx, x);
            fields.emplace_back(ny, y);
            fields.emplace_back(nxy, xy);
            return;
        }
        std::vector<double> rr(mesh_.count4), pp(mesh_.count4), rp(mesh_.count4);
        for (int e = 0; e < mesh_.count4; ++e) {
            const int i = mesh_.count3 + e;
            const Polar p = to_polar(centre4(mesh_, e), x[i], y[i], xy[i] * shear);
            rr[e] = p.rr;
            pp[e] = p.pp;
            rp[e] = p.rp;
        }
        std::string base(nxy);
        fields.emplace_back(std::string(nx).substr(0, std::string(nx).size() - 2) + "rr", rr);
        fields.emplace_back(std::string(ny).substr(0, std::string(ny).size() - 2) + "phiphi", pp);
        fields.emplace_back(base.substr(0, base.size() - 2) + "rphi", rp);
    };
    group("Eps_xx", "Eps_yy", "Gamma_xy", "exx", "eyy", "gamma", 0.5);
    fields.emplace_back("Eps_intensity", field("eps_i"));
    if (plastSolved_) {
        group("Eps_p_xx", "Eps_p_yy", "Gamma_p_xy", "exx_p", "eyy_p", "gamma_p", 0.5);
        fields.emplace_back("Eps_p_intensity", field("eps_p_i"));
        fields.emplace_back("Psi", field("psi"));
        fields.emplace_back("E_c", field("E_c"));
        fields.emplace_back("nu_c", field("nu_c"));
    }
    group("Sigma_xx", "Sigma_yy", "Tau_xy", "sxx", "syy", "tau", 1.0);
    fields.emplace_back("Sigma_intensity", field("sig_i"));
    f << "FIELD FieldData " << fields.size();
    for (auto& p : fields) {
        f << "\n" << p.first << " 1 " << p.second.size() << " float\n";
        for (double x : p.second) f << x << " ";
    }
    std::vector<double> uv = field("uv");
    f << "\nPOINT_DATA " << mesh_.nodeCount << "\nSCALARS NodeID int 1\nLOOKUP_TABLE my_table";
    for (int i = 0; i < mesh_.nodeCount; ++i) f << "\n" << i;
    f << "\nFIELD FieldData2 1\nDisplacement 3 " << mesh_.nodeCount << " float\n";
    for (int i = 0; i < mesh_.nodeCount; ++i) f << uv[2 * i] << " " << uv[2 * i + 1] << " 0 ";
}

// ------------------------------------------------------------ SparseSLAE --

SparseSLAE::SparseSLAE(Mesh& mesh, int dim_, int device) : dim(dim_) {
    if (dim_ != 2) throw std::invalid_argument("SparseSLAE: only dim = 2 (2D displacements) is supported");
    cp_context* ctx = nullptr;
    cp_instance* inst = nullptr;
    auto fail = [&](int st) {
        std::string msg = std::string("cuplast: ") + cp_status_string(st);
        if (ctx && *cp_context_last_error(ctx)) msg += std::string(": ") + cp_context_last_error(ctx);
        if (inst) cp_instance_destroy(inst);
        if (ctx) cp_context_destroy(ctx);
        throw std::runtime_error(msg);
    };
    int st = cp_context_create(device, &ctx);
    if (st) fail(st);
    std::vector<double> xy(2 * (size_t)mesh.nodeCount);
    for (int i = 0; i < mesh.nodeCount; ++i) {
        xy[2 * i] = mesh.node[i].x;
        xy[2 * i + 1] = mesh.node[i].y;
    }
    cp_mesh_view v{mesh.nodeCount, xy.data(), mesh.count3, mesh.elem3, mesh.count4, mesh.elem4, mesh.count8,
                   mesh.elem8};
    cp_material mat{};
    mat.E = 1.0;
    mat.nu = 0.3;
    mat.h = 1.0;
    mat.rho = 1.0;
    st = cp_instance_create(ctx, &v, &mat, &inst);
    if (st) fail(st);
    long long nnz = 0, nadj = 0;
    cp_instance_sizes(inst, nullptr, nullptr, &nnz, &nadj);
    N = 2 * mesh.nodeCount;
    rows = new int[N + 1];
    cols = new int[nnz];
    adj = new int[nadj + 1];
    adjPos = new int[mesh.nodeCount + 1];
    data = new double[nnz]();
    rp = new double[N]();
    st = cp_get_csr(inst, rows, cols, adjPos, adj, nullptr);
    if (st) fail(st);
    cp_instance_destroy(inst);
    cp_context_destroy(ctx);
}

SparseSLAE::~SparseSLAE() {
    delete[] rp;
    delete[] data;
    delete[] rows;
    delete[] cols;
    delete[] adj;
    delete[] adjPos;
}

}  // namespace cuplast
