// ibpm_gpu.cc -- the reference's solver classes, with the reference headers'
// signatures, forwarding to libibpm_b200 (include/ibpm_b200.h).
//
// Linked instead of IBSolver.o ProjectionSolver.o CholeskySolver.o
// ConjugateGradientSolver.o EllipticSolver.o EllipticSolver2d.o
// NavierStokesModel.o Regularizer.o, next to the reference's other objects
// (Grid, Geometry, State, Scalar, Flux, BaseFlow, the outputs, ...) and its
// unmodified src/ibpm.cc, it makes the reference CLI run its time step on the
// GPU.  The classes are the reference's own declarations
// (src/IBSolver.h:20-222, src/ProjectionSolver.h:54-126,
// src/CholeskySolver.h:37-79, src/ConjugateGradientSolver.h:28-57,
// src/EllipticSolver.h:26-76, src/EllipticSolver2d.h:26-100,
// src/NavierStokesModel.h:35-122, src/Regularizer.h:50-89); what each object
// needs on the device (a time-step context, an elliptic solver) lives in side
// tables keyed by the object, created on first use.
//
// Behaviour kept from the reference: advance(State&) leaves the host State
// valid after every step (omega, q, f, timestep, time); the Cholesky factors
// are read and written in the reference's .cholesky files; moving bodies use CG
// with the solver's tolerance.  The host Geometry still moves the bodies
// (NavierStokesModel::updateOperators at each sub-step time, so stateful
// motions see the reference's call sequence) and the device receives the
// points and velocities (ibg_set_step_kinematics).
// Not available: a base flow that moves (the CLI's -ubf) and grids with a
// shifted inner domain (xShift, yShift != 0) exit with a message, as the
// reference does on configuration errors; advance(State&, Bu) and a
// stand-alone advanceSubstep call exit the same way (the device step has no
// control input and runs whole steps).
// IBG_DROPIN_PRECISION=fp32_refined in the environment selects the FP32
// transforms with one FP64-residual refinement per solve.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <map>
#include <string>
#include <vector>

#include "BC.h"
#include "BaseFlow.h"
#include "CholeskySolver.h"
#include "ConjugateGradientSolver.h"
#include "EllipticSolver.h"
#include "EllipticSolver2d.h"
#include "Geometry.h"
#include "IBSolver.h"
#include "NavierStokesModel.h"
#include "ProjectionSolver.h"
#include "Regularizer.h"
#include "State.h"
#include "VectorOperations.h"
#include "ibpm_b200.h"

namespace ibpm {

namespace {

[[noreturn]] void die(const std::string& m) {
    std::cerr << "ibpm_b200: " << m << std::endl;
    exit(1);
}
void check(int status, ibg_context* ctx, const char* where) {
    if (status < 0) die(std::string(where) + ": " + ibg_last_error(ctx));
}

// --- reference containers <-> the device layouts (which are the reference's own) ---
std::vector<double> pack(const Scalar& s) {
    const Grid& g = s.getGrid();
    std::vector<double> v((size_t)g.Ngrid() * (g.Nx() - 1) * (g.Ny() - 1));
    size_t k = 0;
    for (int lev = 0; lev < g.Ngrid(); ++lev)
        for (int i = 1; i < g.Nx(); ++i)
            for (int j = 1; j < g.Ny(); ++j) v[k++] = s(lev, i, j);
    return v;
}
void unpack(const std::vector<double>& v, Scalar& s) {
    const Grid& g = s.getGrid();
    size_t k = 0;
    for (int lev = 0; lev < g.Ngrid(); ++lev)
        for (int i = 1; i < g.Nx(); ++i)
            for (int j = 1; j < g.Ny(); ++j) s(lev, i, j) = v[k++];
}
std::vector<double> pack(const Flux& q) {
    const int L = q.getGrid().Ngrid();
    const size_t n = (size_t)q.end();
    std::vector<double> v(L * n);
    for (int lev = 0; lev < L; ++lev)
        for (Flux::index i = q.begin(); i != q.end(); ++i) v[lev * n + i] = q(lev, i);
    return v;
}
void unpack(const std::vector<double>& v, Flux& q) {
    const int L = q.getGrid().Ngrid();
    const size_t n = (size_t)q.end();
    for (int lev = 0; lev < L; ++lev)
        for (Flux::index i = q.begin(); i != q.end(); ++i) q(lev, i) = v[lev * n + i];
}
std::vector<double> pack(const BoundaryVector& b) {
    std::vector<double> v((size_t)b.end());
    for (BoundaryVector::index i = b.begin(); i != b.end(); ++i) v[i] = b(i);
    return v;
}
void unpack(const std::vector<double>& v, BoundaryVector& b) {
    for (BoundaryVector::index i = b.begin(); i != b.end(); ++i) b(i) = v[i];
}

ibg_grid grid_desc(const Grid& g) {
    // the device nests the inner domains without shift, as the CLI's default xshift = yshift = 0
    if (g.NxExt() != (int)floor(g.Nx() / 4 + 0.5) || g.NyExt() != (int)floor(g.Ny() / 4 + 0.5))
        die("grids with a shifted inner domain are not supported");
    ibg_grid d;
    d.nx = g.Nx();
    d.ny = g.Ny();
    d.ngrid = g.Ngrid();
    d.length = g.Nx() * g.Dx();
    d.xoffset = g.getXEdge(0, 0);
    d.yoffset = g.getYEdge(0, 0);
    return d;
}

int precision_from_env() {
    const char* p = getenv("IBG_DROPIN_PRECISION");
    if (!p || !*p || !strcmp(p, "fp64")) return IBG_PRECISION_FP64;
    if (!strcmp(p, "fp32_refined")) return IBG_PRECISION_FP32_REFINED;
    if (!strcmp(p, "fp32")) return IBG_PRECISION_FP32;
    die(std::string("IBG_DROPIN_PRECISION must be fp64, fp32_refined or fp32, not ") + p);
}

// what a model needs to build device contexts
struct ModelInfo {
    const Grid* grid = nullptr;
    const Geometry* geom = nullptr;
    const BaseFlow* baseflow = nullptr;  // nullptr: no base flow (the linear models)
    double Re = 1.0;
    ibg_context* ops = nullptr;           // operator context (B, C, refreshState, regularizer)
};
std::map<const NavierStokesModel*, ModelInfo> g_models;
std::map<const Geometry*, const NavierStokesModel*> g_model_of_geometry;

// the bodies at their current positions, as one device body that the device does not move
ibg_context* make_context(const ModelInfo& m, double dt, int scheme, double tol, int precision) {
    const Geometry& geo = *m.geom;
    const int n = geo.getNumPoints();
    if (n < 1) die("the geometry has no boundary points");
    if (m.baseflow && !m.baseflow->isStationary()) die("a moving base flow (-ubf) is not supported");
    BoundaryVector pts = geo.getPoints();
    std::vector<double> xy(2 * (size_t)n);
    for (int p = 0; p < n; ++p) {
        xy[2 * p] = pts(X, p);
        xy[2 * p + 1] = pts(Y, p);
    }
    ibg_body body{};
    body.npoints = n;
    body.xy = xy.data();
    body.motion = IBG_MOTION_NONE;
    ibg_params prm{};
    prm.Re = m.Re;
    prm.dt = dt;
    prm.scheme = scheme;
    prm.cg_tol = tol;
    prm.cg_max_iter = 0;
    prm.u_mag = m.baseflow ? m.baseflow->getMag() : 0.0;
    prm.alpha = m.baseflow ? m.baseflow->getAlpha() : 0.0;
    prm.precision = precision;
    prm.device = -1;
    prm.cg_precond = IBG_PRECOND_NONE;
    prm.pc_refresh = 0;
    prm.cg_graph = 1;
    prm.pc_fallback_iter = 0;
    const ibg_grid gd = grid_desc(*m.grid);
    ibg_context* ctx = nullptr;
    if (ibg_create(&gd, 1, &body, &prm, nullptr, &ctx) < 0) die(ibg_last_error(nullptr));
    if (!geo.isStationary()) {
        check(ibg_set_external_kinematics(ctx), ctx, "ibg_set_external_kinematics");
        BoundaryVector vel = geo.getVelocities();
        check(ibg_set_step_kinematics(ctx, -1, pack(pts).data(), pack(vel).data()), ctx, "ibg_set_step_kinematics");
    }
    return ctx;
}

// the device regularizer at the host Geometry's current configuration
void sync_bodies(ibg_context* ctx, const Geometry& geo) {
    if (geo.isStationary()) return;
    BoundaryVector pts = geo.getPoints(), vel = geo.getVelocities();
    check(ibg_set_step_kinematics(ctx, -1, pack(pts).data(), pack(vel).data()), ctx, "ibg_set_step_kinematics");
}

ibg_context* model_ops(const NavierStokesModel* model) {
    auto it = g_models.find(model);
    if (it == g_models.end()) die("NavierStokesModel used before construction");
    ModelInfo& m = it->second;
    if (!m.ops) m.ops = make_context(m, 1.0, IBG_SCHEME_EULER, 1e-7, IBG_PRECISION_FP64);
    sync_bodies(m.ops, *m.geom);
    return m.ops;
}

// per time stepper: its device context and the variant data handed to it
struct SolverInfo {
    const NavierStokesModel* model = nullptr;
    ibg_context* ctx = nullptr;
    int scheme = IBG_SCHEME_RK3;
    double dt = 0.0;
    bool variant_set = false;
};
std::map<const IBSolver*, SolverInfo> g_solvers;

int scheme_of(Scheme::SchemeType s) {
    switch (s) {
        case Scheme::EULER: return IBG_SCHEME_EULER;
        case Scheme::AB2: return IBG_SCHEME_AB2;
        case Scheme::RK3: return IBG_SCHEME_RK3;
        case Scheme::RK3b: return IBG_SCHEME_RK3B;
    }
    return IBG_SCHEME_RK3;
}

}  // namespace

// ===========================================================================
// NavierStokesModel (src/NavierStokesModel.h:35-122)
// ===========================================================================
NavierStokesModel::NavierStokesModel(const Grid& grid, const Geometry& geometry, double Reynolds,
                                     const BaseFlow& q_potential)
    : _grid(grid), _geometry(geometry), _regularizer(grid, geometry), _baseFlow(q_potential),
      _ReynoldsNumber(Reynolds), _poisson(grid), _hasBeenInitialized(false) {
    ModelInfo& m = g_models[this];
    m.grid = &_grid;
    m.geom = &_geometry;
    m.baseflow = &_baseFlow;
    m.Re = Reynolds;
    g_model_of_geometry[&geometry] = this;
}

NavierStokesModel::NavierStokesModel(const Grid& grid, const Geometry& geometry, double Reynolds)
    : _grid(grid), _geometry(geometry), _regularizer(grid, geometry), _baseFlow(grid), _ReynoldsNumber(Reynolds),
      _poisson(grid), _hasBeenInitialized(false) {
    _baseFlow.setFlux(0.);
    ModelInfo& m = g_models[this];
    m.grid = &_grid;
    m.geom = &_geometry;
    m.baseflow = nullptr;
    m.Re = Reynolds;
    g_model_of_geometry[&geometry] = this;
}

NavierStokesModel::~NavierStokesModel() {
    auto it = g_models.find(this);
    if (it != g_models.end()) {
        if (it->second.ops) ibg_destroy(it->second.ops);
        g_models.erase(it);
    }
    g_model_of_geometry.erase(&_geometry);
}

void NavierStokesModel::init() { _hasBeenInitialized = true; }
bool NavierStokesModel::isTimeDependent() const { return !_geometry.isStationary() || !_baseFlow.isStationary(); }
bool NavierStokesModel::geTimeDependent() const { return !_geometry.isStationary(); }
bool NavierStokesModel::bfTimeDependent() const { return !_baseFlow.isStationary(); }
int NavierStokesModel::getNumPoints() const { return _geometry.getNumPoints(); }
double NavierStokesModel::getAlpha() const { return 1. / _ReynoldsNumber; }

BoundaryVector NavierStokesModel::getConstraints() const {
    // body velocities minus the base flow at the boundary points
    BoundaryVector b = _geometry.getVelocities();
    b -= getBaseFlowBoundaryVelocities();
    return b;
}

BoundaryVector NavierStokesModel::getBaseFlowBoundaryVelocities() const {
    return _regularizer.toBoundary(_baseFlow.getFlux());
}

void NavierStokesModel::updateOperators(double time) {
    if (bfTimeDependent()) die("a moving base flow (-ubf) is not supported");
    if (geTimeDependent()) {
        _geometry.moveBodies(time);
        auto it = g_models.find(this);
        if (it != g_models.end() && it->second.ops) sync_bodies(it->second.ops, _geometry);
    }
}

void NavierStokesModel::B(const BoundaryVector& f, Scalar& omega) const {
    ibg_context* ctx = model_ops(this);
    std::vector<double> w((size_t)_grid.Ngrid() * (_grid.Nx() - 1) * (_grid.Ny() - 1));
    check(ibg_model_B(ctx, pack(f).data(), w.data()), ctx, "NavierStokesModel::B");
    unpack(w, omega);
}

void NavierStokesModel::C(const Scalar& omega, BoundaryVector& f) const {
    ibg_context* ctx = model_ops(this);
    std::vector<double> out((size_t)f.end());
    check(ibg_model_C(ctx, pack(omega).data(), out.data()), ctx, "NavierStokesModel::C");
    unpack(out, f);
}

void NavierStokesModel::computeFluxWithoutBaseFlow(const Scalar& omega, Flux& q) const {
    Scalar psi = vorticityToStreamfunction(omega);
    Curl(psi, q);
}

void NavierStokesModel::computeFlux(const Scalar& omega, Flux& q) const {
    // q = Curl(L^-1(-omega)) + q0 on the device (model->refreshState)
    ibg_context* ctx = model_ops(this);
    long long ns = 0, nf = 0;
    int nb = 0;
    ibg_sizes(ctx, &ns, &nf, &nb);
    std::vector<double> w = pack(omega), qq((size_t)nf), f((size_t)nb, 0.0);
    check(ibg_set_state(ctx, w.data(), nullptr, f.data(), 0, 0.0), ctx, "NavierStokesModel::computeFlux");
    int ts = 0;
    double t = 0.0;
    check(ibg_get_state(ctx, nullptr, qq.data(), nullptr, &ts, &t), ctx, "NavierStokesModel::computeFlux");
    unpack(qq, q);
}

void NavierStokesModel::refreshState(State& x) const { computeFlux(x.omega, x.q); }

Scalar NavierStokesModel::vorticityToStreamfunction(const Scalar& omega) const {
    ibg_context* ctx = model_ops(this);
    std::vector<double> f = pack(omega), u(f.size());
    for (double& v : f) v = -v;
    check(ibg_poisson_solve(ctx, f.data(), u.data()), ctx, "NavierStokesModel::vorticityToStreamfunction");
    Scalar psi(_grid);
    unpack(u, psi);
    return psi;
}

// ===========================================================================
// Regularizer (src/Regularizer.h:50-89): the device regularizer of the model
// that owns the geometry
// ===========================================================================
Regularizer::Regularizer(const Grid& grid, const Geometry& geometry) : _grid(grid), _geometry(geometry) {}

void Regularizer::update() {}

Flux Regularizer::toFlux(const BoundaryVector& u) const {
    auto it = g_model_of_geometry.find(&_geometry);
    if (it == g_model_of_geometry.end()) die("Regularizer without a NavierStokesModel");
    ibg_context* ctx = model_ops(it->second);
    Flux q(_grid);
    std::vector<double> out((size_t)_grid.Ngrid() * q.end());
    check(ibg_reg_to_flux(ctx, pack(u).data(), out.data()), ctx, "Regularizer::toFlux");
    unpack(out, q);
    return q;
}

BoundaryVector Regularizer::toBoundary(const Flux& q) const {
    auto it = g_model_of_geometry.find(&_geometry);
    if (it == g_model_of_geometry.end()) die("Regularizer without a NavierStokesModel");
    ibg_context* ctx = model_ops(it->second);
    BoundaryVector f(_geometry.getNumPoints());
    std::vector<double> qq = pack(q), out((size_t)f.end());
    check(ibg_reg_to_boundary(ctx, qq.data(), out.data()), ctx, "Regularizer::toBoundary");
    unpack(out, f);
    return f;
}

// ===========================================================================
// EllipticSolver, PoissonSolver, HelmholtzSolver (src/EllipticSolver.h:26-76)
// ===========================================================================
namespace {
struct EllipticInfo {
    ibg_grid grid{};
    int helmholtz = 0;
    double alpha = 0.0;
    ibg_elliptic* h = nullptr;
};
std::map<const void*, EllipticInfo> g_elliptic;

ibg_elliptic* elliptic_handle(const void* key) {
    EllipticInfo& e = g_elliptic[key];
    if (!e.h && ibg_elliptic_create(&e.grid, e.helmholtz, e.alpha, nullptr, &e.h) < 0)
        die(std::string("ibg_elliptic_create: ") + ibg_elliptic_last_error(nullptr));
    return e.h;
}
void elliptic_release(const void* key) {
    auto it = g_elliptic.find(key);
    if (it == g_elliptic.end()) return;
    if (it->second.h) ibg_elliptic_destroy(it->second.h);
    g_elliptic.erase(it);
}
}  // namespace

EllipticSolver::EllipticSolver(const Grid& grid) : _ngrid(grid.Ngrid()), _dx(grid.Dx()) {
    g_elliptic[this].grid = grid_desc(grid);
}
EllipticSolver::~EllipticSolver() { elliptic_release(this); }
void EllipticSolver::init() { elliptic_handle(this); }

void EllipticSolver::solve(const Scalar& f, Scalar& u) const {
    ibg_elliptic* h = elliptic_handle(this);
    std::vector<double> in = pack(f), out(in.size());
    if (ibg_elliptic_solve(h, in.data(), out.data()) < 0)
        die(std::string("EllipticSolver::solve: ") + ibg_elliptic_last_error(h));
    unpack(out, u);
}

Scalar EllipticSolver::solve(const Scalar& f) const {
    Scalar u(f.getGrid());
    solve(f, u);
    return u;
}

PoissonSolver::PoissonSolver(const Grid& grid) : EllipticSolver(grid), _nx(grid.Nx()), _ny(grid.Ny()) {
    g_elliptic[this].helmholtz = 0;
}
EllipticSolver2d* PoissonSolver::create2dSolver(double dx) { return new PoissonSolver2d(_nx, _ny, dx); }

HelmholtzSolver::HelmholtzSolver(const Grid& grid, double alpha)
    : EllipticSolver(grid), _nx(grid.Nx()), _ny(grid.Ny()), _alpha(alpha) {
    g_elliptic[this].helmholtz = 1;
    g_elliptic[this].alpha = alpha;
}
EllipticSolver2d* HelmholtzSolver::create2dSolver(double dx) { return new HelmholtzSolver2d(_nx, _ny, dx, _alpha); }

// ===========================================================================
// EllipticSolver2d, PoissonSolver2d, HelmholtzSolver2d (src/EllipticSolver2d.h:26-100):
// one level of nx x ny cells of size dx on the device; boundary values enter
// through getRHS as in the reference (src/EllipticSolver2d.cc:125-185)
// ===========================================================================
EllipticSolver2d::EllipticSolver2d(int nx, int ny, double dx) : _nx(nx), _ny(ny), _dx(dx), _FFTWPlan(nullptr) {
    EllipticInfo& e = g_elliptic[this];
    e.grid.nx = nx;
    e.grid.ny = ny;
    e.grid.ngrid = 1;
    e.grid.length = nx * dx;
    e.grid.xoffset = 0.0;
    e.grid.yoffset = 0.0;
}
EllipticSolver2d::~EllipticSolver2d() { elliptic_release(this); }

void EllipticSolver2d::solve(const Array2d& f, Array2d& u) const {
    ibg_elliptic* h = elliptic_handle(this);
    std::vector<double> in((size_t)(_nx - 1) * (_ny - 1)), out(in.size());
    size_t k = 0;
    for (int i = 1; i < _nx; ++i)
        for (int j = 1; j < _ny; ++j) in[k++] = f(i, j);
    if (ibg_elliptic_solve(h, in.data(), out.data()) < 0)
        die(std::string("EllipticSolver2d::solve: ") + ibg_elliptic_last_error(h));
    k = 0;
    for (int i = 1; i < _nx; ++i)
        for (int j = 1; j < _ny; ++j) u(i, j) = out[k++];
}

void EllipticSolver2d::solve(const Array2d& f, const BC& bc, Array2d& u) const {
    Array2d rhs(_nx - 1, _ny - 1, 1, 1);
    getRHS(f, bc, rhs);
    solve(rhs, u);
}

EllipticSolver2d::Array2d EllipticSolver2d::getLaplacianEigenvalues() const {
    // the 5-point Laplacian's Dirichlet eigenvalues (src/EllipticSolver2d.cc:42-54)
    Array2d eig(_nx - 1, _ny - 1, 1, 1);
    const double pi = 4. * atan(1.);
    for (int i = 1; i < _nx; ++i)
        for (int j = 1; j < _ny; ++j)
            eig(i, j) = 2. * (cos(pi * i / _nx) + cos(pi * j / _ny) - 2.) / (_dx * _dx);
    return eig;
}

PoissonSolver2d::PoissonSolver2d(int nx, int ny, double dx) : EllipticSolver2d(nx, ny, dx) {
    g_elliptic[this].helmholtz = 0;
}

// the right-hand side minus the boundary values' part of the Laplacian:
// coef = 1 / dx^2 (Poisson) or alpha / dx^2 (Helmholtz)
static void lift_boundary(const EllipticSolver2d::Array2d& f, const BC& bc, EllipticSolver2d::Array2d& rhs, int nx,
                          int ny, double coef) {
    for (int i = 1; i < nx; ++i)
        for (int j = 1; j < ny; ++j) rhs(i, j) = f(i, j);
    for (int i = 1; i < nx; ++i) {
        rhs(i, 1) -= bc.bottom(i) * coef;
        rhs(i, ny - 1) -= bc.top(i) * coef;
    }
    for (int j = 1; j < ny; ++j) {
        rhs(1, j) -= bc.left(j) * coef;
        rhs(nx - 1, j) -= bc.right(j) * coef;
    }
}

void PoissonSolver2d::getRHS(const Array2d& f, const BC& bc, Array2d& rhs) const {
    lift_boundary(f, bc, rhs, _nx, _ny, 1. / (_dx * _dx));
}

HelmholtzSolver2d::HelmholtzSolver2d(int nx, int ny, double dx, double alpha)
    : EllipticSolver2d(nx, ny, dx), _alpha(alpha) {
    g_elliptic[this].helmholtz = 1;
    g_elliptic[this].alpha = alpha;
}

void HelmholtzSolver2d::getRHS(const Array2d& f, const BC& bc, Array2d& rhs) const {
    lift_boundary(f, bc, rhs, _nx, _ny, _alpha / (_dx * _dx));
}

// ===========================================================================
// ProjectionSolver, CholeskySolver, ConjugateGradientSolver
// (src/ProjectionSolver.h:54-126): a device context with one Euler sub-step of
// time step beta, so that its projection is A = 1 - (beta / 2 Re) L, B = beta B
// ===========================================================================
namespace {
struct ProjectionInfo {
    const NavierStokesModel* model = nullptr;
    double beta = 0.0;
    double tol = 1e-7;
    ibg_context* ctx = nullptr;
};
std::map<const ProjectionSolver*, ProjectionInfo> g_projection;

ibg_context* projection_ctx(const ProjectionSolver* p) {
    ProjectionInfo& pi = g_projection[p];
    if (!pi.ctx) {
        auto it = g_models.find(pi.model);
        if (it == g_models.end()) die("ProjectionSolver without a NavierStokesModel");
        pi.ctx = make_context(it->second, pi.beta, IBG_SCHEME_EULER, pi.tol, IBG_PRECISION_FP64);
    }
    auto it = g_models.find(pi.model);
    if (it != g_models.end()) sync_bodies(pi.ctx, *it->second.geom);
    return pi.ctx;
}
// Scalar values on the grid of a projection solver's model
size_t scalar_size(const ProjectionSolver* p) {
    const Grid& g = *g_models[g_projection[p].model].grid;
    return (size_t)g.Ngrid() * (g.Nx() - 1) * (g.Ny() - 1);
}
bool rename_file(const std::string& from, const std::string& to) { return std::rename(from.c_str(), to.c_str()) == 0; }
bool copy_file(const std::string& from, const std::string& to) {
    FILE* a = fopen(from.c_str(), "rb");
    if (!a) return false;
    FILE* b = fopen(to.c_str(), "wb");
    if (!b) {
        fclose(a);
        return false;
    }
    char buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), a)) > 0) fwrite(buf, 1, n, b);
    fclose(a);
    fclose(b);
    return true;
}
}  // namespace

ProjectionSolver::ProjectionSolver(const Grid& grid, const NavierStokesModel& model, double beta)
    : _beta(beta), _grid(grid), _model(model), _helmholtz(grid, -beta / 2. * model.getAlpha()) {
    ProjectionInfo& pi = g_projection[this];
    pi.model = &model;
    pi.beta = beta;
}
ProjectionSolver::~ProjectionSolver() {
    auto it = g_projection.find(this);
    if (it != g_projection.end()) {
        if (it->second.ctx) ibg_destroy(it->second.ctx);
        g_projection.erase(it);
    }
}
void ProjectionSolver::init() {}
bool ProjectionSolver::save(const std::string&) { return false; }
bool ProjectionSolver::load(const std::string&) { return false; }

void ProjectionSolver::solve(const Scalar& a, const BoundaryVector& b, Scalar& omega, BoundaryVector& f) {
    ibg_context* ctx = projection_ctx(this);
    std::vector<double> aa = pack(a), bb = pack(b), w(aa.size()), ff = pack(f);
    check(ibg_projection_solve(ctx, 0, aa.data(), bb.data(), w.data(), ff.data()), ctx, "ProjectionSolver::solve");
    unpack(w, omega);
    unpack(ff, f);
}

void ProjectionSolver::Ainv(const Scalar& b, Scalar& y) {
    ibg_context* ctx = projection_ctx(this);
    std::vector<double> in = pack(b), out(in.size());
    check(ibg_helmholtz_solve(ctx, -_beta / 2. * _model.getAlpha(), in.data(), out.data()), ctx,
          "ProjectionSolver::Ainv");
    unpack(out, y);
}

void ProjectionSolver::B(const BoundaryVector& f, Scalar& y) {
    _model.B(f, y);
    y *= _beta;
}

void ProjectionSolver::C(const Scalar& x, BoundaryVector& y) { _model.C(x, y); }

void ProjectionSolver::M(const BoundaryVector& f, BoundaryVector& y) {
    Scalar t(_grid);
    B(f, t);
    Ainv(t, t);
    C(t, y);
}

BoundaryVector ProjectionSolver::M(const BoundaryVector& f) {
    BoundaryVector y(f.getNumPoints());
    M(f, y);
    return y;
}

CholeskySolver::CholeskySolver(const Grid& grid, const NavierStokesModel& model, double beta)
    : ProjectionSolver(grid, model, beta), _numPoints(model.getNumPoints()), _size(2 * model.getNumPoints()),
      _alphaBeta(model.getAlpha() * beta), _hasBeenInitialized(false) {}
CholeskySolver::~CholeskySolver() {}

void CholeskySolver::init() {
    ibg_context* ctx = projection_ctx(this);
    check(ibg_init(ctx), ctx, "CholeskySolver::init");
    _hasBeenInitialized = true;
}

// <basename>.cholesky in the reference's format (src/CholeskySolver.cc:113-198);
// the device writes <basename>_01.cholesky for its one sub-step
bool CholeskySolver::save(const std::string& basename) {
    ibg_context* ctx = projection_ctx(this);
    if (ibg_save(ctx, basename.c_str()) != 1) return false;
    return rename_file(basename + "_01.cholesky", basename + ".cholesky");
}

bool CholeskySolver::load(const std::string& basename) {
    ibg_context* ctx = projection_ctx(this);
    const std::string tmp = basename + "_01.cholesky";
    if (!copy_file(basename + ".cholesky", tmp)) return false;
    const int s = ibg_load(ctx, basename.c_str());
    std::remove(tmp.c_str());
    _hasBeenInitialized = (s == 1);
    return s == 1;
}

// x = M^-1 b: the projection with a = 0 gives f = M^-1 (C 0 - b) = -M^-1 b
void CholeskySolver::Minv(const BoundaryVector& b, BoundaryVector& x) {
    ibg_context* ctx = projection_ctx(this);
    std::vector<double> zero(scalar_size(this), 0.0), w(zero.size());
    std::vector<double> bb = pack(b), ff((size_t)x.end(), 0.0);
    check(ibg_projection_solve(ctx, 0, zero.data(), bb.data(), w.data(), ff.data()), ctx, "CholeskySolver::Minv");
    for (double& v : ff) v = -v;
    unpack(ff, x);
}

ConjugateGradientSolver::ConjugateGradientSolver(const Grid& grid, const NavierStokesModel& model, double beta,
                                                 double tolerance)
    : ProjectionSolver(grid, model, beta), _toleranceSquared(tolerance * tolerance) {
    g_projection[this].tol = tolerance;
}

// CG from the warm start x (src/ConjugateGradientSolver.cc:35-65), on the device
void ConjugateGradientSolver::Minv(const BoundaryVector& b, BoundaryVector& x) {
    ibg_context* ctx = projection_ctx(this);
    std::vector<double> zero(scalar_size(this), 0.0), w(zero.size());
    std::vector<double> bb = pack(b), ff = pack(x);
    for (double& v : ff) v = -v;
    check(ibg_projection_solve(ctx, 0, zero.data(), bb.data(), w.data(), ff.data()), ctx,
          "ConjugateGradientSolver::Minv");
    for (double& v : ff) v = -v;
    unpack(ff, x);
}

// ===========================================================================
// IBSolver and its subclasses (src/IBSolver.h:20-222)
// ===========================================================================
namespace {
SolverInfo& solver_info(const IBSolver* s) { return g_solvers[s]; }
}  // namespace

IBSolver::IBSolver(const Grid& grid, NavierStokesModel& model, double dt, Scheme::SchemeType scheme)
    : _grid(grid), _scheme(scheme), _name(_scheme.name()), _dt(dt), _model(model), _Nprev(grid), _Ntemp(grid),
      _oldSaved(false), _solver(), _tol(1e-7) {
    SolverInfo& si = solver_info(this);
    si.model = &model;
    si.scheme = scheme_of(scheme);
    si.dt = dt;
}

IBSolver::IBSolver(const Grid& grid, NavierStokesModel& model, double dt, Scheme::SchemeType scheme, double tol)
    : _grid(grid), _scheme(scheme), _name(_scheme.name()), _dt(dt), _model(model), _Nprev(grid), _Ntemp(grid),
      _oldSaved(false), _solver(), _tol(tol) {
    SolverInfo& si = solver_info(this);
    si.model = &model;
    si.scheme = scheme_of(scheme);
    si.dt = dt;
}

IBSolver::~IBSolver() {
    auto it = g_solvers.find(this);
    if (it != g_solvers.end()) {
        if (it->second.ctx) ibg_destroy(it->second.ctx);
        g_solvers.erase(it);
    }
}

namespace {
ibg_context* solver_ctx(const IBSolver* s, double tol) {
    SolverInfo& si = solver_info(s);
    if (!si.ctx) {
        auto it = g_models.find(si.model);
        if (it == g_models.end()) die("IBSolver without a NavierStokesModel");
        std::cerr << (it->second.geom->isStationary() ? "Using Cholesky solver for projection step (GPU)"
                                                      : "Using ConjugateGradient solver for projection step (GPU)")
                  << std::endl;
        si.ctx = make_context(it->second, si.dt, si.scheme, tol, precision_from_env());
    }
    return si.ctx;
}
}  // namespace

void IBSolver::init() {
    ibg_context* ctx = solver_ctx(this, _tol);
    check(ibg_init(ctx), ctx, "IBSolver::init");
}

void IBSolver::reset() { _oldSaved = false; }

bool IBSolver::load(const string& basename) {
    ibg_context* ctx = solver_ctx(this, _tol);
    return ibg_load(ctx, basename.c_str()) == 1;
}

bool IBSolver::save(const string& basename) {
    ibg_context* ctx = solver_ctx(this, _tol);
    return ibg_save(ctx, basename.c_str()) == 1;
}

string IBSolver::getName() { return _name; }
double IBSolver::getTimestep() { return _dt; }

void IBSolver::setTol(double tol) {
    _tol = tol;
    // the next use builds the device context with the new tolerance
    SolverInfo& si = solver_info(this);
    if (si.ctx) ibg_destroy(si.ctx);
    si.ctx = nullptr;
    si.variant_set = false;
}

ProjectionSolver* IBSolver::createSolver(double beta) {
    if (_model.geTimeDependent()) return new ConjugateGradientSolver(_grid, _model, beta, _tol);
    return new CholeskySolver(_grid, _model, beta);
}
void IBSolver::createAllSolvers() {
    for (size_t i = 0; i < _solver.size(); ++i) _solver[i] = createSolver((_scheme.an(i) + _scheme.bn(i)) * _dt);
}
void IBSolver::deleteAllSolvers() {
    for (ProjectionSolver* p : _solver) delete p;
    _solver.clear();
}

// One whole step on the device: the host State goes up, the step runs, and
// omega, q, f, timestep and time come back (src/IBSolver.cc:142-149).
void IBSolver::advance(State& x) {
    ibg_context* ctx = solver_ctx(this, _tol);
    SolverInfo& si = solver_info(this);
    if (!si.variant_set) {
        // the variants hand the device their base states or filter through N
        N(x);
        si.variant_set = true;
    }
    std::vector<double> w = pack(x.omega), q = pack(x.q), f = pack(x.f);
    check(ibg_set_state(ctx, w.data(), q.data(), f.data(), x.timestep, x.time), ctx, "IBSolver::advance");
    if (_model.geTimeDependent()) {
        // the host Geometry moves to each sub-step time (NavierStokesModel::updateOperators)
        for (int k = 0; k < _scheme.nsteps(); ++k) {
            _model.updateOperators(x.time + _scheme.cn(k) * _dt);
            const Geometry* geo = g_models[&_model].geom;
            BoundaryVector pts = geo->getPoints(), vel = geo->getVelocities();
            check(ibg_set_step_kinematics(ctx, k, pack(pts).data(), pack(vel).data()), ctx, "IBSolver::advance");
        }
    }
    check(ibg_advance(ctx, 1), ctx, "IBSolver::advance");
    int ts = 0;
    double t = 0.0;
    check(ibg_get_state(ctx, w.data(), q.data(), f.data(), &ts, &t), ctx, "IBSolver::advance");
    unpack(w, x.omega);
    unpack(q, x.q);
    unpack(f, x.f);
    x.timestep = ts;
    x.time = t;
    _oldSaved = true;
}

void IBSolver::advance(State&, const Scalar&) { die("advance(State&, Bu): the device step has no control input"); }

void IBSolver::advanceSubstep(State&, const Scalar&, int) {
    die("advanceSubstep: the device runs whole steps (use advance)");
}

// N(x) of each model on the device.  The first evaluation also hands the device
// the base state (linearized models) or the filter (SFD) that its own steps use.
Scalar NonlinearIBSolver::N(const State& x) const {
    ibg_context* ctx = solver_ctx(this, _tol);
    std::vector<double> out((size_t)_grid.Ngrid() * (_grid.Nx() - 1) * (_grid.Ny() - 1));
    check(ibg_nonlinear(ctx, pack(x.q).data(), pack(x.omega).data(), out.data()), ctx, "NonlinearIBSolver::N");
    Scalar g(_grid);
    unpack(out, g);
    return g;
}

namespace {
// Curl(CrossProduct(q1, w1)) + Curl(CrossProduct(q2, w2)) on the device
Scalar linear_N(ibg_context* ctx, const Grid& grid, const State& a, const State& b) {
    const size_t n = (size_t)grid.Ngrid() * (grid.Nx() - 1) * (grid.Ny() - 1);
    std::vector<double> g1(n), g2(n);
    check(ibg_nonlinear(ctx, pack(a.q).data(), pack(b.omega).data(), g1.data()), ctx, "N");
    check(ibg_nonlinear(ctx, pack(b.q).data(), pack(a.omega).data(), g2.data()), ctx, "N");
    for (size_t k = 0; k < n; ++k) g1[k] += g2[k];
    Scalar g(grid);
    unpack(g1, g);
    return g;
}
}  // namespace

Scalar LinearizedIBSolver::N(const State& x) const {
    ibg_context* ctx = solver_ctx(this, _tol);
    if (!g_solvers[this].variant_set)
        check(ibg_set_linearized(ctx, 1, pack(_x0.omega).data(), pack(_x0.q).data()), ctx, "ibg_set_linearized");
    return linear_N(ctx, _grid, _x0, x);
}

Scalar LinearizedPeriodicIBSolver::N(const State& x) const {
    ibg_context* ctx = solver_ctx(this, _tol);
    if (!g_solvers[this].variant_set) {
        std::vector<double> w, q;
        for (int k = 0; k < _period; ++k) {
            std::vector<double> wk = pack(_x0periodic[k].omega), qk = pack(_x0periodic[k].q);
            w.insert(w.end(), wk.begin(), wk.end());
            q.insert(q.end(), qk.begin(), qk.end());
        }
        check(ibg_set_linearized(ctx, _period, w.data(), q.data()), ctx, "ibg_set_linearized");
    }
    return linear_N(ctx, _grid, _x0periodic[x.timestep % _period], x);
}

Scalar AdjointIBSolver::N(const State& x) const {
    ibg_context* ctx = solver_ctx(this, _tol);
    if (!g_solvers[this].variant_set)
        check(ibg_set_adjoint(ctx, pack(_x0.omega).data(), pack(_x0.q).data()), ctx, "ibg_set_adjoint");
    // Laplacian(CrossProduct(q0, q)) - Curl(CrossProduct(q, omega0)): the flux-flux
    // cross product is the reference's host operator, the rest runs on the device
    const size_t n = (size_t)_grid.Ngrid() * (_grid.Nx() - 1) * (_grid.Ny() - 1);
    Scalar c = CrossProduct(_x0.q, x.q);
    std::vector<double> lap(n), cur(n);
    check(ibg_laplacian(ctx, pack(c).data(), lap.data()), ctx, "AdjointIBSolver::N");
    check(ibg_nonlinear(ctx, pack(x.q).data(), pack(_x0.omega).data(), cur.data()), ctx, "AdjointIBSolver::N");
    for (size_t k = 0; k < n; ++k) lap[k] -= cur[k];
    Scalar g(_grid);
    unpack(lap, g);
    return g;
}

Scalar SFDSolver::N(const State& x) const {
    ibg_context* ctx = solver_ctx(this, _tol);
    if (!g_solvers[this].variant_set)
        check(ibg_set_sfd(ctx, _chi, _Delta, pack(_xhat.omega).data()), ctx, "ibg_set_sfd");
    const size_t n = (size_t)_grid.Ngrid() * (_grid.Nx() - 1) * (_grid.Ny() - 1);
    std::vector<double> g(n), w = pack(x.omega), wh(n);
    check(ibg_nonlinear(ctx, pack(x.q).data(), w.data(), g.data()), ctx, "SFDSolver::N");
    check(ibg_get_sfd_state(ctx, wh.data()), ctx, "SFDSolver::N");
    for (size_t k = 0; k < n; ++k) g[k] -= _chi * (w[k] - wh[k]);
    Scalar out(_grid);
    unpack(g, out);
    return out;
}

void SFDSolver::advanceSubstep(State&, const Scalar&, int) {
    die("SFDSolver::advanceSubstep: the device runs whole steps (use advance)");
}

// the filtered state: read from <icFile>_xhat if it exists (src/IBSolver.cc:298-316);
// the device takes it at the first step
void SFDSolver::loadFilteredState(string icFile) {
    const string xhatFile = icFile + "_xhat";
    _xhat.omega = 0.;
    _xhat.f = 0.;
    _xhat.q = 0.;
    if (xhatFile != "_xhat") {
        std::cout << "Loading initial condition from file: " << xhatFile << std::endl;
        if (!_xhat.load(xhatFile)) std::cout << "  (failed: setting xhat = x)" << std::endl;
    } else {
        std::cout << "Setting xhat = x" << std::endl;
    }
    _xhatSaved = true;
}

// the device's filtered vorticity, written as a restart file (src/IBSolver.cc:290-296)
void SFDSolver::saveFilteredState(string outdir, string name, string numDigitInFileName) {
    ibg_context* ctx = solver_ctx(this, _tol);
    std::vector<double> wh((size_t)_grid.Ngrid() * (_grid.Nx() - 1) * (_grid.Ny() - 1));
    check(ibg_get_sfd_state(ctx, wh.data()), ctx, "SFDSolver::saveFilteredState");
    unpack(wh, _xhat.omega);
    long long ns = 0, nf = 0;
    int nb = 0;
    double t = 0.0;
    ibg_sizes(ctx, &ns, &nf, &nb);
    std::vector<double> f((size_t)nb);
    check(ibg_get_boundary_force(ctx, f.data(), &_xhat.timestep, &t), ctx, "SFDSolver::saveFilteredState");
    _xhat.time = t;
    const string formatString = outdir + name + numDigitInFileName + ".bin" + "_xhat";
    char filename[256];
    snprintf(filename, sizeof(filename), formatString.c_str(), _xhat.timestep);
    _xhat.save(filename);
}

}  // namespace ibpm
