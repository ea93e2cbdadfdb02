// refops.cc -- extern "C" bridge exposing the reference's hot-path operators
// to ctypes, so that the numpy restatement (oracle/ibpm_oracle.py) can be
// pinned operator by operator against the reference itself.
//
// TEST INFRASTRUCTURE ONLY; built into oracle/_ref/libibpm_refops.so by
// oracle/Makefile from the reference sources.  Arrays use the reference
// layouts: Scalar = [lev][i-1][j-1] (src/Scalar.h:76-90), Flux = [lev][index]
// (src/Flux.h:176-185), BoundaryVector = [fx..., fy...] (src/BoundaryVector.h:65-69),
// BC ring of 2(nx+ny) values (src/BC.h).
#include "ibpm.h"
#include "ProjectionSolver.h"
#include "CholeskySolver.h"
#include "ConjugateGradientSolver.h"
#include "EllipticSolver.h"
#include "EllipticSolver2d.h"
#include "Regularizer.h"
#include <cmath>
#include <limits>

using namespace ibpm;

namespace {
Grid mkgrid(const int* gi, const double* gd) {
    return Grid(gi[0], gi[1], gi[2], gd[0], gd[1], gd[2]);
}
void toScalar(const double* p, Scalar& s) {
    int k = 0;
    for (int l = 0; l < s.Ngrid(); ++l)
        for (int i = 1; i < s.Nx(); ++i)
            for (int j = 1; j < s.Ny(); ++j) s(l, i, j) = p[k++];
}
void fromScalar(const Scalar& s, double* p) {
    int k = 0;
    for (int l = 0; l < s.Ngrid(); ++l)
        for (int i = 1; i < s.Nx(); ++i)
            for (int j = 1; j < s.Ny(); ++j) p[k++] = s(l, i, j);
}
void toFlux(const double* p, Flux& q) {
    int k = 0;
    for (int l = 0; l < q.Ngrid(); ++l)
        for (int ind = q.begin(); ind != q.end(); ++ind) q(l, ind) = p[k++];
}
void fromFlux(const Flux& q, double* p) {
    int k = 0;
    for (int l = 0; l < q.Ngrid(); ++l)
        for (int ind = q.begin(); ind != q.end(); ++ind) p[k++] = q(l, ind);
}
void toBV(const double* p, BoundaryVector& b) {
    for (int i = 0; i < b.end(); ++i) b(i) = p[i];
}
void fromBV(const BoundaryVector& b, double* p) {
    for (int i = 0; i < b.end(); ++i) p[i] = b(i);
}
Geometry mkgeom(int npts, const double* xy) {
    Geometry g;
    RigidBody body;
    for (int i = 0; i < npts; ++i) body.addPoint(xy[2 * i], xy[2 * i + 1]);
    g.addBody(body);
    return g;
}
const double NaN = std::numeric_limits<double>::quiet_NaN();
// ProjectionSolver::M is protected; this subclass only exposes it.
struct MApply : public CholeskySolver {
    MApply(const Grid& g, const NavierStokesModel& m, double beta) : CholeskySolver(g, m, beta) {}
    BoundaryVector apply(const BoundaryVector& f) { return M(f); }
};
}  // namespace

extern "C" {

// gi = {nx, ny, ngrid}, gd = {length, xoffset, yoffset}
void refops_coarsify(const int* gi, const double* gd, double* s) {
    Grid g = mkgrid(gi, gd);
    Scalar a(g); toScalar(s, a); a.coarsify(); fromScalar(a, s);
}

void refops_getbc(const int* gi, const double* gd, const double* s, int lev, double* bc_out) {
    Grid g = mkgrid(gi, gd);
    Scalar a(g); toScalar(s, a);
    BC bc(g.Nx(), g.Ny());
    a.getBC(lev, bc);
    int nx = g.Nx(), ny = g.Ny();
    // ring order of src/BC.h: left(0..ny-1) ... expressed via accessors
    for (int j = 0; j <= ny; ++j) bc_out[j] = bc.left(j);
    for (int i = 0; i <= nx; ++i) bc_out[ny + i] = bc.top(i);
    for (int j = ny; j >= 0; --j) bc_out[2 * ny + nx - j] = bc.right(j);
    for (int i = nx; i >= 1; --i) bc_out[2 * (nx + ny) - i] = bc.bottom(i);
}

void refops_curl_flux(const int* gi, const double* gd, const double* q, double* w) {
    Grid g = mkgrid(gi, gd);
    Flux a(g); toFlux(q, a);
    Scalar o(g); Curl(a, o); fromScalar(o, w);
}

void refops_curl_scalar(const int* gi, const double* gd, const double* s, double* q) {
    Grid g = mkgrid(gi, gd);
    Scalar a(g); toScalar(s, a);
    Flux o(g); Curl(a, o); fromFlux(o, q);
}

void refops_laplacian(const int* gi, const double* gd, const double* s, double* out) {
    Grid g = mkgrid(gi, gd);
    Scalar a(g); toScalar(s, a);
    Scalar o(g); Laplacian(a, o); fromScalar(o, out);
}

void refops_flux_to_velocity(const int* gi, const double* gd, const double* q, double* u, double* v) {
    Grid g = mkgrid(gi, gd);
    Flux a(g); toFlux(q, a);
    Scalar su(g), sv(g);
    su = NaN; sv = NaN;
    FluxToVelocity(a, su, sv);
    fromScalar(su, u); fromScalar(sv, v);
}

void refops_velocity_to_flux(const int* gi, const double* gd, const double* u, const double* v, double* q) {
    Grid g = mkgrid(gi, gd);
    Scalar su(g), sv(g); toScalar(u, su); toScalar(v, sv);
    Flux o(g); o = NaN;
    VelocityToFlux(su, sv, o); fromFlux(o, q);
}

void refops_cross_product(const int* gi, const double* gd, const double* q, const double* w, double* out) {
    Grid g = mkgrid(gi, gd);
    Flux a(g); toFlux(q, a);
    Scalar o(g); toScalar(w, o);
    Flux c = CrossProduct(a, o); fromFlux(c, out);
}

// NonlinearIBSolver::N (src/IBSolver.cc:205-209)
void refops_nonlinear(const int* gi, const double* gd, const double* q, const double* w, double* out) {
    Grid g = mkgrid(gi, gd);
    Flux a(g); toFlux(q, a);
    Scalar o(g); toScalar(w, o);
    Flux c = CrossProduct(a, o);
    Scalar n = Curl(c); fromScalar(n, out);
}

// kind 0 = Poisson, 1 = Helmholtz (1 + alpha L)
void refops_elliptic(const int* gi, const double* gd, int kind, double alpha, const double* f, double* u) {
    Grid g = mkgrid(gi, gd);
    Scalar a(g); toScalar(f, a);
    Scalar o(g);
    if (kind == 0) { PoissonSolver s(g); s.solve(a, o); }
    else { HelmholtzSolver s(g, alpha); s.solve(a, o); }
    fromScalar(o, u);
}

// single-level 2-D solve; bc_ring may be NULL (zero boundary values)
void refops_elliptic2d(int nx, int ny, double dx, int kind, double alpha,
                       const double* f, const double* bc_ring, double* u) {
    Array::Array2<double> fa(nx - 1, ny - 1, 1, 1), ua(nx - 1, ny - 1, 1, 1);
    int k = 0;
    for (int i = 1; i < nx; ++i) for (int j = 1; j < ny; ++j) fa(i, j) = f[k++];
    EllipticSolver2d* s;
    if (kind == 0) s = new PoissonSolver2d(nx, ny, dx);
    else s = new HelmholtzSolver2d(nx, ny, dx, alpha);
    if (bc_ring) {
        BC bc(nx, ny);
        for (int j = 0; j <= ny; ++j) bc.left(j) = bc_ring[j];
        for (int i = 0; i <= nx; ++i) bc.top(i) = bc_ring[ny + i];
        for (int j = ny; j >= 0; --j) bc.right(j) = bc_ring[2 * ny + nx - j];
        for (int i = nx; i >= 1; --i) bc.bottom(i) = bc_ring[2 * (nx + ny) - i];
        s->solve(fa, bc, ua);
    } else {
        s->solve(fa, ua);
    }
    delete s;
    k = 0;
    for (int i = 1; i < nx; ++i) for (int j = 1; j < ny; ++j) u[k++] = ua(i, j);
}

// raw 2-D RODFT00 through the shim's plan API (row-major n0 x n1)
void refops_dst2d(int n0, int n1, const double* in, double* out) {
    double* buf = new double[(size_t)n0 * n1];
    for (int k = 0; k < n0 * n1; ++k) buf[k] = in[k];
    fftw_plan p = fftw_plan_r2r_2d(n0, n1, buf, buf, FFTW_RODFT00, FFTW_RODFT00, FFTW_EXHAUSTIVE);
    fftw_execute(p);
    fftw_destroy_plan(p);
    for (int k = 0; k < n0 * n1; ++k) out[k] = buf[k];
    delete[] buf;
}

// Regularizer::toFlux / toBoundary over a single body of npts points (xy interleaved)
void refops_reg_toflux(const int* gi, const double* gd, int npts, const double* xy,
                       const double* f, double* q) {
    Grid g = mkgrid(gi, gd);
    Geometry geo = mkgeom(npts, xy);
    Regularizer r(g, geo); r.update();
    BoundaryVector b(npts); toBV(f, b);
    Flux o = r.toFlux(b); fromFlux(o, q);
}

void refops_reg_toboundary(const int* gi, const double* gd, int npts, const double* xy,
                           const double* q, double* f) {
    Grid g = mkgrid(gi, gd);
    Geometry geo = mkgeom(npts, xy);
    Regularizer r(g, geo); r.update();
    Flux a(g); toFlux(q, a);
    BoundaryVector o = r.toBoundary(a); fromBV(o, f);
}

// ProjectionSolver::solve with a fixed body (use_cg = 0: CholeskySolver,
// 1: ConjugateGradientSolver with tolerance tol, starting from f_inout).
void refops_projection(const int* gi, const double* gd, int npts, const double* xy,
                       double Re, double beta, int use_cg, double tol,
                       const double* a, const double* b, double* omega, double* f_inout) {
    Grid g = mkgrid(gi, gd);
    Geometry geo = mkgeom(npts, xy);
    NavierStokesModel model(g, geo, Re);
    model.init();
    ProjectionSolver* s;
    if (use_cg) s = new ConjugateGradientSolver(g, model, beta, tol);
    else s = new CholeskySolver(g, model, beta);
    s->init();
    Scalar sa(g), so(g); toScalar(a, sa);
    BoundaryVector bb(npts), ff(npts); toBV(b, bb); toBV(f_inout, ff);
    s->solve(sa, bb, so, ff);
    fromScalar(so, omega); fromBV(ff, f_inout);
    delete s;
}

// M = C A^-1 B applied to one boundary vector (src/ProjectionSolver.cc:96-101)
void refops_apply_m(const int* gi, const double* gd, int npts, const double* xy,
                    double Re, double beta, const double* f, double* y) {
    Grid g = mkgrid(gi, gd);
    Geometry geo = mkgeom(npts, xy);
    NavierStokesModel model(g, geo, Re);
    model.init();
    MApply s(g, model, beta);
    BoundaryVector ff(npts), yy(npts); toBV(f, ff);
    yy = s.apply(ff);
    fromBV(yy, y);
}

// kind 0 InnerProduct(Scalar, Scalar), 1 FineGridInnerProduct(Scalar, Scalar),
// 2 InnerProduct(Flux, Flux), 3 FineGridInnerProduct(Flux, Flux) (src/VectorOperations.cc:222-412)
void refops_inner_product(const int* gi, const double* gd, int kind, const double* a, const double* b, double* out) {
    Grid g = mkgrid(gi, gd);
    if (kind < 2) {
        Scalar x(g), y(g); toScalar(a, x); toScalar(b, y);
        *out = kind == 0 ? InnerProduct(x, y) : FineGridInnerProduct(x, y);
    } else {
        Flux x(g), y(g); toFlux(a, x); toFlux(b, y);
        *out = kind == 2 ? InnerProduct(x, y) : FineGridInnerProduct(x, y);
    }
}

}  // extern "C"
