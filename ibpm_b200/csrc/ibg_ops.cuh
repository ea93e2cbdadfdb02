// ibg_ops.cuh -- launchers for the stencil, regularizer and body kernels.
#pragma once
#include "ibg_internal.cuh"

namespace ibg {

// Rigid-body motion on the device: motion 0 = none, 1 = fixed (x, y, theta),
// 2 = pitch/plunge with p = (A_theta, 2 pi f_theta, phi_theta, A_y, 2 pi f_y, phi_y).
// A rigid body's motion on the device: p holds the geometry file's numbers
// (PITCHPLUNGE frequencies times 2 pi; the Eldredge family's normalisers
// maxG appended after them), trows / trow0 the rows of its motion table in
// the context's table (7 doubles a row: t x y theta xdot ydot thetadot).
struct BodyDev {
    double xc, yc;
    int motion;
    double p[14];
    int trows, trow0;
};
// Running integrals of the motions whose transformation depends on the times
// they were called at (src/FixedVelocity.h:42-50, src/Eldredge2.h:52-71,
// src/EldredgeCombined2.h:64-87): position integrals, the integral of G, and
// the last time.
struct MotionState {
    double ix, iy, ith, ig, told;
};
bool motion_is_stateful(int motion);

// Regularizer association slots: up to kSlots level-0 fluxes per boundary component.
constexpr int kSlots = 16;
struct RegSlots {
    int* idx = nullptr;     // [2 npts][kSlots] flux index (level 0)
    double* w = nullptr;    // [2 npts][kSlots] weight delta(dx) delta(dy)
    int* n = nullptr;       // [2 npts] number of slots used
    const double* pts = nullptr;  // [npts][2] the boundary points the slots were built from
    // the smear's fixed summation order, rebuilt with the slots: own[e] is the number of entries
    // (component, slot) holding the flux of entry e when e is the first of them in component order,
    // 0 otherwise; contrib[e] lists them (entry indices c * kSlots + k, in component order)
    int* own = nullptr;           // [2 npts][kSlots]
    int* contrib = nullptr;       // [2 npts][kSlots][kMaxContrib]
};
constexpr int kMaxContrib = 16;

template <typename T>
void launch_nonlinear(const GridDev& g, const T* q, const T* w, T* U, T* V, T* C, T* N, int batch, size_t sstride,
                      size_t fstride, cudaStream_t st);
template <typename T>
void launch_curl_flux(const GridDev& g, const T* C, T* N, cudaStream_t st);
// the nonlinear term without its curl (node velocities, cross-product fluxes of every level) ...
template <typename T>
void launch_nonlinear_flux(const GridDev& g, const T* q, const T* w, T* U, T* V, T* C, int batch, size_t sstride,
                           size_t fstride, cudaStream_t st);
// ... and the curl fused with the right-hand side: N = Curl(C), a = launch_rhs's a
template <typename T>
void launch_curl_rhs(const GridDev& g, const T* C, T* N, const T* w, const T* Nprev, T* a, double c1, double an,
                     double bn, double dt, cudaStream_t st);
template <typename T>
void launch_rhs(const GridDev& g, const T* w, const T* N, const T* Nprev, T* a, double c1, double an, double bn,
                double dt, cudaStream_t st);
template <typename T>
void launch_laplacian(const GridDev& g, const T* w, T* out, cudaStream_t st);
void launch_reg_gather(const GridDev& g, int ncomp, const RegSlots& s, const double* q0, double* out,
                       cudaStream_t st);
template <typename T>
// q = Curl(psi) + q0, q0 the uniform flow (u0, v0) dx_lev, or the field q0f (every level) when given
void launch_refresh_flux(const GridDev& g, const T* psi, T* q, double u0, double v0, const double* q0f,
                         cudaStream_t st);
// FluxToVelocity: node velocities u, v of every level (0 where undefined)
void launch_flux_to_vel(const GridDev& g, const double* q, double* u, double* v, cudaStream_t st);
// Moving-frame base flow at time *time_ptr + toff: the flow's velocities
// (xdot', ydot', thetadot') into out[3], the flux field q0 (all levels) from
// them, and the constraints b = body velocity - E(q0).
void launch_frame_flow(const BodyDev* bf, MotionState* ms, const double* mtab, const double* time_ptr, double toff,
                       double magBF, double alphaBF, double* out, cudaStream_t st);
void launch_frame_flux(const GridDev& g, const double* fv, double xc, double yc, double* q0, cudaStream_t st);
void launch_bcon_field(int ncomp, const RegSlots& s, const double* vel, const double* q0, double h, double* bcon,
                       cudaStream_t st);
// Geometry::moveBodies at time *time_ptr + toff: advance the history of the
// stateful motions (one thread per body), then move every point.
void launch_motion_state(int nbodies, const BodyDev* bodies, const double* time_ptr, double toff, MotionState* ms,
                         cudaStream_t st);
void launch_kinematics(int npts, const double* ref_xy, const int* body_of, const BodyDev* bodies,
                       const MotionState* ms, const double* mtab, const double* time_ptr, double toff, double* pts,
                       double* vel, cudaStream_t st);
void launch_reg_update(const GridDev& g, int npts, const double* pts, const double* vel, RegSlots& s, double* bcon,
                       double u0, double v0, double* flux0, cudaStream_t st);
template <typename T>
void launch_reg_interp(const GridDev& g, int ncomp, const RegSlots& s, const T* psi, size_t sstride, int batch,
                       const double* bcon, double* out, size_t ostride, cudaStream_t st);
// Regularizer::toFlux without the dx factor: flux0 (level 0) += sum of weight * f over the
// associations; launch_reg_zero clears the entries the smear touched
void launch_reg_smear(int ncomp, const RegSlots& s, double h, const double* f, double* flux0, cudaStream_t st);
void launch_reg_zero(int ncomp, const RegSlots& s, double* flux0, cudaStream_t st);
template <typename T>
void launch_smear_bf(const GridDev& g, int ncomp, const RegSlots& s, const double* f, double* flux0, T* Bf,
                     double beta, cudaStream_t st);
template <typename T>
void launch_smear_bf_unit(const GridDev& g, int ncomp, int col0, int batch, const RegSlots& s, double* flux0,
                          size_t fstride, T* Bf, size_t sstride, double beta, cudaStream_t st);

// the other N(x) forms (FP64 only)
void launch_nonlinear_lin(const GridDev& g, const double* q, const double* w, const double* qb, const double* wb,
                          int period, const int* ts0, const int* count, double* U, double* V, double* C, double* N,
                          cudaStream_t st);
void launch_flux_cross(const GridDev& g, const double* q1, const double* q2, double* out, cudaStream_t st);
void launch_sub(size_t n, const double* a, const double* b, double* out, cudaStream_t st);
void launch_sfd(size_t n, const double* w, double* what, double* rprev, double* N, double chi, double Delta,
                double an, double bn, double dt, bool first, cudaStream_t st);

}  // namespace ibg
