// ops.cu -- stencil, nonlinear, regularizer and kinematics kernels.
//
// Reference functions replaced (paths inside the reference project):
//   k_node_vel     FluxToXVelocity / FluxToYVelocity  src/VectorOperations.cc:488-667
//                  and the products of CrossProduct     src/VectorOperations.cc:438-457
//   k_cross_flux   XVelocityToFlux / YVelocityToFlux  src/VectorOperations.cc:669-916
//   k_curl_flux    Curl(Flux)                          src/VectorOperations.cc:33-54
//   k_rhs          IBSolver::advanceSubstep RHS        src/IBSolver.cc:168-183
//                  with Laplacian = -Curl(Curl())      src/VectorOperations.cc:63-146
//   k_refresh_flux computeFlux = Curl(psi) + q0         src/NavierStokesModel.cc:114-125
//   k_kinematics   RigidBody::moveBody + Motion        src/RigidBody.cc:586-609, src/Motion.h subclasses
//   k_motion_state the history of FixedVelocity / Eldredge2 / EldredgeCombined2
//   k_frame_flow / k_frame_flux / k_bcon_field  BaseFlow::moveFlow (moving frame), getConstraints
//   k_reg_update   Regularizer::update                 src/Regularizer.cc:54-90
//   k_reg_interp   Regularizer::toBoundary o Curl(psi) src/Regularizer.cc:111-128
//   k_reg_smear/k_bf  Regularizer::toFlux, Curl, *beta  src/Regularizer.cc:92-109, src/ProjectionSolver.cc:87-90
#include "ibg_internal.cuh"
#include "ibg_ops.cuh"
#include "../../include/ibpm_b200.h"

namespace ibg {

template <typename T>
__device__ __forceinline__ T qx_at(const T* q_lev, const GridDev& g, int i, int j) {
    return q_lev[(size_t)i * g.ny + j];
}
template <typename T>
__device__ __forceinline__ T qy_at(const T* q_lev, const GridDev& g, int i, int j) {
    return q_lev[(size_t)g.nXf + (size_t)i * (g.ny + 1) + j];
}

// ---------------------------------------------------------------------------
// node velocities times vorticity: U = -(u w), V = v w on every node where
// the reference defines u, v (coarse overlap interior nodes are never read
// downstream and are written as zero).
// ---------------------------------------------------------------------------
// velocities (u, v) at node (i, j) of level `lev` from the fluxes of that level (ql) and of the
// next finer one (FluxToXVelocity / FluxToYVelocity, src/VectorOperations.cc:224-368); du / dv
// false where the reference leaves the value undefined (coarse overlap interior)
template <typename T>
__device__ __forceinline__ void node_uv(const GridDev& g, const T* ql, int lev, int i, int j, T& u, T& v, bool& du,
                                        bool& dv) {
    const int nx = g.nx, ny = g.ny, nx2 = g.nxe, ny2 = g.nye;
    u = (T)0;
    v = (T)0;
    du = dv = true;
    if (lev == 0) {
        const T o2d = (T)(1.0 / (2 * g.dx));
        u = (qx_at(ql, g, i, j) + qx_at(ql, g, i, j - 1)) * o2d;
        v = (qy_at(ql, g, i - 1, j) + qy_at(ql, g, i, j)) * o2d;
    } else {
        const T bydx = (T)(1.0 / lev_dx(g, lev));
        const T* qf = ql - g.F1;
        const int il = nx2, ir = nx / 2 + nx2, jb = ny2, jt = ny / 2 + ny2;
        // ---- u (x-velocity) regions B, C, D, E, F
        if (i < il || i > ir || j < jb || j > jt || ((i == il || i == ir) && j > jb && j < jt)) {
            u = (qx_at(ql, g, i, j) + qx_at(ql, g, i, j - 1)) * (T)0.5 * bydx;
        } else if ((j == jb || j == jt) && i > il && i < ir) {
            const int ii = (i - nx2) * 2;
            if (j == jb)
                u = (qx_at(ql, g, i, jb - 1) * (T)2 / (T)3 + qx_at(qf, g, ii, 0) * (T)1 / (T)3 +
                     (qx_at(qf, g, ii - 1, 0) + qx_at(qf, g, ii + 1, 0)) * (T)1 / (T)6) * bydx;
            else
                u = (qx_at(ql, g, i, jt) * (T)2 / (T)3 + qx_at(qf, g, ii, ny - 1) * (T)1 / (T)3 +
                     (qx_at(qf, g, ii - 1, ny - 1) + qx_at(qf, g, ii + 1, ny - 1)) * (T)1 / (T)6) * bydx;
        } else if ((i == il || i == ir) && (j == jb || j == jt)) {
            if (j == jb) {
                const T fv = (i == il) ? qx_at(qf, g, 1, 0) : qx_at(qf, g, nx - 1, 0);
                u = (qx_at(ql, g, i, j - 1) * (T)8 / (T)15 + qx_at(ql, g, i, j) * (T)6 / (T)15 + fv * (T)2 / (T)15) * bydx;
            } else {
                const T fv = (i == il) ? qx_at(qf, g, 1, ny - 1) : qx_at(qf, g, nx - 1, ny - 1);
                u = (qx_at(ql, g, i, j) * (T)8 / (T)15 + qx_at(ql, g, i, j - 1) * (T)6 / (T)15 + fv * (T)2 / (T)15) * bydx;
            }
        } else {
            du = false;
        }
        // ---- v (y-velocity): B (bottom/top borders), C (left/right), D, E, F
        if (j < jb || j > jt || i < il || i > ir || ((j == jb || j == jt) && i > il && i < ir)) {
            v = (qy_at(ql, g, i, j) + qy_at(ql, g, i - 1, j)) * (T)0.5 * bydx;
        } else if ((i == il || i == ir) && j > jb && j < jt) {
            const int jj = (j - ny2) * 2;
            if (i == il)
                v = (qy_at(ql, g, il - 1, j) * (T)2 / (T)3 + qy_at(qf, g, 0, jj) * (T)1 / (T)3 +
                     (qy_at(qf, g, 0, jj - 1) + qy_at(qf, g, 0, jj + 1)) * (T)1 / (T)6) * bydx;
            else
                v = (qy_at(ql, g, ir, j) * (T)2 / (T)3 + qy_at(qf, g, nx - 1, jj) * (T)1 / (T)3 +
                     (qy_at(qf, g, nx - 1, jj - 1) + qy_at(qf, g, nx - 1, jj + 1)) * (T)1 / (T)6) * bydx;
        } else if ((i == il || i == ir) && (j == jb || j == jt)) {
            if (i == il) {
                const T fv = (j == jb) ? qy_at(qf, g, 0, 1) : qy_at(qf, g, 0, ny - 1);
                v = (qy_at(ql, g, i - 1, j) * (T)8 / (T)15 + qy_at(ql, g, i, j) * (T)6 / (T)15 + fv * (T)2 / (T)15) * bydx;
            } else {
                const T fv = (j == jb) ? qy_at(qf, g, nx - 1, 1) : qy_at(qf, g, nx - 1, ny - 1);
                v = (qy_at(ql, g, i, j) * (T)8 / (T)15 + qy_at(ql, g, i - 1, j) * (T)6 / (T)15 + fv * (T)2 / (T)15) * bydx;
            }
        } else {
            dv = false;
        }
    }
}

template <typename T>
__global__ void k_node_vel(GridDev g, const T* __restrict__ q, const T* __restrict__ w, T* __restrict__ U,
                           T* __restrict__ V, size_t sstride, size_t fstride) {
    pdl_enter();
    // blockIdx.y: level, blockIdx.z: batch item (32-bit index arithmetic within a level)
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= g.N1) return;
    const int lev = blockIdx.y;
    const size_t tid = (size_t)lev * g.N1 + r;
    const size_t sb = (size_t)blockIdx.z * sstride, fb = (size_t)blockIdx.z * fstride;
    const int i = r / g.NJ + 1, j = r % g.NJ + 1;
    T u, v;
    bool du, dv;
    node_uv(g, q + fb + (size_t)lev * g.F1, lev, i, j, u, v, du, dv);
    const T wv = w[sb + tid];
    U[sb + tid] = du ? (u * wv) * (T)-1 : (T)0;
    V[sb + tid] = dv ? v * wv : (T)0;
}

// FluxToVelocity (src/VectorOperations.cc:924-927): u and v at every node of every level, 0 on the
// coarse interior overlap nodes the reference leaves undefined
__global__ void k_flux_to_vel(GridDev g, const double* __restrict__ q, double* __restrict__ u,
                              double* __restrict__ v) {
    pdl_enter();
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (size_t)g.L * g.N1) return;
    const int lev = (int)(tid / g.N1);
    const int r = (int)(tid % g.N1);
    const int i = r / g.NJ + 1, j = r % g.NJ + 1;
    double uu, vv;
    bool du, dv;
    node_uv(g, q + (size_t)lev * g.F1, lev, i, j, uu, vv, du, dv);
    u[tid] = du ? uu : 0.0;
    v[tid] = dv ? vv : 0.0;
}

// LinearizedIBSolver / LinearizedPeriodicIBSolver node products (src/IBSolver.cc:211-216, 224-232):
// CrossProduct(q0, omega) + CrossProduct(q, omega0) before the flux stencils (which are linear),
// with the base state of phase (timestep % period); the step counter lives on the device
// (ts0 = timestep at the last state upload, count = steps since then).
__global__ void k_node_vel_lin(GridDev g, const double* __restrict__ q, const double* __restrict__ w,
                               const double* __restrict__ qb, const double* __restrict__ wb, int period,
                               const int* __restrict__ ts0, const int* __restrict__ count, double* __restrict__ U,
                               double* __restrict__ V) {
    pdl_enter();
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t total = (size_t)g.L * g.N1;
    if (tid >= total) return;
    const int phase = ((*ts0 + *count) % period + period) % period;
    const double* q0 = qb + (size_t)phase * g.L * g.F1;
    const double* w0 = wb + (size_t)phase * total;
    const int lev = (int)(tid / g.N1);
    const int r = (int)(tid % g.N1);
    const int i = r / g.NJ + 1, j = r % g.NJ + 1;
    double u, v, ub, vb;
    bool du, dv;
    node_uv(g, q + (size_t)lev * g.F1, lev, i, j, u, v, du, dv);
    node_uv(g, q0 + (size_t)lev * g.F1, lev, i, j, ub, vb, du, dv);
    const double wv = w[tid], w0v = w0[tid];
    U[tid] = du ? (ub * wv) * -1.0 + (u * w0v) * -1.0 : 0.0;
    V[tid] = dv ? vb * wv + v * w0v : 0.0;
}

// CrossProduct(Flux q1, Flux q2) = u1 v2 - u2 v1 at the nodes (src/VectorOperations.cc:465-486);
// the coarse overlap interior, undefined here as in the reference, is then filled by coarsify
__global__ void k_flux_cross(GridDev g, const double* __restrict__ q1, const double* __restrict__ q2,
                             double* __restrict__ out) {
    pdl_enter();
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (size_t)g.L * g.N1) return;
    const int lev = (int)(tid / g.N1);
    const int r = (int)(tid % g.N1);
    const int i = r / g.NJ + 1, j = r % g.NJ + 1;
    double u1, v1, u2, v2;
    bool du, dv;
    node_uv(g, q1 + (size_t)lev * g.F1, lev, i, j, u1, v1, du, dv);
    node_uv(g, q2 + (size_t)lev * g.F1, lev, i, j, u2, v2, du, dv);
    out[tid] = (du && dv) ? u1 * v2 - u2 * v1 : 0.0;
}

__global__ void k_sub(size_t n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out) {
    pdl_enter();
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = a[t] - b[t];
}

// SFDSolver (src/IBSolver.cc:238-283): N -= chi (omega - omega_hat), then the filtered state
// advances from the vorticity at the start of the sub-step:
// rhs = (omega - omega_hat) / Delta, omega_hat += dt (an rhs + bn rhs_prev), rhs_prev = rhs
__global__ void k_sfd(size_t n, const double* __restrict__ w, double* __restrict__ what, double* __restrict__ rprev,
                      double* __restrict__ N, double chi, double Delta, double an, double bn, double dt,
                      int first) {
    pdl_enter();
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double d = w[t] - what[t];
    N[t] = N[t] - chi * d;
    const double rhs = d / Delta;
    double a = an * rhs;
    if (bn != 0.0) a += bn * (first ? rhs : rprev[t]);
    a *= dt;
    what[t] = what[t] + a;
    rprev[t] = rhs;
}

// ---------------------------------------------------------------------------
// cross-product fluxes of one level: x part from V (XVelocityToFlux), y part
// from U (YVelocityToFlux).  Coarse-level interior fluxes over the finer
// domain are sums of the finer level's fluxes, so levels run fine to coarse.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_cross_flux(GridDev g, int lev, const T* __restrict__ U, const T* __restrict__ V, T* __restrict__ C,
                             size_t sstride, size_t fstride) {
    pdl_enter();
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= g.F1) return;
    const size_t sb = (size_t)blockIdx.y * sstride, fb = (size_t)blockIdx.y * fstride;
    const int nx = g.nx, ny = g.ny, nx2 = g.nxe, ny2 = g.nye, L = g.L;
    const T dx = (T)lev_dx(g, lev);
    T* Cl = C + fb + (size_t)lev * g.F1;
    const T* Cf = Cl - g.F1;  // finer level (lev >= 1)
    T out;
    if (tid < g.nXf) {
        const int i = tid / ny, j = tid % ny;
        const T* p = V + sb + (size_t)lev * g.N1;
        const T* c = (lev < L - 1) ? V + sb + (size_t)(lev + 1) * g.N1 : nullptr;
        if (i == 0 || i == nx) {
            if (lev == L - 1) {
                out = (T)0;
            } else {
                const int ic = (i == 0) ? nx2 : nx / 2 + nx2;
                const int jj = j / 2 + ny2;
                if ((j & 1) == 0)
                    out = ((T)0.75 * node(c, g, ic, jj) + (T)0.25 * node(c, g, ic, jj + 1)) * dx;
                else
                    out = ((T)0.25 * node(c, g, ic, jj) + (T)0.75 * node(c, g, ic, jj + 1)) * dx;
            }
        } else if (j == 0 || j == ny - 1) {
            const int jn = (j == 0) ? 1 : ny - 1;
            if (lev == L - 1) {
                out = node(p, g, i, jn) * (T)0.5 * dx;
            } else {
                const int jc = (j == 0) ? ny2 : ny / 2 + ny2;
                const int ii = i / 2 + nx2;
                if ((i & 1) == 0)
                    out = (node(p, g, i, jn) + node(c, g, ii, jc)) * (T)0.5 * dx;
                else
                    out = ((T)0.5 * node(p, g, i, jn) + (T)0.25 * node(c, g, ii, jc) + (T)0.25 * node(c, g, ii + 1, jc)) * dx;
            }
        } else if (lev > 0 && j >= ny2 && j < ny / 2 + ny2 && i > nx2 && i < nx / 2 + nx2) {
            const int ii = 2 * (i - nx2), jj = 2 * (j - ny2);
            out = qx_at(Cf, g, ii, jj) + qx_at(Cf, g, ii, jj + 1);
        } else {
            out = (node(p, g, i, j) + node(p, g, i, j + 1)) * (T)0.5 * dx;
        }
    } else {
        const int t = tid - g.nXf;
        const int i = t / (ny + 1), j = t % (ny + 1);
        const T* p = U + sb + (size_t)lev * g.N1;
        const T* c = (lev < L - 1) ? U + sb + (size_t)(lev + 1) * g.N1 : nullptr;
        if (j == 0 || j == ny) {
            if (lev == L - 1) {
                out = (T)0;
            } else {
                const int jc = (j == 0) ? ny2 : ny / 2 + ny2;
                const int ii = i / 2 + nx2;
                if ((i & 1) == 0)
                    out = ((T)0.75 * node(c, g, ii, jc) + (T)0.25 * node(c, g, ii + 1, jc)) * dx;
                else
                    out = ((T)0.25 * node(c, g, ii, jc) + (T)0.75 * node(c, g, ii + 1, jc)) * dx;
            }
        } else if (i == 0 || i == nx - 1) {
            const int in_ = (i == 0) ? 1 : nx - 1;
            if (lev == L - 1) {
                out = node(p, g, in_, j) * (T)0.5 * dx;
            } else {
                const int ic = (i == 0) ? nx2 : nx / 2 + nx2;
                const int jj = j / 2 + ny2;
                if ((j & 1) == 0)
                    out = (node(p, g, in_, j) + node(c, g, ic, jj)) * (T)0.5 * dx;
                else
                    out = ((T)0.5 * node(p, g, in_, j) + (T)0.25 * node(c, g, ic, jj) + (T)0.25 * node(c, g, ic, jj + 1)) * dx;
            }
        } else if (lev > 0 && i >= nx2 && i < nx / 2 + nx2 && j > ny2 && j < ny / 2 + ny2) {
            const int ii = 2 * (i - nx2), jj = 2 * (j - ny2);
            out = qy_at(Cf, g, ii, jj) + qy_at(Cf, g, ii + 1, jj);
        } else {
            out = (node(p, g, i, j) + node(p, g, i + 1, j)) * (T)0.5 * dx;
        }
    }
    Cl[tid] = out;
}

// Curl of a Flux on every level (no inter-level coupling)
template <typename T>
__global__ void k_curl_flux(GridDev g, const T* __restrict__ C, T* __restrict__ N, size_t sstride, size_t fstride) {
    pdl_enter();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;  // blockIdx.y: level, blockIdx.z: batch item
    if (r >= g.N1) return;
    const int lev = blockIdx.y;
    const size_t tid = (size_t)lev * g.N1 + r;
    const size_t sb = (size_t)blockIdx.z * sstride, fb = (size_t)blockIdx.z * fstride;
    const int i = r / g.NJ + 1, j = r % g.NJ + 1;
    const T* ql = C + fb + (size_t)lev * g.F1;
    const double dxl = lev_dx(g, lev);
    const T bydx2 = (T)(1. / (dxl * dxl));
    N[sb + tid] = (qy_at(ql, g, i, j) - qy_at(ql, g, i - 1, j) + qx_at(ql, g, i, j - 1) - qx_at(ql, g, i, j)) * bydx2;
}

// a = omega + dt (c1 L omega + an N + bn Nprev)
template <typename T>
__global__ void k_rhs(GridDev g, const T* __restrict__ w, const T* __restrict__ N, const T* __restrict__ Nprev,
                      T* __restrict__ a, T c1, T an, T bn, T dt, int lap_only) {
    pdl_enter();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;  // blockIdx.y: level
    if (r >= g.N1) return;
    const int lev = blockIdx.y;
    const size_t tid = (size_t)lev * g.N1 + r;
    const int i = r / g.NJ + 1, j = r % g.NJ + 1;
    const T* f = w + (size_t)lev * g.N1;
    const T* c = (lev < g.L - 1) ? w + (size_t)(lev + 1) * g.N1 : nullptr;
    const T p = node(f, g, i, j);
    const T pe = node_bc(f, c, g, i + 1, j), pw = node_bc(f, c, g, i - 1, j);
    const T pn = node_bc(f, c, g, i, j + 1), ps = node_bc(f, c, g, i, j - 1);
    const T qy_ij = p - pe, qy_im = pw - p, qx_jm = p - ps, qx_ij = pn - p;
    const double dxl = lev_dx(g, lev);
    const T bydx2 = (T)(1. / (dxl * dxl));
    const T lap = ((qy_ij - qy_im + qx_jm - qx_ij) * bydx2) * (T)-1;
    if (lap_only) {
        a[tid] = lap;
        return;
    }
    T v = lap * c1;
    v = v + an * N[tid];
    if (Nprev) v = v + bn * Nprev[tid];
    v = v * dt;
    a[tid] = v + p;
}

// k_curl_flux and k_rhs of one sub-step in one launch: N = Curl(C) is stored (the next sub-step's
// N_prev) and used at once.  The same operations in the same order as the two kernels, so the same
// results.  Nprev may be N itself (the first step of a multistep scheme).
template <typename T>
__global__ void k_curl_rhs(GridDev g, const T* __restrict__ C, T* N, const T* __restrict__ w, const T* Nprev,
                           T* __restrict__ a, T c1, T an, T bn, T dt) {
    pdl_enter();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;  // blockIdx.y: level
    if (r >= g.N1) return;
    const int lev = blockIdx.y;
    const size_t tid = (size_t)lev * g.N1 + r;
    const int i = r / g.NJ + 1, j = r % g.NJ + 1;
    const double dxl = lev_dx(g, lev);
    const T bydx2 = (T)(1. / (dxl * dxl));
    const T* ql = C + (size_t)lev * g.F1;
    const T nv = (qy_at(ql, g, i, j) - qy_at(ql, g, i - 1, j) + qx_at(ql, g, i, j - 1) - qx_at(ql, g, i, j)) * bydx2;
    N[tid] = nv;
    const T* f = w + (size_t)lev * g.N1;
    const T* c = (lev < g.L - 1) ? w + (size_t)(lev + 1) * g.N1 : nullptr;
    const T p = node(f, g, i, j);
    const T pe = node_bc(f, c, g, i + 1, j), pw = node_bc(f, c, g, i - 1, j);
    const T pn = node_bc(f, c, g, i, j + 1), ps = node_bc(f, c, g, i, j - 1);
    const T qy_ij = p - pe, qy_im = pw - p, qx_jm = p - ps, qx_ij = pn - p;
    const T lap = ((qy_ij - qy_im + qx_jm - qx_ij) * bydx2) * (T)-1;
    T v = lap * c1;
    v = v + an * nv;
    if (Nprev) v = v + bn * (Nprev == N ? nv : Nprev[tid]);
    v = v * dt;
    a[tid] = v + p;
}

// Curl of a Scalar (with boundary values from the next coarser level) at a
// flux index of level lev.
template <typename T>
__device__ __forceinline__ T curl_scalar_at(const GridDev& g, const T* f, const T* c, int idx) {
    if (idx < g.nXf) {
        const int i = idx / g.ny, j = idx % g.ny;
        return node_bc(f, c, g, i, j + 1) - node_bc(f, c, g, i, j);
    }
    const int t = idx - g.nXf;
    const int i = t / (g.ny + 1), j = t % (g.ny + 1);
    return node_bc(f, c, g, i, j) - node_bc(f, c, g, i + 1, j);
}

// q = Curl(psi) + q0 on every level
template <typename T>
__global__ void k_refresh_flux(GridDev g, const T* __restrict__ psi, T* __restrict__ q, double u0, double v0,
                               const double* __restrict__ q0f) {
    pdl_enter();
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;  // blockIdx.y: level
    if (idx >= g.F1) return;
    const int lev = blockIdx.y;
    const size_t tid = (size_t)lev * g.F1 + idx;
    const T* f = psi + (size_t)lev * g.N1;
    const T* c = (lev < g.L - 1) ? psi + (size_t)(lev + 1) * g.N1 : nullptr;
    const double dxl = lev_dx(g, lev);
    const T base = q0f ? (T)q0f[tid] : (T)((idx < g.nXf ? u0 : v0) * dxl);
    q[tid] = curl_scalar_at(g, f, c, idx) + base;
}

// ---------------------------------------------------------------------------
// bodies
// ---------------------------------------------------------------------------
__host__ __device__ inline bool motion_is_stateful_dev(int motion) {
    return motion == IBG_MOTION_FIXEDVEL || motion == IBG_MOTION_ELDREDGE2 || motion == IBG_MOTION_ELDREDGECOMBINED2;
}
bool motion_is_stateful(int motion) { return motion_is_stateful_dev(motion); }

// G(t) = log(cosh(a(t - t1)) cosh(a(t - t4)) / (cosh(a(t - t2)) cosh(a(t - t3)))) and dG/dt of
// Eldredge's smoothed ramp (src/EldredgeManeuver.h:56-59), with q = (a, t1, t2, t3, t4)
__device__ __forceinline__ double eld_G(const double* q, double t) {
    const double a = q[0];
    return log((cosh(a * (t - q[1])) * cosh(a * (t - q[4]))) / (cosh(a * (t - q[2])) * cosh(a * (t - q[3]))));
}
__device__ __forceinline__ double eld_dG(const double* q, double t) {
    const double a = q[0];
    return a * (tanh(a * (t - q[1])) - tanh(a * (t - q[2])) - tanh(a * (t - q[3])) + tanh(a * (t - q[4])));
}

// The reference's Motion objects that keep a running integral update it on
// every getTransformation call; a second call at the same time adds nothing.
__device__ void advance_history(const BodyDev& b, MotionState& s, double t) {
    if (!motion_is_stateful_dev(b.motion)) return;
    double dtt = t - s.told;
    if (b.motion == IBG_MOTION_FIXEDVEL) {  // src/FixedVelocity.h:42-48
        if (dtt > 1) dtt = 0.;
        s.ix = s.ix + b.p[0] * dtt;
        s.iy = s.iy + b.p[1] * dtt;
        s.ith = s.ith + b.p[2] * dtt;
    } else {  // src/Eldredge2.h:62-66, src/EldredgeCombined2.h:81-85 (G of the plunge ramp a)
        s.ig = s.ig + eld_G(b.p + 1, t) * dtt;
    }
    s.told = t;
}

// one thread per body
__global__ void k_motion_state(int nbodies, const BodyDev* __restrict__ bodies, const double* __restrict__ time_ptr,
                               double toff, MotionState* __restrict__ ms) {
    pdl_enter();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nbodies) return;
    const BodyDev& b = bodies[k];
    if (!motion_is_stateful_dev(b.motion)) return;
    MotionState s = ms[k];
    advance_history(b, s, *time_ptr + toff);
    ms[k] = s;
}

// Motion::getTransformation(t): (x, y, theta, xdot, ydot, thetadot) of the body frame.
__device__ void body_frame(const BodyDev& b, const MotionState& s, const double* __restrict__ mtab, double t,
                           double& x, double& y, double& th, double& xd, double& yd, double& thd) {
    const double pi = 3.141592653589793;  // 4 atan(1), as the reference computes it
    x = y = th = xd = yd = thd = 0.0;
    const double* p = b.p;
    switch (b.motion) {
        case IBG_MOTION_FIXED:  // src/FixedPosition.h:42-44
            x = p[0]; y = p[1]; th = p[2];
            break;
        case IBG_MOTION_PITCHPLUNGE:  // src/PitchPlunge.h:52-58 (frequencies already times 2 pi)
            y = p[3] * sin(p[4] * t + p[5]);
            yd = p[3] * p[4] * cos(p[4] * t + p[5]);
            th = p[0] * sin(p[1] * t + p[2]);
            thd = p[0] * p[1] * cos(p[1] * t + p[2]);
            break;
        case IBG_MOTION_FIXEDVEL:  // src/FixedVelocity.h:49
            x = s.ix; y = s.iy; th = s.ith;
            xd = p[0]; yd = p[1]; thd = p[2];
            break;
        case IBG_MOTION_SIGMOIDALSTEP: {  // src/SigmoidalStep.h:41-51: AMP, DUR, t0
            const double arg = ((12. * (t - p[2]) / p[1]) - 6.);
            const double coeff = 12. / (p[1] * sqrt(pi));
            th = (1. / 2) * p[0] * (pi / 180) * (1. + erf(arg));
            thd = p[0] * (pi / 180) * coeff * exp(-arg * arg);
            break;
        }
        case IBG_MOTION_LAGSTEP1:    // src/LagStep1.h:41-62: AMP, PW, TAU, T0
        case IBG_MOTION_LAGSTEP2: {  // src/LagStep2.h:41-62
            const double ampr = p[0] * (pi / 180), PW = p[1], TAU = p[2], td = t - p[3];
            double a = 0., ad = 0.;
            if (td > 0 && td <= PW) {
                if (b.motion == IBG_MOTION_LAGSTEP1) {
                    a = td + TAU * exp(-td / TAU) - TAU;
                    ad = 1 - exp(-td / TAU);
                } else {
                    a = td + (2 * TAU + td) * exp(-td / TAU) - 2 * TAU;
                    ad = 1. - (1. + td / TAU) * exp(-td / TAU);
                }
            } else if (td > PW) {
                if (b.motion == IBG_MOTION_LAGSTEP1) {
                    a = PW + TAU * exp(-td / TAU) - TAU * exp(-(td - PW) / TAU);
                    ad = -1. * exp(-td / TAU) + exp(-(td - PW) / TAU);
                } else {
                    a = PW + (2 * TAU + td) * exp(-td / TAU) + (PW - 2 * TAU) * exp(-(td - PW) / TAU) -
                        td * exp(-(td - PW) / TAU);
                    ad = -(1. + td / TAU) * exp(-td / TAU) + (1. + (td - PW) / TAU) * exp(-(td - PW) / TAU);
                }
            }
            th = a * ampr / PW;
            thd = ad * ampr / PW;
            break;
        }
        case IBG_MOTION_ELDREDGE: {  // src/EldredgeManeuver.h:48-61: pitch; p[6] = maxG
            const double ampr = p[0] * (pi / 180);
            th = eld_G(p + 1, t) * ampr / p[6];
            thd = eld_dG(p + 1, t) * ampr / p[6];
            break;
        }
        case IBG_MOTION_ELDREDGE1:  // src/Eldredge1.h:46-56: plunge
            y = eld_G(p + 1, t) * p[0] / p[6];
            yd = eld_dG(p + 1, t) * p[0] / p[6];
            break;
        case IBG_MOTION_ELDREDGE2:  // src/Eldredge2.h:52-71: plunge velocity G, position its integral
            y = s.ig * p[0] / p[6];
            yd = eld_G(p + 1, t) * p[0] / p[6];
            break;
        case IBG_MOTION_ELDREDGECOMBINED2: {  // src/EldredgeCombined2.h:64-87; p[12] = maxGa, p[13] = maxGb
            const double ampr = p[6] * (pi / 180);
            y = s.ig * p[0] / p[12];
            th = eld_G(p + 7, t) * ampr / p[13];
            yd = eld_G(p + 1, t) * p[0] / p[12];
            thd = eld_dG(p + 7, t) * ampr / p[13];
            break;
        }
        case IBG_MOTION_FILE:
        case IBG_MOTION_FILE_PERIODIC: {  // src/MotionFile.h:90-115, src/MotionFilePeriodic.h:91-117
            const double tt = b.motion == IBG_MOTION_FILE_PERIODIC ? fmod(t, p[0]) : t;
            const double* r = mtab + 7 * (size_t)b.trow0;
            const int n = b.trows;
            // the interval [t_i, t_i+1) holding tt: the last row with t_i <= tt, unless it is the last row
            // (rows are non-decreasing in t, so that interval is the reference's scan result)
            if (n < 2 || !(tt >= r[0])) break;
            int lo = 0, hi = n - 1;  // r[7 lo] <= tt
            while (hi - lo > 1) {
                const int mid = (lo + hi) / 2;
                if (r[7 * mid] <= tt) lo = mid; else hi = mid;
            }
            if (r[7 * hi] <= tt) break;  // tt at or past the last row
            const double* r0 = r + 7 * lo;
            const double* r1 = r0 + 7;
            const double al = (tt - r0[0]) / (r1[0] - r0[0]);
            x = al * r1[1] + (1 - al) * r0[1];
            y = al * r1[2] + (1 - al) * r0[2];
            th = al * r1[3] + (1 - al) * r0[3];
            xd = al * r1[4] + (1 - al) * r0[4];
            yd = al * r1[5] + (1 - al) * r0[5];
            thd = al * r1[6] + (1 - al) * r0[6];
            break;
        }
        default:
            break;
    }
}

__global__ void k_kinematics(int npts, const double* __restrict__ ref_xy, const int* __restrict__ body_of,
                             const BodyDev* __restrict__ bodies, const MotionState* __restrict__ ms,
                             const double* __restrict__ mtab, const double* __restrict__ time_ptr, double toff,
                             double* __restrict__ pts, double* __restrict__ vel) {
    pdl_enter();
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npts) return;
    const int k = body_of[p];
    const BodyDev& b = bodies[k];
    const double rx = ref_xy[2 * p], ry = ref_xy[2 * p + 1];
    if (b.motion == IBG_MOTION_NONE) {
        pts[2 * p] = rx;
        pts[2 * p + 1] = ry;
        vel[2 * p] = 0.0;
        vel[2 * p + 1] = 0.0;
        return;
    }
    const double t = *time_ptr + toff;
    double x, y, th, xd, yd, thd;
    body_frame(b, ms[k], mtab, t, x, y, th, xd, yd, thd);
    // TangentSE2::mapPosition / mapVelocity about the centre (src/TangentSE2.h:83-107)
    const double a = rx - b.xc, bb = ry - b.yc;
    const double c = cos(th), s = sin(th);
    pts[2 * p] = (x + a * c - bb * s) + b.xc;
    pts[2 * p + 1] = (y + a * s + bb * c) + b.yc;
    vel[2 * p] = -a * s * thd - bb * c * thd + xd;
    vel[2 * p + 1] = a * c * thd - bb * s * thd + yd;
}

// ---------------------------------------------------------------------------
// moving-frame base flow: the body's motion carried by the base flow
// (src/BaseFlow.cc:114-150 setAlphaMag / moveFlow, src/Flux.cc:101-129 setFlow)
// ---------------------------------------------------------------------------
// One thread: out = (xdot', ydot', thetadot') of the flow seen from the body.
__global__ void k_frame_flow(const BodyDev* __restrict__ bf, MotionState* __restrict__ ms,
                             const double* __restrict__ mtab, const double* __restrict__ time_ptr, double toff,
                             double magBF, double alphaBF, double* __restrict__ out) {
    pdl_enter();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double t = *time_ptr + toff;
    const BodyDev b = *bf;
    MotionState s = *ms;
    advance_history(b, s, t);
    *ms = s;
    double x, y, th, xd, yd, thd;
    body_frame(b, s, mtab, t, x, y, th, xd, yd, thd);
    // setAlphaMag: the free stream relative to the moving body, in the body's frame
    const double xdT = xd - magBF * cos(alphaBF);
    const double ydT = yd - magBF * sin(alphaBF);
    const double gamma = atan2(ydT, -1. * xdT);
    const double alpha = -1. * th - gamma;
    const double mag = sqrt(xdT * xdT + ydT * ydT);
    out[0] = mag * cos(alpha);
    out[1] = mag * sin(alpha);
    out[2] = -1. * thd;
}

// Flux::setFlow: q0 = ((xdot' - thetadot' (y - yc)) dx, (ydot' + thetadot' (x - xc)) dx) at every flux of
// every level, at the flux positions of Grid::getXEdge / getXCenter with zero shift (src/Grid.cc:104-139)
__global__ void k_frame_flux(GridDev g, const double* __restrict__ fv, double xc, double yc, double* __restrict__ q0) {
    pdl_enter();
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= (size_t)g.L * g.F1) return;
    const int lev = (int)(tid / g.F1);
    const int idx = (int)(tid % g.F1);
    const double dxl = lev_dx(g, lev);
    const double offx = g.x0 + 0.5 * (0.0 - 1) * ((1 << lev) - 1) * (g.nx * g.dx);
    const double offy = g.y0 + 0.5 * (0.0 - 1) * ((1 << lev) - 1) * (g.ny * g.dx);
    const double xdot = fv[0], ydot = fv[1], thdot = fv[2];
    if (idx < g.nXf) {
        const int j = idx % g.ny;
        const double yd = (offy + (j + 0.5) * dxl) - yc;
        q0[tid] = (xdot - thdot * yd) * dxl;
    } else {
        const int i = (idx - g.nXf) / (g.ny + 1);
        const double xd = (offx + (i + 0.5) * dxl) - xc;
        q0[tid] = (ydot + thdot * xd) * dxl;
    }
}

// getConstraints with a base-flow field: b_c = body velocity - Regularizer::toBoundary(q0)_c
// (src/NavierStokesModel.cc:86-91, src/Regularizer.cc:111-128)
__global__ void k_bcon_field(int ncomp, const int* __restrict__ sidx, const double* __restrict__ sw,
                             const int* __restrict__ sn, const double* __restrict__ vel, const double* __restrict__ q0,
                             double h, double* __restrict__ bcon) {
    pdl_enter();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncomp) return;
    const int npts = ncomp / 2, dir = c / npts, p = c % npts;
    double e = 0.0;
    const int n = sn[c];
    for (int k = 0; k < n; ++k) e = e + sw[(size_t)c * kSlots + k] * q0[sidx[(size_t)c * kSlots + k]];
    bcon[c] = vel[2 * p + dir] - e / h;
}

__device__ __forceinline__ double delta_fn(double r) {
    if (r > 1.5) return 0.0;
    if (r <= 0.5) return (1 + sqrt(1 - 3 * r * r)) / 3;
    return (5 - 3 * r - sqrt(1 - 3 * (1 - r) * (1 - r))) / 6;
}

// Association slots per boundary component c = dir*npts + p: the level-0
// fluxes within 1.5 cells in both directions (3 x 3 in exact arithmetic, up to
// 4 x 4 when rounding puts a flux at exactly 1.5 cells), in increasing flux
// index, and
// the constraint b_c = body velocity - E(q0)_c.
__global__ void k_reg_update(GridDev g, int npts, const double* __restrict__ pts, const double* __restrict__ vel,
                             int* __restrict__ sidx, double* __restrict__ sw, int* __restrict__ sn,
                             double* __restrict__ bcon, double u0, double v0) {
    pdl_enter();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= 2 * npts) return;
    const int dir = c / npts, p = c % npts;
    const double h = g.dx;
    const double px = pts[2 * p], py = pts[2 * p + 1];
    const double offx = dir == 0 ? 0.0 : 0.5, offy = dir == 0 ? 0.5 : 0.0;
    const int ni = dir == 0 ? g.nx + 1 : g.nx;
    const int nj = dir == 0 ? g.ny : g.ny + 1;
    const int base = dir == 0 ? 0 : g.nXf;
    const int stride = dir == 0 ? g.ny : g.ny + 1;
    const int ic = (int)floor((px - g.x0) / h - offx);
    const int jc = (int)floor((py - g.y0) / h - offy);
    int n = 0;
    double e = 0.0;
    const double q0 = (dir == 0 ? u0 : v0) * h;
    for (int i = ic - 1; i <= ic + 2; ++i) {
        if (i < 0 || i >= ni) continue;
        // flux position as Flux::x (getXEdge / getXCenter): x0 + i dx or x0 + (i + .5) dx
        const double fx = dir == 0 ? __dadd_rn(g.x0, __dmul_rn((double)i, h))
                                   : __dadd_rn(g.x0, __dmul_rn((double)i + 0.5, h));
        const double dxn = fabs(fx - px) / h;
        if (!(dxn < 1.5)) continue;
        for (int j = jc - 1; j <= jc + 2; ++j) {
            if (j < 0 || j >= nj) continue;
            const double fy = dir == 0 ? __dadd_rn(g.y0, __dmul_rn((double)j + 0.5, h))
                                       : __dadd_rn(g.y0, __dmul_rn((double)j, h));
            const double dyn = fabs(fy - py) / h;
            if (!(dyn < 1.5)) continue;
            if (n < kSlots) {
                const double wgt = delta_fn(dxn) * delta_fn(dyn);
                sidx[c * kSlots + n] = base + i * stride + j;
                sw[c * kSlots + n] = wgt;
                e = e + wgt * q0;
                ++n;
            }
        }
    }
    sn[c] = n;
    const double velc = vel[2 * p + dir];
    bcon[c] = velc - e / h;
}

// rhs_c = E(Curl(psi))_c - b_c  (C operator of the projection, batched)
template <typename T>
__global__ void k_reg_interp(GridDev g, int ncomp, const int* __restrict__ sidx, const double* __restrict__ sw,
                             const int* __restrict__ sn, const T* __restrict__ psi, size_t sstride,
                             const double* __restrict__ bcon, double* __restrict__ out, size_t ostride) {
    pdl_enter();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncomp) return;
    const T* f = psi + (size_t)blockIdx.y * sstride;
    const T* cc = g.L > 1 ? f + g.N1 : nullptr;
    double acc = 0.0;
    const int n = sn[c];
    for (int k = 0; k < n; ++k) acc = acc + sw[c * kSlots + k] * (double)curl_scalar_at(g, f, cc, sidx[c * kSlots + k]);
    double v = acc / g.dx;
    if (bcon) v = v - bcon[c];
    out[(size_t)blockIdx.y * ostride + c] = v;
}

// smear: flux0[idx] += w f_c (atomic; flux0 is kept zero between uses)
// The smear's summation order (Regularizer::toFlux, src/Regularizer.cc:92-109),
// rebuilt whenever the slots are: the thread of each (component, slot) entry
// looks for the entries of the other components of the same direction that
// hold the same flux (only points within 3.5 cells can: each reaches 1.5
// cells).  The first of them in component order -- the order of the
// reference's association list (src/Regularizer.cc:54-90) -- records how many
// there are and which, in that order; the others record 0.
__global__ void k_reg_owners(int ncomp, const int* __restrict__ sidx, const int* __restrict__ sn,
                             const double* __restrict__ pts, double h, int* __restrict__ own,
                             int* __restrict__ contrib) {
    pdl_enter();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = t / kSlots, k = t % kSlots;
    if (c >= ncomp) return;
    if (k >= sn[c]) {
        own[t] = 0;
        return;
    }
    const int npts = ncomp / 2, dir = c / npts, p = c % npts;
    const int j = sidx[t];
    const double px = pts[2 * p], py = pts[2 * p + 1], lim = 3.5 * h;
    int cnt = 0;
    for (int q = 0; q < npts; ++q) {
        if (fabs(pts[2 * q] - px) > lim || fabs(pts[2 * q + 1] - py) > lim) continue;
        const int c2 = dir * npts + q;
        const int n2 = sn[c2];
        for (int k2 = 0; k2 < n2; ++k2) {
            if (sidx[c2 * kSlots + k2] != j) continue;
            if (c2 < c) {  // an earlier component writes this flux
                own[t] = 0;
                return;
            }
            if (cnt < kMaxContrib) contrib[(size_t)t * kMaxContrib + cnt] = c2 * kSlots + k2;
            ++cnt;
            break;
        }
    }
    own[t] = cnt;
}

// Regularizer::toFlux without the dx factor: the first entry of each flux writes
// the sum over its entries in the recorded order, starting from zero, products
// rounded before the sum as the reference's host arithmetic does.  No atomics,
// so the result is the same in every run.  (A flux reached by more than
// kMaxContrib entries is summed by scanning the points again, in the same order.)
__global__ void k_reg_smear(int ncomp, const int* __restrict__ sidx, const double* __restrict__ sw,
                            const int* __restrict__ sn, const int* __restrict__ own,
                            const int* __restrict__ contrib, const double* __restrict__ pts, double h,
                            const double* __restrict__ f, double* __restrict__ flux0) {
    pdl_enter();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = t / kSlots, k = t % kSlots;
    if (c >= ncomp || k >= sn[c]) return;
    const int cnt = own[t];
    if (cnt == 0) return;
    double sum = 0.0;
    if (cnt <= kMaxContrib) {
        const int* lst = contrib + (size_t)t * kMaxContrib;
        for (int q = 0; q < cnt; ++q) {
            const int e = lst[q];
            sum = __dadd_rn(sum, __dmul_rn(sw[e], f[e / kSlots]));
        }
    } else {
        const int npts = ncomp / 2, dir = c / npts, p = c % npts;
        const int j = sidx[t];
        const double px = pts[2 * p], py = pts[2 * p + 1], lim = 3.5 * h;
        for (int q = 0; q < npts; ++q) {
            if (fabs(pts[2 * q] - px) > lim || fabs(pts[2 * q + 1] - py) > lim) continue;
            const int c2 = dir * npts + q;
            const int n2 = sn[c2];
            for (int k2 = 0; k2 < n2; ++k2) {
                if (sidx[c2 * kSlots + k2] != j) continue;
                sum = __dadd_rn(sum, __dmul_rn(sw[c2 * kSlots + k2], f[c2]));
                break;
            }
        }
    }
    flux0[sidx[t]] = sum;
}

// batched smear of unit vectors: item b carries e_{col0+b}
__global__ void k_reg_smear_unit(int ncomp, int col0, const int* __restrict__ sidx, const double* __restrict__ sw,
                                 const int* __restrict__ sn, double* __restrict__ flux0, size_t fstride) {
    pdl_enter();
    const int b = blockIdx.x;
    const int c = col0 + b;
    const int k = threadIdx.x;
    if (c >= ncomp || k >= sn[c]) return;
    flux0[(size_t)b * fstride + sidx[c * kSlots + k]] = sw[c * kSlots + k];
}

__global__ void k_reg_zero(int ncomp, int col0, int unit, const int* __restrict__ sidx, const int* __restrict__ sn,
                           double* __restrict__ flux0, size_t fstride) {
    pdl_enter();
    if (unit) {
        const int b = blockIdx.x, c = col0 + b, k = threadIdx.x;
        if (c >= ncomp || k >= sn[c]) return;
        flux0[(size_t)b * fstride + sidx[c * kSlots + k]] = 0.0;
        return;
    }
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = t / kSlots, k = t % kSlots;
    if (c >= ncomp || k >= sn[c]) return;
    flux0[sidx[c * kSlots + k]] = 0.0;
}

// Bf on level 0: beta * Curl(flux0 * dx); coarser levels of Bf stay zero
template <typename T>
__global__ void k_bf(GridDev g, const double* __restrict__ flux0, size_t fstride, T* __restrict__ Bf, size_t sstride,
                     double beta) {
    pdl_enter();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= g.N1) return;
    const double* q = flux0 + (size_t)blockIdx.y * fstride;
    const int i = r / g.NJ + 1, j = r % g.NJ + 1;
    const double h = g.dx;
    const double bydx2 = 1. / (h * h);
    const double qyij = qy_at(q, g, i, j) * h, qyim = qy_at(q, g, i - 1, j) * h;
    const double qxjm = qx_at(q, g, i, j - 1) * h, qxij = qx_at(q, g, i, j) * h;
    Bf[(size_t)blockIdx.y * sstride + r] = (T)(((qyij - qyim + qxjm - qxij) * bydx2) * beta);
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
static inline unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

template <typename T>
void launch_nonlinear_flux(const GridDev& g, const T* q, const T* w, T* U, T* V, T* C, int batch, size_t sstride,
                           size_t fstride, cudaStream_t st) {
    launch_k(k_node_vel<T>, dim3(nblk(g.N1, 256), (unsigned)g.L, batch), 256, 0, st, g, q, w, U, V, sstride, fstride);
    for (int lev = 0; lev < g.L; ++lev)
        launch_k(k_cross_flux<T>, dim3(nblk(g.F1, 256), batch), 256, 0, st, g, lev, U, V, C, sstride, fstride);
}

template <typename T>
void launch_nonlinear(const GridDev& g, const T* q, const T* w, T* U, T* V, T* C, T* N, int batch, size_t sstride,
                      size_t fstride, cudaStream_t st) {
    launch_nonlinear_flux<T>(g, q, w, U, V, C, batch, sstride, fstride, st);
    launch_k(k_curl_flux<T>, dim3(nblk(g.N1, 256), (unsigned)g.L, batch), 256, 0, st, g, C, N, sstride, fstride);
}

template <typename T>
void launch_curl_rhs(const GridDev& g, const T* C, T* N, const T* w, const T* Nprev, T* a, double c1, double an,
                     double bn, double dt, cudaStream_t st) {
    launch_k(k_curl_rhs<T>, dim3(nblk(g.N1, 256), (unsigned)g.L), 256, 0, st, g, C, N, w, Nprev, a, (T)c1, (T)an, (T)bn,
             (T)dt);
}

void launch_nonlinear_lin(const GridDev& g, const double* q, const double* w, const double* qb, const double* wb,
                          int period, const int* ts0, const int* count, double* U, double* V, double* C, double* N,
                          cudaStream_t st) {
    const size_t S = (size_t)g.L * g.N1, F = (size_t)g.L * g.F1;
    launch_k(k_node_vel_lin, nblk(S, 256), 256, 0, st, g, q, w, qb, wb, period, ts0, count, U, V);
    for (int lev = 0; lev < g.L; ++lev)
        launch_k(k_cross_flux<double>, dim3(nblk(g.F1, 256), 1), 256, 0, st, g, lev, U, V, C, S, F);
    launch_k(k_curl_flux<double>, dim3(nblk(g.N1, 256), (unsigned)g.L, 1), 256, 0, st, g, C, N, S, F);
}

void launch_flux_cross(const GridDev& g, const double* q1, const double* q2, double* out, cudaStream_t st) {
    const size_t S = (size_t)g.L * g.N1;
    launch_k(k_flux_cross, nblk(S, 256), 256, 0, st, g, q1, q2, out);
}

void launch_sub(size_t n, const double* a, const double* b, double* out, cudaStream_t st) {
    launch_k(k_sub, nblk(n, 256), 256, 0, st, n, a, b, out);
}

void launch_sfd(size_t n, const double* w, double* what, double* rprev, double* N, double chi, double Delta,
                double an, double bn, double dt, bool first, cudaStream_t st) {
    launch_k(k_sfd, nblk(n, 256), 256, 0, st, n, w, what, rprev, N, chi, Delta, an, bn, dt, first ? 1 : 0);
}

template <typename T>
void launch_curl_flux(const GridDev& g, const T* C, T* N, cudaStream_t st) {
    const size_t S = (size_t)g.L * g.N1;
    launch_k(k_curl_flux<T>, dim3(nblk(g.N1, 256), (unsigned)g.L, 1), 256, 0, st, g, C, N, S, (size_t)g.L * g.F1);
}

template <typename T>
void launch_rhs(const GridDev& g, const T* w, const T* N, const T* Nprev, T* a, double c1, double an, double bn,
                double dt, cudaStream_t st) {
    launch_k(k_rhs<T>, dim3(nblk(g.N1, 256), (unsigned)g.L), 256, 0, st, g, w, N, Nprev, a, (T)c1, (T)an, (T)bn, (T)dt, 0);
}

template <typename T>
void launch_laplacian(const GridDev& g, const T* w, T* out, cudaStream_t st) {
    launch_k(k_rhs<T>, dim3(nblk(g.N1, 256), (unsigned)g.L), 256, 0, st, g, w, nullptr, nullptr, out, (T)0, (T)0, (T)0,
             (T)0, 1);
}

// E applied to given level-0 fluxes (Regularizer::toBoundary)
__global__ void k_reg_gather(int ncomp, const int* __restrict__ sidx, const double* __restrict__ sw,
                             const int* __restrict__ sn, const double* __restrict__ q0, double dx,
                             double* __restrict__ out) {
    pdl_enter();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncomp) return;
    double acc = 0.0;
    for (int k = 0; k < sn[c]; ++k) acc = acc + sw[c * kSlots + k] * q0[sidx[c * kSlots + k]];
    out[c] = acc / dx;
}

void launch_reg_gather(const GridDev& g, int ncomp, const RegSlots& s, const double* q0, double* out,
                       cudaStream_t st) {
    launch_k(k_reg_gather, nblk(ncomp, 128), 128, 0, st, ncomp, s.idx, s.w, s.n, q0, g.dx, out);
}

template <typename T>
void launch_refresh_flux(const GridDev& g, const T* psi, T* q, double u0, double v0, const double* q0f,
                         cudaStream_t st) {
    launch_k(k_refresh_flux<T>, dim3(nblk(g.F1, 256), (unsigned)g.L), 256, 0, st, g, psi, q, u0, v0, q0f);
}

void launch_flux_to_vel(const GridDev& g, const double* q, double* u, double* v, cudaStream_t st) {
    const size_t S = (size_t)g.L * g.N1;
    launch_k(k_flux_to_vel, nblk(S, 256), 256, 0, st, g, q, u, v);
}

void launch_frame_flow(const BodyDev* bf, MotionState* ms, const double* mtab, const double* time_ptr, double toff,
                       double magBF, double alphaBF, double* out, cudaStream_t st) {
    launch_k(k_frame_flow, 1, 32, 0, st, bf, ms, mtab, time_ptr, toff, magBF, alphaBF, out);
}

void launch_frame_flux(const GridDev& g, const double* fv, double xc, double yc, double* q0, cudaStream_t st) {
    const size_t F = (size_t)g.L * g.F1;
    launch_k(k_frame_flux, nblk(F, 256), 256, 0, st, g, fv, xc, yc, q0);
}

void launch_bcon_field(int ncomp, const RegSlots& s, const double* vel, const double* q0, double h, double* bcon,
                       cudaStream_t st) {
    launch_k(k_bcon_field, nblk(ncomp, 128), 128, 0, st, ncomp, s.idx, s.w, s.n, vel, q0, h, bcon);
}

void launch_motion_state(int nbodies, const BodyDev* bodies, const double* time_ptr, double toff, MotionState* ms,
                         cudaStream_t st) {
    launch_k(k_motion_state, nblk(nbodies, 32), 32, 0, st, nbodies, bodies, time_ptr, toff, ms);
}

void launch_kinematics(int npts, const double* ref_xy, const int* body_of, const BodyDev* bodies,
                       const MotionState* ms, const double* mtab, const double* time_ptr, double toff, double* pts,
                       double* vel, cudaStream_t st) {
    launch_k(k_kinematics, nblk(npts, 128), 128, 0, st, npts, ref_xy, body_of, bodies, ms, mtab, time_ptr, toff, pts, vel);
}

void launch_reg_update(const GridDev& g, int npts, const double* pts, const double* vel, RegSlots& s, double* bcon,
                       double u0, double v0, double* flux0, cudaStream_t st) {
    // flux0 is zero outside the current slots' flux indices (launch_smear_bf): clear the old ones first
    if (flux0)
        launch_k(k_reg_zero, nblk((size_t)2 * npts * kSlots, 128), 128, 0, st, 2 * npts, 0, 0, (const int*)s.idx,
                 (const int*)s.n, flux0, (size_t)0);
    launch_k(k_reg_update, nblk(2 * npts, 128), 128, 0, st, g, npts, pts, vel, s.idx, s.w, s.n, bcon, u0, v0);
    launch_k(k_reg_owners, nblk((size_t)2 * npts * kSlots, 128), 128, 0, st, 2 * npts, (const int*)s.idx,
             (const int*)s.n, pts, g.dx, s.own, s.contrib);
}

template <typename T>
void launch_reg_interp(const GridDev& g, int ncomp, const RegSlots& s, const T* psi, size_t sstride, int batch,
                       const double* bcon, double* out, size_t ostride, cudaStream_t st) {
    launch_k(k_reg_interp<T>, dim3(nblk(ncomp, 128), batch), 128, 0, st, g, ncomp, s.idx, s.w, s.n, psi, sstride, bcon, out,
                                                                    ostride);
}

// flux0 is zero outside the current slots' flux indices.  Every such index has one owner, which
// writes the full sum, so a smear overwrites exactly the indices the previous smear with the same
// slots wrote and needs no clearing; launch_reg_update clears the old indices before the slots move.
template <typename T>
void launch_smear_bf(const GridDev& g, int ncomp, const RegSlots& s, const double* f, double* flux0, T* Bf,
                     double beta, cudaStream_t st) {
    launch_k(k_reg_smear, nblk((size_t)ncomp * kSlots, 128), 128, 0, st, ncomp, (const int*)s.idx,
             (const double*)s.w, (const int*)s.n, (const int*)s.own, (const int*)s.contrib, s.pts, g.dx, f, flux0);
    launch_k(k_bf<T>, dim3(nblk(g.N1, 256), 1), 256, 0, st, g, flux0, 0, Bf, 0, beta);
}

void launch_reg_smear(int ncomp, const RegSlots& s, double h, const double* f, double* flux0, cudaStream_t st) {
    launch_k(k_reg_smear, nblk((size_t)ncomp * kSlots, 128), 128, 0, st, ncomp, (const int*)s.idx,
             (const double*)s.w, (const int*)s.n, (const int*)s.own, (const int*)s.contrib, s.pts, h, f, flux0);
}
void launch_reg_zero(int ncomp, const RegSlots& s, double* flux0, cudaStream_t st) {
    launch_k(k_reg_zero, nblk((size_t)ncomp * kSlots, 128), 128, 0, st, ncomp, 0, 0, s.idx, s.n, flux0, 0);
}

template <typename T>
void launch_smear_bf_unit(const GridDev& g, int ncomp, int col0, int batch, const RegSlots& s, double* flux0,
                          size_t fstride, T* Bf, size_t sstride, double beta, cudaStream_t st) {
    launch_k(k_reg_smear_unit, batch, 32, 0, st, ncomp, col0, s.idx, s.w, s.n, flux0, fstride);
    launch_k(k_bf<T>, dim3(nblk(g.N1, 256), batch), 256, 0, st, g, flux0, fstride, Bf, sstride, beta);
    launch_k(k_reg_zero, batch, 32, 0, st, ncomp, col0, 1, s.idx, s.n, flux0, fstride);
}

#define IBG_INST(T)                                                                                            \
    template void launch_nonlinear<T>(const GridDev&, const T*, const T*, T*, T*, T*, T*, int, size_t, size_t, \
                                      cudaStream_t);                                                           \
    template void launch_curl_flux<T>(const GridDev&, const T*, T*, cudaStream_t);                             \
    template void launch_nonlinear_flux<T>(const GridDev&, const T*, const T*, T*, T*, T*, int, size_t, size_t, \
                                           cudaStream_t);                                                      \
    template void launch_curl_rhs<T>(const GridDev&, const T*, T*, const T*, const T*, T*, double, double,     \
                                     double, double, cudaStream_t);                                            \
    template void launch_rhs<T>(const GridDev&, const T*, const T*, const T*, T*, double, double, double,      \
                                double, cudaStream_t);                                                         \
    template void launch_laplacian<T>(const GridDev&, const T*, T*, cudaStream_t);                             \
    template void launch_refresh_flux<T>(const GridDev&, const T*, T*, double, double, const double*, cudaStream_t);          \
    template void launch_reg_interp<T>(const GridDev&, int, const RegSlots&, const T*, size_t, int,            \
                                       const double*, double*, size_t, cudaStream_t);                          \
    template void launch_smear_bf<T>(const GridDev&, int, const RegSlots&, const double*, double*, T*, double, \
                                     cudaStream_t);                                                            \
    template void launch_smear_bf_unit<T>(const GridDev&, int, int, int, const RegSlots&, double*, size_t, T*, \
                                          size_t, double, cudaStream_t);
IBG_INST(double)
IBG_INST(float)

}  // namespace ibg
