// kernels_step.cuh -- eddy viscosity, wall model and the fused RHS + RK3 stage kernel.
#pragma once

#include "dfdm_common.cuh"

namespace dfdm {

// Everything a step kernel reads besides the fields.  Metric arrays are offset so index -1 is valid.
template <typename T> struct StepArgs {
    Dims d;
    Metric1D<T> my, mz;          // y and z metrics in the storage type
    Metric1D<double> myd, mzd;   // the same in double (wall model, reductions)
    T nu, inv_dx, inv_dx2, dx2;
    T dPdx, dPdz;
    T w_adv;                     // 0.5 skew-symmetric, 0 divergence form
    int nwl;                     // divergence-form wall band (adv_wall_layers)
    int wm;                      // flat-wall EQWM on both no-slip walls
    int sgs_model;               // 1 Vreman, 2 AMD
    T C_amd, c_V;
    double nu_d, Ly, yg2, ygtop; // wall distances of the first centres: yg(2), Ly - yg(nyg-1)
};

// ---------------------------------------------------------------------------------------------------------------
// Reichardt law and the Newton solve for u_tau (src/wallmodel.f90:29-74), always in double.
__device__ __forceinline__ void reichardt_uplus(double yplus, double &uplus, double &duplus) {
    const double kappa = 0.41, A1 = 11.0, A2 = 0.33;
    const double c_buf = 5.2 - log(kappa) / kappa;
    double a1i = 1.0 / A1;
    double e1 = exp(-yplus * a1i);
    double e2 = exp(-A2 * yplus);
    uplus = log(1.0 + kappa * yplus) / kappa + c_buf * (1.0 - e1 - yplus * a1i * e2);
    duplus = 1.0 / (1.0 + kappa * yplus) + c_buf * (a1i * e1 - a1i * e2 + yplus * a1i * A2 * e2);
}
__device__ __forceinline__ double solve_u_tau(double u_ref, double y_ref, double nu_l) {
    double u_tau = fmax(1e-3 * u_ref, sqrt(nu_l * u_ref / fmax(y_ref, 1e-14)));
    for (int iter = 1; iter <= 20; ++iter) {   // n_iter_wm = 20, bounded
        double yplus = u_tau * y_ref / nu_l, uplus, duplus;
        reichardt_uplus(yplus, uplus, duplus);
        double f = u_ref / fmax(u_tau, 1e-20) - uplus;
        double fp = -u_ref / fmax(u_tau * u_tau, 1e-20) - duplus * y_ref / nu_l;
        double u_tau_new = u_tau - f / (fp + copysign(1e-14, fp));
        u_tau_new = fmin(fmax(u_tau_new, 0.1 * u_tau), 10.0 * u_tau);
        if (fabs(u_tau_new - u_tau) < 1e-6 * u_tau_new) { u_tau = u_tau_new; break; }
        u_tau = u_tau_new;
    }
    return u_tau;
}

// ---------------------------------------------------------------------------------------------------------------
// Eddy viscosity at the cell centres: compute_vreman pass 1 (src/sgs_model.f90:118-223) with the AMD
// (Rozema et al. 2015) or Vreman (2004) closure and the wall-modelled first-cell gradient override (:158-172).
// Ghost values are implied by the read rules (sgs_fill_ghosts, :458-531).
template <typename T>
__global__ void __launch_bounds__(256) k_sgs(StepArgs<T> a, const T *__restrict__ U, const T *__restrict__ V,
                                             const T *__restrict__ W, T *__restrict__ nut) {
    const Dims &d = a.d;
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= d.Nx || j >= d.Ny) return;
    typedef Arith<T> A;
    const Metric1D<T> &my = a.my, &mz = a.mz;
    int im = wrap(i - 1, d.Nx), ip = wrap(i + 1, d.Nx), km = wrap(k - 1, d.Nz), kp = wrap(k + 1, d.Nz);
    T dz_c = mz.dc[k], dz2 = dz_c * dz_c;
    T inv_dz_k = A::inv(mz.dc, mz.idc, k), inv_zg_km = A::inv(mz.df, mz.idf, k - 1), inv_zg_kp = A::inv(mz.df, mz.idf, k);
    T dy_c = my.dc[j], dy2_c = dy_c * dy_c;
    T inv_yg_jm = A::inv(my.df, my.idf, j - 1), inv_yg_jp = A::inv(my.df, my.idf, j), inv_dy_j = A::inv(my.dc, my.idc, j);
    T inv_dx = a.inv_dx, dx2 = a.dx2;
    T Uc = __ldg(U + idx3(d, i, j, k));
    T a11 = (Uc - __ldg(U + idx3(d, im, j, k))) * inv_dx;
    T a21 = T(0.5) * ((Uc - ld_yc(U, d, i, j - 1, k)) * inv_yg_jm + (ld_yc(U, d, i, j + 1, k) - Uc) * inv_yg_jp);
    T a31 = T(0.5) * ((Uc - __ldg(U + idx3(d, i, j, km))) * inv_zg_km + (__ldg(U + idx3(d, i, j, kp)) - Uc) * inv_zg_kp);
    T Vc = ld_yf(V, d, i, j, k);
    T a12 = T(0.5) * ((Vc - ld_yf(V, d, im, j, k)) + (ld_yf(V, d, ip, j, k) - Vc)) * inv_dx;
    T a22 = (Vc - ld_yf(V, d, i, j - 1, k)) * inv_dy_j;
    T a32 = T(0.5) * ((Vc - ld_yf(V, d, i, j, km)) * inv_zg_km + (ld_yf(V, d, i, j, kp) - Vc) * inv_zg_kp);
    T Wc = __ldg(W + idx3(d, i, j, k));
    T a13 = T(0.5) * ((Wc - __ldg(W + idx3(d, im, j, k))) + (__ldg(W + idx3(d, ip, j, k)) - Wc)) * inv_dx;
    T a23 = T(0.5) * ((Wc - ld_yc(W, d, i, j - 1, k)) * inv_yg_jm + (ld_yc(W, d, i, j + 1, k) - Wc) * inv_yg_jp);
    T a33 = (Wc - __ldg(W + idx3(d, i, j, km))) * inv_dz_k;
    if (a.wm && (j == 0 || j == d.Ny - 1)) {
        double y_w = (j == 0) ? a.yg2 : a.ygtop;
        double u_c = 0.5 * ((double)__ldg(U + idx3(d, im, j, k)) + (double)Uc);
        double w_c = 0.5 * ((double)__ldg(W + idx3(d, i, j, km)) + (double)Wc);
        double u_mag = sqrt(u_c * u_c + w_c * w_c);
        if (u_mag > 1e-14) {
            double u_tau = solve_u_tau(u_mag, y_w, a.nu_d);
            double fac_w = ((j == 0) ? 1.0 : -1.0) * u_tau / (0.41 * y_w * u_mag);
            a21 = (T)(fac_w * u_c);
            a23 = (T)(fac_w * w_c);
        }
    }
    T b11 = dx2 * (a11 * a11) + dy2_c * (a21 * a21) + dz2 * (a31 * a31);
    T b22 = dx2 * (a12 * a12) + dy2_c * (a22 * a22) + dz2 * (a32 * a32);
    T b33 = dx2 * (a13 * a13) + dy2_c * (a23 * a23) + dz2 * (a33 * a33);
    T b12 = dx2 * (a11 * a12) + dy2_c * (a21 * a22) + dz2 * (a31 * a32);
    T b13 = dx2 * (a11 * a13) + dy2_c * (a21 * a23) + dz2 * (a31 * a33);
    T b23 = dx2 * (a12 * a13) + dy2_c * (a22 * a23) + dz2 * (a32 * a33);
    T alpha_sq = a11 * a11 + a12 * a12 + a13 * a13 + a21 * a21 + a22 * a22 + a23 * a23 + a31 * a31 + a32 * a32 + a33 * a33;
    T nu_t = T(0);
    if (a.sgs_model == 2) {
        T amd_num = -(b11 * a11 + b22 * a22 + b33 * a33 + b12 * (a12 + a21) + b13 * (a13 + a31) + b23 * (a23 + a32));
        if (alpha_sq > T(1e-20) && amd_num > T(1e-12) * (dx2 + dy2_c + dz2) * alpha_sq * sqrt(alpha_sq))
            nu_t = a.C_amd * amd_num / alpha_sq;
    } else {
        T B_beta = b11 * b22 - b12 * b12 + b11 * b33 - b13 * b13 + b22 * b33 - b23 * b23;
        if (alpha_sq > T(1e-20) && B_beta > T(0)) nu_t = a.c_V * sqrt(B_beta / alpha_sq);
    }
    nut[idx3(d, i, j, k)] = nu_t;
}

// ---------------------------------------------------------------------------------------------------------------
// Flat-wall EQWM state, one plane per wall (iw = 0 bottom, 1 top), index (iw*Nz + k)*Nx + i.
struct WallState {
    double *tau_x, *tau_z;                       // wall shear at U faces / W faces
    double *ux, *wx, *tx, *uz, *wz, *tz;         // filtered velocity and u_tau (wmf_* of src/global.f90:343)
};

// update_wm_filter (src/wallmodel.f90:397-439): one thread per (i,k), both walls, U-face and W-face sets.
template <typename T>
__global__ void k_wm_filter(StepArgs<T> a, WallState ws, const T *__restrict__ U, const T *__restrict__ W, int seed,
                            double dt, double Tf_fac) {
    const Dims &d = a.d;
    int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (i >= d.Nx) return;
    const double kap = 0.41;
    int im = wrap(i - 1, d.Nx), km = wrap(k - 1, d.Nz);
    for (int iw = 0; iw < 2; ++iw) {
        int jm = (iw == 0) ? 0 : d.Ny - 1;
        double ym = fmax((iw == 0) ? a.yg2 : a.ygtop, 1e-14);
        long long p = ((long long)iw * d.Nz + k) * d.Nx + i;
        double eps = 1.0;
        if (!seed && ws.tx[p] > 0.0) eps = fmin(1.0, dt * kap * ws.tx[p] / (Tf_fac * ym));
        ws.ux[p] = (1.0 - eps) * ws.ux[p] + eps * (double)U[idx3(d, i, jm, k)];
        ws.wx[p] = (1.0 - eps) * ws.wx[p] + eps * 0.5 * ((double)W[idx3(d, i, jm, km)] + (double)W[idx3(d, i, jm, k)]);
        eps = 1.0;
        if (!seed && ws.tz[p] > 0.0) eps = fmin(1.0, dt * kap * ws.tz[p] / (Tf_fac * ym));
        ws.uz[p] = (1.0 - eps) * ws.uz[p] + eps * 0.5 * ((double)U[idx3(d, im, jm, k)] + (double)U[idx3(d, i, jm, k)]);
        ws.wz[p] = (1.0 - eps) * ws.wz[p] + eps * (double)W[idx3(d, i, jm, k)];
    }
}

// compute_flat_wall_eqwm (src/wallmodel.f90:442-583), smooth Reichardt law, matching height = first centre.
template <typename T>
__global__ void k_wall_model(StepArgs<T> a, WallState ws, const T *__restrict__ U, const T *__restrict__ W, int filter) {
    const Dims &d = a.d;
    int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (i >= d.Nx) return;
    int im = wrap(i - 1, d.Nx), km = wrap(k - 1, d.Nz);
    for (int iw = 0; iw < 2; ++iw) {
        int jw = (iw == 0) ? 0 : d.Ny - 1;
        double y_match = fmax((iw == 0) ? a.yg2 : a.ygtop, 1e-14);
        long long p = ((long long)iw * d.Nz + k) * d.Nx + i;
        // U faces
        double Uw = (double)U[idx3(d, i, jw, k)];
        double W_at = 0.5 * ((double)W[idx3(d, i, jw, km)] + (double)W[idx3(d, i, jw, k)]);
        double u_ref = sqrt(Uw * Uw + W_at * W_at), u_match = u_ref, num = Uw;
        if (filter) { u_match = sqrt(ws.ux[p] * ws.ux[p] + ws.wx[p] * ws.wx[p]); num = ws.ux[p]; u_ref = u_match; }
        double u_tau = solve_u_tau(u_match, y_match, a.nu_d);
        ws.tx[p] = u_tau;
        double tv = u_tau * u_tau * num / fmax(u_ref, 1e-30);
        ws.tau_x[p] = (iw == 0) ? tv : -tv;
        // W faces
        double uc = 0.5 * ((double)U[idx3(d, im, jw, k)] + Uw);
        double Ww = (double)W[idx3(d, i, jw, k)];
        u_ref = sqrt(uc * uc + Ww * Ww); u_match = u_ref; num = Ww;
        if (filter) { u_match = sqrt(ws.uz[p] * ws.uz[p] + ws.wz[p] * ws.wz[p]); num = ws.wz[p]; u_ref = u_match; }
        u_tau = solve_u_tau(u_match, y_match, a.nu_d);
        ws.tz[p] = u_tau;
        tv = u_tau * u_tau * num / fmax(u_ref, 1e-30);
        ws.tau_z[p] = (iw == 0) ? tv : -tv;
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Right-hand sides (src/equations.f90), evaluated in the reference's expression order at one index (i,j,k).
template <typename T> struct Fields {
    const T *__restrict__ U; const T *__restrict__ V; const T *__restrict__ W; const T *__restrict__ nut;
};

template <typename T, bool LES>
__device__ __forceinline__ T rhs_u_at(const StepArgs<T> &a, const Fields<T> &f, const double *__restrict__ tau_x,
                                      int i, int j, int k) {
    const Dims &d = a.d;
    typedef Arith<T> A;
    const Metric1D<T> &my = a.my, &mz = a.mz;
    int im = wrap(i - 1, d.Nx), ip = wrap(i + 1, d.Nx), km = wrap(k - 1, d.Nz), kp = wrap(k + 1, d.Nz);
    const T *U = f.U, *V = f.V, *W = f.W;
    T Uc = __ldg(U + idx3(d, i, j, k)), Uim = __ldg(U + idx3(d, im, j, k)), Uip = __ldg(U + idx3(d, ip, j, k));
    T Ujm = ld_yc(U, d, i, j - 1, k), Ujp = ld_yc(U, d, i, j + 1, k);
    T Ukm = __ldg(U + idx3(d, i, j, km)), Ukp = __ldg(U + idx3(d, i, j, kp));
    bool wm_band = a.wm && (j + 2 <= 1 + a.nwl || j + 2 >= d.Ny + 2 - a.nwl);
    T wa = wm_band ? T(0) : a.w_adv, wd = T(1) - wa;
    // -d(uu)/dx
    T t1 = T(0.5) * (Uc + Uip), t0 = T(0.5) * (Uim + Uc);
    T r = -(wd * (t1 * t1 - t0 * t0) + wa * Uc * (t1 - t0)) * a.inv_dx;
    // -d(uv)/dy: u at y faces j-1, j (weighted), v at x faces (plain average)
    {
        T u1 = my.w0[j] * Uc + my.w1[j] * Ujp, u0 = my.w0[j - 1] * Ujm + my.w1[j - 1] * Uc;
        T v1 = T(0.5) * (ld_yf(V, d, i, j, k) + ld_yf(V, d, ip, j, k));
        T v0 = T(0.5) * (ld_yf(V, d, i, j - 1, k) + ld_yf(V, d, ip, j - 1, k));
        r = r - A::div(wd * (u1 * v1 - u0 * v0) + wa * T(0.5) * (v0 + v1) * (u1 - u0), my.dc, my.idc, j);
    }
    // -d(uw)/dz
    {
        T u1 = mz.w0[k] * Uc + mz.w1[k] * Ukp, u0 = mz.w0[k - 1] * Ukm + mz.w1[k - 1] * Uc;
        T w1 = T(0.5) * (__ldg(W + idx3(d, i, j, k)) + __ldg(W + idx3(d, ip, j, k)));
        T w0 = T(0.5) * (__ldg(W + idx3(d, i, j, km)) + __ldg(W + idx3(d, ip, j, km)));
        r = r - A::div(wd * (u1 * w1 - u0 * w0) + wa * T(0.5) * (w0 + w1) * (u1 - u0), mz.dc, mz.idc, k);
    }
    // viscous: d(2 nu_x du/dx)/dx + d(nu_y (du/dy + dv/dx))/dy + d(nu_z (du/dz + dw/dx))/dz + dPdx
    T inv_dz3 = A::inv(mz.dc, mz.idc, k), inv_dy3 = A::inv(my.dc, my.idc, j);
    T nu = a.nu;
    T nu_x1 = nu, nu_x2 = nu, nu_y1 = nu, nu_y2 = nu, nu_z1 = nu, nu_z2 = nu;
    if (LES) {
        const T *N = f.nut;
        T n_c = ld_nu(N, d, i, j, k), n_p = ld_nu(N, d, ip, j, k);
        nu_x1 = nu + n_c; nu_x2 = nu + n_p;
        if (!(d.yper == 0 && j == 0))
            nu_y1 = nu + T(0.5) * (my.w0[j - 1] * ld_nu(N, d, i, j - 1, k) + my.w1[j - 1] * n_c +
                                   my.w0[j - 1] * ld_nu(N, d, ip, j - 1, k) + my.w1[j - 1] * n_p);
        if (!(d.yper == 0 && j == d.Ny - 1))
            nu_y2 = nu + T(0.5) * (my.w0[j] * n_c + my.w1[j] * ld_nu(N, d, i, j + 1, k) +
                                   my.w0[j] * n_p + my.w1[j] * ld_nu(N, d, ip, j + 1, k));
        nu_z1 = nu + T(0.5) * (mz.w0[k - 1] * (ld_nu(N, d, i, j, km) + ld_nu(N, d, ip, j, km)) + mz.w1[k - 1] * (n_c + n_p));
        nu_z2 = nu + T(0.5) * (mz.w0[k] * (n_c + n_p) + mz.w1[k] * (ld_nu(N, d, i, j, kp) + ld_nu(N, d, ip, j, kp)));
    }
    T tj = A::div(Ujp - Uc, my.df, my.idf, j), tjm = A::div(Uc - Ujm, my.df, my.idf, j - 1);
    T fy2 = nu_y2 * (tj + (ld_yf(V, d, ip, j, k) - ld_yf(V, d, i, j, k)) * a.inv_dx);
    T fy1 = nu_y1 * (tjm + (ld_yf(V, d, ip, j - 1, k) - ld_yf(V, d, i, j - 1, k)) * a.inv_dx);
    if (a.wm) {
        if (j == 0) fy1 = (T)tau_x[(long long)k * d.Nx + i];
        if (j == d.Ny - 1) fy2 = (T)tau_x[((long long)d.Nz + k) * d.Nx + i];
    }
    T tk = A::div(Ukp - Uc, mz.df, mz.idf, k), tkm = A::div(Uc - Ukm, mz.df, mz.idf, k - 1);
    T fz2 = nu_z2 * (tk + (__ldg(W + idx3(d, ip, j, k)) - __ldg(W + idx3(d, i, j, k))) * a.inv_dx);
    T fz1 = nu_z1 * (tkm + (__ldg(W + idx3(d, ip, j, km)) - __ldg(W + idx3(d, i, j, km))) * a.inv_dx);
    r = r + T(2) * a.inv_dx2 * (nu_x2 * (Uip - Uc) - nu_x1 * (Uc - Uim)) + inv_dy3 * (fy2 - fy1) + inv_dz3 * (fz2 - fz1) + a.dPdx;
    return r;
}

template <typename T, bool LES>
__device__ __forceinline__ T rhs_v_at(const StepArgs<T> &a, const Fields<T> &f, int i, int j, int k) {
    const Dims &d = a.d;
    typedef Arith<T> A;
    const Metric1D<T> &my = a.my, &mz = a.mz;
    int im = wrap(i - 1, d.Nx), ip = wrap(i + 1, d.Nx), km = wrap(k - 1, d.Nz), kp = wrap(k + 1, d.Nz);
    const T *U = f.U, *V = f.V, *W = f.W;
    T wa = a.w_adv, wd = T(1) - wa;
    T Vc = ld_yf(V, d, i, j, k), Vjm = ld_yf(V, d, i, j - 1, k), Vjp = ld_yf(V, d, i, j + 1, k);
    T Vim = ld_yf(V, d, im, j, k), Vip = ld_yf(V, d, ip, j, k);
    T Vkm = ld_yf(V, d, i, j, km), Vkp = ld_yf(V, d, i, j, kp);
    // -d(vv)/dy
    T t1 = T(0.5) * (Vc + Vjp), t0 = T(0.5) * (Vjm + Vc);
    T r = -A::div(wd * (t1 * t1 - t0 * t0) + wa * Vc * (t1 - t0), my.df, my.idf, j);
    // -d(uv)/dx: u at y face j (weighted), v at x faces
    T Uc = __ldg(U + idx3(d, i, j, k)), Um = __ldg(U + idx3(d, im, j, k));
    T Ucp = ld_yc(U, d, i, j + 1, k), Ump = ld_yc(U, d, im, j + 1, k);
    {
        T u1 = my.w0[j] * Uc + my.w1[j] * Ucp, u0 = my.w0[j] * Um + my.w1[j] * Ump;
        T v1 = T(0.5) * (Vc + Vip), v0 = T(0.5) * (Vim + Vc);
        r = r - (wd * (u1 * v1 - u0 * v0) + wa * T(0.5) * (u0 + u1) * (v1 - v0)) * a.inv_dx;
    }
    // -d(vw)/dz: v at z faces (weighted), w at y face j (weighted)
    T Wc = __ldg(W + idx3(d, i, j, k)), Wjp = ld_yc(W, d, i, j + 1, k);
    T Wkm = __ldg(W + idx3(d, i, j, km)), Wkmjp = ld_yc(W, d, i, j + 1, km);
    {
        T v1 = mz.w0[k] * Vc + mz.w1[k] * Vkp, v0 = mz.w0[k - 1] * Vkm + mz.w1[k - 1] * Vc;
        T w1 = my.w0[j] * Wc + my.w1[j] * Wjp, w0 = my.w0[j] * Wkm + my.w1[j] * Wkmjp;
        r = r - A::div(wd * (v1 * w1 - v0 * w0) + wa * T(0.5) * (w0 + w1) * (v1 - v0), mz.dc, mz.idc, k);
    }
    // viscous
    T inv_dz3 = A::inv(mz.dc, mz.idc, k);
    T inv_dzg1 = A::inv(mz.df, mz.idf, k - 1), inv_dzg2 = A::inv(mz.df, mz.idf, k);
    T inv_dy1 = A::inv(my.dc, my.idc, j), inv_dy2 = A::inv(my.dc, my.idc, j + 1), inv_dy3 = A::inv(my.df, my.idf, j);
    T two_inv_dy3 = T(2) * inv_dy3;
    T nu = a.nu;
    T nu_x1 = nu, nu_x2 = nu, nu_y1 = nu, nu_y2 = nu, nu_z1 = nu, nu_z2 = nu;
    if (LES) {
        const T *N = f.nut;
        T n_c = ld_nu(N, d, i, j, k), n_jp = ld_nu(N, d, i, j + 1, k);
        T w0 = my.w0[j], w1 = my.w1[j];
        nu_x1 = nu + T(0.5) * (w0 * ld_nu(N, d, im, j, k) + w1 * ld_nu(N, d, im, j + 1, k) + w0 * n_c + w1 * n_jp);
        nu_x2 = nu + T(0.5) * (w0 * n_c + w1 * n_jp + w0 * ld_nu(N, d, ip, j, k) + w1 * ld_nu(N, d, ip, j + 1, k));
        nu_y1 = nu + n_c;
        nu_y2 = nu + n_jp;
        nu_z1 = nu + mz.w0[k - 1] * (w0 * ld_nu(N, d, i, j, km) + w1 * ld_nu(N, d, i, j + 1, km)) + mz.w1[k - 1] * (w0 * n_c + w1 * n_jp);
        nu_z2 = nu + mz.w0[k] * (w0 * n_c + w1 * n_jp) + mz.w1[k] * (w0 * ld_nu(N, d, i, j, kp) + w1 * ld_nu(N, d, i, j + 1, kp));
    }
    T fx2 = nu_x2 * ((Vip - Vc) * a.inv_dx + (Ucp - Uc) * inv_dy3);
    T fx1 = nu_x1 * ((Vc - Vim) * a.inv_dx + (Ump - Um) * inv_dy3);
    T fz2 = nu_z2 * ((Vkp - Vc) * inv_dzg2 + (Wjp - Wc) * inv_dy3);
    T fz1 = nu_z1 * ((Vc - Vkm) * inv_dzg1 + (Wkmjp - Wkm) * inv_dy3);
    r = r + a.inv_dx * (fx2 - fx1) + two_inv_dy3 * (nu_y2 * (Vjp - Vc) * inv_dy2 - nu_y1 * (Vc - Vjm) * inv_dy1) + inv_dz3 * (fz2 - fz1);
    return r;
}

template <typename T, bool LES>
__device__ __forceinline__ T rhs_w_at(const StepArgs<T> &a, const Fields<T> &f, const double *__restrict__ tau_z,
                                      int i, int j, int k) {
    const Dims &d = a.d;
    typedef Arith<T> A;
    const Metric1D<T> &my = a.my, &mz = a.mz;
    int im = wrap(i - 1, d.Nx), ip = wrap(i + 1, d.Nx), km = wrap(k - 1, d.Nz), kp = wrap(k + 1, d.Nz);
    const T *U = f.U, *V = f.V, *W = f.W;
    bool wm_band = a.wm && (j + 2 <= 1 + a.nwl || j + 2 >= d.Ny + 2 - a.nwl);
    T wa = wm_band ? T(0) : a.w_adv, wd = T(1) - wa;
    T Wc = __ldg(W + idx3(d, i, j, k)), Wkm = __ldg(W + idx3(d, i, j, km)), Wkp = __ldg(W + idx3(d, i, j, kp));
    T Wim = __ldg(W + idx3(d, im, j, k)), Wip = __ldg(W + idx3(d, ip, j, k));
    T Wjm = ld_yc(W, d, i, j - 1, k), Wjp = ld_yc(W, d, i, j + 1, k);
    // -d(ww)/dz
    T t1 = T(0.5) * (Wc + Wkp), t0 = T(0.5) * (Wkm + Wc);
    T r = -A::div(wd * (t1 * t1 - t0 * t0) + wa * Wc * (t1 - t0), mz.df, mz.idf, k);
    // -d(uw)/dx: u at z face k (weighted), w at x faces
    T Uc = __ldg(U + idx3(d, i, j, k)), Um = __ldg(U + idx3(d, im, j, k));
    T Ukp = __ldg(U + idx3(d, i, j, kp)), Umkp = __ldg(U + idx3(d, im, j, kp));
    {
        T u1 = mz.w0[k] * Uc + mz.w1[k] * Ukp, u0 = mz.w0[k] * Um + mz.w1[k] * Umkp;
        T w1 = T(0.5) * (Wc + Wip), w0 = T(0.5) * (Wim + Wc);
        r = r - (wd * (u1 * w1 - u0 * w0) + wa * T(0.5) * (u0 + u1) * (w1 - w0)) * a.inv_dx;
    }
    // -d(vw)/dy: v at z face k (weighted), w at y faces (weighted)
    T Vc = ld_yf(V, d, i, j, k), Vkp = ld_yf(V, d, i, j, kp), Vjm = ld_yf(V, d, i, j - 1, k), Vjmkp = ld_yf(V, d, i, j - 1, kp);
    {
        T v1 = mz.w0[k] * Vc + mz.w1[k] * Vkp, v0 = mz.w0[k] * Vjm + mz.w1[k] * Vjmkp;
        T w1 = my.w0[j] * Wc + my.w1[j] * Wjp, w0 = my.w0[j - 1] * Wjm + my.w1[j - 1] * Wc;
        r = r - A::div(wd * (v1 * w1 - v0 * w0) + wa * T(0.5) * (v0 + v1) * (w1 - w0), my.dc, my.idc, j);
    }
    // viscous
    T inv_dz1 = A::inv(mz.dc, mz.idc, k), inv_dz2 = A::inv(mz.dc, mz.idc, k + 1), inv_dz3 = A::inv(mz.df, mz.idf, k);
    T two_inv_dz3 = T(2) * inv_dz3;
    T inv_dy3 = A::inv(my.dc, my.idc, j);
    T nu = a.nu;
    T nu_x1 = nu, nu_x2 = nu, nu_y1 = nu, nu_y2 = nu, nu_z1 = nu, nu_z2 = nu;
    if (LES) {
        const T *N = f.nut;
        T n_c = ld_nu(N, d, i, j, k), n_kp = ld_nu(N, d, i, j, kp);
        T z0 = mz.w0[k], z1 = mz.w1[k];
        nu_x1 = nu + T(0.5) * (z0 * (n_c + ld_nu(N, d, im, j, k)) + z1 * (n_kp + ld_nu(N, d, im, j, kp)));
        nu_x2 = nu + T(0.5) * (z0 * (n_c + ld_nu(N, d, ip, j, k)) + z1 * (n_kp + ld_nu(N, d, ip, j, kp)));
        if (!(d.yper == 0 && j == 0))
            nu_y1 = nu + z0 * (my.w0[j - 1] * ld_nu(N, d, i, j - 1, k) + my.w1[j - 1] * n_c) +
                    z1 * (my.w0[j - 1] * ld_nu(N, d, i, j - 1, kp) + my.w1[j - 1] * n_kp);
        if (!(d.yper == 0 && j == d.Ny - 1))
            nu_y2 = nu + z0 * (my.w0[j] * n_c + my.w1[j] * ld_nu(N, d, i, j + 1, k)) +
                    z1 * (my.w0[j] * n_kp + my.w1[j] * ld_nu(N, d, i, j + 1, kp));
        nu_z1 = nu + n_c;
        nu_z2 = nu + n_kp;
    }
    T tj = A::div(Wjp - Wc, my.df, my.idf, j), tjm = A::div(Wc - Wjm, my.df, my.idf, j - 1);
    T fy2 = nu_y2 * (tj + (Vkp - Vc) * inv_dz3);
    T fy1 = nu_y1 * (tjm + (Vjmkp - Vjm) * inv_dz3);
    if (a.wm) {
        if (j == 0) fy1 = (T)tau_z[(long long)k * d.Nx + i];
        if (j == d.Ny - 1) fy2 = (T)tau_z[((long long)d.Nz + k) * d.Nx + i];
    }
    T fx2 = nu_x2 * ((Wip - Wc) * a.inv_dx + (Ukp - Uc) * inv_dz3);
    T fx1 = nu_x1 * ((Wc - Wim) * a.inv_dx + (Umkp - Um) * inv_dz3);
    r = r + a.inv_dx * (fx2 - fx1) + inv_dy3 * (fy2 - fy1) +
        two_inv_dz3 * (nu_z2 * (Wkp - Wc) * inv_dz2 - nu_z1 * (Wc - Wkm) * inv_dz1) + a.dPdz;
    return r;
}

// Fused stage kernel: the three right-hand sides at (i,j,k) and the Butcher-form RK3 update
// (src/time_integration.f90:255-259, :393-397, :525-532).  Stage 1 also writes the base state uo and F1.
//   s = 1: u* = uo + (dt a11) F1                 (F1 = rhs, uo = u)
//   s = 2: u* = uo + dt (a21 F1 + a22 rhs)
//   s = 3: u* = uo + dt (a31 F1 + a33 rhs)        (a32 = 0, so F2 is never needed)
struct StageCoef {
    int stage;       // 1, 2 or 3
    double dt_a11;   // dt*rk_coef(1,1), stage 1
    double dt;       // dt, stages 2 and 3
    double c1, c2;   // rk_coef(s,1) and rk_coef(s,s), stages 2 and 3
};

template <typename T, bool LES>
__global__ void __launch_bounds__(256) k_stage(StepArgs<T> a, Fields<T> f, const double *__restrict__ tau_x,
                                               const double *__restrict__ tau_z, StageCoef sc,
                                               T *__restrict__ uo, T *__restrict__ vo, T *__restrict__ wo,
                                               T *__restrict__ f1u, T *__restrict__ f1v, T *__restrict__ f1w,
                                               T *__restrict__ us, T *__restrict__ vs, T *__restrict__ wsf,
                                               T *__restrict__ rhs_only) {
    const Dims &d = a.d;
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= d.Nx || j >= d.Ny) return;
    long long p = idx3(d, i, j, k);
    T ru = rhs_u_at<T, LES>(a, f, tau_x, i, j, k);
    T rw = rhs_w_at<T, LES>(a, f, tau_z, i, j, k);
    bool vrow = j < d.NyV;
    T rv = vrow ? rhs_v_at<T, LES>(a, f, i, j, k) : T(0);
    if (rhs_only) {   // unit entry point: F = rhs, no update
        rhs_only[p] = ru; rhs_only[d.cells + p] = rv; rhs_only[2 * d.cells + p] = rw;
        return;
    }
    if (sc.stage == 1) {
        T u0 = f.U[p], w0 = f.W[p];
        T c = (T)sc.dt_a11;
        uo[p] = u0; f1u[p] = ru; us[p] = u0 + c * ru;
        wo[p] = w0; f1w[p] = rw; wsf[p] = w0 + c * rw;
        if (vrow) { T v0 = f.V[p]; vo[p] = v0; f1v[p] = rv; vs[p] = v0 + c * rv; }
    } else {
        T c1 = (T)sc.c1, c2 = (T)sc.c2, dtt = (T)sc.dt;
        us[p] = uo[p] + dtt * (c1 * f1u[p] + c2 * ru);
        wsf[p] = wo[p] + dtt * (c1 * f1w[p] + c2 * rw);
        if (vrow) vs[p] = vo[p] + dtt * (c1 * f1v[p] + c2 * rv);
    }
}

}  // namespace dfdm
