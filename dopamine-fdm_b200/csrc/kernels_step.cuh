// kernels_step.cuh -- eddy viscosity, wall model and the fused RHS + RK3 stage kernel.
#pragma once

#include "dfdm_common.cuh"
#include "f32x2.cuh"

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
    // Streamwise base profile: U is stored as U - ub(j) (FP32-mixed; all zeros in FP64).  ub is exactly
    // representable in the storage type; ubd is the same profile in double.
    const T *ub;
    const double *ubd;
    // advection_scheme = 2: the dissipative terms of k_adv_hybrid_faces (u, v, w blocks of `cells`), added to the
    // right-hand sides; null otherwise
    const T *adv;
    // fused correction of the previous stage (CORR kernels): its potential phi; the plane loads then hold u* and
    // the loader forms u = u* - grad(phi) exactly as k_correct does
    const T *phi;
    // FP32: the eight z metrics of every plane in AxisLocal<F2>::load8 order, 8 consecutive values per plane (one
    // 32-byte bulk copy per plane for the TMA stage kernel); null in FP64
    const float *zm8;
    // LES with the wall model: the first-cell gradient factor of every wall cell, (iw*Nz + k)*Nx + i, written by
    // k_wall_sgs from the velocity the eddy viscosity is computed from (NaN where the override does not apply);
    // null: nut_at solves for it in place
    const double *wfac;
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

// The wall-modelled first-cell gradient override of compute_vreman (src/sgs_model.f90:158-172): the factor
// u_tau/(kappa y_w |u|) (signed by the wall) that replaces du/dy and dw/dy by fac*u_c and fac*w_c, with u_tau from the
// Reichardt law at the first-cell velocity magnitude; NaN where |u| <= 1e-14 and the gradients are kept.
__device__ __forceinline__ double wall_gradient_factor(double u_c, double w_c, bool lower, double y_w, double nu) {
    double u_mag = sqrt(u_c * u_c + w_c * w_c);
    if (!(u_mag > 1e-14)) return __longlong_as_double(0x7ff8000000000000LL);
    double u_tau = solve_u_tau(u_mag, y_w, nu);
    return (lower ? 1.0 : -1.0) * u_tau / (0.41 * y_w * u_mag);
}

// ---------------------------------------------------------------------------------------------------------------
// Eddy viscosity at one cell centre: compute_vreman pass 1 (src/sgs_model.f90:118-223) with the AMD
// (Rozema et al. 2015) or Vreman (2004) closure and the wall-modelled first-cell gradient override (:158-172).
// Ghost values come from the neighbourhood accessor (sgs_fill_ghosts' rules, :458-531).
template <typename T, typename Q>
__device__ __forceinline__ T nut_at(const StepArgs<T> &a, const Q &q, int i, int j, int k) {
    const Dims &d = a.d;
    typedef Arith<T> A;
    const Metric1D<T> &my = a.my, &mz = a.mz;
    T dz_c = mz.dc[k], dz2 = dz_c * dz_c;
    T inv_dz_k = A::inv(mz.dc, mz.idc, k), inv_zg_km = A::inv(mz.df, mz.idf, k - 1), inv_zg_kp = A::inv(mz.df, mz.idf, k);
    T dy_c = my.dc[j], dy2_c = dy_c * dy_c;
    T inv_yg_jm = A::inv(my.df, my.idf, j - 1), inv_yg_jp = A::inv(my.df, my.idf, j), inv_dy_j = A::inv(my.dc, my.idc, j);
    T inv_dx = a.inv_dx, dx2 = a.dx2;
    T Uc = q.U(0, 0, 0), Um = q.U(-1, 0, 0);
    T a11 = (Uc - Um) * inv_dx;
    T a21 = T(0.5) * ((Uc - q.U(0, -1, 0)) * inv_yg_jm + (q.U(0, 1, 0) - Uc) * inv_yg_jp);
    T a31 = T(0.5) * ((Uc - q.U(0, 0, -1)) * inv_zg_km + (q.U(0, 0, 1) - Uc) * inv_zg_kp);
    T Vc = q.V(0, 0, 0);
    T a12 = T(0.5) * ((Vc - q.V(-1, 0, 0)) + (q.V(1, 0, 0) - Vc)) * inv_dx;
    T a22 = (Vc - q.V(0, -1, 0)) * inv_dy_j;
    T a32 = T(0.5) * ((Vc - q.V(0, 0, -1)) * inv_zg_km + (q.V(0, 0, 1) - Vc) * inv_zg_kp);
    T Wc = q.W(0, 0, 0), Wkm = q.W(0, 0, -1);
    T a13 = T(0.5) * ((Wc - q.W(-1, 0, 0)) + (q.W(1, 0, 0) - Wc)) * inv_dx;
    T a23 = T(0.5) * ((Wc - q.W(0, -1, 0)) * inv_yg_jm + (q.W(0, 1, 0) - Wc) * inv_yg_jp);
    T a33 = (Wc - Wkm) * inv_dz_k;
    if (a.wm && (j == 0 || j == d.Ny - 1)) {
        double u_c = 0.5 * ((double)Um + (double)Uc);
        double w_c = 0.5 * ((double)Wkm + (double)Wc);
        double fac_w;
        if (a.wfac) {
            fac_w = a.wfac[((j == 0 ? 0 : d.Nz) + k) * d.Nx + i];   // NaN: no override
        } else {
            fac_w = wall_gradient_factor(u_c, w_c, j == 0, (j == 0) ? a.yg2 : a.ygtop, a.nu_d);
        }
        if (!isnan(fac_w)) {
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
    return nu_t;
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
                            double dt_fixed, const double *__restrict__ dtp, double Tf_fac) {
    pdl_enter();
    const Dims &d = a.d;
    const double dt = dtp ? *dtp : dt_fixed;   // adaptive time step: from device memory
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
        const double ubm = a.ubd[jm];
        ws.ux[p] = (1.0 - eps) * ws.ux[p] + eps * ((double)U[idx3(d, i, jm, k)] + ubm);
        ws.wx[p] = (1.0 - eps) * ws.wx[p] + eps * 0.5 * ((double)W[idx3(d, i, jm, km)] + (double)W[idx3(d, i, jm, k)]);
        eps = 1.0;
        if (!seed && ws.tz[p] > 0.0) eps = fmin(1.0, dt * kap * ws.tz[p] / (Tf_fac * ym));
        ws.uz[p] = (1.0 - eps) * ws.uz[p] + eps * 0.5 * (((double)U[idx3(d, im, jm, k)] + ubm) + ((double)U[idx3(d, i, jm, k)] + ubm));
        ws.wz[p] = (1.0 - eps) * ws.wz[p] + eps * (double)W[idx3(d, i, jm, k)];
    }
}

// compute_flat_wall_eqwm (src/wallmodel.f90:442-583), smooth Reichardt law, matching height = first centre.
template <typename T>
__global__ void k_wall_model(StepArgs<T> a, WallState ws, const T *__restrict__ U, const T *__restrict__ W, int filter) {
    pdl_enter();
    const Dims &d = a.d;
    int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (i >= d.Nx) return;
    int im = wrap(i - 1, d.Nx), km = wrap(k - 1, d.Nz);
    for (int iw = 0; iw < 2; ++iw) {
        int jw = (iw == 0) ? 0 : d.Ny - 1;
        double y_match = fmax((iw == 0) ? a.yg2 : a.ygtop, 1e-14);
        long long p = ((long long)iw * d.Nz + k) * d.Nx + i;
        // U faces
        const double ubw = a.ubd[jw];
        double Uw = (double)U[idx3(d, i, jw, k)] + ubw;
        double W_at = 0.5 * ((double)W[idx3(d, i, jw, km)] + (double)W[idx3(d, i, jw, k)]);
        double u_ref = sqrt(Uw * Uw + W_at * W_at), u_match = u_ref, num = Uw;
        if (filter) { u_match = sqrt(ws.ux[p] * ws.ux[p] + ws.wx[p] * ws.wx[p]); num = ws.ux[p]; u_ref = u_match; }
        double u_tau = solve_u_tau(u_match, y_match, a.nu_d);
        ws.tx[p] = u_tau;
        double tv = u_tau * u_tau * num / fmax(u_ref, 1e-30);
        ws.tau_x[p] = (iw == 0) ? tv : -tv;
        // W faces
        double uc = 0.5 * (((double)U[idx3(d, im, jw, k)] + ubw) + Uw);
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
// Metric values around one index p of an axis: weights of faces p-1 and p, widths and spacings at p-1, p, p+1.
// FP32 reads them once per thread (y) or once per plane (z) and keeps them in registers; FP64 reads them where
// they are used (its registers are taken by the double-precision stencil) and divides exactly, as Arith does.
template <typename T> struct AxisLocal;
template <> struct AxisLocal<float> {
    float w0m_, w1m_, w0_, w1_, idc_, idcp_, idfm_, idf_;
    __device__ __forceinline__ void load(const Metric1D<float> &m, int p) {
        w0m_ = __ldg(m.w0 + p - 1); w1m_ = __ldg(m.w1 + p - 1); w0_ = __ldg(m.w0 + p); w1_ = __ldg(m.w1 + p);
        idc_ = __ldg(m.idc + p); idcp_ = __ldg(m.idc + p + 1); idfm_ = __ldg(m.idf + p - 1); idf_ = __ldg(m.idf + p);
    }
    __device__ __forceinline__ float w0m() const { return w0m_; }
    __device__ __forceinline__ float w1m() const { return w1m_; }
    __device__ __forceinline__ float w0() const { return w0_; }
    __device__ __forceinline__ float w1() const { return w1_; }
    __device__ __forceinline__ float divc(float x) const { return x * idc_; }
    __device__ __forceinline__ float divf(float x) const { return x * idf_; }
    __device__ __forceinline__ float divfm(float x) const { return x * idfm_; }
    __device__ __forceinline__ float invc() const { return idc_; }
    __device__ __forceinline__ float invcp() const { return idcp_; }
    __device__ __forceinline__ float invf() const { return idf_; }
    __device__ __forceinline__ float invfm() const { return idfm_; }
};
template <> struct AxisLocal<F2> {   // packed pairs: the same metrics broadcast to both lanes, read once
    F2 w0m_, w1m_, w0_, w1_, idc_, idcp_, idfm_, idf_;
    __device__ __forceinline__ void load(const Metric1D<float> &m, int p) {
        w0m_ = F2(__ldg(m.w0 + p - 1)); w1m_ = F2(__ldg(m.w1 + p - 1)); w0_ = F2(__ldg(m.w0 + p)); w1_ = F2(__ldg(m.w1 + p));
        idc_ = F2(__ldg(m.idc + p)); idcp_ = F2(__ldg(m.idc + p + 1)); idfm_ = F2(__ldg(m.idf + p - 1)); idf_ = F2(__ldg(m.idf + p));
    }
    // the same eight values staged by metric_src (w0, w1 at p-1 and p; idc at p, p+1; idf at p-1, p)
    __device__ __forceinline__ void load8(const float *z) {
        w0m_ = F2(z[0]); w1m_ = F2(z[1]); w0_ = F2(z[2]); w1_ = F2(z[3]);
        idc_ = F2(z[4]); idcp_ = F2(z[5]); idfm_ = F2(z[6]); idf_ = F2(z[7]);
    }
    // the address of staged value t (0..7) of point p, in the order of load8
    static __device__ __forceinline__ const float *metric_src(const Metric1D<float> &m, int p, int t) {
        switch (t) {
        case 0: return m.w0 + p - 1;
        case 1: return m.w1 + p - 1;
        case 2: return m.w0 + p;
        case 3: return m.w1 + p;
        case 4: return m.idc + p;
        case 5: return m.idc + p + 1;
        case 6: return m.idf + p - 1;
        default: return m.idf + p;
        }
    }
    __device__ __forceinline__ F2 w0m() const { return w0m_; }
    __device__ __forceinline__ F2 w1m() const { return w1m_; }
    __device__ __forceinline__ F2 w0() const { return w0_; }
    __device__ __forceinline__ F2 w1() const { return w1_; }
    __device__ __forceinline__ P2 divc(F2 x) const { return x * idc_; }
    __device__ __forceinline__ P2 divf(F2 x) const { return x * idf_; }
    __device__ __forceinline__ P2 divfm(F2 x) const { return x * idfm_; }
    __device__ __forceinline__ F2 invc() const { return idc_; }
    __device__ __forceinline__ F2 invcp() const { return idcp_; }
    __device__ __forceinline__ F2 invf() const { return idf_; }
    __device__ __forceinline__ F2 invfm() const { return idfm_; }
};
template <> struct AxisLocal<double> {
    const Metric1D<double> *m;   // the kernel argument's metric (stays in the parameter bank once inlined)
    int p;
    __device__ __forceinline__ void load(const Metric1D<double> &m_, int p_) { m = &m_; p = p_; }
    __device__ __forceinline__ double w0m() const { return m->w0[p - 1]; }
    __device__ __forceinline__ double w1m() const { return m->w1[p - 1]; }
    __device__ __forceinline__ double w0() const { return m->w0[p]; }
    __device__ __forceinline__ double w1() const { return m->w1[p]; }
    __device__ __forceinline__ double divc(double x) const { return x / m->dc[p]; }
    __device__ __forceinline__ double divf(double x) const { return x / m->df[p]; }
    __device__ __forceinline__ double divfm(double x) const { return x / m->df[p - 1]; }
    __device__ __forceinline__ double invc() const { return 1.0 / m->dc[p]; }
    __device__ __forceinline__ double invcp() const { return 1.0 / m->dc[p + 1]; }
    __device__ __forceinline__ double invf() const { return 1.0 / m->df[p]; }
    __device__ __forceinline__ double invfm() const { return 1.0 / m->df[p - 1]; }
};

// The gradient factor of the eddy viscosity's wall override for every wall cell (wall_gradient_factor), from the
// velocity the eddy viscosity is then computed from: U and W as stored, or (CORR) the previous stage's u* with its
// projection applied exactly as the stage kernels' loaders apply it.  One thread per (i, k) of both walls: the
// Reichardt solve runs once per wall cell here instead of on the critical path of every tile that holds the cell.
template <typename T, bool CORR>
__global__ void k_wall_sgs(StepArgs<T> a, const T *__restrict__ U, const T *__restrict__ W, const T *__restrict__ phi,
                           double *__restrict__ wfac) {
    pdl_enter();
    const Dims &d = a.d;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y;
    if (i >= d.Nx) return;
    const int im = wrap(i - 1, d.Nx), ip = wrap(i + 1, d.Nx), km = wrap(k - 1, d.Nz), kp = wrap(k + 1, d.Nz);
    for (int iw = 0; iw < 2; ++iw) {
        const int j = iw ? d.Ny - 1 : 0;
        T u0 = U[idx3(d, im, j, k)], u1 = U[idx3(d, i, j, k)], w0 = W[idx3(d, i, j, km)], w1 = W[idx3(d, i, j, k)];
        if constexpr (CORR) {
            const T pm = phi[idx3(d, im, j, k)], pc = phi[idx3(d, i, j, k)], pp = phi[idx3(d, ip, j, k)];
            const T pkm = phi[idx3(d, i, j, km)], pkp = phi[idx3(d, i, j, kp)];
            u0 = u0 - (pc - pm) * a.inv_dx;
            u1 = u1 - (pp - pc) * a.inv_dx;
            w0 = w0 - (pc - pkm) * Arith<T>::inv(a.mz.df, a.mz.idf, km);
            w1 = w1 - (pkp - pc) * Arith<T>::inv(a.mz.df, a.mz.idf, k);
        }
        const T ubj = a.ub[j];
        const T Um = u0 + ubj, Uc = u1 + ubj;   // as TileQ::U forms them
        const double u_c = 0.5 * ((double)Um + (double)Uc);
        const double w_c = 0.5 * ((double)w0 + (double)w1);
        wfac[((long long)iw * d.Nz + k) * d.Nx + i] = wall_gradient_factor(u_c, w_c, iw == 0, iw ? a.ygtop : a.yg2, a.nu_d);
    }
}

// Wall-model flux of the cell at t (plain types) or of the cells at t and t+1 (packed pairs), from double.
template <typename T> __device__ __forceinline__ T wall_flux(const double *t) { return (T)t[0]; }
template <> __device__ __forceinline__ F2 wall_flux<F2>(const double *t) { return F2::pair((float)t[0], (float)t[1]); }

// Right-hand sides (src/equations.f90), evaluated in the reference's expression order at one index (i,j,k).
// `q` is a neighbourhood accessor: q.U(di,dj,dk) is U at (i+di, j+dj, k+dk) with every boundary rule already
// applied (periodic wraps, no-slip mirror, zero wall faces, zero nu_t ghosts), so the formulas below see the
// same values the reference reads from its ghosted arrays.
template <typename T, bool LES, bool WM, typename Q, typename SA>
__device__ __forceinline__ T rhs_u_at(const SA &a, const Q &q, const AxisLocal<T> &Y, const AxisLocal<T> &Z,
                                    const double *__restrict__ tau_x, int i, int j, int k) {
    const Dims &d = a.d;
    T Uc = q.U(0, 0, 0), Uim = q.U(-1, 0, 0), Uip = q.U(1, 0, 0);
    T Ujm = q.U(0, -1, 0), Ujp = q.U(0, 1, 0), Ukm = q.U(0, 0, -1), Ukp = q.U(0, 0, 1);
    bool wm_band = WM && a.wm && (j + 2 <= 1 + a.nwl || j + 2 >= d.Ny + 2 - a.nwl);
    T wa = wm_band ? T(0) : a.w_adv, wd = T(1) - wa;
    // -d(uu)/dx
    T r;
    if constexpr (Fp32Forms<T>::value) {
        // FP32: t1^2 - t0^2 = (t1 - t0)(t1 + t0) with t1 - t0 from the stored deviations (no cancellation)
        T dlt = T(0.5) * (q.Ud(1, 0, 0) - q.Ud(-1, 0, 0));
        T sum = T(0.5) * (Uip + Uim) + Uc;
        r = -dlt * (wd * sum + wa * Uc) * a.inv_dx;
    } else {
        T t1 = T(0.5) * (Uc + Uip), t0 = T(0.5) * (Uim + Uc);
        r = -(wd * (t1 * t1 - t0 * t0) + wa * Uc * (t1 - t0)) * a.inv_dx;
    }
    // -d(uv)/dy: u at y faces j-1, j (weighted), v at x faces (plain average)
    T V00 = q.V(0, 0, 0), V10 = q.V(1, 0, 0), V0m = q.V(0, -1, 0), V1m = q.V(1, -1, 0);
    {
        T u1 = Y.w0() * Uc + Y.w1() * Ujp, u0 = Y.w0m() * Ujm + Y.w1m() * Uc;
        T v1 = T(0.5) * (V00 + V10), v0 = T(0.5) * (V0m + V1m);
        r = r - Y.divc(wd * (u1 * v1 - u0 * v0) + wa * T(0.5) * (v0 + v1) * (u1 - u0));
    }
    // -d(uw)/dz
    T W00 = q.W(0, 0, 0), W10 = q.W(1, 0, 0), W0m = q.W(0, 0, -1), W1m = q.W(1, 0, -1);
    {
        T u1 = Z.w0() * Uc + Z.w1() * Ukp, u0 = Z.w0m() * Ukm + Z.w1m() * Uc;
        T w1 = T(0.5) * (W00 + W10), w0 = T(0.5) * (W0m + W1m);
        if constexpr (Fp32Forms<T>::value) {
            // u1 w1 - u0 w0 = u1 (w1 - w0) + w0 (u1 - u0); u1 - u0 from deviations (same row: the profile cancels)
            T Udc = q.Ud(0, 0, 0);
            T du = (Z.w0() * Udc + Z.w1() * q.Ud(0, 0, 1)) - (Z.w0m() * q.Ud(0, 0, -1) + Z.w1m() * Udc);
            r = r - Z.divc(wd * (u1 * (w1 - w0) + w0 * du) + wa * T(0.5) * (w0 + w1) * du);
        } else {
            r = r - Z.divc(wd * (u1 * w1 - u0 * w0) + wa * T(0.5) * (w0 + w1) * (u1 - u0));
        }
    }
    // viscous: d(2 nu_x du/dx)/dx + d(nu_y (du/dy + dv/dx))/dy + d(nu_z (du/dz + dw/dx))/dz + dPdx
    T inv_dz3 = Z.invc(), inv_dy3 = Y.invc();
    T nu = a.nu;
    T nu_x1 = nu, nu_x2 = nu, nu_y1 = nu, nu_y2 = nu, nu_z1 = nu, nu_z2 = nu;
    if (LES) {
        T n_c = q.N(0, 0, 0), n_p = q.N(1, 0, 0);
        nu_x1 = nu + n_c; nu_x2 = nu + n_p;
        if (!(d.yper == 0 && j == 0))
            nu_y1 = nu + T(0.5) * (Y.w0m() * q.N(0, -1, 0) + Y.w1m() * n_c + Y.w0m() * q.N(1, -1, 0) + Y.w1m() * n_p);
        if (!(d.yper == 0 && j == d.Ny - 1))
            nu_y2 = nu + T(0.5) * (Y.w0() * n_c + Y.w1() * q.N(0, 1, 0) + Y.w0() * n_p + Y.w1() * q.N(1, 1, 0));
        nu_z1 = nu + T(0.5) * (Z.w0m() * (q.N(0, 0, -1) + q.N(1, 0, -1)) + Z.w1m() * (n_c + n_p));
        nu_z2 = nu + T(0.5) * (Z.w0() * (n_c + n_p) + Z.w1() * (q.N(0, 0, 1) + q.N(1, 0, 1)));
    }
    T tj = Y.divf(Ujp - Uc), tjm = Y.divfm(Uc - Ujm);
    T fy2 = nu_y2 * (tj + (V10 - V00) * a.inv_dx);
    T fy1 = nu_y1 * (tjm + (V1m - V0m) * a.inv_dx);
    if (WM && a.wm) {
        if (j == 0) fy1 = wall_flux<T>(tau_x + k * d.Nx + i);
        if (j == d.Ny - 1) fy2 = wall_flux<T>(tau_x + (d.Nz + k) * d.Nx + i);
    }
    T dUkp = Ukp - Uc, dUkm = Uc - Ukm, dUip = Uip - Uc, dUim = Uc - Uim;
    if constexpr (Fp32Forms<T>::value) {   // x and z differences of U from the deviations
        T Udc = q.Ud(0, 0, 0);
        dUkp = q.Ud(0, 0, 1) - Udc; dUkm = Udc - q.Ud(0, 0, -1);
        dUip = q.Ud(1, 0, 0) - Udc; dUim = Udc - q.Ud(-1, 0, 0);
    }
    T tk = Z.divf(dUkp), tkm = Z.divfm(dUkm);
    T fz2 = nu_z2 * (tk + (W10 - W00) * a.inv_dx);
    T fz1 = nu_z1 * (tkm + (W1m - W0m) * a.inv_dx);
    r = r + T(2) * a.inv_dx2 * (nu_x2 * dUip - nu_x1 * dUim) + inv_dy3 * (fy2 - fy1) + inv_dz3 * (fz2 - fz1) + a.dPdx;
    return r;
}

template <typename T, bool LES, bool WM, typename Q, typename SA>
__device__ __forceinline__ T rhs_v_at(const SA &a, const Q &q, const AxisLocal<T> &Y, const AxisLocal<T> &Z, int i, int j, int k) {
    const Dims &d = a.d;
    (void)i; (void)d;
    T wa = a.w_adv, wd = T(1) - wa;
    T Vc = q.V(0, 0, 0), Vjm = q.V(0, -1, 0), Vjp = q.V(0, 1, 0);
    T Vim = q.V(-1, 0, 0), Vip = q.V(1, 0, 0), Vkm = q.V(0, 0, -1), Vkp = q.V(0, 0, 1);
    // -d(vv)/dy
    T t1 = T(0.5) * (Vc + Vjp), t0 = T(0.5) * (Vjm + Vc);
    T r = -Y.divf(wd * (t1 * t1 - t0 * t0) + wa * Vc * (t1 - t0));
    // -d(uv)/dx: u at y face j (weighted), v at x faces
    T Uc = q.U(0, 0, 0), Um = q.U(-1, 0, 0), Ucp = q.U(0, 1, 0), Ump = q.U(-1, 1, 0);
    {
        T u1 = Y.w0() * Uc + Y.w1() * Ucp, u0 = Y.w0() * Um + Y.w1() * Ump;
        T v1 = T(0.5) * (Vc + Vip), v0 = T(0.5) * (Vim + Vc);
        if constexpr (Fp32Forms<T>::value) {   // u1 v1 - u0 v0 = u1 (v1 - v0) + v0 (u1 - u0), u1 - u0 from deviations
            T du = Y.w0() * (q.Ud(0, 0, 0) - q.Ud(-1, 0, 0)) + Y.w1() * (q.Ud(0, 1, 0) - q.Ud(-1, 1, 0));
            r = r - (wd * (u1 * (v1 - v0) + v0 * du) + wa * T(0.5) * (u0 + u1) * (v1 - v0)) * a.inv_dx;
        } else {
            r = r - (wd * (u1 * v1 - u0 * v0) + wa * T(0.5) * (u0 + u1) * (v1 - v0)) * a.inv_dx;
        }
    }
    // -d(vw)/dz: v at z faces (weighted), w at y face j (weighted)
    T Wc = q.W(0, 0, 0), Wjp = q.W(0, 1, 0), Wkm = q.W(0, 0, -1), Wkmjp = q.W(0, 1, -1);
    {
        T v1 = Z.w0() * Vc + Z.w1() * Vkp, v0 = Z.w0m() * Vkm + Z.w1m() * Vc;
        T w1 = Y.w0() * Wc + Y.w1() * Wjp, w0 = Y.w0() * Wkm + Y.w1() * Wkmjp;
        r = r - Z.divc(wd * (v1 * w1 - v0 * w0) + wa * T(0.5) * (w0 + w1) * (v1 - v0));
    }
    // viscous
    T inv_dz3 = Z.invc();
    T inv_dzg1 = Z.invfm(), inv_dzg2 = Z.invf();
    T inv_dy1 = Y.invc(), inv_dy2 = Y.invcp(), inv_dy3 = Y.invf();
    T two_inv_dy3 = T(2) * inv_dy3;
    T nu = a.nu;
    T nu_x1 = nu, nu_x2 = nu, nu_y1 = nu, nu_y2 = nu, nu_z1 = nu, nu_z2 = nu;
    if (LES) {
        T n_c = q.N(0, 0, 0), n_jp = q.N(0, 1, 0);
        T w0 = Y.w0(), w1 = Y.w1();
        nu_x1 = nu + T(0.5) * (w0 * q.N(-1, 0, 0) + w1 * q.N(-1, 1, 0) + w0 * n_c + w1 * n_jp);
        nu_x2 = nu + T(0.5) * (w0 * n_c + w1 * n_jp + w0 * q.N(1, 0, 0) + w1 * q.N(1, 1, 0));
        nu_y1 = nu + n_c;
        nu_y2 = nu + n_jp;
        nu_z1 = nu + Z.w0m() * (w0 * q.N(0, 0, -1) + w1 * q.N(0, 1, -1)) + Z.w1m() * (w0 * n_c + w1 * n_jp);
        nu_z2 = nu + Z.w0() * (w0 * n_c + w1 * n_jp) + Z.w1() * (w0 * q.N(0, 0, 1) + w1 * q.N(0, 1, 1));
    }
    T fx2 = nu_x2 * ((Vip - Vc) * a.inv_dx + (Ucp - Uc) * inv_dy3);
    T fx1 = nu_x1 * ((Vc - Vim) * a.inv_dx + (Ump - Um) * inv_dy3);
    T fz2 = nu_z2 * ((Vkp - Vc) * inv_dzg2 + (Wjp - Wc) * inv_dy3);
    T fz1 = nu_z1 * ((Vc - Vkm) * inv_dzg1 + (Wkmjp - Wkm) * inv_dy3);
    r = r + a.inv_dx * (fx2 - fx1) + two_inv_dy3 * (nu_y2 * (Vjp - Vc) * inv_dy2 - nu_y1 * (Vc - Vjm) * inv_dy1) + inv_dz3 * (fz2 - fz1);
    return r;
}

template <typename T, bool LES, bool WM, typename Q, typename SA>
__device__ __forceinline__ T rhs_w_at(const SA &a, const Q &q, const AxisLocal<T> &Y, const AxisLocal<T> &Z,
                                    const double *__restrict__ tau_z, int i, int j, int k) {
    const Dims &d = a.d;
    bool wm_band = WM && a.wm && (j + 2 <= 1 + a.nwl || j + 2 >= d.Ny + 2 - a.nwl);
    T wa = wm_band ? T(0) : a.w_adv, wd = T(1) - wa;
    T Wc = q.W(0, 0, 0), Wkm = q.W(0, 0, -1), Wkp = q.W(0, 0, 1);
    T Wim = q.W(-1, 0, 0), Wip = q.W(1, 0, 0), Wjm = q.W(0, -1, 0), Wjp = q.W(0, 1, 0);
    // -d(ww)/dz
    T t1 = T(0.5) * (Wc + Wkp), t0 = T(0.5) * (Wkm + Wc);
    T r = -Z.divf(wd * (t1 * t1 - t0 * t0) + wa * Wc * (t1 - t0));
    // -d(uw)/dx: u at z face k (weighted), w at x faces
    T Uc = q.U(0, 0, 0), Um = q.U(-1, 0, 0), Ukp = q.U(0, 0, 1), Umkp = q.U(-1, 0, 1);
    {
        T u1 = Z.w0() * Uc + Z.w1() * Ukp, u0 = Z.w0() * Um + Z.w1() * Umkp;
        T w1 = T(0.5) * (Wc + Wip), w0 = T(0.5) * (Wim + Wc);
        if constexpr (Fp32Forms<T>::value) {   // u1 w1 - u0 w0 = u1 (w1 - w0) + w0 (u1 - u0), u1 - u0 from deviations
            T du = Z.w0() * (q.Ud(0, 0, 0) - q.Ud(-1, 0, 0)) + Z.w1() * (q.Ud(0, 0, 1) - q.Ud(-1, 0, 1));
            r = r - (wd * (u1 * (w1 - w0) + w0 * du) + wa * T(0.5) * (u0 + u1) * (w1 - w0)) * a.inv_dx;
        } else {
            r = r - (wd * (u1 * w1 - u0 * w0) + wa * T(0.5) * (u0 + u1) * (w1 - w0)) * a.inv_dx;
        }
    }
    // -d(vw)/dy: v at z face k (weighted), w at y faces (weighted)
    T Vc = q.V(0, 0, 0), Vkp = q.V(0, 0, 1), Vjm = q.V(0, -1, 0), Vjmkp = q.V(0, -1, 1);
    {
        T v1 = Z.w0() * Vc + Z.w1() * Vkp, v0 = Z.w0() * Vjm + Z.w1() * Vjmkp;
        T w1 = Y.w0() * Wc + Y.w1() * Wjp, w0 = Y.w0m() * Wjm + Y.w1m() * Wc;
        r = r - Y.divc(wd * (v1 * w1 - v0 * w0) + wa * T(0.5) * (v0 + v1) * (w1 - w0));
    }
    // viscous
    T inv_dz1 = Z.invc(), inv_dz2 = Z.invcp(), inv_dz3 = Z.invf();
    T two_inv_dz3 = T(2) * inv_dz3;
    T inv_dy3 = Y.invc();
    T nu = a.nu;
    T nu_x1 = nu, nu_x2 = nu, nu_y1 = nu, nu_y2 = nu, nu_z1 = nu, nu_z2 = nu;
    if (LES) {
        T n_c = q.N(0, 0, 0), n_kp = q.N(0, 0, 1);
        T z0 = Z.w0(), z1 = Z.w1();
        nu_x1 = nu + T(0.5) * (z0 * (n_c + q.N(-1, 0, 0)) + z1 * (n_kp + q.N(-1, 0, 1)));
        nu_x2 = nu + T(0.5) * (z0 * (n_c + q.N(1, 0, 0)) + z1 * (n_kp + q.N(1, 0, 1)));
        if (!(d.yper == 0 && j == 0))
            nu_y1 = nu + z0 * (Y.w0m() * q.N(0, -1, 0) + Y.w1m() * n_c) + z1 * (Y.w0m() * q.N(0, -1, 1) + Y.w1m() * n_kp);
        if (!(d.yper == 0 && j == d.Ny - 1))
            nu_y2 = nu + z0 * (Y.w0() * n_c + Y.w1() * q.N(0, 1, 0)) + z1 * (Y.w0() * n_kp + Y.w1() * q.N(0, 1, 1));
        nu_z1 = nu + n_c;
        nu_z2 = nu + n_kp;
    }
    T tj = Y.divf(Wjp - Wc), tjm = Y.divfm(Wc - Wjm);
    T fy2 = nu_y2 * (tj + (Vkp - Vc) * inv_dz3);
    T fy1 = nu_y1 * (tjm + (Vjmkp - Vjm) * inv_dz3);
    if (WM && a.wm) {
        if (j == 0) fy1 = wall_flux<T>(tau_z + k * d.Nx + i);
        if (j == d.Ny - 1) fy2 = wall_flux<T>(tau_z + (d.Nz + k) * d.Nx + i);
    }
    T fx2 = nu_x2 * ((Wip - Wc) * a.inv_dx + (Ukp - Uc) * inv_dz3);
    T fx1 = nu_x1 * ((Wc - Wim) * a.inv_dx + (Umkp - Um) * inv_dz3);
    r = r + a.inv_dx * (fx2 - fx1) + inv_dy3 * (fy2 - fy1) +
        two_inv_dz3 * (nu_z2 * (Wkp - Wc) * inv_dz2 - nu_z1 * (Wc - Wkm) * inv_dz1) + a.dPdz;
    return r;
}

// Stage coefficients of the Butcher-form RK3 update (src/time_integration.f90:255-259, :393-397, :525-532):
//   s = 1: u* = uo + (dt a11) F1                 (F1 = rhs, uo = u)
//   s = 2: u* = uo + dt (a21 F1 + a22 rhs)
//   s = 3: u* = uo + dt (a31 F1 + a33 rhs)        (a32 = 0, so F2 is never needed)
struct StageCoef {
    int stage;       // 1, 2 or 3
    double dt_a11;   // dt*rk_coef(1,1), stage 1
    double dt;       // dt, stages 2 and 3
    double c1, c2;   // rk_coef(s,1) and rk_coef(s,s), stages 2 and 3
    int incr;        // store the increment du = dt (c1 F1 + c2 rhs) instead of u* = uo + du; uo is not read
    const double *dtp = nullptr;   // adaptive time step: dt is dtp[0] (device memory) and dt_a11, dt are not used
    int no_uo = 0;                 // stage 1: the step-start velocity stays in U (fused corrections), uo is not written
};

// Shared-memory neighbourhood of one thread: three z-planes (k-1, k, k+1) of each field, each plane a
// (TX+2) x (TY+2) tile with a one-cell halo in x and y.
template <typename T, int PX> struct TileQ {
    const T *u[3], *v[3], *w[3], *n[3];
    int c;       // local index of the centre cell
    T ub[3];     // streamwise base profile of rows j-1, j, j+1 (mirrored on wall ghost rows)
    // U (total) and Ud (stored deviation from the base profile; equal to U in FP64, where the profile is zero)
    __device__ __forceinline__ T U(int di, int dj, int dk) const { return u[dk + 1][c + dj * PX + di] + ub[dj + 1]; }
    __device__ __forceinline__ T Ud(int di, int dj, int dk) const { return u[dk + 1][c + dj * PX + di]; }
    __device__ __forceinline__ T V(int di, int dj, int dk) const { return v[dk + 1][c + dj * PX + di]; }
    __device__ __forceinline__ T W(int di, int dj, int dk) const { return w[dk + 1][c + dj * PX + di]; }
    __device__ __forceinline__ T N(int di, int dj, int dk) const { return n[dk + 1][c + dj * PX + di]; }
};

// The same neighbourhood for a pair of x-neighbour cells (c, c+1) in FP32 shared planes; c is even and so is the
// row pitch PX, so a pair at an even x-offset is one 8-byte shared load.
template <int PX> struct TileQ2 {
    const float *u[3], *v[3], *w[3], *n[3];
    int c;
    F2 ub[3];
    static __device__ __forceinline__ F2 ld(const float *pl, int off) {
        if ((off & 1) == 0) return F2(*reinterpret_cast<const float2 *>(pl + off));
        return F2::pair(pl[off], pl[off + 1]);
    }
    __device__ __forceinline__ F2 U(int di, int dj, int dk) const { return ld(u[dk + 1] + c, dj * PX + di) + ub[dj + 1]; }
    __device__ __forceinline__ F2 Ud(int di, int dj, int dk) const { return ld(u[dk + 1] + c, dj * PX + di); }
    __device__ __forceinline__ F2 V(int di, int dj, int dk) const { return ld(v[dk + 1] + c, dj * PX + di); }
    __device__ __forceinline__ F2 W(int di, int dj, int dk) const { return ld(w[dk + 1] + c, dj * PX + di); }
    __device__ __forceinline__ F2 N(int di, int dj, int dk) const { return ld(n[dk + 1] + c, dj * PX + di); }
};



// One thread's cell (i, j, k) from the shared-memory neighbourhood q: the three right-hand sides and the RK3 stage
// update (or, with rhs_only, the right-hand sides themselves).  Shared by the one-cell stage kernels.
template <typename T, bool LES, bool WM, bool HYB, typename Q>
__device__ __forceinline__ void stage_cell(const StepArgs<T> &a, const Q &q, const AxisLocal<T> &Y,
                                           const double *__restrict__ tau_x, const double *__restrict__ tau_z,
                                           const StageCoef &sc, int i, int j, int k, T *__restrict__ uo,
                                           T *__restrict__ vo, T *__restrict__ wo, T *__restrict__ f1u,
                                           T *__restrict__ f1v, T *__restrict__ f1w, T *__restrict__ us,
                                           T *__restrict__ vs, T *__restrict__ wsf, T *__restrict__ rhs_only) {
    const Dims &d = a.d;
    const int p = k * (d.Nx * d.Ny) + j * d.Nx + i;
    const bool vrow = j < d.NyV;
    const bool upd = !rhs_only && sc.stage != 1;
    T ou = T(0), ov = T(0), ow = T(0), fu = T(0), fv = T(0), fw = T(0);
    if (upd) {   // issue the base-state and F1 loads before the arithmetic
        if (!sc.incr) { ou = uo[p]; ow = wo[p]; if (vrow) ov = vo[p]; }
        fu = f1u[p]; fw = f1w[p];
        if (vrow) fv = f1v[p];
    }
    AxisLocal<T> Z;
    Z.load(a.mz, k);
    T ru = rhs_u_at<T, LES, WM>(a, q, Y, Z, tau_x, i, j, k);
    T rw = rhs_w_at<T, LES, WM>(a, q, Y, Z, tau_z, i, j, k);
    T rv = vrow ? rhs_v_at<T, LES, WM>(a, q, Y, Z, i, j, k) : T(0);
    if constexpr (HYB) {
        ru = ru + a.adv[p]; rw = rw + a.adv[2 * d.cells + p];
        if (vrow) rv = rv + a.adv[d.cells + p];
    }
    if (rhs_only) {
        rhs_only[p] = ru; rhs_only[d.cells + p] = rv; rhs_only[2 * d.cells + p] = rw;
    } else if (sc.stage == 1) {
        T c = (T)(sc.dtp ? *sc.dtp * (8.0 / 15.0) : sc.dt_a11);
        T u0 = q.Ud(0, 0, 0), w0 = q.W(0, 0, 0);   // U as stored (deviation from the base profile)
        f1u[p] = ru; us[p] = u0 + c * ru;
        f1w[p] = rw; wsf[p] = w0 + c * rw;
        if (!sc.no_uo) { uo[p] = u0; wo[p] = w0; }
        if (vrow) {
            T v0 = q.V(0, 0, 0);
            f1v[p] = rv; vs[p] = v0 + c * rv;
            if (!sc.no_uo) vo[p] = v0;
        }
    } else {
        T c1 = (T)sc.c1, c2 = (T)sc.c2, dtt = (T)(sc.dtp ? *sc.dtp : sc.dt);   // with sc.incr the base stays zero: du
        us[p] = ou + dtt * (c1 * fu + c2 * ru);
        wsf[p] = ow + dtt * (c1 * fw + c2 * rw);
        if (vrow) vs[p] = ov + dtt * (c1 * fv + c2 * rv);
    }
}

// Tiled kernels (KIND 0: fused stage, KIND 1: eddy viscosity, KIND 2: fused stage adding the dissipative terms of
// advection_scheme = 2 from StepArgs::adv), 2.5-D blocked: a block owns a TX x TY column of
// (i,j) cells and marches through a chunk of kc z-planes.  Each z-plane of U, V, W (and nu_t) is copied from HBM
// once per block, with its one-cell halo, into one of four rotating shared planes by cp.async: the copies of
// plane k+2 are in flight while the cells of plane k are evaluated, and one barrier per plane suffices.  After
// its copies land, each thread adds the streamwise base profile to the U elements it copied and applies the wall
// rules (no-slip mirror of U and W, zero V and nu_t on the ghost rows).  Every thread then evaluates the three
// right-hand sides of its cell from shared memory and writes the RK3 update (or, with rhs_only, the right-hand
// sides themselves for the unit entry point; with KIND 1, nu_t).
// WM = false compiles the flat-wall model out; with WM = true the runtime flag StepArgs::wm decides (the FP64 form
// always takes that variant: without the branches its register allocation spills).
// CORR (stages 2 and 3 of a step whose stage kernel is the only reader of the corrected velocity): U, V, W are the
// previous stage's u*, and the loader applies that stage's projection, u = u* - grad(phi) with StepArgs::phi, to
// every plane element it copies, before the wall rules -- the arithmetic of k_correct, so the values are the ones
// k_correct would have stored.  phi planes rotate through five more shared planes and are copied two planes ahead
// of the velocity planes (a plane's w correction needs phi of the plane above), so they have landed, and passed a
// barrier, before the plane that needs them is corrected.
template <typename T, bool LES, bool WM, int TX, int TY, int KIND, bool CORR = false, class BC>
__device__ __forceinline__ void k_tiled_body(const BC &bc, const StepArgs<T> &a, const T *__restrict__ U, const T *__restrict__ V,
                                                  const T *__restrict__ W, const T *__restrict__ NU,
                                                  const double *__restrict__ tau_x, const double *__restrict__ tau_z,
                                                  const StageCoef &sc, const int kc, T *__restrict__ uo, T *__restrict__ vo,
                                                  T *__restrict__ wo, T *__restrict__ f1u, T *__restrict__ f1v,
                                                  T *__restrict__ f1w, T *__restrict__ us, T *__restrict__ vs,
                                                  T *__restrict__ wsf, T *__restrict__ rhs_only, T *__restrict__ nut_out) {
    constexpr int PX = TX + 2, PY = TY + 2, PS = PX * PY, NT = TX * TY;
    constexpr int NF = LES ? 4 : 3;
    constexpr int PER = (PS + NT - 1) / NT;   // plane elements per thread
    __shared__ __align__(16) T sm[NF][4][PS];
    constexpr int PXP = PX + 1, PSP = PXP * (PY + 1), PERP = (PSP + NT - 1) / NT;   // phi tile: one more column, row
    __shared__ __align__(16) T smp[CORR ? 5 : 1][CORR ? PSP : 1];
    const Dims &d = a.d;
    const int Nx = d.Nx, Ny = d.Ny, Nz = d.Nz;
    const int i0 = bc.idx().x * TX, j0 = bc.idx().y * TY;
    const int k0 = bc.idx().z * kc, kend = min(k0 + kc, Nz);
    const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
    const int i = i0 + tx, j = j0 + ty;
    const bool active = i < Nx && j < Ny;
    const int plane = Nx * Ny;

    // This thread's share of a plane: offsets within the plane (or -1), the wall rule and the base profile.
    int off[PER];
    bool ghost[PER];   // wall ghost row: mirror U/W, zero V/nu_t
    int pix[CORR ? PER : 1];    // CORR: phi-tile index of the element
    T iyq[CORR ? PER : 1];      // CORR: 1/(centre spacing) of its row for the v correction, 0 where v is not corrected
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        int e = threadIdx.x + q * NT;
        off[q] = -1; ghost[q] = false;
        if (e < PS) {
            int jj = e / PX, ii = e - jj * PX;
            int gi = i0 - 1 + ii;
            gi = gi < 0 ? gi + Nx : gi;
            while (gi >= Nx) gi -= Nx;
            int gj = j0 - 1 + jj, g;
            if (d.yper) {
                g = gj < 0 ? gj + Ny : gj;
                while (g >= Ny) g -= Ny;
            } else {
                g = gj < 0 ? 0 : (gj >= Ny ? Ny - 1 : gj);
                ghost[q] = (gj < 0 || gj >= Ny);
            }
            off[q] = g * Nx + gi;
            if constexpr (CORR) {
                pix[q] = jj * PXP + ii;
                iyq[q] = (ghost[q] || g >= d.NyV) ? T(0) : Arith<T>::inv(a.my.df, a.my.idf, g);
            }
        }
    }
    int offp[CORR ? PERP : 1];   // CORR: this thread's share of a phi plane (same row and column rules)
    if constexpr (CORR) {
#pragma unroll
        for (int q = 0; q < PERP; ++q) {
            int e = threadIdx.x + q * NT;
            offp[q] = -1;
            if (e < PSP) {
                int jj = e / PXP, ii = e - jj * PXP;
                int gi = i0 - 1 + ii;
                gi = gi < 0 ? gi + Nx : gi;
                while (gi >= Nx) gi -= Nx;
                int gj = j0 - 1 + jj, g;
                if (d.yper) { g = gj < 0 ? gj + Ny : gj; while (g >= Ny) g -= Ny; }
                else g = gj < 0 ? 0 : (gj >= Ny ? Ny - 1 : gj);
                offp[q] = g * Nx + gi;
            }
        }
    }
    auto issue_phi = [&](int k) {   // phi plane k into phi slot (k - k0 + 1) % 5
        if constexpr (CORR) {
            const int kw = k < 0 ? k + Nz : (k >= Nz ? k - Nz : k), slot = (k - k0 + 1) % 5;
#pragma unroll
            for (int q = 0; q < PERP; ++q)
                if (offp[q] >= 0) cp_async<sizeof(T)>(&smp[slot][threadIdx.x + q * NT], a.phi + kw * plane + offp[q]);
        }
    };
    auto issue = [&](int slot, int k) {
        int kw = k < 0 ? k + Nz : (k >= Nz ? k - Nz : k);
        const int kb = kw * plane;
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            if (off[q] < 0) continue;
            const int o = kb + off[q], e = threadIdx.x + q * NT;
            cp_async<sizeof(T)>(&sm[0][slot][e], U + o);
            cp_async<sizeof(T)>(&sm[2][slot][e], W + o);
            if (!ghost[q]) {
                cp_async<sizeof(T)>(&sm[1][slot][e], V + o);
                if (LES) cp_async<sizeof(T)>(&sm[NF - 1][slot][e], NU + o);
            }
        }
    };
    auto fix = [&](int slot, int k) {   // after the copies of plane k (and, CORR, phi k and k+1) have landed
        if constexpr (CORR) {   // project_velocity of the previous stage (k_correct's arithmetic)
            const int kw = k < 0 ? k + Nz : (k >= Nz ? k - Nz : k);
            const int p0 = (k - k0 + 1) % 5, p1 = (k - k0 + 2) % 5;
            const T iz = Arith<T>::inv(a.mz.df, a.mz.idf, kw);
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                if (off[q] < 0) continue;
                const int e = threadIdx.x + q * NT;
                const T pc = smp[p0][pix[q]], pxp = smp[p0][pix[q] + 1], pzp = smp[p1][pix[q]];
                sm[0][slot][e] = sm[0][slot][e] - (pxp - pc) * a.inv_dx;
                sm[2][slot][e] = sm[2][slot][e] - (pzp - pc) * iz;
                if (iyq[q] != T(0)) sm[1][slot][e] = sm[1][slot][e] - (smp[p0][pix[q] + PXP] - pc) * iyq[q];
            }
        }
#pragma unroll
        for (int q = 0; q < PER; ++q) {   // wall ghost rows
            if (off[q] < 0 || !ghost[q]) continue;
            const int e = threadIdx.x + q * NT;
            sm[0][slot][e] = -sm[0][slot][e];   // deviation mirrored; the row profile is mirrored in TileQ::ub
            sm[2][slot][e] = -sm[2][slot][e];
            sm[1][slot][e] = T(0);
            if (LES) sm[NF - 1][slot][e] = T(0);
        }
    };
    // base profile of the thread's rows j-1, j, j+1 (a wall ghost row carries minus its mirror row's profile)
    T ubr[3];
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj) {
        int gj = min(j, Ny - 1) + dj;
        T sgn = T(1);
        if (d.yper) { gj = gj < 0 ? gj + Ny : (gj >= Ny ? gj - Ny : gj); }
        else if (gj < 0 || gj >= Ny) { gj = gj < 0 ? 0 : Ny - 1; sgn = T(-1); }
        ubr[dj + 1] = sgn * __ldg(a.ub + gj);
    }

    AxisLocal<T> Y;   // this thread's y metrics (FP32: read here once for every plane)
    Y.load(a.my, min(j, Ny - 1));

    // planes k0-1, k0, k0+1 into slots 0, 1, 2; plane k lives in slot (k - k0 + 1) & 3 (CORR: phi k0-1 .. k0+2)
    issue(0, k0 - 1); issue(1, k0); issue(2, k0 + 1);
    issue_phi(k0 - 1); issue_phi(k0); issue_phi(k0 + 1); issue_phi(k0 + 2); issue_phi(k0 + 3);
    cp_async_commit();
    cp_async_wait_all();
    if (CORR) __syncthreads();   // phi elements copied by other threads
    fix(0, k0 - 1); fix(1, k0); fix(2, k0 + 1);
    __syncthreads();
    const int cloc = (ty + 1) * PX + tx + 1;
    for (int k = k0; k < kend; ++k) {
        const bool more = k + 2 <= kend;
        const int snext = (k - k0 + 3) & 3;
        if (more) { issue(snext, k + 2); issue_phi(k + 4); }
        cp_async_commit();
        const int sm_ = (k - k0) & 3, s0 = (k - k0 + 1) & 3, sp = (k - k0 + 2) & 3;
        if (active) {
            const int p = k * plane + j * Nx + i;
            TileQ<T, PX> q;
            q.c = cloc;
            q.ub[0] = ubr[0]; q.ub[1] = ubr[1]; q.ub[2] = ubr[2];
            q.u[0] = sm[0][sm_]; q.u[1] = sm[0][s0]; q.u[2] = sm[0][sp];
            q.v[0] = sm[1][sm_]; q.v[1] = sm[1][s0]; q.v[2] = sm[1][sp];
            q.w[0] = sm[2][sm_]; q.w[1] = sm[2][s0]; q.w[2] = sm[2][sp];
            q.n[0] = sm[NF - 1][sm_]; q.n[1] = sm[NF - 1][s0]; q.n[2] = sm[NF - 1][sp];
            if (KIND == 1) {
                nut_out[p] = nut_at<T>(a, q, i, j, k);
            } else {
                stage_cell<T, LES, WM, KIND == 2>(a, q, Y, tau_x, tau_z, sc, i, j, k, uo, vo, wo, f1u, f1v, f1w, us, vs,
                                                  wsf, rhs_only);
            }
        }
        cp_async_wait_all();
        if (more) fix(snext, k + 2);   // CORR: phi k+2 and k+3 were copied one and two iterations ago
        __syncthreads();
    }
}
template <typename T, bool LES, bool WM, int TX, int TY, int KIND, bool CORR = false>
__global__ void __launch_bounds__(TX *TY, sizeof(T) == 4 ? 3 : 2) k_tiled(StepArgs<T> a, const T *__restrict__ U, const T *__restrict__ V,
                                                  const T *__restrict__ W, const T *__restrict__ NU,
                                                  const double *__restrict__ tau_x, const double *__restrict__ tau_z,
                                                  StageCoef sc, int kc, T *__restrict__ uo, T *__restrict__ vo,
                                                  T *__restrict__ wo, T *__restrict__ f1u, T *__restrict__ f1v,
                                                  T *__restrict__ f1w, T *__restrict__ us, T *__restrict__ vs,
                                                  T *__restrict__ wsf, T *__restrict__ rhs_only, T *__restrict__ nut_out) {
    pdl_enter();
    k_tiled_body<T, LES, WM, TX, TY, KIND, CORR>(HwBlock(), a, U, V, W, NU, tau_x, tau_z, sc, kc, uo, vo, wo, f1u, f1v, f1w, us, vs, wsf, rhs_only, nut_out);
}


// One thread's pair of cells (i, i+1) of plane k from the shared-memory neighbourhood q: the three right-hand sides
// and the RK3 stage update (or, with rhs_only, the right-hand sides themselves).  zm holds the eight z metrics of
// plane k (AxisLocal<F2>::load8 order).  Shared by the packed stage kernels.
template <bool LES, bool WM, bool HYB, int PX>
__device__ __forceinline__ void stage_pair(const StepArgs<float> &a, const TileQ2<PX> &q, const AxisLocal<F2> &Y,
                                           const float *zm, const double *__restrict__ tau_x,
                                           const double *__restrict__ tau_z, const StageCoef &sc, int i, int j, int k,
                                           float *__restrict__ uo, float *__restrict__ vo, float *__restrict__ wo,
                                           float *__restrict__ f1u, float *__restrict__ f1v, float *__restrict__ f1w,
                                           float *__restrict__ us, float *__restrict__ vs, float *__restrict__ wsf,
                                           float *__restrict__ rhs_only) {
    const Dims &d = a.d;
    const int p = k * (d.Nx * d.Ny) + j * d.Nx + i;
    const bool vrow = j < d.NyV;
    const bool upd = !rhs_only && sc.stage != 1;
    auto ld2 = [&](const float *b) { return F2(*reinterpret_cast<const float2 *>(b + p)); };
    auto st2 = [&](float *b, F2 x) { *reinterpret_cast<float2 *>(b + p) = x.v; };
    F2 ou(0.0f), ov(0.0f), ow(0.0f), fu(0.0f), fv(0.0f), fw(0.0f);
    if (upd) {
        if (!sc.incr) { ou = ld2(uo); ow = ld2(wo); if (vrow) ov = ld2(vo); }
        fu = ld2(f1u); fw = ld2(f1w);
        if (vrow) fv = ld2(f1v);
    }
    AxisLocal<F2> Z;
    Z.load8(zm);
    F2 ru = rhs_u_at<F2, LES, WM>(a, q, Y, Z, tau_x, i, j, k);
    F2 rw = rhs_w_at<F2, LES, WM>(a, q, Y, Z, tau_z, i, j, k);
    F2 rv = vrow ? rhs_v_at<F2, LES, WM>(a, q, Y, Z, i, j, k) : F2(0.0f);
    if constexpr (HYB) {
        ru = ru + ld2(a.adv); rw = rw + ld2(a.adv + 2 * d.cells);
        if (vrow) rv = rv + ld2(a.adv + d.cells);
    }
    if (rhs_only) {
        st2(rhs_only, ru); st2(rhs_only + d.cells, rv); st2(rhs_only + 2 * d.cells, rw);
    } else if (sc.stage == 1) {
        const F2 c = F2(sc.dtp ? *sc.dtp * (8.0 / 15.0) : sc.dt_a11);
        F2 u0 = q.Ud(0, 0, 0), w0 = q.W(0, 0, 0);
        st2(f1u, ru); st2(us, u0 + c * ru);
        st2(f1w, rw); st2(wsf, w0 + c * rw);
        if (!sc.no_uo) { st2(uo, u0); st2(wo, w0); }
        if (vrow) {
            F2 v0 = q.V(0, 0, 0);
            st2(f1v, rv); st2(vs, v0 + c * rv);
            if (!sc.no_uo) st2(vo, v0);
        }
    } else {
        const F2 c1 = F2(sc.c1), c2 = F2(sc.c2), dtt = F2(sc.dtp ? *sc.dtp : sc.dt);
        st2(us, ou + dtt * (c1 * fu + c2 * ru));
        st2(wsf, ow + dtt * (c1 * fw + c2 * rw));
        if (vrow) st2(vs, ov + dtt * (c1 * fv + c2 * rv));
    }
}

// FP32 stage kernel with two x-neighbour cells per thread, computed with the packed FP32x2 instructions (F2).  Same
// loader, ghost rules and RK3 epilogue as k_tiled<float, LES, WM, ..., 0>; a block owns 64 x TY cells, one warp
// per row of 32 cell pairs; HYB adds the dissipative terms of advection_scheme = 2 (StepArgs::adv); CORR fuses
// the previous stage's correction into the loader as k_tiled does.  It needs ~118 registers: capping it at 96 or 80 (for more resident warps) spills
// 170-300 bytes, so it runs 2 blocks of 256 threads per SM.  Shared rows hold cells i0-2 .. i0+65 (pitch 68), so every pair starts at an even index.
template <bool LES, bool WM, int TY = 8, bool HYB = false, bool CORR = false, class BC>
__device__ __forceinline__ void k_tiled2_body(const BC &bc, const StepArgs<float> &a, const float *__restrict__ U, const float *__restrict__ V,
                                                   const float *__restrict__ W, const float *__restrict__ NU,
                                                   const double *__restrict__ tau_x, const double *__restrict__ tau_z,
                                                   const StageCoef &sc, const int kc, float *__restrict__ uo, float *__restrict__ vo,
                                                   float *__restrict__ wo, float *__restrict__ f1u, float *__restrict__ f1v,
                                                   float *__restrict__ f1w, float *__restrict__ us, float *__restrict__ vs,
                                                   float *__restrict__ wsf, float *__restrict__ rhs_only) {
    constexpr int TXC = 64, NT = 32 * TY;
    constexpr int PX = TXC + 4, PY = TY + 2, PS = PX * PY;
    constexpr int NF = LES ? 4 : 3;
    // the loader moves element pairs (columns 2m, 2m+1 of a tile row: even global x, so one 8-byte copy)
    constexpr int PS2 = PS / 2, PER = (PS2 + NT - 1) / NT;
    __shared__ __align__(16) float sm[NF][4][PS];
    // CORR phi tile: two more columns (an even pitch keeps pairs aligned) and one more row
    constexpr int PXP = PX + 2, PSP2 = PXP * (PY + 1) / 2, PERP = (PSP2 + NT - 1) / NT;
    __shared__ __align__(16) float smp[CORR ? 5 : 1][CORR ? 2 * PSP2 : 2];
    // the z metrics of planes k .. k+2 (AxisLocal<F2>::load8 order), copied with the planes: under the streaming
    // tile copies the metric tables do not stay in L1, and every thread needs them at the start of its plane
    __shared__ float zmr[4][8];
    const Dims &d = a.d;
    const int Nx = d.Nx, Ny = d.Ny, Nz = d.Nz;
    const int i0 = bc.idx().x * TXC, j0 = bc.idx().y * TY;
    const int k0 = bc.idx().z * kc, kend = min(k0 + kc, Nz);
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int i = i0 + 2 * tx, j = j0 + ty;
    const bool active = i < Nx && j < Ny;   // Nx is even: the pair's second cell is in range too
    const int plane = Nx * Ny;

    int off[PER];       // global offset of the pair's first element within a plane, or -1
    bool ghost[PER];
    int pix[CORR ? PER : 1];      // CORR: phi-tile index of the pair
    float iyq[CORR ? PER : 1];    // CORR: 1/(centre spacing) of its row for the v correction, 0 where v is not corrected
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        int e2 = threadIdx.x + q * NT;
        off[q] = -1; ghost[q] = false;
        if (e2 < PS2) {
            int jj = e2 / (PX / 2), ii = 2 * (e2 - jj * (PX / 2));
            int gi = i0 - 2 + ii;
            gi = gi < 0 ? gi + Nx : gi;
            while (gi >= Nx) gi -= Nx;
            int gj = j0 - 1 + jj, g;
            if (d.yper) {
                g = gj < 0 ? gj + Ny : gj;
                while (g >= Ny) g -= Ny;
            } else {
                g = gj < 0 ? 0 : (gj >= Ny ? Ny - 1 : gj);
                ghost[q] = (gj < 0 || gj >= Ny);
            }
            off[q] = g * Nx + gi;
            if constexpr (CORR) {
                pix[q] = jj * PXP + ii;
                iyq[q] = (ghost[q] || g >= d.NyV) ? 0.0f : Arith<float>::inv(a.my.df, a.my.idf, g);
            }
        }
    }
    int offp[CORR ? PERP : 1];   // CORR: this thread's pairs of a phi plane (same row and column rules)
    if constexpr (CORR) {
#pragma unroll
        for (int q = 0; q < PERP; ++q) {
            int e2 = threadIdx.x + q * NT;
            offp[q] = -1;
            if (e2 < PSP2) {
                int jj = e2 / (PXP / 2), ii = 2 * (e2 - jj * (PXP / 2));
                int gi = i0 - 2 + ii;
                gi = gi < 0 ? gi + Nx : gi;
                while (gi >= Nx) gi -= Nx;
                int gj = j0 - 1 + jj, g;
                if (d.yper) { g = gj < 0 ? gj + Ny : gj; while (g >= Ny) g -= Ny; }
                else g = gj < 0 ? 0 : (gj >= Ny ? Ny - 1 : gj);
                offp[q] = g * Nx + gi;
            }
        }
    }
    auto issue_phi = [&](int k) {   // phi plane k into phi slot (k - k0 + 1) % 5
        if constexpr (CORR) {
            const int kw = k < 0 ? k + Nz : (k >= Nz ? k - Nz : k), slot = (k - k0 + 1) % 5;
#pragma unroll
            for (int q = 0; q < PERP; ++q)
                if (offp[q] >= 0) cp_async<8>(&smp[slot][2 * (threadIdx.x + q * NT)], a.phi + kw * plane + offp[q]);
        }
    };
    auto issue_z = [&](int k) {   // the z metrics of plane k (k0 <= k < kend) into zmr[(k - k0) & 3]
        if (threadIdx.x < 8) cp_async<4>(&zmr[(k - k0) & 3][threadIdx.x], AxisLocal<F2>::metric_src(a.mz, k, threadIdx.x));
    };
    auto issue = [&](int slot, int k) {
        int kw = k < 0 ? k + Nz : (k >= Nz ? k - Nz : k);
        const int kb = kw * plane;
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            if (off[q] < 0) continue;
            const int o = kb + off[q], e = 2 * (threadIdx.x + q * NT);
            cp_async<8>(&sm[0][slot][e], U + o);
            cp_async<8>(&sm[2][slot][e], W + o);
            if (!ghost[q]) {
                cp_async<8>(&sm[1][slot][e], V + o);
                if (LES) cp_async<8>(&sm[NF - 1][slot][e], NU + o);
            }
        }
    };
    auto fix = [&](int slot, int k) {
        if constexpr (CORR) {   // project_velocity of the previous stage (k_correct's arithmetic, lane by lane)
            const int kw = k < 0 ? k + Nz : (k >= Nz ? k - Nz : k);
            const int p0 = (k - k0 + 1) % 5, p1 = (k - k0 + 2) % 5;
            const float iz = Arith<float>::inv(a.mz.df, a.mz.idf, kw);
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                if (off[q] < 0) continue;
                const int e = 2 * (threadIdx.x + q * NT);
                const float2 pc = *reinterpret_cast<const float2 *>(&smp[p0][pix[q]]);
                const float pn = smp[p0][pix[q] + 2];
                const float2 pz = *reinterpret_cast<const float2 *>(&smp[p1][pix[q]]);
                float2 *u2 = reinterpret_cast<float2 *>(&sm[0][slot][e]), *w2 = reinterpret_cast<float2 *>(&sm[2][slot][e]);
                float2 u = *u2, w = *w2;
                u.x = u.x - (pc.y - pc.x) * a.inv_dx; u.y = u.y - (pn - pc.y) * a.inv_dx;
                w.x = w.x - (pz.x - pc.x) * iz; w.y = w.y - (pz.y - pc.y) * iz;
                *u2 = u; *w2 = w;
                if (iyq[q] != 0.0f) {
                    const float2 py = *reinterpret_cast<const float2 *>(&smp[p0][pix[q] + PXP]);
                    float2 *v2 = reinterpret_cast<float2 *>(&sm[1][slot][e]);
                    float2 v = *v2;
                    v.x = v.x - (py.x - pc.x) * iyq[q]; v.y = v.y - (py.y - pc.y) * iyq[q];
                    *v2 = v;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            if (off[q] < 0 || !ghost[q]) continue;
            const int e = 2 * (threadIdx.x + q * NT);
            float2 *u2 = reinterpret_cast<float2 *>(&sm[0][slot][e]), *w2 = reinterpret_cast<float2 *>(&sm[2][slot][e]);
            const float2 u = *u2, w = *w2;
            *u2 = make_float2(-u.x, -u.y);
            *w2 = make_float2(-w.x, -w.y);
            *reinterpret_cast<float2 *>(&sm[1][slot][e]) = make_float2(0.0f, 0.0f);
            if (LES) *reinterpret_cast<float2 *>(&sm[NF - 1][slot][e]) = make_float2(0.0f, 0.0f);
        }
    };
    F2 ubr[3];
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj) {
        int gj = min(j, Ny - 1) + dj;
        float sgn = 1.0f;
        if (d.yper) { gj = gj < 0 ? gj + Ny : (gj >= Ny ? gj - Ny : gj); }
        else if (gj < 0 || gj >= Ny) { gj = gj < 0 ? 0 : Ny - 1; sgn = -1.0f; }
        ubr[dj + 1] = F2(sgn * __ldg(a.ub + gj));
    }
    AxisLocal<F2> Y;
    Y.load(a.my, min(j, Ny - 1));

    issue(0, k0 - 1); issue(1, k0); issue(2, k0 + 1);
    issue_phi(k0 - 1); issue_phi(k0); issue_phi(k0 + 1); issue_phi(k0 + 2); issue_phi(k0 + 3);
    issue_z(k0);
    if (k0 + 1 < kend) issue_z(k0 + 1);
    cp_async_commit();
    cp_async_wait_all();
    if (CORR) __syncthreads();   // phi elements copied by other threads
    fix(0, k0 - 1); fix(1, k0); fix(2, k0 + 1);
    __syncthreads();
    const int cloc = (ty + 1) * PX + 2 + 2 * tx;
    for (int k = k0; k < kend; ++k) {
        const bool more = k + 2 <= kend;
        const int snext = (k - k0 + 3) & 3;
        if (more) { issue(snext, k + 2); issue_phi(k + 4); }
        if (k + 2 < kend) issue_z(k + 2);
        cp_async_commit();
        const int sm_ = (k - k0) & 3, s0 = (k - k0 + 1) & 3, sp = (k - k0 + 2) & 3;
        if (active) {
            TileQ2<PX> q;
            q.c = cloc;
            q.ub[0] = ubr[0]; q.ub[1] = ubr[1]; q.ub[2] = ubr[2];
            q.u[0] = sm[0][sm_]; q.u[1] = sm[0][s0]; q.u[2] = sm[0][sp];
            q.v[0] = sm[1][sm_]; q.v[1] = sm[1][s0]; q.v[2] = sm[1][sp];
            q.w[0] = sm[2][sm_]; q.w[1] = sm[2][s0]; q.w[2] = sm[2][sp];
            q.n[0] = sm[NF - 1][sm_]; q.n[1] = sm[NF - 1][s0]; q.n[2] = sm[NF - 1][sp];
            stage_pair<LES, WM, HYB>(a, q, Y, zmr[(k - k0) & 3], tau_x, tau_z, sc, i, j, k, uo, vo, wo, f1u, f1v, f1w,
                                     us, vs, wsf, rhs_only);
        }
        cp_async_wait_all();
        if (more) fix(snext, k + 2);   // CORR: phi k+2 and k+3 were copied one and two iterations ago
        __syncthreads();
    }
}
template <bool LES, bool WM, int TY = 8, bool HYB = false, bool CORR = false>
__global__ void __launch_bounds__(32 * TY, 512 / (32 * TY)) k_tiled2(StepArgs<float> a, const float *__restrict__ U, const float *__restrict__ V,
                                                   const float *__restrict__ W, const float *__restrict__ NU,
                                                   const double *__restrict__ tau_x, const double *__restrict__ tau_z,
                                                   StageCoef sc, int kc, float *__restrict__ uo, float *__restrict__ vo,
                                                   float *__restrict__ wo, float *__restrict__ f1u, float *__restrict__ f1v,
                                                   float *__restrict__ f1w, float *__restrict__ us, float *__restrict__ vs,
                                                   float *__restrict__ wsf, float *__restrict__ rhs_only) {
    pdl_enter();
    k_tiled2_body<LES, WM, TY, HYB, CORR>(HwBlock(), a, U, V, W, NU, tau_x, tau_z, sc, kc, uo, vo, wo, f1u, f1v, f1w, us, vs, wsf, rhs_only);
}

}  // namespace dfdm
