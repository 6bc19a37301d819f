// dfdm_oracle.cpp -- TEST INFRASTRUCTURE ONLY: the CPU FP64 oracle of the dopamine-fdm single-phase RK3 step.
//
// This file restates, in C++, the reference's Fortran algorithm for one time step, following its loops, array
// shapes (one rank, column-major, explicit lower bounds) and expression order, so that the GPU library can be
// checked against it. It is the checker, never the product: only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg may load it. Nothing in the shipped library calls it, and the library fails loudly when its
// own CUDA code is missing instead of falling back here.
//
// Parity status: the reference (Fortran + MPI + FFTW + LAPACK) cannot be built in this environment and ships no
// golden vectors for this path, so this restatement is pinned against the reference's own regression invariants
// (max|div| after a projection, periodic/wall ghost identities, restart = uninterrupted) and against analytic
// known answers (manufactured Poisson modes, Taylor-Green decay) in tests/, plus numpy's FFT and scipy's LAPACK
// zgtsv for the third-party arithmetic.  Against reference OUTPUTS it is "parity unpinned".
//
// Reference files followed (paths inside the dopamine-fdm project):
//   src/time_integration.f90:120-713  compute_time_step_RK3 (Butcher-form RK3, stage order, constant flux)
//   src/equations.f90:25-721          compute_rhs_u / compute_rhs_v / compute_rhs_w
//   src/interpolation.f90:13-88       interpolate_x / _y / _z
//   src/sgs_model.f90:73-338,458-531  compute_vreman (AMD and Vreman), sgs_fill_ghosts
//   src/wallmodel.f90:29-74,397-583   Reichardt law, Newton solve, update_wm_filter, compute_flat_wall_eqwm
//   src/boundary_conditions.f90:186-804 apply_boundary_conditions and the periodic / Robin rules
//   src/projection.f90:21-639         divergence, solve_poisson_equation (CPU chain), projection, P save
//   src/initialization.f90:243-274,326-345,417-539,629-660  centres, dx, kxx/kzz/kyy, Dyy, weights, RK
//   src/monitor.f90:463-523           compute_bulk_velocity (compensated sums: the reference's order is unspecified)
// Third-party arithmetic restated from its published algorithm: FFTW3's complex DFT (here a mixed-radix
// Cooley-Tukey FFT) and LAPACK zgtsv (Gaussian elimination with partial pivoting, LAPACK 3.x).

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <algorithm>
#include <limits>
#include "dfdm.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef std::complex<double> cplx;

// A Fortran-style 3-D array with explicit lower and upper bounds, column-major.
struct A3 {
    int l1 = 1, u1 = 0, l2 = 1, u2 = 0, l3 = 1, u3 = 0;
    long n1 = 0, n2 = 0, n3 = 0;
    std::vector<double> d;
    void init(int a1, int b1, int a2, int b2, int a3, int b3) {
        l1 = a1; u1 = b1; l2 = a2; u2 = b2; l3 = a3; u3 = b3;
        n1 = b1 - a1 + 1; n2 = b2 - a2 + 1; n3 = b3 - a3 + 1;
        d.assign((size_t)(n1 * n2 * n3), 0.0);
    }
    inline double &operator()(int i, int j, int k) {
        return d[(size_t)((i - l1) + n1 * ((j - l2) + n2 * (long)(k - l3)))];
    }
    inline double operator()(int i, int j, int k) const {
        return d[(size_t)((i - l1) + n1 * ((j - l2) + n2 * (long)(k - l3)))];
    }
    size_t size() const { return d.size(); }
};

// ---------------------------------------------------------------------------------------------------------------
// FFT: mixed-radix Cooley-Tukey (radix 2, 3, 4 and a plain DFT for any other prime), forward sign -1, unnormalised,
// the same convention as FFTW_FORWARD / FFTW_BACKWARD.
struct FFTPlan {
    int n = 0;
    std::vector<int> factors;
    std::vector<cplx> tw;  // exp(-2 pi i k / n), k = 0..n-1
    // Per recursion level fi (sub-length len = n / twstride, radix r, m = len / r): the table entries the
    // butterflies use, gathered once so that the inner loops index without a modulo. tw1[fi][q*m + k] =
    // tw[(q k twstride) mod n] (twiddles), tw2[fi][q*r + s] = tw[(q s m twstride) mod n] (the radix-r DFT).
    std::vector<std::vector<cplx>> tw1, tw2;
    void init(int n_) {
        n = n_;
        factors.clear();
        int m = n;
        while (m % 4 == 0) { factors.push_back(4); m /= 4; }
        while (m % 2 == 0) { factors.push_back(2); m /= 2; }
        while (m % 3 == 0) { factors.push_back(3); m /= 3; }
        for (int p = 5; m > 1; p += 2) while (m % p == 0) { factors.push_back(p); m /= p; }
        tw.resize(n);
        const double pi = 4.0 * std::atan(1.0);
        for (int k = 0; k < n; ++k) {
            double a = -2.0 * pi * (double)k / (double)n;
            tw[k] = cplx(std::cos(a), std::sin(a));
        }
        tw1.assign(factors.size(), {});
        tw2.assign(factors.size(), {});
        long twstride = 1;
        for (size_t fi = 0; fi < factors.size(); ++fi) {
            int r = factors[fi];
            long len = n / twstride, mm = len / r;
            tw1[fi].resize((size_t)(r * mm));
            tw2[fi].resize((size_t)(r * r));
            for (int q = 0; q < r; ++q) {
                for (long k = 0; k < mm; ++k) tw1[fi][(size_t)(q * mm + k)] = tw[(size_t)((long)q * k * twstride % n)];
                for (int s2 = 0; s2 < r; ++s2) tw2[fi][(size_t)(q * r + s2)] = tw[(size_t)((long)q * s2 * mm * twstride % n)];
            }
            twstride *= r;
        }
    }
    // recursive decimation in time on strided input
    void rec(const cplx *in, long istride, cplx *out, int len, int fi, bool inverse) const {
        if (len == 1) { out[0] = in[0]; return; }
        int r = factors[fi];
        int m = len / r;
        for (int q = 0; q < r; ++q)
            rec(in + q * istride, istride * r, out + q * m, m, fi + 1, inverse);
        cplx tmp_s[16], res_s[16];
        std::vector<cplx> tmp_v, res_v;
        cplx *tmp = tmp_s, *res = res_s;
        if (r > 16) { tmp_v.resize(r); res_v.resize(r); tmp = tmp_v.data(); res = res_v.data(); }
        const cplx *t1 = tw1[fi].data(), *t2 = tw2[fi].data();
        for (int k = 0; k < m; ++k) {
            for (int q = 0; q < r; ++q) {
                cplx w = t1[q * m + k];
                if (inverse) w = std::conj(w);
                tmp[q] = out[q * m + k] * w;
            }
            for (int s = 0; s < r; ++s) {
                cplx acc(0.0, 0.0);
                for (int q = 0; q < r; ++q) {
                    cplx w = t2[q * r + s];
                    if (inverse) w = std::conj(w);
                    acc += tmp[q] * w;
                }
                res[s] = acc;
            }
            for (int s = 0; s < r; ++s) out[s * m + k] = res[s];
        }
    }
    void exec(cplx *data, long stride, bool inverse) const {
        std::vector<cplx> in(n), out(n);
        for (int i = 0; i < n; ++i) in[i] = data[i * stride];
        rec(in.data(), 1, out.data(), n, 0, inverse);
        for (int i = 0; i < n; ++i) data[i * stride] = out[i];
    }
};

// LAPACK zgtsv restated (Gaussian elimination with partial pivoting on a tridiagonal system, one right-hand
// side). dl(1:n-1), d(1:n), du(1:n-1) are destroyed. Returns info (0 ok, k>0 singular pivot). Counts row
// interchanges in *swaps so the tests can show that the pressure operator never pivots.
static inline double cabs1(cplx z) { return std::fabs(z.real()) + std::fabs(z.imag()); }
int zgtsv(int n, cplx *dl, cplx *d, cplx *du, cplx *b, long *swaps) {
    // 0-based: dl[k] couples row k+1 to column k
    for (int k = 0; k < n - 1; ++k) {
        if (dl[k] == cplx(0.0, 0.0)) {
            if (d[k] == cplx(0.0, 0.0)) return k + 1;
        } else if (cabs1(d[k]) >= cabs1(dl[k])) {
            cplx mult = dl[k] / d[k];
            d[k + 1] = d[k + 1] - mult * du[k];
            b[k + 1] = b[k + 1] - mult * b[k];
            if (k < n - 2) dl[k] = cplx(0.0, 0.0);
        } else {
            if (swaps) ++*swaps;
            cplx mult = d[k] / dl[k];
            d[k] = dl[k];
            cplx temp = d[k + 1];
            d[k + 1] = du[k] - mult * temp;
            if (k < n - 2) {
                dl[k] = du[k + 1];
                du[k + 1] = -mult * dl[k];
            }
            du[k] = temp;
            temp = b[k];
            b[k] = b[k + 1];
            b[k + 1] = temp - mult * b[k + 1];
        }
    }
    if (d[n - 1] == cplx(0.0, 0.0)) return n;
    b[n - 1] = b[n - 1] / d[n - 1];
    if (n > 1) b[n - 2] = (b[n - 2] - du[n - 2] * b[n - 1]) / d[n - 2];
    for (int k = n - 3; k >= 0; --k) b[k] = (b[k] - du[k] * b[k + 1] - dl[k] * b[k + 2]) / d[k];
    return 0;
}

// ---------------------------------------------------------------------------------------------------------------
struct Oracle {
    // grid (one rank): face counts and derived sizes
    int nx, ny, nz, nxg, nyg, nzg, nxm, nym, nzm;
    int x_bc_type, y_bc_type, z_bc_type, bc_face_ylo, bc_face_yhi;
    std::vector<double> x, y, z, xg, yg, zg;   // 1-based storage: x[1..nx]
    double dx, dz, Lx, Ly, Lz;
    int nxp, nzp;                              // Fourier lengths
    std::vector<double> kxx, kzz, kyy;         // 0-based mode index
    std::vector<double> Dyy_d, Dyy_l, Dyy_u;   // Dyy(j,j), Dyy(j,j-1), Dyy(j,j+1), index j (1-based)
    // 4-wall duct (z_bc_type 1 with y walls): Dzz rows 2..nzg-1 (1-based index k), and the eigenbasis of
    // S = W^(1/2) Dzz W^(-1/2): lambda_z ascending, Qz(k, m) = Qz[k * nzm + m] orthonormal, sqrt_w_z(k)
    std::vector<double> Dzz_d, Dzz_l, Dzz_u, lambda_z, Qz, sqrt_w_z;
    std::vector<double> wy0, wy1, wz0, wz1;    // weight_y_0(1:ny), weight_z_0(1:nz), 1-based
    double rk_t[4], rk_coef[4][4];
    dfdm_params prm;
    int nwl;                                   // resolved adv_wall_layers
    int wm_filter_mode;
    double t;
    double dPdx, dPdz;

    A3 U, V, W, P, Uo, Vo, Wo, nu_t, term_1, term_2, rhs_p;
    A3 Fu[4], Fv[4], Fw[4];
    A3 tau_x, tau_z, wmf_ux, wmf_wx, wmf_tx, wmf_uz, wmf_wz, wmf_tz;
    bool wmf_seeded = false;
    FFTPlan fx, fz, fy;
    long gtsv_swaps = 0;
    int last_info = 0;

    const double pi = 4.0 * std::atan(1.0);

    // ---- set-up: src/initialization.f90:243-274 (centres), :326-345 (dx, nxp), :417-489 (k^2), :497-539 (Dyy),
    //      :629-660 (weights, RK), src/wallmodel.f90 j_match (flag 1: j_match = 2, nyg-1)
    int setup(const dfdm_grid *g, const dfdm_params *p) {
        nx = g->nx; ny = g->ny; nz = g->nz;
        x_bc_type = g->x_bc_type; y_bc_type = g->y_bc_type; z_bc_type = g->z_bc_type;
        bc_face_ylo = g->bc_face_ylo; bc_face_yhi = g->bc_face_yhi;
        prm = *p;
        nxm = nx - 1; nym = ny - 1; nzm = nz - 1;
        nxg = nxm + 2; nyg = nym + 2; nzg = nzm + 2;
        x.assign(nx + 1, 0.0); y.assign(ny + 1, 0.0); z.assign(nz + 1, 0.0);
        for (int i = 1; i <= nx; ++i) x[i] = g->x[i - 1];
        for (int j = 1; j <= ny; ++j) y[j] = g->y[j - 1];
        for (int k = 1; k <= nz; ++k) z[k] = g->z[k - 1];
        auto centres = [](const std::vector<double> &f, int n, std::vector<double> &c) {
            int nm = n - 1;
            std::vector<double> m(nm + 1);
            for (int i = 1; i <= nm; ++i) m[i] = 0.5 * (f[i] + f[i + 1]);
            c.assign(nm + 3, 0.0);
            for (int i = 1; i <= nm; ++i) c[i + 1] = m[i];
            c[1] = m[1] - 2.0 * (m[1] - f[1]);
            c[nm + 2] = m[nm] + 2.0 * (f[n] - m[nm]);
        };
        centres(x, nx, xg); centres(y, ny, yg); centres(z, nz, zg);
        double dxmin = 1e300, dzmin = 1e300;
        for (int i = 1; i <= nxg - 1; ++i) dxmin = std::min(dxmin, xg[i + 1] - xg[i]);
        for (int k = 1; k <= nzg - 1; ++k) dzmin = std::min(dzmin, zg[k + 1] - zg[k]);
        Lx = x[nx] - x[1]; Ly = y[ny] - y[1]; Lz = z[nz] - z[1];
        dx = dxmin; dz = dzmin;
        // x periodic: the last interior cell duplicates the first (nxp = nxm - 1); inflow/outflow x (x_bc_type 1,
        // the DCT-IV path): all nxm cells (src/initialization.f90:330-336)
        nxp = x_bc_type == 0 ? nxm - 1 : nxm;
        nzp = z_bc_type == 0 ? nzm - 1 : nzm;   // z periodic; a z wall keeps every point (:338-345)
        int mx = nxp - 1, mz = nzp - 1;
        kxx.assign(mx + 1, 0.0); kzz.assign(mz + 1, 0.0);
        int cx = (int)std::ceil((double)nxp / 2.0), cz = (int)std::ceil((double)nzp / 2.0);
        if (x_bc_type == 0) {
            for (int i = 0; i <= cx; ++i)
                kxx[i] = 2.0 * (std::cos(2.0 * pi * (double)i / (double)nxp) - 1.0) / std::pow(dx, 2.0);
            for (int i = cx + 1; i <= mx; ++i)
                kxx[i] = 2.0 * (std::cos(2.0 * pi * (double)(-nxp + i) / (double)nxp) - 1.0) / std::pow(dx, 2.0);
        } else {   // DCT-IV (quarter-wave) modified wavenumber (src/initialization.f90:455-457)
            for (int i = 0; i <= mx; ++i)
                kxx[i] = 2.0 * (std::cos(pi * (double)(2 * i + 1) / (2.0 * (double)nxp)) - 1.0) / std::pow(dx, 2.0);
            dct_cos.assign((size_t)8 * nxp, 0.0);
            for (int m = 0; m < 8 * nxp; ++m) dct_cos[m] = std::cos(pi * (double)m / (4.0 * (double)nxp));
        }
        if (z_bc_type == 0) {
            for (int k = 0; k <= cz; ++k)
                kzz[k] = 2.0 * (std::cos(2.0 * pi * (double)k / (double)nzp) - 1.0) / std::pow(dz, 2.0);
            for (int k = cz + 1; k <= mz; ++k)
                kzz[k] = 2.0 * (std::cos(2.0 * pi * (double)(-nzp + k) / (double)nzp) - 1.0) / std::pow(dz, 2.0);
        } else {
            setup_duct();
        }
        if (y_bc_type == 0) {
            int nyp = nym - 1;
            kyy.assign(nyp, 0.0);
            double dy = y[2] - y[1];
            int cy = (int)std::ceil((double)nyp / 2.0);
            for (int j = 0; j <= cy && j < nyp; ++j)
                kyy[j] = 2.0 * (std::cos(2.0 * pi * (double)j / (double)nyp) - 1.0) / std::pow(dy, 2.0);
            for (int j = cy + 1; j <= nyp - 1; ++j)
                kyy[j] = 2.0 * (std::cos(2.0 * pi * (double)(-nyp + j) / (double)nyp) - 1.0) / std::pow(dy, 2.0);
            fy.init(nyp);
        }
        // Dyy (src/initialization.f90:507-535)
        Dyy_d.assign(nyg + 1, 0.0); Dyy_l.assign(nyg + 1, 0.0); Dyy_u.assign(nyg + 1, 0.0);
        for (int j = 3; j <= nyg - 2; ++j) {
            double a = 1.0 / (y[j] - y[j - 1]) / (yg[j + 1] - yg[j]);
            double b = 1.0 / (y[j] - y[j - 1]) * (-1.0 / (yg[j + 1] - yg[j]) - 1.0 / (yg[j] - yg[j - 1]));
            double c = 1.0 / (y[j] - y[j - 1]) / (yg[j] - yg[j - 1]);
            Dyy_u[j] = a; Dyy_l[j] = c; Dyy_d[j] = b;
        }
        {
            int j = 2;
            double a = 1.0 / (y[j] - y[j - 1]) / (yg[j + 1] - yg[j]);
            double b = 1.0 / (y[j] - y[j - 1]) * (-1.0 / (yg[j + 1] - yg[j]) - 1.0 / (yg[j] - yg[j - 1]));
            double c = 1.0 / (y[j] - y[j - 1]) / (yg[j] - yg[j - 1]);
            Dyy_d[2] = b + c; Dyy_u[2] = a;
            j = nyg - 1;
            a = 1.0 / (y[j] - y[j - 1]) / (yg[j + 1] - yg[j]);
            b = 1.0 / (y[j] - y[j - 1]) * (-1.0 / (yg[j + 1] - yg[j]) - 1.0 / (yg[j] - yg[j - 1]));
            c = 1.0 / (y[j] - y[j - 1]) / (yg[j] - yg[j - 1]);
            Dyy_d[nyg - 1] = a + b; Dyy_l[nyg - 1] = c;
        }
        // weights (src/initialization.f90:633-644)
        wy0.assign(ny + 1, 0.0); wy1.assign(ny + 1, 0.0); wz0.assign(nz + 1, 0.0); wz1.assign(nz + 1, 0.0);
        for (int j = 1; j <= ny; ++j) { wy0[j] = (yg[j + 1] - y[j]) / (yg[j + 1] - yg[j]); wy1[j] = 1.0 - wy0[j]; }
        for (int k = 1; k <= nz; ++k) wz0[k] = 0.5;
        for (int k = 1; k <= std::min(nz, nzg - 1); ++k) wz0[k] = (zg[k + 1] - z[k]) / (zg[k + 1] - zg[k]);
        for (int k = 1; k <= nz; ++k) wz1[k] = 1.0 - wz0[k];
        // RK3 (src/initialization.f90:650-660)
        std::memset(rk_coef, 0, sizeof(rk_coef));
        rk_t[1] = 8.0 / 15.0; rk_t[2] = 2.0 / 3.0; rk_t[3] = 1.0;
        rk_coef[1][1] = 8.0 / 15.0; rk_coef[2][1] = 1.0 / 4.0; rk_coef[2][2] = 5.0 / 12.0;
        rk_coef[3][1] = 1.0 / 4.0; rk_coef[3][2] = 0.0; rk_coef[3][3] = 3.0 / 4.0;
        // automatic defaults (src/input_output.f90:938-940, :967-970)
        nwl = prm.adv_wall_layers;
        if (nwl < 0) { nwl = 0; if (prm.flat_wall_model_flag > 0 && prm.advection_scheme != 1) nwl = 8; }
        wm_filter_mode = prm.wm_filter_mode;
        if (wm_filter_mode < 0) { wm_filter_mode = 0; if (prm.flat_wall_model_flag > 0 && z_bc_type == 0) wm_filter_mode = 1; }
        dPdx = prm.dPdx; dPdz = prm.dPdz;
        t = 0.0;
        // arrays (src/initialization.f90:204-219, :662-678, :723-742)
        U.init(1, nx, 1, nyg, 1, nzg); V.init(1, nxg, 1, ny, 1, nzg); W.init(1, nxg, 1, nyg, 1, nz);
        P.init(1, nxg, 1, nyg, 1, nzg); nu_t.init(1, nxg, 1, nyg, 1, nzg);
        Uo.init(1, nx, 1, nyg, 1, nzg); Vo.init(1, nxg, 1, ny, 1, nzg); Wo.init(1, nxg, 1, nyg, 1, nz);
        term_1.init(1, nxg, 1, nyg, 1, nzg); term_2.init(1, nxg, 1, nyg, 1, nzg);
        rhs_p.init(2, nxg, 2, nyg - 1, 2, nzg);
        for (int s = 1; s <= 3; ++s) {
            Fu[s].init(2, nx - 1, 2, nyg - 1, 2, nzg - 1);
            Fv[s].init(2, nxg - 1, 2, ny - 1, 2, nzg - 1);
            Fw[s].init(2, nxg - 1, 2, nyg - 1, 2, nz - 1);
        }
        tau_x.init(1, nx, 1, 2, 1, nzg); tau_z.init(1, nxg, 1, 2, 1, nz);
        wmf_ux.init(1, nx, 1, 2, 1, nzg); wmf_wx.init(1, nx, 1, 2, 1, nzg); wmf_tx.init(1, nx, 1, 2, 1, nzg);
        wmf_uz.init(1, nxg, 1, 2, 1, nz); wmf_wz.init(1, nxg, 1, 2, 1, nz); wmf_tz.init(1, nxg, 1, 2, 1, nz);
        if (x_bc_type == 0) fx.init(nxp);
        if (z_bc_type == 0) fz.init(nzp);
        return 0;
    }

    // Dzz with z walls (src/initialization.f90:543-572, the construction of Dyy on the z grid) and the duct's
    // eigenbasis (:579-618): S = W^(1/2) Dzz W^(-1/2), W = diag of the interior cell widths, is symmetric
    // tridiagonal with S's diagonal = Dzz's and S(k,k+1) = 1 / ((zg(k+2) - zg(k+1)) sqrt(w(k) w(k+1))).  The
    // reference diagonalises it with LAPACK dstev, which runs the implicit QL/QR iteration on the tridiagonal matrix
    // (dsteqr); this restates that method (implicit QL with Wilkinson shifts, Bowdler, Martin, Reinsch and Wilkinson,
    // Numer. Math. 11, 1968) and sorts the pairs ascending as dstev returns them.  A dense cyclic Jacobi iteration was
    // tried first: its rounding grows with the number of rotations (2e-13 relative in the eigenvalues at 511 cells).
    // Eigenvector signs may differ from dstev's; the solve does not depend on them.
    void setup_duct() {
        Dzz_d.assign(nzg + 1, 0.0); Dzz_l.assign(nzg + 1, 0.0); Dzz_u.assign(nzg + 1, 0.0);
        auto abc = [&](int k, double &a, double &b, double &c) {
            a = 1.0 / (z[k] - z[k - 1]) / (zg[k + 1] - zg[k]);
            b = 1.0 / (z[k] - z[k - 1]) * (-1.0 / (zg[k + 1] - zg[k]) - 1.0 / (zg[k] - zg[k - 1]));
            c = 1.0 / (z[k] - z[k - 1]) / (zg[k] - zg[k - 1]);
        };
        for (int k = 3; k <= nzg - 2; ++k) { double a, b, c; abc(k, a, b, c); Dzz_u[k] = a; Dzz_l[k] = c; Dzz_d[k] = b; }
        { double a, b, c; abc(2, a, b, c); Dzz_d[2] = b + c; Dzz_u[2] = a; }
        { double a, b, c; abc(nzg - 1, a, b, c); Dzz_d[nzg - 1] = a + b; Dzz_l[nzg - 1] = c; }
        const int n = nzm;
        std::vector<double> w(n);
        sqrt_w_z.assign(n, 0.0);
        for (int k = 0; k < n; ++k) { w[k] = z[k + 2] - z[k + 1]; sqrt_w_z[k] = std::sqrt(w[k]); }
        // diag dg[k], off-diagonal sub[k] between k and k+1 (sub[n-1] = 0); V accumulates the rotations
        std::vector<double> dg(n), sub(n, 0.0), V((size_t)n * n, 0.0);
        for (int k = 0; k < n; ++k) { dg[k] = Dzz_d[k + 2]; V[(size_t)k * n + k] = 1.0; }
        for (int k = 0; k + 1 < n; ++k) sub[k] = 1.0 / ((zg[k + 3] - zg[k + 2]) * std::sqrt(w[k] * w[k + 1]));
        const double eps = std::numeric_limits<double>::epsilon();
        for (int l = 0; l < n; ++l) {
            int iter = 0;
            while (true) {
                int m = l;
                while (m < n - 1 && std::fabs(sub[m]) > eps * (std::fabs(dg[m]) + std::fabs(dg[m + 1]))) ++m;
                if (m == l) break;
                if (++iter > 100) { std::fprintf(stderr, "oracle: the duct's z operator did not converge\n"); std::abort(); }
                const double g0 = (dg[l + 1] - dg[l]) / (2.0 * sub[l]);
                const double r0 = std::sqrt(g0 * g0 + 1.0);
                double g = dg[m] - dg[l] + sub[l] / (g0 + std::copysign(r0, g0));
                double s = 1.0, c = 1.0, p = 0.0;
                int i = m - 1;
                for (; i >= l; --i) {
                    const double f = s * sub[i], b = c * sub[i];
                    const double r = std::sqrt(f * f + g * g);
                    sub[i + 1] = r;
                    if (r == 0.0) { dg[i + 1] -= p; sub[m] = 0.0; break; }
                    s = f / r; c = g / r;
                    const double gg = dg[i + 1] - p;
                    const double rr = (dg[i] - gg) * s + 2.0 * c * b;
                    p = s * rr;
                    dg[i + 1] = gg + p;
                    g = c * rr - b;
                    for (int k = 0; k < n; ++k) {
                        const double vk1 = V[(size_t)k * n + i + 1], vk = V[(size_t)k * n + i];
                        V[(size_t)k * n + i + 1] = s * vk + c * vk1;
                        V[(size_t)k * n + i] = c * vk - s * vk1;
                    }
                }
                if (i >= l) continue;   // split at a vanished rotation: iterate on the smaller block
                dg[l] -= p; sub[l] = g; sub[m] = 0.0;
            }
        }
        std::vector<int> order(n);
        for (int m = 0; m < n; ++m) order[m] = m;
        std::sort(order.begin(), order.end(), [&](int i, int j) { return dg[i] < dg[j]; });
        lambda_z.assign(n, 0.0); Qz.assign((size_t)n * n, 0.0);
        for (int m = 0; m < n; ++m) {
            lambda_z[m] = dg[order[m]];
            for (int k = 0; k < n; ++k) Qz[(size_t)k * n + m] = V[(size_t)k * n + order[m]];
        }
    }

    // DCT-IV of one x line, unnormalised (FFTW REDFT11, which the reference's CPU build plans; its GPU build forms the
    // same coefficients through a zero-padded 4N-point FFT, src/poisson_gpu.f90:139-180):
    //   Y_k = 2 sum_n x_n cos(pi (2n+1)(2k+1) / (4N)),  k = 0..N-1.
    // Computed by the definition with the cosines tabulated at the exact multiples m = (2n+1)(2k+1) mod 8N of pi/(4N).
    // It is its own inverse up to 2N.
    std::vector<double> dct_cos;   // cos(pi m / (4 nxp)), m = 0..8 nxp - 1
    void dct4(const double *in, double *out) const {
        const long N = nxp, P = 8 * N;
        for (long k = 0; k < N; ++k) {
            double acc = 0.0;
            for (long n = 0; n < N; ++n) acc += in[n] * dct_cos[(size_t)(((2 * n + 1) * (2 * k + 1)) % P)];
            out[k] = 2.0 * acc;
        }
    }

    // ---- boundary conditions (src/boundary_conditions.f90:186-260, one rank) ----
    void periodic_x(A3 &F, int id) {   // :263-342, self-paired rank
        for (int k = F.l3; k <= F.u3; ++k)
            for (int j = F.l2; j <= F.u2; ++j) {
                if (id == 1) { F(1, j, k) = F(nx - 1, j, k); }
                else { F(1, j, k) = F(nxg - 2, j, k); }
            }
        for (int k = F.l3; k <= F.u3; ++k)
            for (int j = F.l2; j <= F.u2; ++j) {
                if (id == 1) { F(nx, j, k) = F(2, j, k); }
                else { F(nxg - 1, j, k) = F(2, j, k); }
            }
        if (id != 1)
            for (int k = F.l3; k <= F.u3; ++k)
                for (int j = F.l2; j <= F.u2; ++j) F(nxg, j, k) = F(3, j, k);
    }
    void periodic_z(A3 &F, int id) {   // :580-601
        for (int j = F.l2; j <= F.u2; ++j)
            for (int i = F.l1; i <= F.u1; ++i) {
                if (id == 3) F(i, j, 1) = F(i, j, nz - 1); else F(i, j, 1) = F(i, j, nzg - 2);
            }
        for (int j = F.l2; j <= F.u2; ++j)
            for (int i = F.l1; i <= F.u1; ++i) {
                if (id == 3) F(i, j, nz) = F(i, j, 2); else F(i, j, nzg - 1) = F(i, j, 2);
            }
        if (id != 3)
            for (int j = F.l2; j <= F.u2; ++j)
                for (int i = F.l1; i <= F.u1; ++i) F(i, j, nzg) = F(i, j, 3);
    }
    void periodic_y(A3 &F, int id) {   // :762-781
        for (int k = F.l3; k <= F.u3; ++k)
            for (int i = F.l1; i <= F.u1; ++i) {
                if (id == 1) { F(i, 1, k) = F(i, ny - 1, k); }
                else { F(i, 1, k) = F(i, nyg - 2, k); }
            }
        for (int k = F.l3; k <= F.u3; ++k)
            for (int i = F.l1; i <= F.u1; ++i) {
                if (id == 1) F(i, ny, k) = F(i, 2, k); else F(i, nyg - 1, k) = F(i, 2, k);
            }
        if (id != 1)
            for (int k = F.l3; k <= F.u3; ++k)
                for (int i = F.l1; i <= F.u1; ++i) F(i, nyg, k) = F(i, 3, k);
    }
    // apply_Robin_bc_y with alpha = 0 (no-slip mirror; compute_constant_alpha and compute_flat_wall_eqwm both
    // set alpha = 0 on a no-slip wall, src/wallmodel.f90:483,504,726-741)
    void robin_y(A3 &F, int id) {     // :784-804
        const double alpha = 0.0;
        for (int k = F.l3; k <= F.u3; ++k)
            for (int i = F.l1; i <= F.u1; ++i) {
                if (id == 1) {
                    F(i, 1, k) = alpha * F(i, 2, k) / (y[2] - y[1]) / (alpha / (y[2] - y[1]) + 1.0);
                } else {
                    F(i, 1, k) = (2.0 * alpha / (yg[2] - yg[1]) - 1.0) * F(i, 2, k) / (2.0 * alpha / (yg[2] - yg[1]) + 1.0);
                }
            }
        for (int k = F.l3; k <= F.u3; ++k)
            for (int i = F.l1; i <= F.u1; ++i) {
                if (id == 1) {
                    F(i, ny, k) = alpha * F(i, ny - 1, k) / (y[ny] - y[ny - 1]) / (alpha / (y[ny] - y[ny - 1]) + 1.0);
                } else {
                    F(i, nyg, k) = (2.0 * alpha / (yg[nyg] - yg[nyg - 1]) - 1.0) * F(i, nyg - 1, k) /
                                   (2.0 * alpha / (yg[nyg] - yg[nyg - 1]) + 1.0);
                }
            }
    }
    void apply_boundary_conditions() {
        // exchange_velocity_halos: no-op at one rank
        periodic_x(U, 1); periodic_x(V, 2); periodic_x(W, 2);
        periodic_z(U, 1); periodic_z(V, 2); periodic_z(W, 3);
        if (y_bc_type == 0) { periodic_y(U, 2); periodic_y(V, 1); periodic_y(W, 2); }
        else { robin_y(U, 2); robin_y(V, 1); robin_y(W, 2); }
        periodic_x(U, 1); periodic_x(V, 2); periodic_x(W, 2);
        periodic_z(U, 1); periodic_z(V, 2); periodic_z(W, 3);
    }

    // ---- interpolation (src/interpolation.f90) writing into term arrays with the reference's sections ----
    // x, faces<->centres, uniform: ui(1:n1-1) = 0.5*(u(1:n1-1)+u(2:n1))
    void interp_x(const A3 &u, A3 &ui) {
        for (int k = u.l3; k <= u.u3; ++k)
            for (int j = u.l2; j <= u.u2; ++j)
                for (int i = 1; i <= u.u1 - 1; ++i) ui(i, j, k) = 0.5 * (u(i, j, k) + u(i + 1, j, k));
    }
    void interp_y(const A3 &u, A3 &ui, int di) {
        int n2 = u.u2;
        for (int k = u.l3; k <= u.u3; ++k)
            for (int j = 1; j <= n2 - 1; ++j)
                for (int i = u.l1; i <= u.u1; ++i) {
                    if (di == 1) ui(i, j, k) = 0.5 * (u(i, j, k) + u(i, j + 1, k));
                    else ui(i, j, k) = wy0[j] * u(i, j, k) + wy1[j] * u(i, j + 1, k);
                }
    }
    void interp_z(const A3 &u, A3 &ui, int di) {
        int n3 = u.u3;
        for (int k = 1; k <= n3 - 1; ++k)
            for (int j = u.l2; j <= u.u2; ++j)
                for (int i = u.l1; i <= u.u1; ++i) {
                    if (di == 2) ui(i, j, k) = wz0[k] * u(i, j, k) + wz1[k] * u(i, j, k + 1);
                    else ui(i, j, k) = 0.5 * (u(i, j, k) + u(i, j, k + 1));
                }
    }

    bool wall_lo() const { return y_bc_type == 1 && bc_face_ylo == 1; }
    bool wall_hi() const { return y_bc_type == 1 && bc_face_yhi == 1; }

    // ---- compute_rhs_u (src/equations.f90:25-257) ----
    // ---- advection_scheme = 2: upwind-biased dissipation (src/adv_hybrid.f90), beta = adv_beta0 (no solid) ----
    // adv_wsel (:88-103): stencil weights of the dissipative flux for s(-2:3)
    static void adv_wsel(int o, double w[6]) {
        static const double w5[6] = {1.0, -5.0, 10.0, -10.0, 5.0, -1.0}, w3[6] = {0.0, -1.0, 3.0, -3.0, 1.0, 0.0};
        for (int q = 0; q < 6; ++q) w[q] = (o == 5) ? w5[q] / 60.0 : (o == 3) ? w3[q] / 12.0 : 0.0;
    }
    // adv_dflux (:106-117)
    static double adv_dflux(double a, double b, double c, double d, double e, double f, double uc, double beta,
                            const double w[6]) {
        return beta * std::fabs(uc) * (w[0] * a + w[1] * b + w[2] * c + w[3] * d + w[4] * e + w[5] * f);
    }
    // adv_ord_y (:120-133): order usable for the face between rows m and m+1 of 1..n
    static int adv_ord_y(int m, int n, int ord) {
        if (ord == 5 && m - 2 >= 1 && m + 3 <= n) return 5;
        if (m - 1 >= 1 && m + 2 <= n) return 3;
        return 0;
    }
    // the padded copies of pad_field_dev (src/halo_pad.f90:185-240) on one rank: x and z extended periodically
    double pad(const A3 &F, int i, int j, int k) const {
        const int Nc = nx - 2, Nzc = nz - 2;
        const int iw = 2 + (((i - 2) % Nc) + Nc) % Nc, kw = 2 + (((k - 2) % Nzc) + Nzc) % Nzc;
        return F(iw, j, kw);
    }
    // adv_add_u / adv_add_v / adv_add_w (:136-282): rhs += -d/dx_j of the dissipative fluxes.  `comp` 0 u, 1 v, 2 w.
    void adv_add(int comp, A3 &rhs) {
        const int n = prm.adv_order;
        double wx[6];
        adv_wsel(n, wx);
        const double inv_dx = 1.0 / dx, bt = prm.adv_beta0;
        const A3 &F = comp == 0 ? U : comp == 1 ? V : W;
        const int ihi = comp == 0 ? nx - 1 : nxg - 1, jhi = comp == 1 ? ny - 1 : nyg - 1, khi = comp == 2 ? nz - 1 : nzg - 1;
        const int ny_f = comp == 1 ? ny : nyg;   // rows of the advected field
#pragma omp parallel for
        for (int k = 2; k <= khi; ++k)
            for (int j = 2; j <= jhi; ++j)
                for (int i = 2; i <= ihi; ++i) {
                    double dyj, dzk;
                    if (comp == 1) dyj = 1.0 / (yg[j + 1] - yg[j]); else dyj = 1.0 / (y[j] - y[j - 1]);
                    if (comp == 2) dzk = 1.0 / (zg[k + 1] - zg[k]); else dzk = 1.0 / (z[k] - z[k - 1]);
                    double r = 0.0, wy[6];   // per thread: the y order changes near the ends
                    for (int m = 0; m <= 1; ++m) {
                        const double sg = 2.0 * m - 1.0;
                        const int ii = i - 1 + m, jj = j - 1 + m, kk = k - 1 + m;
                        // the convecting velocity at the face, at the advected field's position
                        double ucx, ucy, ucz;
                        if (comp == 0) {
                            ucx = 0.5 * (pad(U, ii, j, k) + pad(U, ii + 1, j, k));
                            ucy = 0.5 * (pad(V, i, jj, k) + pad(V, i + 1, jj, k));
                            ucz = 0.5 * (pad(W, i, j, kk) + pad(W, i + 1, j, kk));
                        } else if (comp == 1) {
                            ucx = 0.5 * (pad(U, ii, j, k) + pad(U, ii, j + 1, k));
                            ucy = 0.5 * (pad(V, i, jj, k) + pad(V, i, jj + 1, k));
                            ucz = 0.5 * (pad(W, i, j, kk) + pad(W, i, j + 1, kk));
                        } else {
                            ucx = 0.5 * (pad(U, ii, j, k) + pad(U, ii, j, k + 1));
                            ucy = 0.5 * (pad(V, i, jj, k) + pad(V, i, jj, k + 1));
                            ucz = 0.5 * (pad(W, i, j, kk) + pad(W, i, j, kk + 1));
                        }
                        r = r - sg * adv_dflux(pad(F, ii - 2, j, k), pad(F, ii - 1, j, k), pad(F, ii, j, k), pad(F, ii + 1, j, k),
                                               pad(F, ii + 2, j, k), pad(F, ii + 3, j, k), ucx, bt, wx) * inv_dx;
                        adv_wsel(adv_ord_y(jj, ny_f, n), wy);
                        r = r - sg * adv_dflux(pad(F, i, std::max(jj - 2, 1), k), pad(F, i, std::max(jj - 1, 1), k), pad(F, i, jj, k),
                                               pad(F, i, jj + 1, k), pad(F, i, std::min(jj + 2, ny_f), k),
                                               pad(F, i, std::min(jj + 3, ny_f), k), ucy, bt, wy) * dyj;
                        r = r - sg * adv_dflux(pad(F, i, j, kk - 2), pad(F, i, j, kk - 1), pad(F, i, j, kk), pad(F, i, j, kk + 1),
                                               pad(F, i, j, kk + 2), pad(F, i, j, kk + 3), ucz, bt, wx) * dzk;
                    }
                    rhs(i, j, k) = rhs(i, j, k) + r;
                }
    }

    void compute_rhs_u(A3 &rhs_u) {
        bool wlo = wall_lo(), whi = wall_hi();
        bool wm_lo = wlo && prm.flat_wall_model_flag > 0, wm_hi = whi && prm.flat_wall_model_flag > 0;
        double inv_dx = 1.0 / dx, inv_dx2 = inv_dx * inv_dx;
        double w_adv = (prm.advection_scheme == 1) ? 0.0 : 0.5;
        auto blend = [&](int j, double &wa, double &wd) {
            bool wcell = (wm_lo && j <= 1 + nwl) || (wm_hi && j >= nyg - nwl);
            wa = wcell ? 0.0 : w_adv; wd = 1.0 - wa;
        };
        interp_x(U, term_1);
#pragma omp parallel for
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j) {
                double wa, wd; blend(j, wa, wd);
                for (int i = 2; i <= nx - 1; ++i)
                    rhs_u(i, j, k) = -(wd * (term_1(i, j, k) * term_1(i, j, k) - term_1(i - 1, j, k) * term_1(i - 1, j, k)) +
                                       wa * U(i, j, k) * (term_1(i, j, k) - term_1(i - 1, j, k))) * inv_dx;
            }
        interp_y(U, term_1, 2);   // term_1(1:nx,:,:)
        interp_x(V, term_2);      // term_2(:,1:ny,:)
#pragma omp parallel for
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j) {
                double wa, wd; blend(j, wa, wd);
                for (int i = 2; i <= nx - 1; ++i)
                    rhs_u(i, j, k) = rhs_u(i, j, k) - (wd * (term_1(i, j, k) * term_2(i, j, k) - term_1(i, j - 1, k) * term_2(i, j - 1, k)) +
                                                       wa * 0.5 * (term_2(i, j - 1, k) + term_2(i, j, k)) * (term_1(i, j, k) - term_1(i, j - 1, k))) /
                                                          (y[j] - y[j - 1]);
            }
        interp_z(U, term_1, 2);
        interp_x(W, term_2);
#pragma omp parallel for
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j) {
                double wa, wd; blend(j, wa, wd);
                for (int i = 2; i <= nx - 1; ++i)
                    rhs_u(i, j, k) = rhs_u(i, j, k) - (wd * (term_1(i, j, k) * term_2(i, j, k) - term_1(i, j, k - 1) * term_2(i, j, k - 1)) +
                                                       wa * 0.5 * (term_2(i, j, k - 1) + term_2(i, j, k)) * (term_1(i, j, k) - term_1(i, j, k - 1))) /
                                                          (z[k] - z[k - 1]);
            }
        if (prm.advection_scheme == 2) adv_add(0, rhs_u);   // src/equations.f90:149
        // viscous terms
#pragma omp parallel for
        for (int k = 1; k <= nzg; ++k)
            for (int j = 1; j <= nyg - 1; ++j)
                for (int i = 1; i <= nx; ++i) term_1(i, j, k) = (U(i, j + 1, k) - U(i, j, k)) / (yg[j + 1] - yg[j]);
#pragma omp parallel for
        for (int k = 1; k <= nzg - 1; ++k)
            for (int j = 1; j <= nyg; ++j)
                for (int i = 1; i <= nx; ++i) term_2(i, j, k) = (U(i, j, k + 1) - U(i, j, k)) / (zg[k + 1] - zg[k]);
#pragma omp parallel for
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j) {
                double dz_3 = z[k] - z[k - 1], inv_dz3 = 1.0 / dz_3;
                double dy_3 = y[j] - y[j - 1], inv_dy3 = 1.0 / dy_3;
                for (int i = 2; i <= nx - 1; ++i) {
                    double nu = prm.nu;
                    double nu_x1 = nu + nu_t(i, j, k);
                    double nu_x2 = nu + nu_t(i + 1, j, k);
                    double nu_y1, nu_y2;
                    if (wlo && j - 1 == 1) nu_y1 = nu;
                    else nu_y1 = nu + 0.5 * (wy0[j - 1] * nu_t(i, j - 1, k) + wy1[j - 1] * nu_t(i, j, k) +
                                             wy0[j - 1] * nu_t(i + 1, j - 1, k) + wy1[j - 1] * nu_t(i + 1, j, k));
                    if (whi && j + 1 == nyg) nu_y2 = nu;
                    else nu_y2 = nu + 0.5 * (wy0[j] * nu_t(i, j, k) + wy1[j] * nu_t(i, j + 1, k) +
                                             wy0[j] * nu_t(i + 1, j, k) + wy1[j] * nu_t(i + 1, j + 1, k));
                    double nu_z1 = nu + 0.5 * (wz0[k - 1] * (nu_t(i, j, k - 1) + nu_t(i + 1, j, k - 1)) +
                                               wz1[k - 1] * (nu_t(i, j, k) + nu_t(i + 1, j, k)));
                    double nu_z2 = nu + 0.5 * (wz0[k] * (nu_t(i, j, k) + nu_t(i + 1, j, k)) +
                                               wz1[k] * (nu_t(i, j, k + 1) + nu_t(i + 1, j, k + 1)));
                    double fy2 = nu_y2 * (term_1(i, j, k) + (V(i + 1, j, k) - V(i, j, k)) * inv_dx);
                    double fy1 = nu_y1 * (term_1(i, j - 1, k) + (V(i + 1, j - 1, k) - V(i, j - 1, k)) * inv_dx);
                    if (prm.flat_wall_model_flag > 0) {
                        if (wlo && j == 2) fy1 = tau_x(i, 1, k);
                        if (whi && j == nyg - 1) fy2 = tau_x(i, 2, k);
                    }
                    double fz2 = nu_z2 * (term_2(i, j, k) + (W(i + 1, j, k) - W(i, j, k)) * inv_dx);
                    double fz1 = nu_z1 * (term_2(i, j, k - 1) + (W(i + 1, j, k - 1) - W(i, j, k - 1)) * inv_dx);
                    rhs_u(i, j, k) = rhs_u(i, j, k) +
                                     2.0 * inv_dx2 * (nu_x2 * (U(i + 1, j, k) - U(i, j, k)) - nu_x1 * (U(i, j, k) - U(i - 1, j, k))) +
                                     inv_dy3 * (fy2 - fy1) + inv_dz3 * (fz2 - fz1) + dPdx;
                }
            }
    }

    // ---- compute_rhs_v (src/equations.f90:261-485) ----
    void compute_rhs_v(A3 &rhs_v) {
        double inv_dx = 1.0 / dx;
        double w_adv = (prm.advection_scheme == 1) ? 0.0 : 0.5;
        double wa = w_adv, wd = 1.0 - wa;   // wcell is set only by z walls, absent on this path
        interp_y(V, term_1, 1);
#pragma omp parallel for
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= ny - 1; ++j)
                for (int i = 2; i <= nxg - 1; ++i)
                    rhs_v(i, j, k) = -(wd * (term_1(i, j, k) * term_1(i, j, k) - term_1(i, j - 1, k) * term_1(i, j - 1, k)) +
                                       wa * V(i, j, k) * (term_1(i, j, k) - term_1(i, j - 1, k))) / (yg[j + 1] - yg[j]);
        interp_y(U, term_1, 2);
        interp_x(V, term_2);
#pragma omp parallel for
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= ny - 1; ++j)
                for (int i = 2; i <= nxg - 1; ++i)
                    rhs_v(i, j, k) = rhs_v(i, j, k) - (wd * (term_1(i, j, k) * term_2(i, j, k) - term_1(i - 1, j, k) * term_2(i - 1, j, k)) +
                                                       wa * 0.5 * (term_1(i - 1, j, k) + term_1(i, j, k)) * (term_2(i, j, k) - term_2(i - 1, j, k))) * inv_dx;
        interp_z(V, term_1, 2);
        interp_y(W, term_2, 2);
#pragma omp parallel for
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= ny - 1; ++j)
                for (int i = 2; i <= nxg - 1; ++i)
                    rhs_v(i, j, k) = rhs_v(i, j, k) - (wd * (term_1(i, j, k) * term_2(i, j, k) - term_1(i, j, k - 1) * term_2(i, j, k - 1)) +
                                                       wa * 0.5 * (term_2(i, j, k - 1) + term_2(i, j, k)) * (term_1(i, j, k) - term_1(i, j, k - 1))) /
                                                          (z[k] - z[k - 1]);
        if (prm.advection_scheme == 2) adv_add(1, rhs_v);   // src/equations.f90:373
#pragma omp parallel for
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= ny - 1; ++j) {
                double dz_3 = z[k] - z[k - 1], inv_dz3 = 1.0 / dz_3;
                double inv_dzg1 = 1.0 / (zg[k] - zg[k - 1]), inv_dzg2 = 1.0 / (zg[k + 1] - zg[k]);
                double dy_1 = y[j] - y[j - 1], dy_2 = y[j + 1] - y[j], dy_3 = yg[j + 1] - yg[j];
                double inv_dy1 = 1.0 / dy_1, inv_dy2 = 1.0 / dy_2, inv_dy3 = 1.0 / dy_3, two_inv_dy3 = 2.0 * inv_dy3;
                for (int i = 2; i <= nxg - 1; ++i) {
                    double nu = prm.nu;
                    double nu_x1 = nu + 0.5 * (wy0[j] * nu_t(i - 1, j, k) + wy1[j] * nu_t(i - 1, j + 1, k) +
                                               wy0[j] * nu_t(i, j, k) + wy1[j] * nu_t(i, j + 1, k));
                    double nu_x2 = nu + 0.5 * (wy0[j] * nu_t(i, j, k) + wy1[j] * nu_t(i, j + 1, k) +
                                               wy0[j] * nu_t(i + 1, j, k) + wy1[j] * nu_t(i + 1, j + 1, k));
                    double nu_y1 = nu + nu_t(i, j, k);
                    double nu_y2 = nu + nu_t(i, j + 1, k);
                    double nu_z1 = nu + wz0[k - 1] * (wy0[j] * nu_t(i, j, k - 1) + wy1[j] * nu_t(i, j + 1, k - 1)) +
                                   wz1[k - 1] * (wy0[j] * nu_t(i, j, k) + wy1[j] * nu_t(i, j + 1, k));
                    double nu_z2 = nu + wz0[k] * (wy0[j] * nu_t(i, j, k) + wy1[j] * nu_t(i, j + 1, k)) +
                                   wz1[k] * (wy0[j] * nu_t(i, j, k + 1) + wy1[j] * nu_t(i, j + 1, k + 1));
                    double fx2 = nu_x2 * ((V(i + 1, j, k) - V(i, j, k)) * inv_dx + (U(i, j + 1, k) - U(i, j, k)) * inv_dy3);
                    double fx1 = nu_x1 * ((V(i, j, k) - V(i - 1, j, k)) * inv_dx + (U(i - 1, j + 1, k) - U(i - 1, j, k)) * inv_dy3);
                    double fz2 = nu_z2 * ((V(i, j, k + 1) - V(i, j, k)) * inv_dzg2 + (W(i, j + 1, k) - W(i, j, k)) * inv_dy3);
                    double fz1 = nu_z1 * ((V(i, j, k) - V(i, j, k - 1)) * inv_dzg1 + (W(i, j + 1, k - 1) - W(i, j, k - 1)) * inv_dy3);
                    rhs_v(i, j, k) = rhs_v(i, j, k) + inv_dx * (fx2 - fx1) +
                                     two_inv_dy3 * (nu_y2 * (V(i, j + 1, k) - V(i, j, k)) * inv_dy2 - nu_y1 * (V(i, j, k) - V(i, j - 1, k)) * inv_dy1) +
                                     inv_dz3 * (fz2 - fz1);
                }
            }
    }

    // ---- compute_rhs_w (src/equations.f90:489-721) ----
    void compute_rhs_w(A3 &rhs_w) {
        bool wlo = wall_lo(), whi = wall_hi();
        bool wm_lo = wlo && prm.flat_wall_model_flag > 0, wm_hi = whi && prm.flat_wall_model_flag > 0;
        double inv_dx = 1.0 / dx;
        double w_adv = (prm.advection_scheme == 1) ? 0.0 : 0.5;
        auto blend = [&](int j, double &wa, double &wd) {
            bool wcell = (wm_lo && j <= 1 + nwl) || (wm_hi && j >= nyg - nwl);
            wa = wcell ? 0.0 : w_adv; wd = 1.0 - wa;
        };
        interp_z(W, term_1, 1);
#pragma omp parallel for
        for (int k = 2; k <= nz - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j) {
                double wa, wd; blend(j, wa, wd);
                for (int i = 2; i <= nxg - 1; ++i)
                    rhs_w(i, j, k) = -(wd * (term_1(i, j, k) * term_1(i, j, k) - term_1(i, j, k - 1) * term_1(i, j, k - 1)) +
                                       wa * W(i, j, k) * (term_1(i, j, k) - term_1(i, j, k - 1))) / (zg[k + 1] - zg[k]);
            }
        interp_z(U, term_1, 2);
        interp_x(W, term_2);
#pragma omp parallel for
        for (int k = 2; k <= nz - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j) {
                double wa, wd; blend(j, wa, wd);
                for (int i = 2; i <= nxg - 1; ++i)
                    rhs_w(i, j, k) = rhs_w(i, j, k) - (wd * (term_1(i, j, k) * term_2(i, j, k) - term_1(i - 1, j, k) * term_2(i - 1, j, k)) +
                                                       wa * 0.5 * (term_1(i - 1, j, k) + term_1(i, j, k)) * (term_2(i, j, k) - term_2(i - 1, j, k))) * inv_dx;
            }
        interp_z(V, term_1, 2);
        interp_y(W, term_2, 2);
#pragma omp parallel for
        for (int k = 2; k <= nz - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j) {
                double wa, wd; blend(j, wa, wd);
                for (int i = 2; i <= nxg - 1; ++i)
                    rhs_w(i, j, k) = rhs_w(i, j, k) - (wd * (term_1(i, j, k) * term_2(i, j, k) - term_1(i, j - 1, k) * term_2(i, j - 1, k)) +
                                                       wa * 0.5 * (term_1(i, j - 1, k) + term_1(i, j, k)) * (term_2(i, j, k) - term_2(i, j - 1, k))) /
                                                          (y[j] - y[j - 1]);
            }
        if (prm.advection_scheme == 2) adv_add(2, rhs_w);   // src/equations.f90:602
#pragma omp parallel for
        for (int k = 1; k <= nz; ++k)
            for (int j = 1; j <= nyg - 1; ++j)
                for (int i = 1; i <= nxg; ++i) term_1(i, j, k) = (W(i, j + 1, k) - W(i, j, k)) / (yg[j + 1] - yg[j]);
#pragma omp parallel for
        for (int k = 2; k <= nz - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j) {
                double dz_1 = z[k] - z[k - 1], dz_2 = z[k + 1] - z[k], dz_3 = zg[k + 1] - zg[k];
                double inv_dz1 = 1.0 / dz_1, inv_dz2 = 1.0 / dz_2, inv_dz3 = 1.0 / dz_3, two_inv_dz3 = 2.0 * inv_dz3;
                double dy_3 = y[j] - y[j - 1], inv_dy3 = 1.0 / dy_3;
                for (int i = 2; i <= nxg - 1; ++i) {
                    double nu = prm.nu;
                    double nu_x1 = nu + 0.5 * (wz0[k] * (nu_t(i, j, k) + nu_t(i - 1, j, k)) +
                                               wz1[k] * (nu_t(i, j, k + 1) + nu_t(i - 1, j, k + 1)));
                    double nu_x2 = nu + 0.5 * (wz0[k] * (nu_t(i, j, k) + nu_t(i + 1, j, k)) +
                                               wz1[k] * (nu_t(i, j, k + 1) + nu_t(i + 1, j, k + 1)));
                    double nu_y1, nu_y2;
                    if (wlo && j - 1 == 1) nu_y1 = nu;
                    else nu_y1 = nu + wz0[k] * (wy0[j - 1] * nu_t(i, j - 1, k) + wy1[j - 1] * nu_t(i, j, k)) +
                                 wz1[k] * (wy0[j - 1] * nu_t(i, j - 1, k + 1) + wy1[j - 1] * nu_t(i, j, k + 1));
                    if (whi && j + 1 == nyg) nu_y2 = nu;
                    else nu_y2 = nu + wz0[k] * (wy0[j] * nu_t(i, j, k) + wy1[j] * nu_t(i, j + 1, k)) +
                                 wz1[k] * (wy0[j] * nu_t(i, j, k + 1) + wy1[j] * nu_t(i, j + 1, k + 1));
                    double nu_z1 = nu + nu_t(i, j, k);
                    double nu_z2 = nu + nu_t(i, j, k + 1);
                    double fy2 = nu_y2 * (term_1(i, j, k) + (V(i, j, k + 1) - V(i, j, k)) * inv_dz3);
                    double fy1 = nu_y1 * (term_1(i, j - 1, k) + (V(i, j - 1, k + 1) - V(i, j - 1, k)) * inv_dz3);
                    if (prm.flat_wall_model_flag > 0) {
                        if (wlo && j == 2) fy1 = tau_z(i, 1, k);
                        if (whi && j == nyg - 1) fy2 = tau_z(i, 2, k);
                    }
                    double fx2 = nu_x2 * ((W(i + 1, j, k) - W(i, j, k)) * inv_dx + (U(i, j, k + 1) - U(i, j, k)) * inv_dz3);
                    double fx1 = nu_x1 * ((W(i, j, k) - W(i - 1, j, k)) * inv_dx + (U(i - 1, j, k + 1) - U(i - 1, j, k)) * inv_dz3);
                    rhs_w(i, j, k) = rhs_w(i, j, k) + inv_dx * (fx2 - fx1) + inv_dy3 * (fy2 - fy1) +
                                     two_inv_dz3 * (nu_z2 * (W(i, j, k + 1) - W(i, j, k)) * inv_dz2 - nu_z1 * (W(i, j, k) - W(i, j, k - 1)) * inv_dz1) +
                                     dPdz;
                }
            }
    }

    // ---- wall model (src/wallmodel.f90) ----
    static constexpr double kappa_wm = 0.41, B_wm = 5.2, REICH_A1 = 11.0, REICH_A2 = 0.33;
    static void reichardt_uplus(double yplus, double &uplus, double &duplus) {
        const double c_buf = B_wm - std::log(kappa_wm) / kappa_wm;
        double a1i = 1.0 / REICH_A1;
        double e1 = std::exp(-yplus * a1i);
        double e2 = std::exp(-REICH_A2 * yplus);
        uplus = std::log(1.0 + kappa_wm * yplus) / kappa_wm + c_buf * (1.0 - e1 - yplus * a1i * e2);
        duplus = 1.0 / (1.0 + kappa_wm * yplus) + c_buf * (a1i * e1 - a1i * e2 + yplus * a1i * REICH_A2 * e2);
    }
    static double solve_u_tau_reichardt(double u_ref, double y_ref, double nu_l) {
        double u_tau = std::max(1e-3 * u_ref, std::sqrt(nu_l * u_ref / std::max(y_ref, 1e-14)));
        for (int iter = 1; iter <= 20; ++iter) {
            double yplus = u_tau * y_ref / nu_l, uplus, duplus;
            reichardt_uplus(yplus, uplus, duplus);
            double f = u_ref / std::max(u_tau, 1e-20) - uplus;
            double fp = -u_ref / std::max(u_tau * u_tau, 1e-20) - duplus * y_ref / nu_l;
            double u_tau_new = u_tau - f / (fp + std::copysign(1e-14, fp));
            u_tau_new = std::min(std::max(u_tau_new, 0.1 * u_tau), 10.0 * u_tau);
            if (std::fabs(u_tau_new - u_tau) < 1e-6 * u_tau_new) { u_tau = u_tau_new; break; }
            u_tau = u_tau_new;
        }
        return u_tau;
    }
    void update_wm_filter() {   // :397-439
        if (wm_filter_mode != 1) return;
        bool seed = !wmf_seeded;
        double kap = kappa_wm;
        for (int iw = 1; iw <= 2; ++iw) {
            int jm = (iw == 1) ? 2 : nyg - 1;
            double ym = std::max((iw == 1) ? yg[jm] : Ly - yg[jm], 1e-14);
            for (int k = 2; k <= nzg - 1; ++k)
                for (int i = 2; i <= nx - 1; ++i) {
                    double eps = 1.0;
                    if (!seed && wmf_tx(i, iw, k) > 0.0) eps = std::min(1.0, dt() * kap * wmf_tx(i, iw, k) / (prm.wm_filter_Tf_fac * ym));
                    wmf_ux(i, iw, k) = (1.0 - eps) * wmf_ux(i, iw, k) + eps * U(i, jm, k);
                    wmf_wx(i, iw, k) = (1.0 - eps) * wmf_wx(i, iw, k) + eps * 0.5 * (W(i, jm, k - 1) + W(i, jm, k));
                }
            for (int k = 2; k <= nz - 1; ++k)
                for (int i = 2; i <= nxg - 1; ++i) {
                    double eps = 1.0;
                    if (!seed && wmf_tz(i, iw, k) > 0.0) eps = std::min(1.0, dt() * kap * wmf_tz(i, iw, k) / (prm.wm_filter_Tf_fac * ym));
                    wmf_uz(i, iw, k) = (1.0 - eps) * wmf_uz(i, iw, k) + eps * 0.5 * (U(i - 1, jm, k) + U(i, jm, k));
                    wmf_wz(i, iw, k) = (1.0 - eps) * wmf_wz(i, iw, k) + eps * W(i, jm, k);
                }
        }
        wmf_seeded = true;
    }
    void compute_wall_model() {   // :197-233 -> compute_flat_wall_eqwm :442-583 (smooth law, no MOST)
        if (y_bc_type != 1 || prm.flat_wall_model_flag != 1) return;   // constant alpha = 0: nothing else to do
        double y_match_lo = std::max(yg[2], 1e-14), y_match_hi = std::max(Ly - yg[nyg - 1], 1e-14);
        int jlo = 2, jhi = nyg - 1;
        for (int k = 2; k <= nzg - 1; ++k)
            for (int i = 2; i <= nx - 1; ++i) {
                for (int iw = 1; iw <= 2; ++iw) {
                    int jw = (iw == 1) ? 2 : nyg - 1, jm = (iw == 1) ? jlo : jhi;
                    double W_at_pt = 0.5 * (W(i, jw, k - 1) + W(i, jw, k));
                    double u_ref = std::sqrt(U(i, jw, k) * U(i, jw, k) + W_at_pt * W_at_pt);
                    double W_match = 0.5 * (W(i, jm, k - 1) + W(i, jm, k));
                    double u_match = std::sqrt(U(i, jm, k) * U(i, jm, k) + W_match * W_match);
                    double num = U(i, jw, k);
                    if (wm_filter_mode == 1) {
                        u_match = std::sqrt(wmf_ux(i, iw, k) * wmf_ux(i, iw, k) + wmf_wx(i, iw, k) * wmf_wx(i, iw, k));
                        num = wmf_ux(i, iw, k); u_ref = u_match;
                    }
                    double u_tau = solve_u_tau_reichardt(u_match, (iw == 1) ? y_match_lo : y_match_hi, prm.nu);
                    wmf_tx(i, iw, k) = u_tau;
                    double tv = u_tau * u_tau * num / std::max(u_ref, 1e-30);
                    tau_x(i, iw, k) = (iw == 1) ? tv : -tv;
                }
            }
        for (int iw = 1; iw <= 2; ++iw) {
            for (int k = 1; k <= nzg; ++k) { tau_x(1, iw, k) = tau_x(2, iw, k); tau_x(nx, iw, k) = tau_x(nx - 1, iw, k); }
            for (int i = 1; i <= nx; ++i) { tau_x(i, iw, 1) = tau_x(i, iw, 2); tau_x(i, iw, nzg) = tau_x(i, iw, nzg - 1); }
        }
        for (int k = 2; k <= nz - 1; ++k)
            for (int i = 2; i <= nxg - 1; ++i) {
                for (int iw = 1; iw <= 2; ++iw) {
                    int jw = (iw == 1) ? 2 : nyg - 1, jm = (iw == 1) ? jlo : jhi;
                    double uc = 0.5 * (U(i - 1, jw, k) + U(i, jw, k));
                    double u_ref = std::sqrt(uc * uc + W(i, jw, k) * W(i, jw, k));
                    double ucm = 0.5 * (U(i - 1, jm, k) + U(i, jm, k));
                    double u_match = std::sqrt(ucm * ucm + W(i, jm, k) * W(i, jm, k));
                    double num = W(i, jw, k);
                    if (wm_filter_mode == 1) {
                        u_match = std::sqrt(wmf_uz(i, iw, k) * wmf_uz(i, iw, k) + wmf_wz(i, iw, k) * wmf_wz(i, iw, k));
                        num = wmf_wz(i, iw, k); u_ref = u_match;
                    }
                    double u_tau = solve_u_tau_reichardt(u_match, (iw == 1) ? y_match_lo : y_match_hi, prm.nu);
                    wmf_tz(i, iw, k) = u_tau;
                    double tv = u_tau * u_tau * num / std::max(u_ref, 1e-30);
                    tau_z(i, iw, k) = (iw == 1) ? tv : -tv;
                }
            }
        for (int iw = 1; iw <= 2; ++iw) {
            for (int k = 1; k <= nz; ++k) { tau_z(1, iw, k) = tau_z(2, iw, k); tau_z(nxg, iw, k) = tau_z(nxg - 1, iw, k); }
            for (int i = 1; i <= nxg; ++i) { tau_z(i, iw, 1) = tau_z(i, iw, 2); tau_z(i, iw, nz) = tau_z(i, iw, nz - 1); }
        }
    }

    // ---- SGS eddy viscosity: compute_vreman pass 1 (src/sgs_model.f90:118-223) and ghosts (:458-531) ----
    void compute_sgs_model() {
        if (prm.sgs_model == 0) return;
        bool use_amd = prm.sgs_model == 2;
        double c_V = 2.5 * prm.Cs_vreman * prm.Cs_vreman;
        bool wm_lo = prm.flat_wall_model_flag > 0 && y_bc_type == 1 && bc_face_ylo == 1;
        bool wm_hi = prm.flat_wall_model_flag > 0 && y_bc_type == 1 && bc_face_yhi == 1;
        double inv_dx = 1.0 / dx, dx2 = dx * dx;
#pragma omp parallel for
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j) {
                double dz_c = z[k] - z[k - 1], dz2 = dz_c * dz_c, inv_dz_k = 1.0 / dz_c;
                double inv_zg_km = 1.0 / (zg[k] - zg[k - 1]), inv_zg_kp = 1.0 / (zg[k + 1] - zg[k]);
                double dy_c = y[j] - y[j - 1], dy2_c = dy_c * dy_c;
                double inv_yg_jm = 1.0 / (yg[j] - yg[j - 1]), inv_yg_jp = 1.0 / (yg[j + 1] - yg[j]);
                double inv_dy_j = 1.0 / dy_c;
                for (int i = 2; i <= nxg - 1; ++i) {
                    double a11 = (U(i, j, k) - U(i - 1, j, k)) * inv_dx;
                    double a21 = 0.5 * ((U(i, j, k) - U(i, j - 1, k)) * inv_yg_jm + (U(i, j + 1, k) - U(i, j, k)) * inv_yg_jp);
                    double a31 = 0.5 * ((U(i, j, k) - U(i, j, k - 1)) * inv_zg_km + (U(i, j, k + 1) - U(i, j, k)) * inv_zg_kp);
                    double a12 = 0.5 * ((V(i, j, k) - V(i - 1, j, k)) + (V(i + 1, j, k) - V(i, j, k))) * inv_dx;
                    double a22 = (V(i, j, k) - V(i, j - 1, k)) * inv_dy_j;
                    double a32 = 0.5 * ((V(i, j, k) - V(i, j, k - 1)) * inv_zg_km + (V(i, j, k + 1) - V(i, j, k)) * inv_zg_kp);
                    double a13 = 0.5 * ((W(i, j, k) - W(i - 1, j, k)) + (W(i + 1, j, k) - W(i, j, k))) * inv_dx;
                    double a23 = 0.5 * ((W(i, j, k) - W(i, j - 1, k)) * inv_yg_jm + (W(i, j + 1, k) - W(i, j, k)) * inv_yg_jp);
                    double a33 = (W(i, j, k) - W(i, j, k - 1)) * inv_dz_k;
                    if ((wm_lo && j == 2) || (wm_hi && j == nyg - 1)) {
                        double y_w = (j == 2) ? yg[2] : Ly - yg[nyg - 1];
                        double u_c = 0.5 * (U(i - 1, j, k) + U(i, j, k));
                        double w_c = 0.5 * (W(i, j, k - 1) + W(i, j, k));
                        double u_mag = std::sqrt(u_c * u_c + w_c * w_c);
                        if (u_mag > 1e-14) {
                            double u_tau = solve_u_tau_reichardt(u_mag, y_w, prm.nu);
                            double fac_w = ((j == 2) ? 1.0 : -1.0) * u_tau / (kappa_wm * y_w * u_mag);
                            a21 = fac_w * u_c;
                            a23 = fac_w * w_c;
                        }
                    }
                    double b11 = dx2 * (a11 * a11) + dy2_c * (a21 * a21) + dz2 * (a31 * a31);
                    double b22 = dx2 * (a12 * a12) + dy2_c * (a22 * a22) + dz2 * (a32 * a32);
                    double b33 = dx2 * (a13 * a13) + dy2_c * (a23 * a23) + dz2 * (a33 * a33);
                    double b12 = dx2 * (a11 * a12) + dy2_c * (a21 * a22) + dz2 * (a31 * a32);
                    double b13 = dx2 * (a11 * a13) + dy2_c * (a21 * a23) + dz2 * (a31 * a33);
                    double b23 = dx2 * (a12 * a13) + dy2_c * (a22 * a23) + dz2 * (a32 * a33);
                    double B_beta = b11 * b22 - b12 * b12 + b11 * b33 - b13 * b13 + b22 * b33 - b23 * b23;
                    double alpha_sq = a11 * a11 + a12 * a12 + a13 * a13 + a21 * a21 + a22 * a22 + a23 * a23 +
                                      a31 * a31 + a32 * a32 + a33 * a33;
                    double nu_t_loc;
                    if (use_amd) {
                        double amd_num = -(b11 * a11 + b22 * a22 + b33 * a33 + b12 * (a12 + a21) + b13 * (a13 + a31) + b23 * (a23 + a32));
                        if (alpha_sq > 1e-20 && amd_num > 1e-12 * (dx2 + dy2_c + dz2) * alpha_sq * std::sqrt(alpha_sq))
                            nu_t_loc = prm.C_amd * amd_num / alpha_sq;
                        else nu_t_loc = 0.0;
                    } else if (alpha_sq > 1e-20 && B_beta > 0.0) {
                        nu_t_loc = c_V * std::sqrt(B_beta / alpha_sq);
                    } else nu_t_loc = 0.0;
                    nu_t(i, j, k) = nu_t_loc;
                }
            }
        // sgs_fill_ghosts (:458-531), one rank, no IBM
        if (y_bc_type == 1 && bc_face_ylo == 1) for (int k = 1; k <= nzg; ++k) for (int i = 1; i <= nxg; ++i) nu_t(i, 1, k) = 0.0;
        if (y_bc_type == 1 && bc_face_yhi == 1) for (int k = 1; k <= nzg; ++k) for (int i = 1; i <= nxg; ++i) nu_t(i, nyg, k) = 0.0;
        if (y_bc_type == 0) {
            for (int k = 1; k <= nzg; ++k) for (int i = 1; i <= nxg; ++i) nu_t(i, 1, k) = nu_t(i, nyg - 2, k);
            for (int k = 1; k <= nzg; ++k) for (int i = 1; i <= nxg; ++i) nu_t(i, nyg - 1, k) = nu_t(i, 2, k);
            for (int k = 1; k <= nzg; ++k) for (int i = 1; i <= nxg; ++i) nu_t(i, nyg, k) = nu_t(i, 3, k);
        }
        for (int k = 1; k <= nzg; ++k) for (int j = 1; j <= nyg; ++j) nu_t(1, j, k) = nu_t(nxg - 2, j, k);
        for (int k = 1; k <= nzg; ++k) for (int j = 1; j <= nyg; ++j) nu_t(nxg - 1, j, k) = nu_t(2, j, k);
        for (int k = 1; k <= nzg; ++k) for (int j = 1; j <= nyg; ++j) nu_t(nxg, j, k) = nu_t(3, j, k);
        periodic_z(nu_t, 4);
    }

    // time step: fixed (prm.dt) or adaptive (cfl_adaptive = 1; src/global.f90:472-478)
    double dt_cur = -1.0;
    int cfl_adaptive = 0;
    double cfl_target = 0.5, cfl_safety = 0.9, dt_min = 1e-10, dt_max = 1e10;
    double dt() const { return dt_cur > 0.0 ? dt_cur : prm.dt; }

    // compute_cfl (src/monitor.f90:304-424) without the IBM, buoyancy, rotation and actuator terms
    void compute_cfl(double &conv_out, double &visc_out) {
        double conv = 0.0, visc = 0.0;
        const double inv_dx = 1.0 / dx, inv_dx2 = inv_dx * inv_dx;
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j) {
                const double inv_dy = 1.0 / std::max(y[j] - y[j - 1], 1e-14), inv_dy2 = inv_dy * inv_dy;
                const double inv_dz = 1.0 / std::max(z[k] - z[k - 1], 1e-14), inv_dz2 = inv_dz * inv_dz;
                for (int i = 2; i <= nxg - 1; ++i) {
                    const double c = std::fabs(0.5 * (U(i, j, k) + U(i - 1, j, k))) * inv_dx +
                                     std::fabs(0.5 * (V(i, j, k) + V(i, j - 1, k))) * inv_dy +
                                     std::fabs(0.5 * (W(i, j, k) + W(i, j, k - 1))) * inv_dz;
                    conv = std::max(conv, c);
                    visc = std::max(visc, (prm.nu + nu_t(i, j, k)) * 2.0 * (inv_dx2 + inv_dy2 + inv_dz2));
                }
            }
        conv_out = conv * dt();
        visc_out = visc * dt();
    }
    // output landing (nsave < 0, chunk_nsave < 0, slice_freq < 0, line_freq < 0, nsteps < 0): the step is shrunk
    // in turn for each target, in select_dt's order tsave_next, chunk_tsave_next, slice_tnext, line_tnext,
    // sim_end_time; NaN: no target in that slot.  A target within 1e-10 of t counts as reached (the tolerance of
    // src/time_integration.f90:597 and src/main.f90:90-91), and the caller moves it on.
    static constexpr int NLAND = 5;
    double t_land[NLAND] = {NAN, NAN, NAN, NAN, NAN};
    bool landing() const {
        for (double v : t_land)
            if (!std::isnan(v)) return true;
        return false;
    }
    double dt_presnap = -1.0;
    // landing_dt (src/monitor.f90:450-458): a remainder below 2 dt is taken in one step, or in two equal halves
    // when it is above dt
    static double landing_dt(double dt_now, double rem) {
        double r = dt_now;
        if (rem < 2.0 * dt_now) {
            r = rem;
            if (rem > dt_now) r = 0.5 * rem;
        }
        return r;
    }
    // select_dt (src/monitor.f90:429-444)
    void select_dt() {
        if (cfl_adaptive == 1) {
            double conv = 0.0, visc = 0.0;
            compute_cfl(conv, visc);
            const double cfl_now = std::max(conv, visc);
            if (cfl_now > 0.0) dt_cur = std::max(dt_min, std::min(dt_max, dt() * cfl_target / cfl_now * cfl_safety));
        }
        dt_presnap = dt();
        for (double tl : t_land)
            if (tl - t > 1e-10) dt_cur = landing_dt(dt(), tl - t);
    }

    // ---- projection (src/projection.f90) ----
    void compute_pseudo_pressure_rhs() {   // :37-63
        double inv_dx_p = 1.0 / dx;
#pragma omp parallel for
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j) {
                double inv_dzk = 1.0 / (z[k] - z[k - 1]);
                double inv_dyj = 1.0 / (y[j] - y[j - 1]);
                for (int i = 2; i <= nxg - 1; ++i)
                    rhs_p(i, j, k) = (U(i, j, k) - U(i - 1, j, k)) * inv_dx_p + (V(i, j, k) - V(i, j - 1, k)) * inv_dyj +
                                     (W(i, j, k) - W(i, j, k - 1)) * inv_dzk;
            }
    }
    // CPU chain of solve_poisson_equation (:100-343), one rank: poisson arrays are (nxp, nym, nzp)
    void solve_poisson_core() {
        long n1 = nxp, n2 = nym, n3 = nzp;
        std::vector<cplx> c((size_t)(n1 * n2 * n3));
        auto id = [&](long i, long j, long k) { return (size_t)(i + n1 * (j + n2 * k)); };
        for (long k = 0; k < n3; ++k)
            for (long j = 0; j < n2; ++j)
                for (long i = 0; i < n1; ++i) c[id(i, j, k)] = cplx(rhs_p((int)i + 2, (int)j + 2, (int)k + 2), 0.0);
        // forward x (batched over (j,k)): FFT, or with inflow/outflow x the real DCT-IV (src/projection.f90:124-130)
        if (x_bc_type == 0) {
#pragma omp parallel for
            for (long jk = 0; jk < n2 * n3; ++jk) fx.exec(&c[(size_t)(jk * n1)], 1, false);
        } else {
#pragma omp parallel for
            for (long jk = 0; jk < n2 * n3; ++jk) {
                std::vector<double> a((size_t)n1), b((size_t)n1);
                for (long i = 0; i < n1; ++i) a[i] = c[(size_t)(jk * n1 + i)].real();
                dct4(a.data(), b.data());
                for (long i = 0; i < n1; ++i) c[(size_t)(jk * n1 + i)] = cplx(b[i], 0.0);
            }
        }
        // then z
        if (z_bc_type == 0) {
#pragma omp parallel for
            for (long ij = 0; ij < n1 * n2; ++ij) fz.exec(&c[(size_t)ij], n1 * n2, false);
        }
        if (z_bc_type == 1 && y_bc_type == 0) {
            // spanwise walls alone (src/projection.f90:136-143, 219-250, 310-316): FFT in y over the nyp independent
            // rows, one z-tridiagonal solve per (kx, ky) with Dzz and kxx + kyy, the (0,0) mode pinned as the y-wall
            // branch pins its own, then the inverse y FFT and / nyp (the row nyp+1 rides through untransformed and
            // is replaced by the periodic y copy below)
            const int nyp = nym - 1, nr = (int)n3;
#pragma omp parallel for
            for (long k = 0; k < n3; ++k)
                for (long i = 0; i < n1; ++i) fy.exec(&c[id(i, 0, k)], n1, false);
            long swaps = 0; int info_max = 0;
#pragma omp parallel for reduction(+ : swaps) reduction(max : info_max)
            for (long j = 0; j < nyp; ++j) {
                std::vector<cplx> DL(nr), D(nr), DU(nr), B(nr);
                for (long i = 0; i < n1; ++i) {
                    for (int k = 2; k <= nzg - 2; ++k) { DL[k - 2] = Dzz_l[k + 1]; DU[k - 2] = Dzz_u[k]; }
                    const double wavenum_sum = kxx[i] + kyy[j];
                    for (int k = 2; k <= nzg - 1; ++k) D[k - 2] = Dzz_d[k] + wavenum_sum;
                    if (x_bc_type == 0 && i == 0 && j == 0) D[0] = 3.0 / 2.0 * D[0];
                    for (int k = 0; k < nr; ++k) B[k] = c[id(i, j, k)];
                    long sw = 0;
                    const int info = zgtsv(nr, DL.data(), D.data(), DU.data(), B.data(), &sw);
                    swaps += sw; info_max = std::max(info_max, info);
                    for (int k = 0; k < nr; ++k) c[id(i, j, k)] = B[k];
                }
            }
            gtsv_swaps += swaps; last_info = info_max;
#pragma omp parallel for
            for (long k = 0; k < n3; ++k)
                for (long i = 0; i < n1; ++i) fy.exec(&c[id(i, 0, k)], n1, true);
            for (long k = 0; k < n3; ++k)
                for (long j = 0; j < nyp; ++j)
                    for (long i = 0; i < n1; ++i) c[id(i, j, k)] = c[id(i, j, k)] / (double)nyp;
        } else if (z_bc_type == 1) {
            // 4-wall duct (src/projection.f90:172-217): per x mode, project onto the eigenbasis after scaling by
            // sqrt(cell width), one y-tridiagonal solve per eigenmode with lambda_z(m) in place of kzz, then
            // unproject and unscale
            const int nr = nym, nm = (int)n3;
            double lmax = 0.0;
            for (int m = 0; m < nm; ++m) lmax = std::max(lmax, std::fabs(lambda_z[m]));
            long swaps = 0; int info_max = 0;
#pragma omp parallel for reduction(+ : swaps) reduction(max : info_max)
            for (long i = 0; i < n1; ++i) {
                std::vector<cplx> zh((size_t)n2 * nm), DL(nr), D(nr), DU(nr), B(nr);
                for (long j = 0; j < n2; ++j)
                    for (int m = 0; m < nm; ++m) {
                        cplx acc(0.0, 0.0);
                        for (int k = 0; k < nm; ++k) acc += c[id(i, j, k)] * sqrt_w_z[k] * Qz[(size_t)k * nm + m];
                        zh[(size_t)(j + n2 * m)] = acc;
                    }
                for (int m = 0; m < nm; ++m) {
                    for (int j = 2; j <= nyg - 2; ++j) { DL[j - 2] = Dyy_l[j + 1]; DU[j - 2] = Dyy_u[j]; }
                    const double wavenum_sum = kxx[i] + lambda_z[m];
                    for (int j = 2; j <= nyg - 1; ++j) D[j - 2] = Dyy_d[j] + wavenum_sum;
                    if (x_bc_type == 0 && i == 0 && std::fabs(lambda_z[m]) < 1e-8 * lmax) D[0] = 3.0 / 2.0 * D[0];
                    for (int j = 0; j < nr; ++j) B[j] = zh[(size_t)(j + n2 * m)];
                    long sw = 0;
                    const int info = zgtsv(nr, DL.data(), D.data(), DU.data(), B.data(), &sw);
                    swaps += sw; info_max = std::max(info_max, info);
                    for (int j = 0; j < nr; ++j) zh[(size_t)(j + n2 * m)] = B[j];
                }
                for (long j = 0; j < n2; ++j)
                    for (int k = 0; k < nm; ++k) {
                        cplx acc(0.0, 0.0);
                        for (int m = 0; m < nm; ++m) acc += zh[(size_t)(j + n2 * m)] * Qz[(size_t)k * nm + m];
                        c[id(i, j, k)] = acc / sqrt_w_z[k];
                    }
            }
            gtsv_swaps += swaps; last_info = info_max;
        } else if (y_bc_type == 0) {
            int nyp = nym - 1;
#pragma omp parallel for
            for (long k = 0; k < n3; ++k)
                for (long i = 0; i < n1; ++i) fy.exec(&c[id(i, 0, k)], n1, false);
#pragma omp parallel for
            for (long k = 0; k < n3; ++k)
                for (long i = 0; i < n1; ++i)
                    for (long j = 0; j < nyp; ++j) {
                        double wavenum_sum = kxx[i] + kyy[j] + kzz[k];
                        if (i == 0 && j == 0 && k == 0) c[id(i, j, k)] = cplx(0.0, 0.0);
                        else c[id(i, j, k)] = c[id(i, j, k)] / wavenum_sum;
                    }
#pragma omp parallel for
            for (long k = 0; k < n3; ++k)
                for (long i = 0; i < n1; ++i) fy.exec(&c[id(i, 0, k)], n1, true);
            for (long k = 0; k < n3; ++k)
                for (long j = 0; j < nyp; ++j)
                    for (long i = 0; i < n1; ++i) c[id(i, j, k)] = c[id(i, j, k)] / (double)nyp;
        } else {
            int nr = nym;
            long swaps = 0; int info_max = 0;
#pragma omp parallel for reduction(+ : swaps) reduction(max : info_max)
            for (long k = 0; k < n3; ++k) {
                std::vector<cplx> DL(nr), D(nr), DU(nr), B(nr);
                for (long i = 0; i < n1; ++i) {
                    double wavenum_sum = kxx[i] + kzz[k];
                    for (int j = 2; j <= nyg - 2; ++j) { DL[j - 2] = Dyy_l[j + 1]; DU[j - 2] = Dyy_u[j]; }
                    for (int j = 2; j <= nyg - 1; ++j) D[j - 2] = Dyy_d[j] + wavenum_sum;
                    if (x_bc_type == 0 && i == 0 && k == 0) D[0] = 3.0 / 2.0 * D[0];
                    for (int j = 0; j < nr; ++j) B[j] = c[id(i, j, k)];
                    long sw = 0;
                    int info = zgtsv(nr, DL.data(), D.data(), DU.data(), B.data(), &sw);
                    swaps += sw; info_max = std::max(info_max, info);
                    for (int j = 0; j < nr; ++j) c[id(i, j, k)] = B[j];
                }
            }
            gtsv_swaps += swaps; last_info = info_max;
        }
        if (z_bc_type == 0) {
#pragma omp parallel for
            for (long ij = 0; ij < n1 * n2; ++ij) fz.exec(&c[(size_t)ij], n1 * n2, true);
        }
        if (x_bc_type == 0) {
#pragma omp parallel for
            for (long jk = 0; jk < n2 * n3; ++jk) fx.exec(&c[(size_t)(jk * n1)], 1, true);
            // a z wall is solved in physical z: no z normalisation (:326-332)
            double norm = z_bc_type == 0 ? (double)((long)nxp * (long)nzp) : (double)nxp;
            for (long k = 0; k < n3; ++k)
                for (long j = 0; j < n2; ++j)
                    for (long i = 0; i < n1; ++i) rhs_p((int)i + 2, (int)j + 2, (int)k + 2) = c[id(i, j, k)].real() / norm;
        } else {   // real part, DCT-IV again, / (2 nxp nzp), or / (2 nxp) with z walls (src/projection.f90:334-343)
            const double norm = z_bc_type == 0 ? 2.0 * (double)nxp * (double)nzp : 2.0 * (double)nxp;
#pragma omp parallel for
            for (long jk = 0; jk < n2 * n3; ++jk) {
                std::vector<double> a((size_t)n1), b((size_t)n1);
                for (long i = 0; i < n1; ++i) a[i] = c[(size_t)(jk * n1 + i)].real();
                dct4(a.data(), b.data());
                const long j = jk % n2, k = jk / n2;
                for (long i = 0; i < n1; ++i) rhs_p((int)i + 2, (int)j + 2, (int)k + 2) = b[i] / norm;
            }
        }
        // apply_periodic_xz_pressure (:441-500), one rank: the x copy only with periodic x (inflow/outflow x leaves
        // the plane nxg as it was)
        if (x_bc_type == 0)
            for (int k = 2; k <= nzg; ++k)
                for (int j = 2; j <= nyg - 1; ++j) rhs_p(nxg - 1, j, k) = rhs_p(2, j, k);
        if (z_bc_type == 0)   // no z copy with a z wall (:473-476)
            for (int j = 2; j <= nyg - 1; ++j)
                for (int i = 2; i <= nxg - 1; ++i) rhs_p(i, j, nzp + 2) = rhs_p(i, j, 2);
        if (y_bc_type == 0)
            for (int k = 2; k <= nzg; ++k)
                for (int i = 2; i <= nxg; ++i) rhs_p(i, nyg - 1, k) = rhs_p(i, 2, k);
        // update_ghost_interior_planes_pressure(_x): no neighbour at one rank
    }
    void finish_pressure_ghosts(A3 &Pf) {   // :388-438
        for (int k = 1; k <= nzg; ++k)
            for (int i = 1; i <= nxg; ++i) { Pf(i, 1, k) = Pf(i, 2, k); Pf(i, nyg, k) = Pf(i, nyg - 1, k); }
        for (int k = 1; k <= nzg; ++k) for (int j = 1; j <= nyg; ++j) Pf(1, j, k) = Pf(nxg - 2, j, k);
        for (int k = 1; k <= nzg; ++k) for (int j = 1; j <= nyg; ++j) Pf(nxg - 1, j, k) = Pf(2, j, k);
        for (int k = 1; k <= nzg; ++k) for (int j = 1; j <= nyg; ++j) Pf(nxg, j, k) = Pf(3, j, k);
        periodic_z(Pf, 4);
    }
    void project_velocity() {   // :551-604, one rank (is_last_x: the nx face is left to the periodic BC)
        double inv_dx_proj = 1.0 / dx;
#pragma omp parallel for
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j)
                for (int i = 2; i <= nx - 1; ++i)
                    U(i, j, k) = U(i, j, k) - (rhs_p(i + 1, j, k) - rhs_p(i, j, k)) * inv_dx_proj;
        for (int j = 2; j <= ny - 1; ++j) {
            double inv_dygj = 1.0 / (yg[j + 1] - yg[j]);
#pragma omp parallel for
            for (int k = 2; k <= nzg - 1; ++k)
                for (int i = 2; i <= nxg - 1; ++i)
                    V(i, j, k) = V(i, j, k) - (rhs_p(i, j + 1, k) - rhs_p(i, j, k)) * inv_dygj;
        }
        for (int k = 2; k <= nz - 1; ++k) {
            double inv_dzgk = 1.0 / (zg[k + 1] - zg[k]);
#pragma omp parallel for
            for (int j = 2; j <= nyg - 1; ++j)
                for (int i = 2; i <= nxg - 1; ++i)
                    W(i, j, k) = W(i, j, k) - (rhs_p(i, j, k + 1) - rhs_p(i, j, k)) * inv_dzgk;
        }
    }
    void compute_projection_step(int rk_step) {
        compute_pseudo_pressure_rhs();
        solve_poisson_core();
        if (rk_step == 3) {
            for (int k = 2; k <= nzg - 1; ++k)
                for (int j = 2; j <= nyg - 1; ++j)
                    for (int i = 2; i <= nxg - 1; ++i) P(i, j, k) = rhs_p(i, j, k) / (dt() * rk_coef[3][3]);
            finish_pressure_ghosts(P);
        }
        project_velocity();
    }

    // ---- compute_bulk_velocity (src/monitor.f90:463-523) ----
    // The reference accumulates the two sums in an unspecified order (an !$acc parallel loop reduction(+:...), then
    // MPI_Allreduce over the ranks), so no one rounding of them is the reference's. This restatement evaluates each
    // sum with Kahan compensation, within a few ulps of its exact value: a sequential sum carries O(sqrt(N) eps)
    // relative error, which the constant-flux shift feeds back into U at every step (on the 128 x 96 x 128 channel
    // a sequential and a compensated oracle differ by 9e-12 relative L2 in V and W after 200 steps).
    double compute_bulk_velocity() {
        int ihi = nxg - 2, jhi = nyg - 1, khi = nzg - 2;
        if (y_bc_type == 0) jhi = nyg - 2;
        double local_sum = 0.0, local_wgt = 0.0, c_sum = 0.0, c_wgt = 0.0;
        for (int k = 2; k <= khi; ++k)
            for (int j = 2; j <= jhi; ++j) {
                double dy_j = (y[j] - y[j - 1]) * (z[k] - z[k - 1]);
                for (int i = 2; i <= ihi; ++i) {
                    const double xs = 0.5 * (U(i, j, k) + U(i - 1, j, k)) * dy_j - c_sum;
                    const double ts = local_sum + xs;
                    c_sum = (ts - local_sum) - xs;
                    local_sum = ts;
                    const double xw = dy_j - c_wgt;
                    const double tw = local_wgt + xw;
                    c_wgt = (tw - local_wgt) - xw;
                    local_wgt = tw;
                }
            }
        return local_sum / std::max(local_wgt, 1e-14);
    }
    // check_divergence (src/projection.f90:607-639)
    double check_divergence() {
        double div = 0.0;
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j)
                for (int i = 2; i <= nxg - 1; ++i)
                    div = std::max(div, std::fabs((U(i, j, k) - U(i - 1, j, k)) / (x[i] - x[i - 1]) +
                                                  (V(i, j, k) - V(i, j - 1, k)) / (y[j] - y[j - 1]) +
                                                  (W(i, j, k) - W(i, j, k - 1)) / (z[k] - z[k - 1])));
        return div;
    }
    // output_monitor (src/monitor.f90:21-102) for one rank, without its printing: out = {t, dt, meanU, maxU,
    // max_divergence, cfl_conv, cfl_visc, mean u_tau lower wall, upper wall (wall_diag_sums, src/wallmodel.f90:700-723;
    // 0 without the y-wall model), NaN flag}.  The CFL numbers are those of the current state.
    void output_monitor(double *out) {
        int bad = 0;
        auto chk = [&](double v) { if (v != v || std::fabs(v) > 1e8) bad = 1; };
        double maxU = 0.0;
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j)
                for (int i = 2; i <= nx - 1; ++i) { chk(U(i, j, k)); maxU = std::max(maxU, std::fabs(U(i, j, k))); }
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= ny - 1; ++j)
                for (int i = 2; i <= nxg - 1; ++i) chk(V(i, j, k));
        for (int k = 2; k <= nz - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j)
                for (int i = 2; i <= nxg - 1; ++i) chk(W(i, j, k));
        double conv = 0.0, visc = 0.0;
        compute_cfl(conv, visc);
        double s1 = 0.0, s2 = 0.0;
        if (y_bc_type == 1 && prm.flat_wall_model_flag > 0) {
            for (int k = 2; k <= nzg - 1; ++k)
                for (int i = 2; i <= nx - 1; ++i) { s1 += wmf_tx(i, 1, k); s2 += wmf_tx(i, 2, k); }
            const double cols = (double)((nx - 2) * (nzg - 2));
            s1 /= cols; s2 /= cols;
        }
        const double vals[10] = {t, dt(), compute_bulk_velocity(), maxU, check_divergence(), conv, visc, s1, s2,
                                 (double)bad};
        for (int q = 0; q < 10; ++q) out[q] = vals[q];
    }
    // volume-weighted 0.5*<|u|^2> over the independent cells with face velocities averaged to centres
    double kinetic_energy() {
        int ihi = nxg - 2, jhi = (y_bc_type == 0) ? nyg - 2 : nyg - 1, khi = nzg - 2;
        long double s = 0.0L, wsum = 0.0L;
        for (int k = 2; k <= khi; ++k)
            for (int j = 2; j <= jhi; ++j) {
                double vol = (y[j] - y[j - 1]) * (z[k] - z[k - 1]) * dx;
                for (int i = 2; i <= ihi; ++i) {
                    double uc = 0.5 * (U(i, j, k) + U(i - 1, j, k));
                    double vc = 0.5 * (V(i, j, k) + V(i, j - 1, k));
                    double wc = 0.5 * (W(i, j, k) + W(i, j, k - 1));
                    s += (long double)(0.5 * (uc * uc + vc * vc + wc * wc) * vol);
                    wsum += (long double)vol;
                }
            }
        return (double)(s / wsum);
    }

    // ---- compute_time_step_RK3 (src/time_integration.f90:120-713), single-phase flag set ----
    void stage_update(int s) {
        double dtc1 = dt() * rk_coef[1][1];
#pragma omp parallel for
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j)
                for (int i = 2; i <= nx - 1; ++i) {
                    if (s == 1) U(i, j, k) = Uo(i, j, k) + dtc1 * Fu[1](i, j, k);
                    else if (s == 2) U(i, j, k) = Uo(i, j, k) + dt() * (rk_coef[2][1] * Fu[1](i, j, k) + rk_coef[2][2] * Fu[2](i, j, k));
                    else U(i, j, k) = Uo(i, j, k) + dt() * (rk_coef[3][1] * Fu[1](i, j, k) + rk_coef[3][2] * Fu[2](i, j, k) + rk_coef[3][3] * Fu[3](i, j, k));
                }
#pragma omp parallel for
        for (int k = 2; k <= nzg - 1; ++k)
            for (int j = 2; j <= ny - 1; ++j)
                for (int i = 2; i <= nxg - 1; ++i) {
                    if (s == 1) V(i, j, k) = Vo(i, j, k) + dtc1 * Fv[1](i, j, k);
                    else if (s == 2) V(i, j, k) = Vo(i, j, k) + dt() * (rk_coef[2][1] * Fv[1](i, j, k) + rk_coef[2][2] * Fv[2](i, j, k));
                    else V(i, j, k) = Vo(i, j, k) + dt() * (rk_coef[3][1] * Fv[1](i, j, k) + rk_coef[3][2] * Fv[2](i, j, k) + rk_coef[3][3] * Fv[3](i, j, k));
                }
#pragma omp parallel for
        for (int k = 2; k <= nz - 1; ++k)
            for (int j = 2; j <= nyg - 1; ++j)
                for (int i = 2; i <= nxg - 1; ++i) {
                    if (s == 1) W(i, j, k) = Wo(i, j, k) + dtc1 * Fw[1](i, j, k);
                    else if (s == 2) W(i, j, k) = Wo(i, j, k) + dt() * (rk_coef[2][1] * Fw[1](i, j, k) + rk_coef[2][2] * Fw[2](i, j, k));
                    else W(i, j, k) = Wo(i, j, k) + dt() * (rk_coef[3][1] * Fw[1](i, j, k) + rk_coef[3][2] * Fw[2](i, j, k) + rk_coef[3][3] * Fw[3](i, j, k));
                }
    }
    void step() {
        compute_sgs_model();
        // dt from the start-of-step velocity, after nu_t (src/time_integration.f90:146-160)
        const bool sel = cfl_adaptive == 1 || landing();
        if (sel) select_dt();
        double to = t;
        Uo.d = U.d; Vo.d = V.d; Wo.d = W.d;
        if (prm.flow_forcing_mode == 0) { dPdx = prm.dPdx; dPdz = prm.dPdz; } else { dPdx = 0.0; dPdz = prm.dPdz; }
        for (int s = 1; s <= 3; ++s) {
            if (s > 1) compute_sgs_model();
            if (s == 1) update_wm_filter();
            compute_wall_model();
            compute_rhs_u(Fu[s]); compute_rhs_v(Fv[s]); compute_rhs_w(Fw[s]);
            stage_update(s);
            t = to + rk_t[s] * dt();
            apply_boundary_conditions();
            compute_projection_step(s);
            apply_boundary_conditions();
        }
        if (prm.flow_forcing_mode == 1) {
            double Ub_now = compute_bulk_velocity();
            double dU = prm.Ub_target - Ub_now;
            for (int k = 2; k <= nzg - 1; ++k)
                for (int j = 2; j <= nyg - 1; ++j)
                    for (int i = 2; i <= nx - 1; ++i) U(i, j, k) = U(i, j, k) + dU;
            apply_boundary_conditions();
        }
        if (sel) dt_cur = dt_presnap;   // dt = dt_presnap (src/time_integration.f90:711)
    }
};

}  // namespace

// ------------------------------------------------------------------------------------------------------------
// C API for the tests (ctypes). Arrays are Fortran-ordered doubles in the reference's one-rank shapes.
extern "C" {

void *orc_create(const dfdm_grid *g, const dfdm_params *p) {
    Oracle *o = new Oracle();
    o->setup(g, p);
    return o;
}
void orc_destroy(void *h) { delete (Oracle *)h; }
void orc_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}
int orc_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
static void copy_in(A3 &a, const double *src) { if (src) std::memcpy(a.d.data(), src, a.size() * sizeof(double)); }
static void copy_out(const A3 &a, double *dst) { if (dst) std::memcpy(dst, a.d.data(), a.size() * sizeof(double)); }
void orc_set_state(void *h, const double *U, const double *V, const double *W, const double *P) {
    Oracle *o = (Oracle *)h;
    copy_in(o->U, U); copy_in(o->V, V); copy_in(o->W, W); copy_in(o->P, P);
}
void orc_get_state(void *h, double *U, double *V, double *W, double *P) {
    Oracle *o = (Oracle *)h;
    copy_out(o->U, U); copy_out(o->V, V); copy_out(o->W, W); copy_out(o->P, P);
}
void orc_get_nu_t(void *h, double *nu_t) { copy_out(((Oracle *)h)->nu_t, nu_t); }
void orc_set_nu_t(void *h, const double *nu_t) { copy_in(((Oracle *)h)->nu_t, nu_t); }
void orc_apply_bc(void *h) { ((Oracle *)h)->apply_boundary_conditions(); }
void orc_step(void *h, int nsteps) { for (int n = 0; n < nsteps; ++n) ((Oracle *)h)->step(); }
double orc_time(void *h) { return ((Oracle *)h)->t; }
double orc_dt(void *h) { return ((Oracle *)h)->dt(); }
void orc_set_adaptive(void *h, int enable, double target, double safety, double dtmin, double dtmax) {
    Oracle *o = (Oracle *)h;
    o->cfl_adaptive = enable ? 1 : 0;
    o->cfl_target = target; o->cfl_safety = safety; o->dt_min = dtmin; o->dt_max = dtmax;
    if (!enable) o->dt_cur = -1.0;
}
void orc_output_monitor(void *h, double *out) { ((Oracle *)h)->output_monitor(out); }
void orc_set_landing(void *h, double t_land) {
    Oracle *o = (Oracle *)h;
    for (double &v : o->t_land) v = NAN;
    o->t_land[0] = t_land;
}
void orc_set_landings(void *h, int n, const double *t_land) {
    Oracle *o = (Oracle *)h;
    for (int q = 0; q < Oracle::NLAND; ++q) o->t_land[q] = q < n ? t_land[q] : NAN;
}
void orc_cfl(void *h, double *conv, double *visc) { ((Oracle *)h)->compute_cfl(*conv, *visc); }
void orc_compute_sgs(void *h) { ((Oracle *)h)->compute_sgs_model(); }
void orc_wall_model(void *h, int update_filter, double *tau_x, double *tau_z) {
    Oracle *o = (Oracle *)h;
    if (update_filter) o->update_wm_filter();
    o->compute_wall_model();
    copy_out(o->tau_x, tau_x); copy_out(o->tau_z, tau_z);
}
void orc_compute_rhs(void *h, double *Fu, double *Fv, double *Fw) {
    Oracle *o = (Oracle *)h;
    if (o->prm.flow_forcing_mode == 0) { o->dPdx = o->prm.dPdx; o->dPdz = o->prm.dPdz; } else { o->dPdx = 0.0; o->dPdz = o->prm.dPdz; }
    o->compute_rhs_u(o->Fu[1]); o->compute_rhs_v(o->Fv[1]); o->compute_rhs_w(o->Fw[1]);
    copy_out(o->Fu[1], Fu); copy_out(o->Fv[1], Fv); copy_out(o->Fw[1], Fw);
}
// rhs_p in/out, shape (2:nxg, 2:nyg-1, 2:nzg)
int orc_solve_poisson(void *h, double *rhs) {
    Oracle *o = (Oracle *)h;
    copy_in(o->rhs_p, rhs);
    o->solve_poisson_core();
    copy_out(o->rhs_p, rhs);
    return o->last_info;
}
void orc_divergence_rhs(void *h, double *rhs) {
    Oracle *o = (Oracle *)h;
    o->compute_pseudo_pressure_rhs();
    copy_out(o->rhs_p, rhs);
}
void orc_projection(void *h, int save_p) {
    Oracle *o = (Oracle *)h;
    o->compute_projection_step(save_p ? 3 : 1);
}
double orc_bulk_velocity(void *h) { return ((Oracle *)h)->compute_bulk_velocity(); }
double orc_max_divergence(void *h) { return ((Oracle *)h)->check_divergence(); }
double orc_kinetic_energy(void *h) { return ((Oracle *)h)->kinetic_energy(); }
long orc_gtsv_swaps(void *h) { return ((Oracle *)h)->gtsv_swaps; }
// grid-derived quantities, for known-answer tests: which = 0 xg, 1 yg, 2 zg (1..n+1 entries), 3 kxx, 4 kzz,
// 5 Dyy diag (index 2..nyg-1), 6 weight_y_0 (1..ny), 7 dx/dz pair, 8/9 Dyy lower/upper; with z walls 10-12 Dzz
// diag/lower/upper (index 2..nzg-1), 13 lambda_z (ascending), 14 sqrt(cell width)
int orc_grid_array(void *h, int which, double *out) {
    Oracle *o = (Oracle *)h;
    switch (which) {
    case 0: for (int i = 1; i <= o->nxg; ++i) out[i - 1] = o->xg[i]; return o->nxg;
    case 1: for (int i = 1; i <= o->nyg; ++i) out[i - 1] = o->yg[i]; return o->nyg;
    case 2: for (int i = 1; i <= o->nzg; ++i) out[i - 1] = o->zg[i]; return o->nzg;
    case 3: for (size_t i = 0; i < o->kxx.size(); ++i) out[i] = o->kxx[i]; return (int)o->kxx.size();
    case 4: for (size_t i = 0; i < o->kzz.size(); ++i) out[i] = o->kzz[i]; return (int)o->kzz.size();
    case 5: for (int j = 2; j <= o->nyg - 1; ++j) out[j - 2] = o->Dyy_d[j]; return o->nyg - 2;
    case 6: for (int j = 1; j <= o->ny; ++j) out[j - 1] = o->wy0[j]; return o->ny;
    case 7: out[0] = o->dx; out[1] = o->dz; return 2;
    case 8: for (int j = 2; j <= o->nyg - 1; ++j) out[j - 2] = o->Dyy_l[j]; return o->nyg - 2;   // Dyy(j, j-1)
    case 9: for (int j = 2; j <= o->nyg - 1; ++j) out[j - 2] = o->Dyy_u[j]; return o->nyg - 2;   // Dyy(j, j+1)
    }
    if (o->z_bc_type != 1) return 0;
    switch (which) {   // the duct's z operator and eigenbasis
    case 10: for (int k = 2; k <= o->nzg - 1; ++k) out[k - 2] = o->Dzz_d[k]; return o->nzg - 2;
    case 11: for (int k = 2; k <= o->nzg - 1; ++k) out[k - 2] = o->Dzz_l[k]; return o->nzg - 2;   // Dzz(k, k-1)
    case 12: for (int k = 2; k <= o->nzg - 1; ++k) out[k - 2] = o->Dzz_u[k]; return o->nzg - 2;   // Dzz(k, k+1)
    case 13: for (int m = 0; m < o->nzm; ++m) out[m] = o->lambda_z[m]; return o->nzm;
    case 14: for (int k = 0; k < o->nzm; ++k) out[k] = o->sqrt_w_z[k]; return o->nzm;
    }
    return 0;
}

// the DCT-IV of one x line of an inflow/outflow-x oracle (nxp values in, nxp out); -1 for a periodic-x oracle
int orc_dct4(void *h, const double *in, double *out) {
    Oracle *o = (Oracle *)h;
    if (o->x_bc_type != 1) return -1;
    o->dct4(in, out);
    return o->nxp;
}
// raw FFT and zgtsv entry points for cross-checks against numpy / scipy
void orc_fft(int n, double *re_im, int inverse) {
    FFTPlan p; p.init(n);
    p.exec((cplx *)re_im, 1, inverse != 0);
}
int orc_zgtsv(int n, double *dl, double *d, double *du, double *b) {
    long sw = 0;
    return zgtsv(n, (cplx *)dl, (cplx *)d, (cplx *)du, (cplx *)b, &sw);
}

}  // extern "C"
