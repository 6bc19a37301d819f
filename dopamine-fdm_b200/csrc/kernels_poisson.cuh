// kernels_poisson.cuh -- the projection: div u*, FFT x / FFT z / y solve, inverse transforms, velocity correction.
//
// Follows compute_projection_step (src/projection.f90:21-34): rhs_p = div u* (no 1/dt, :47-61), the spectral
// Poisson solve of solve_poisson_equation (:100-382; GPU ordering of src/poisson_gpu.f90:230-493: real-to-complex
// x transform, complex z transform, y solve, inverse z, complex-to-real x with 1/(nxp*nzp)), the stage-3 pressure
// save P = phi/(dt*3/4) (:362-380) and project_velocity (:551-604).
#pragma once

#include "dfdm_common.cuh"
#include "fft_smem.cuh"

namespace dfdm {

template <typename T> struct PoissonArgs {
    Dims d;
    Metric1D<T> my, mz;
    T inv_dx;
    double norm;         // nxp*nzp
    double pdiv;         // dt*rk_coef(3,3)
};

// ---- 1. rhs_p = div u* fused with the forward real-to-complex x transform ------------------------------------
// One block transforms `lx` x-lines (line = k*Ny + j).  A real line of length Nx is packed as Nx/2 complex values
// z_n = x_2n + i x_2n+1 (its natural memory layout), transformed with a length-Nx/2 FFT and unpacked:
//   X_k = E_k + W_Nx^k O_k,  E_k = (Z_k + conj Z_{M-k})/2,  O_k = (Z_k - conj Z_{M-k})/(2i),  k = 0..M.
// FROM_DIV = false transforms a given real field instead (unit entry point of the Poisson solve).
template <typename T, bool FROM_DIV>
__global__ void __launch_bounds__(256) k_fwd_x(PoissonArgs<T> a, int lx, const T *__restrict__ U, const T *__restrict__ V,
                                               const T *__restrict__ W, const T *__restrict__ src,
                                               typename cplx_t<T>::type *__restrict__ spec, FFTPlan p,
                                               const typename cplx_t<T>::type *__restrict__ tw,
                                               const typename cplx_t<T>::type *__restrict__ twr) {
    typedef typename cplx_t<T>::type C;
    typedef Arith<T> A;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Dims &d = a.d;
    const int M = d.Nx / 2;
    C *b0 = (C *)smem_raw, *b1 = b0 + (size_t)lx * M;
    const long long nlines_tot = (long long)d.Ny * d.Nz;
    const long long line0 = (long long)blockIdx.x * lx;
    const int nl = (int)min((long long)lx, nlines_tot - line0);
    T *r0 = (T *)b0;
    for (int e = threadIdx.x; e < nl * d.Nx; e += blockDim.x) {
        int ll = e / d.Nx, i = e - ll * d.Nx;
        long long line = line0 + ll;
        int j = (int)(line % d.Ny), k = (int)(line / d.Ny);
        T val;
        if (FROM_DIV) {
            int im = wrap(i - 1, d.Nx), km = wrap(k - 1, d.Nz);
            T inv_dyj = A::inv(a.my.dc, a.my.idc, j), inv_dzk = A::inv(a.mz.dc, a.mz.idc, k);
            val = (__ldg(U + idx3(d, i, j, k)) - __ldg(U + idx3(d, im, j, k))) * a.inv_dx +
                  (ld_yf(V, d, i, j, k) - ld_yf(V, d, i, j - 1, k)) * inv_dyj +
                  (__ldg(W + idx3(d, i, j, k)) - __ldg(W + idx3(d, i, j, km))) * inv_dzk;
        } else {
            val = src[line * d.Nx + i];
        }
        r0[(size_t)ll * d.Nx + i] = val;
    }
    __syncthreads();
    C *res = fft_lines<T, false, false>(b0, b1, nl, M, 1, p, tw);
    for (int e = threadIdx.x; e < nl * (M + 1); e += blockDim.x) {
        int ll = e / (M + 1), kx = e - ll * (M + 1);
        C Zk = res[ll * M + (kx == M ? 0 : kx)];
        C Zm = res[ll * M + (kx == 0 ? 0 : M - kx)];
        T Er = T(0.5) * (Zk.x + Zm.x), Ei = T(0.5) * (Zk.y - Zm.y);
        T Dr = T(0.5) * (Zk.x - Zm.x), Di = T(0.5) * (Zk.y + Zm.y);
        T Or = Di, Oi = -Dr;   // O = D / i
        C w = __ldg(twr + kx);
        C X;
        X.x = Er + (w.x * Or - w.y * Oi);
        X.y = Ei + (w.x * Oi + w.y * Or);
        spec[(line0 + ll) * d.Nxc + kx] = X;
    }
}

// ---- 2. transforms along z (and the periodic-y Poisson solve) on column tiles ---------------------------------
// A block loads `tx` consecutive kx columns of length L (rows at stride rowstride), transforms every column in
// shared memory and stores them back in place.
//   MODE 0: forward FFT along z (rows = kz, one block per (kx tile, j))
//   MODE 1: inverse FFT along z
//   MODE 2: periodic y (rows = j, one block per (kx tile, kz)): forward FFT, divide by kxx+kyy+kzz with the
//           (0,0,0) mode set to zero, inverse FFT, divide by nyp (src/projection.f90:246-273)
template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_col_fft(Dims d, int tx, typename cplx_t<T>::type *__restrict__ spec, FFTPlan p,
                                                 const typename cplx_t<T>::type *__restrict__ tw,
                                                 const double *__restrict__ kxx, const double *__restrict__ kyy,
                                                 const double *__restrict__ kzz) {
    typedef typename cplx_t<T>::type C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *b0 = (C *)smem_raw, *b1 = b0 + (size_t)p.n * tx;
    const int L = p.n;
    const int kx0 = blockIdx.x * tx;
    const int other = blockIdx.y;
    long long base, rowstride;
    if (MODE == 2) { base = (long long)other * d.Ny * d.Nxc; rowstride = d.Nxc; }
    else { base = (long long)other * d.Nxc; rowstride = (long long)d.Ny * d.Nxc; }
    for (int e = threadIdx.x; e < L * tx; e += blockDim.x) {
        int row = e / tx, c = e - row * tx, kx = kx0 + c;
        C v = mkc<T>(T(0), T(0));
        if (kx < d.Nxc) v = spec[base + row * rowstride + kx];
        b0[e] = v;
    }
    __syncthreads();
    C *res;
    if (MODE == 0) res = fft_lines<T, false, true>(b0, b1, tx, 1, tx, p, tw);
    else if (MODE == 1) res = fft_lines<T, true, true>(b0, b1, tx, 1, tx, p, tw);
    else {
        res = fft_lines<T, false, true>(b0, b1, tx, 1, tx, p, tw);
        const int kz = other;
        for (int e = threadIdx.x; e < L * tx; e += blockDim.x) {
            int j = e / tx, c = e - j * tx, kx = kx0 + c;
            if (kx >= d.Nxc) continue;
            double wavenum_sum = kxx[kx] + kyy[j] + kzz[kz];
            C v = res[e];
            if (kx == 0 && j == 0 && kz == 0) { v.x = T(0); v.y = T(0); }
            else { v.x = (T)((double)v.x / wavenum_sum); v.y = (T)((double)v.y / wavenum_sum); }
            res[e] = v;
        }
        __syncthreads();
        C *other_buf = (res == b0) ? b1 : b0;
        res = fft_lines<T, true, true>(res, other_buf, tx, 1, tx, p, tw);
        const double nyp = (double)L;
        for (int e = threadIdx.x; e < L * tx; e += blockDim.x) {
            C v = res[e];
            v.x = (T)((double)v.x / nyp); v.y = (T)((double)v.y / nyp);
            res[e] = v;
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < L * tx; e += blockDim.x) {
        int row = e / tx, c = e - row * tx, kx = kx0 + c;
        if (kx < d.Nxc) spec[base + row * rowstride + kx] = res[e];
    }
}

// ---- 3. wall-bounded y: one tridiagonal system per (kx, kz) ----------------------------------------------------
// (Dyy + kxx + kzz) phi = r with the (0,0) row D(2) scaled by 3/2 (src/projection.f90:275-297, GPU
// src/poisson_gpu.f90:445-489), solved by the no-interchange branch of LAPACK zgtsv in double:
//   m = DL(r-1)/D(r-1),  D(r) = (Dyy(r,r) + lambda) - m DU(r-1),  b(r) = b(r) - m b(r-1)
//   x(n-1) = b(n-1)/D(n-1),  x(r) = (b(r) - DU(r) x(r+1))/D(r)
// The pressure operator is similar to a symmetric negative-definite matrix once the null mode is pinned, so
// elimination without interchanges is stable.  One thread owns one (kx,kz) column; a warp covers 32
// consecutive kx, so every row access is coalesced.  The pivots D(r) stay in shared memory; the eliminated
// right-hand side is written back in place (double in FP64 storage, as zgtsv overwrites B) and re-read by the
// back substitution while it is still in L2.
template <typename T>
__global__ void __launch_bounds__(32) k_ysolve(Dims d, typename cplx_t<T>::type *__restrict__ spec,
                                               const double *__restrict__ kxx, const double *__restrict__ kzz,
                                               const double *__restrict__ lo, const double *__restrict__ di,
                                               const double *__restrict__ up) {
    typedef typename cplx_t<T>::type C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *pv = (double *)smem_raw;   // [Ny][32]
    const int c = threadIdx.x;
    const int kx = blockIdx.x * 32 + c, kz = blockIdx.y;
    if (kx >= d.Nxc) return;
    const int n = d.Ny;
    C *col = spec + (long long)kz * d.Ny * d.Nxc + kx;
    const long long st = d.Nxc;
    const double lam = kxx[kx] + kzz[kz];
    double D = di[0] + lam;
    if (kx == 0 && kz == 0) D = 3.0 / 2.0 * D;
    pv[c] = D;
    C v = col[0];
    double br = (double)v.x, bi = (double)v.y;
    for (int r = 1; r < n; ++r) {
        double m = lo[r] / D;
        D = (di[r] + lam) - m * up[r - 1];
        pv[r * 32 + c] = D;
        v = col[r * st];
        br = (double)v.x - m * br;
        bi = (double)v.y - m * bi;
        if (r < n - 1) { v.x = (T)br; v.y = (T)bi; col[r * st] = v; }
    }
    double xr = br / D, xi = bi / D;
    v.x = (T)xr; v.y = (T)xi;
    col[(n - 1) * st] = v;
    for (int r = n - 2; r >= 0; --r) {
        double u = up[r];
        double p = pv[r * 32 + c];
        v = col[r * st];
        xr = ((double)v.x - u * xr) / p;
        xi = ((double)v.y - u * xi) / p;
        v.x = (T)xr; v.y = (T)xi;
        col[r * st] = v;
    }
}

// ---- 4. inverse complex-to-real x transform, writes the pseudo-pressure phi ----------------------------------
//   Z_k = (X_k + conj X_{M-k}) + i (X_k - conj X_{M-k}) conj(W_Nx^k),  z = IFFT_M(Z),  x_2n = Re z_n, x_2n+1 = Im z_n
// (unnormalised like cufftExecZ2D); the imaginary parts of X_0 and X_M are dropped, as the real part of the
// full complex inverse does; the result is divided by nxp*nzp.
template <typename T>
__global__ void __launch_bounds__(256) k_inv_x(PoissonArgs<T> a, int lx, const typename cplx_t<T>::type *__restrict__ spec,
                                               T *__restrict__ phi, FFTPlan p,
                                               const typename cplx_t<T>::type *__restrict__ tw,
                                               const typename cplx_t<T>::type *__restrict__ twr) {
    typedef typename cplx_t<T>::type C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Dims &d = a.d;
    const int M = d.Nx / 2;
    C *b0 = (C *)smem_raw, *b1 = b0 + (size_t)lx * M;
    const long long nlines_tot = (long long)d.Ny * d.Nz;
    const long long line0 = (long long)blockIdx.x * lx;
    const int nl = (int)min((long long)lx, nlines_tot - line0);
    for (int e = threadIdx.x; e < nl * M; e += blockDim.x) {
        int ll = e / M, kx = e - ll * M;
        const C *row = spec + (line0 + ll) * d.Nxc;
        C X = row[kx], Xm = row[M - kx];
        if (kx == 0) { X.y = T(0); Xm.y = T(0); }
        // E2 = X + conj(Xm), D2 = X - conj(Xm), O2 = D2 * conj(W^k)
        T E2r = X.x + Xm.x, E2i = X.y - Xm.y;
        T D2r = X.x - Xm.x, D2i = X.y + Xm.y;
        C w = __ldg(twr + kx);
        T O2r = D2r * w.x + D2i * w.y, O2i = D2i * w.x - D2r * w.y;
        C Z; Z.x = E2r - O2i; Z.y = E2i + O2r;
        b0[(size_t)ll * M + kx] = Z;
    }
    __syncthreads();
    C *res = fft_lines<T, true, false>(b0, b1, nl, M, 1, p, tw);
    const T *rr = (const T *)res;
    for (int e = threadIdx.x; e < nl * d.Nx; e += blockDim.x) {
        int ll = e / d.Nx, i = e - ll * d.Nx;
        T v = rr[(size_t)ll * d.Nx + i];
        T o;
        if (sizeof(T) == 8) o = (T)((double)v / a.norm);
        else o = v * (T)(1.0 / a.norm);
        phi[(line0 + ll) * d.Nx + i] = o;
    }
}

// ---- 5. project_velocity (src/projection.f90:551-604) and the stage-3 pressure save --------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_correct(PoissonArgs<T> a, const T *__restrict__ phi, const T *__restrict__ us,
                                                 const T *__restrict__ vs, const T *__restrict__ ws, T *__restrict__ U,
                                                 T *__restrict__ V, T *__restrict__ W, T *__restrict__ P) {
    typedef Arith<T> A;
    const Dims &d = a.d;
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= d.Nx || j >= d.Ny) return;
    long long p = idx3(d, i, j, k);
    T pc = __ldg(phi + p);
    T pxp = __ldg(phi + idx3(d, wrap(i + 1, d.Nx), j, k));
    T pzp = __ldg(phi + idx3(d, i, j, wrap(k + 1, d.Nz)));
    U[p] = us[p] - (pxp - pc) * a.inv_dx;
    W[p] = ws[p] - (pzp - pc) * A::inv(a.mz.df, a.mz.idf, k);
    if (j < d.NyV) {
        T pyp = __ldg(phi + idx3(d, i, wrap(j + 1, d.Ny), k));
        V[p] = vs[p] - (pyp - pc) * A::inv(a.my.df, a.my.idf, j);
    }
    if (P) {
        if (sizeof(T) == 8) P[p] = (T)((double)pc / a.pdiv);
        else P[p] = pc * (T)(1.0 / a.pdiv);
    }
}

// phi <- real field for the unit Poisson entry point: nothing to do (k_fwd_x<T,false> reads it directly).

}  // namespace dfdm
