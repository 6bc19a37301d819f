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
    double norm;              // nxp*nzp
    double pdiv;              // dt*rk_coef(3,3)
    const double *dtp;        // adaptive time step: pdiv = dtp[0]*rk_coef(3,3) from device memory (null: fixed dt)
    FastDiv fNx, fNy, fM, fM1;   // division by Nx, Ny, Nx/2, Nx/2+1
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
    pdl_enter();
    typedef typename cplx_t<T>::type C;
    typedef Arith<T> A;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Dims &d = a.d;
    const int Nx = d.Nx, Ny = d.Ny, Nz = d.Nz, M = Nx / 2, plane = Nx * Ny;
    C *b0 = (C *)smem_raw, *b1 = b0 + lx * M;
    const int nlines_tot = Ny * Nz;
    const int line0 = blockIdx.x * lx;
    const int nl = min(lx, nlines_tot - line0);
    T *r0 = (T *)b0;
    for (int e = threadIdx.x; e < nl * Nx; e += blockDim.x) {
        int ll = (int)fdiv((unsigned)e, a.fNx), i = e - ll * Nx;
        int line = line0 + ll;
        T val;
        if (FROM_DIV) {
            int k = (int)fdiv((unsigned)line, a.fNy), j = line - k * Ny;
            int o = k * plane + j * Nx + i;
            int oim = (i == 0) ? o + (Nx - 1) : o - 1;
            int okm = (k == 0) ? o + (Nz - 1) * plane : o - plane;
            T vjm;
            if (j > 0) vjm = __ldg(V + o - Nx);
            else vjm = d.yper ? __ldg(V + o + (Ny - 1) * Nx) : T(0);
            T inv_dyj = A::inv(a.my.dc, a.my.idc, j), inv_dzk = A::inv(a.mz.dc, a.mz.idc, k);
            val = (__ldg(U + o) - __ldg(U + oim)) * a.inv_dx + (__ldg(V + o) - vjm) * inv_dyj +
                  (__ldg(W + o) - __ldg(W + okm)) * inv_dzk;
        } else {
            val = src[line * Nx + i];
        }
        r0[ll * Nx + i] = val;
    }
    __syncthreads();
    C *res = fft_lines<T, false, false>(b0, b1, nl, M, 1, p, tw);
    const int Nxc = d.Nxc;
    for (int e = threadIdx.x; e < nl * (M + 1); e += blockDim.x) {
        int ll = (int)fdiv((unsigned)e, a.fM1), kx = e - ll * (M + 1);
        C Zk = res[ll * M + (kx == M ? 0 : kx)];
        C Zm = res[ll * M + (kx == 0 ? 0 : M - kx)];
        T Er = T(0.5) * (Zk.x + Zm.x), Ei = T(0.5) * (Zk.y - Zm.y);
        T Dr = T(0.5) * (Zk.x - Zm.x), Di = T(0.5) * (Zk.y + Zm.y);
        T Or = Di, Oi = -Dr;   // O = D / i
        C w = __ldg(twr + kx);
        C X;
        X.x = Er + (w.x * Or - w.y * Oi);
        X.y = Ei + (w.x * Oi + w.y * Or);
        spec[(line0 + ll) * Nxc + kx] = X;
    }
}

// ---- 2. transforms along z (and the periodic-y Poisson solve) on column tiles ---------------------------------
// A block loads TX consecutive kx columns of length L (rows at stride rowstride), transforms every column in
// shared memory and stores them back in place.
//   MODE 0: forward FFT along z (rows = kz, one block per (kx tile, j))
//   MODE 1: inverse FFT along z
//   MODE 2: periodic y (rows = j, one block per (kx tile, kz)): forward FFT, divide by kxx+kyy+kzz with the
//           (0,0,0) mode set to zero, inverse FFT, divide by nyp (src/projection.f90:246-273)
template <typename T, int MODE, int TX>
__global__ void __launch_bounds__(256) k_col_fft(Dims d, typename cplx_t<T>::type *__restrict__ spec, FFTPlan p,
                                                 const typename cplx_t<T>::type *__restrict__ tw,
                                                 const double *__restrict__ kxx, const double *__restrict__ kyy,
                                                 const double *__restrict__ kzz) {
    pdl_enter();
    typedef typename cplx_t<T>::type C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L = p.n;
    C *b0 = (C *)smem_raw, *b1 = b0 + L * TX;
    const int kx0 = blockIdx.x * TX;
    const int other = blockIdx.y;
    const int Nxc = d.Nxc;
    int base, rowstride;
    if (MODE == 2) { base = other * d.Ny * Nxc; rowstride = Nxc; }
    else { base = other * Nxc; rowstride = d.Ny * Nxc; }
    for (int e = threadIdx.x; e < L * TX; e += blockDim.x) {
        int row = e / TX, c = e % TX, kx = kx0 + c;
        C v = mkc<T>(T(0), T(0));
        if (kx < Nxc) v = spec[base + row * rowstride + kx];
        b0[e] = v;
    }
    __syncthreads();
    C *res;
    if (MODE == 0) res = fft_lines<T, false, true, TX>(b0, b1, TX, 1, TX, p, tw);
    else if (MODE == 1) res = fft_lines<T, true, true, TX>(b0, b1, TX, 1, TX, p, tw);
    else {
        res = fft_lines<T, false, true, TX>(b0, b1, TX, 1, TX, p, tw);
        const int kz = other;
        for (int e = threadIdx.x; e < L * TX; e += blockDim.x) {
            int j = e / TX, c = e % TX, kx = kx0 + c;
            if (kx >= Nxc) continue;
            double wavenum_sum = kxx[kx] + kyy[j] + kzz[kz];
            C v = res[e];
            if (kx == 0 && j == 0 && kz == 0) { v.x = T(0); v.y = T(0); }
            else { v.x = (T)((double)v.x / wavenum_sum); v.y = (T)((double)v.y / wavenum_sum); }
            res[e] = v;
        }
        __syncthreads();
        C *other_buf = (res == b0) ? b1 : b0;
        res = fft_lines<T, true, true, TX>(res, other_buf, TX, 1, TX, p, tw);
        const double nyp = (double)L;
        for (int e = threadIdx.x; e < L * TX; e += blockDim.x) {
            C v = res[e];
            v.x = (T)((double)v.x / nyp); v.y = (T)((double)v.y / nyp);
            res[e] = v;
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < L * TX; e += blockDim.x) {
        int row = e / TX, c = e % TX, kx = kx0 + c;
        if (kx < Nxc) spec[base + row * rowstride + kx] = res[e];
    }
}

// ---- 3. wall-bounded y: one tridiagonal system per (kx, kz) ----------------------------------------------------
// (Dyy + kxx + kzz) phi = r with the (0,0) row D(2) scaled by 3/2 (src/projection.f90:275-297, GPU
// src/poisson_gpu.f90:445-489), solved by the no-interchange branch of LAPACK zgtsv in double.  The
// elimination pivots D(r) depend only on the mode, so 1/D(r) is tabulated once at set-up (table layout
// (kz, r, kx), double); each solve is then a pair of division-free recurrences
//   b'(r) = b(r) - m(r) b'(r-1),  m(r) = DL(r-1)/D(r-1)          (forward, b' written back in place)
//   x(n-1) = b'(n-1)/D(n-1),  x(r) = (b'(r) - DU(r) x(r+1))/D(r)  (backward)
// The pressure operator is similar to a symmetric negative-definite matrix once the null mode is pinned, so
// elimination without interchanges is stable.  One thread owns one (kx,kz) column and a warp covers 32
// consecutive kx, so every row access is coalesced.  Each sweep keeps two register buffers of CH rows and issues
// the loads of the next chunk before the recurrence of the current one runs, and the per-row coefficients DL and
// DU are read from shared memory.
template <typename T, int CH, class BC>
__device__ __forceinline__ void k_ysolve2_body(const BC &bc, const Dims &d, typename cplx_t<T>::type *__restrict__ spec,
                                                const double *__restrict__ rpiv, const double *__restrict__ lo,
                                                const double *__restrict__ up) {
    typedef typename cplx_t<T>::type C;
    extern __shared__ double sco[];   // DL at [0, n), DU at [n, 2n)
    const int Nxc = d.Nxc, n = d.Ny;
    for (int r = threadIdx.x; r < n; r += blockDim.x) { sco[r] = lo[r]; sco[n + r] = up[r]; }
    __syncthreads();
    const int kx = bc.idx().x * blockDim.x + threadIdx.x, kz = bc.idx().y;
    if (kx >= Nxc) return;
    C *col = spec + kz * n * Nxc + kx;
    const double *rp = rpiv + kz * n * Nxc + kx;
    const double *slo = sco, *sup = sco + n;
    C va[CH], vb[CH];
    double ra[CH], rb[CH];
    auto fload = [&](C *v, double *rv, int r0) {
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            const int r = r0 + q;
            if (r < n) { v[q] = col[r * Nxc]; rv[q] = __ldg(rp + r * Nxc); }
        }
    };
    C v0 = col[0];
    double br = (double)v0.x, bi = (double)v0.y, rprev = __ldg(rp);
    auto fproc = [&](const C *v, const double *rv, int r0) {
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            const int r = r0 + q;
            if (r < n) {
                const double m = slo[r] * rprev;
                br = (double)v[q].x - m * br;
                bi = (double)v[q].y - m * bi;
                if (r < n - 1) { C o; o.x = (T)br; o.y = (T)bi; col[r * Nxc] = o; }
                rprev = rv[q];
            }
        }
    };
    fload(va, ra, 1);
    for (int r0 = 1; r0 < n; r0 += 2 * CH) {
        if (r0 + CH < n) fload(vb, rb, r0 + CH);
        fproc(va, ra, r0);
        if (r0 + CH >= n) break;
        if (r0 + 2 * CH < n) fload(va, ra, r0 + 2 * CH);
        fproc(vb, rb, r0 + CH);
    }
    double xr = br * rprev, xi = bi * rprev;
    {
        C o; o.x = (T)xr; o.y = (T)xi;
        col[(n - 1) * Nxc] = o;
    }
    auto bload = [&](C *v, double *rv, int r0) {
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            const int r = r0 - q;
            if (r >= 0) { v[q] = col[r * Nxc]; rv[q] = __ldg(rp + r * Nxc); }
        }
    };
    auto bproc = [&](const C *v, const double *rv, int r0) {
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            const int r = r0 - q;
            if (r >= 0) {
                xr = ((double)v[q].x - sup[r] * xr) * rv[q];
                xi = ((double)v[q].y - sup[r] * xi) * rv[q];
                C o; o.x = (T)xr; o.y = (T)xi;
                col[r * Nxc] = o;
            }
        }
    };
    bload(va, ra, n - 2);
    for (int r0 = n - 2; r0 >= 0; r0 -= 2 * CH) {
        if (r0 - CH >= 0) bload(vb, rb, r0 - CH);
        bproc(va, ra, r0);
        if (r0 - CH < 0) break;
        if (r0 - 2 * CH >= 0) bload(va, ra, r0 - 2 * CH);
        bproc(vb, rb, r0 - CH);
    }
}
template <typename T, int CH>
__global__ void __launch_bounds__(64) k_ysolve2(Dims d, typename cplx_t<T>::type *__restrict__ spec,
                                                const double *__restrict__ rpiv, const double *__restrict__ lo,
                                                const double *__restrict__ up) {
    pdl_enter();
    k_ysolve2_body<T, CH>(HwBlock(), d, spec, rpiv, lo, up);
}

// The same solve with whole columns staged in shared memory.  k_ysolve2's sweeps wait for one HBM latency per chunk
// of CH rows (2 n / CH waits per column), with too few columns per SM to hide them, and write b' to global memory
// and read it back.  Here a block owns YS_COLS
// consecutive columns of the flattened (kz, kx) index, one thread each; it issues the cp.async copies of all n rows
// of its columns' spectrum and pivots at once (one latency per block), runs both recurrences from shared memory
// (b' rounded to the storage type in place, as k_ysolve2 stores it) and writes each row of x once.  The arithmetic
// is k_ysolve2's, operation for operation.  Shared memory: n * YS_COLS * (sizeof(C) + 8) + 16 n bytes, so that only
// as many columns sweep at once on an SM as their rows fit: the library uses it where at least three blocks fit
// (in FP32 up to Ny ~ 140), k_ysolve2 above.  The grouped launch (kernels_group.cuh) always uses it.
constexpr int YS_COLS = 32;
template <typename T> __host__ __device__ constexpr size_t ysolve3_smem(int n) {
    return (size_t)n * YS_COLS * (sizeof(typename cplx_t<T>::type) + sizeof(double)) + (size_t)2 * n * sizeof(double);
}
template <typename T, class BC>
__device__ __forceinline__ void k_ysolve3_body(const BC &bc, const Dims &d, typename cplx_t<T>::type *__restrict__ spec,
                                                const double *__restrict__ rpiv, const double *__restrict__ lo,
                                                const double *__restrict__ up) {
    typedef typename cplx_t<T>::type C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int Nxc = d.Nxc, n = d.Ny;
    double *piv = reinterpret_cast<double *>(smem_raw);         // [r * YS_COLS + lane]
    double *sco = piv + (size_t)n * YS_COLS;                       // DL at [0, n), DU at [n, 2n)
    C *v = reinterpret_cast<C *>(sco + 2 * n);                     // [r * YS_COLS + lane]
    const int lane = threadIdx.x;
    const int c = bc.idx().x * YS_COLS + lane;
    const bool own = c < Nxc * d.Nz;
    const int kz = own ? c / Nxc : 0, kx = own ? c - kz * Nxc : 0;
    C *col = spec + (size_t)kz * n * Nxc + kx;
    const double *rp = rpiv + (size_t)kz * n * Nxc + kx;
    if (own) {
        for (int r = 0; r < n; ++r) {
            cp_async<sizeof(C)>(v + r * YS_COLS + lane, col + (size_t)r * Nxc);
            cp_async<8>(piv + r * YS_COLS + lane, rp + (size_t)r * Nxc);
        }
    }
    cp_async_commit();
    for (int r = lane; r < n; r += YS_COLS) { sco[r] = lo[r]; sco[n + r] = up[r]; }
    cp_async_wait_all();
    __syncthreads();
    if (!own) return;
    const double *slo = sco, *sup = sco + n;
    C v0 = v[lane];
    double br = (double)v0.x, bi = (double)v0.y, rprev = piv[lane];
#pragma unroll 4
    for (int r = 1; r < n; ++r) {
        const C x = v[r * YS_COLS + lane];
        const double m = slo[r] * rprev;
        br = (double)x.x - m * br;
        bi = (double)x.y - m * bi;
        C o; o.x = (T)br; o.y = (T)bi;
        v[r * YS_COLS + lane] = o;
        rprev = piv[r * YS_COLS + lane];
    }
    double xr = br * rprev, xi = bi * rprev;
    {
        C o; o.x = (T)xr; o.y = (T)xi;
        col[(size_t)(n - 1) * Nxc] = o;
    }
#pragma unroll 4
    for (int r = n - 2; r >= 0; --r) {
        const C x = v[r * YS_COLS + lane];
        const double rv = piv[r * YS_COLS + lane];
        xr = ((double)x.x - sup[r] * xr) * rv;
        xi = ((double)x.y - sup[r] * xi) * rv;
        C o; o.x = (T)xr; o.y = (T)xi;
        col[(size_t)r * Nxc] = o;
    }
}
template <typename T>
__global__ void __launch_bounds__(YS_COLS) k_ysolve3(Dims d, typename cplx_t<T>::type *__restrict__ spec,
                                                     const double *__restrict__ rpiv, const double *__restrict__ lo,
                                                     const double *__restrict__ up) {
    pdl_enter();
    k_ysolve3_body<T>(HwBlock(), d, spec, rpiv, lo, up);
}

// ---- inflow/outflow x: the DCT-IV path of the pressure solve (src/projection.f90:124-130,334-343; GPU
// src/poisson_gpu.f90:139-226) -------------------------------------------------------------------------------------
// The real DCT-IV of every x line, Y_k = 2 sum_n x_n cos(pi (2n+1)(2k+1) / (4N)) (FFTW REDFT11, which the reference's
// CPU build plans and its GPU build forms through a zero-padded 4N-point FFT), as a product with the N x N matrix
// C[k][n] of those coefficients (symmetric; built on the host in FP64 with the angle reduced exactly, stored in the
// context's precision T).  N = nx - 1 is odd and can be prime (257), so the matrix product replaces a fast transform.
// A block stages DCT_LINES lines in shared memory as [n][line] (the lines' values at one n contiguous, read as
// vectors at one address by every thread of a warp); thread t < N produces output t of all of them, reading row n of
// C at consecutive t (coalesced, through L1) and accumulating in T.  Forward: x lines (the real field, x fastest) to
// the spectrum's kx columns (imaginary parts zero, kx = 0..N-1); inverse: the real parts of the spectrum's lines to
// the real field, times 1 / (2 N nzp) (the DCT-IV is its own inverse up to 2N).
constexpr int DCT_LINES = 16, DCT_NMAX = 257, DCT_THREADS = 288;   // lines per block; the longest line; threads
static_assert(DCT_THREADS >= (DCT_NMAX + 31) / 32 * 32, "one thread per output of the longest line");
template <typename T> struct DctVec;
template <> struct DctVec<float> { typedef float4 type; static constexpr int W = 4; };
template <> struct DctVec<double> { typedef double2 type; static constexpr int W = 2; };
template <typename T>
__device__ __forceinline__ void dct_accumulate(T cv, const T *__restrict__ v, T (&acc)[DCT_LINES]) {
    typedef typename DctVec<T>::type V;
    constexpr int W = DctVec<T>::W;
#pragma unroll
    for (int q = 0; q < DCT_LINES / W; ++q) {
        const V x = reinterpret_cast<const V *>(v)[q];
        const T *xs = reinterpret_cast<const T *>(&x);
#pragma unroll
        for (int w = 0; w < W; ++w) acc[q * W + w] = fma(cv, xs[w], acc[q * W + w]);
    }
}
// acc[l] += sum_n col[n * N] * ln[n][l]: the column's coefficients are loaded DCT_AHEAD at a time, one group ahead of
// the group being accumulated (the matrix is shared by every block and mostly served by L1).
constexpr int DCT_AHEAD = 8;
template <typename T>
__device__ __forceinline__ void dct_column(const T *__restrict__ col, int N, const T *__restrict__ ln, T (&acc)[DCT_LINES]) {
    T ca[DCT_AHEAD], cb[DCT_AHEAD];
    auto load = [&](T (&c)[DCT_AHEAD], int n0) {
#pragma unroll
        for (int q = 0; q < DCT_AHEAD; ++q) c[q] = __ldg(col + (size_t)(n0 + q) * N);
    };
    auto proc = [&](const T (&c)[DCT_AHEAD], int n0) {
#pragma unroll
        for (int q = 0; q < DCT_AHEAD; ++q) dct_accumulate<T>(c[q], ln + (n0 + q) * DCT_LINES, acc);
    };
    const int full = N / DCT_AHEAD * DCT_AHEAD;
    int n0 = 0;
    if (full > 0) load(ca, 0);
    for (; n0 + 2 * DCT_AHEAD <= full; n0 += 2 * DCT_AHEAD) {
        load(cb, n0 + DCT_AHEAD);
        proc(ca, n0);
        if (n0 + 2 * DCT_AHEAD < full) load(ca, n0 + 2 * DCT_AHEAD);
        proc(cb, n0 + DCT_AHEAD);
    }
    if (n0 < full) { proc(ca, n0); n0 += DCT_AHEAD; }
    for (; n0 < N; ++n0) dct_accumulate<T>(__ldg(col + (size_t)n0 * N), ln + n0 * DCT_LINES, acc);
}
template <typename T>
__global__ void __launch_bounds__(DCT_THREADS) k_dct_x(Dims d, const T *__restrict__ src, const T *__restrict__ C,
                                                       typename cplx_t<T>::type *__restrict__ spec) {
    pdl_enter();
    __shared__ __align__(16) T ln[DCT_LINES * DCT_NMAX];
    const int N = d.Nx, nlines = d.Ny * d.Nz;
    const int line0 = blockIdx.x * DCT_LINES, nl = min(DCT_LINES, nlines - line0);
    for (int e = threadIdx.x; e < DCT_LINES * N; e += blockDim.x) {
        const int l = e / N, n = e - l * N;
        ln[n * DCT_LINES + l] = l < nl ? src[(size_t)(line0 + l) * N + n] : T(0);
    }
    __syncthreads();
    const int k = threadIdx.x;
    if (k >= N) return;
    T acc[DCT_LINES];
#pragma unroll
    for (int l = 0; l < DCT_LINES; ++l) acc[l] = T(0);
    dct_column<T>(C + k, N, ln, acc);
#pragma unroll
    for (int l = 0; l < DCT_LINES; ++l)
        if (l < nl) spec[(size_t)(line0 + l) * N + k] = mkc<T>(acc[l], T(0));
}
template <typename T>
__global__ void __launch_bounds__(DCT_THREADS) k_idct_x(Dims d, const typename cplx_t<T>::type *__restrict__ spec,
                                                        const T *__restrict__ C, T inv_norm, T *__restrict__ dst) {
    pdl_enter();
    __shared__ __align__(16) T ln[DCT_LINES * DCT_NMAX];
    const int N = d.Nx, nlines = d.Ny * d.Nz;
    const int line0 = blockIdx.x * DCT_LINES, nl = min(DCT_LINES, nlines - line0);
    for (int e = threadIdx.x; e < DCT_LINES * N; e += blockDim.x) {
        const int l = e / N, k = e - l * N;
        ln[k * DCT_LINES + l] = l < nl ? spec[(size_t)(line0 + l) * N + k].x : T(0);
    }
    __syncthreads();
    const int n = threadIdx.x;
    if (n >= N) return;
    T acc[DCT_LINES];
#pragma unroll
    for (int l = 0; l < DCT_LINES; ++l) acc[l] = T(0);
    dct_column<T>(C + n, N, ln, acc);
#pragma unroll
    for (int l = 0; l < DCT_LINES; ++l)
        if (l < nl) dst[(size_t)(line0 + l) * N + n] = acc[l] * inv_norm;
}
// The solved field back into rhs_p's shape for the Poisson-only contexts.  x: with periodic x (xwrap) the copies of
// apply_periodic_xz_pressure (rhs_p(nxg-1) = rhs_p(2)) and of the next wrap for the plane nxg, as k_pack_rhs_p
// writes them; with inflow/outflow x the plane nxg is left alone.  z: with periodic z (zwrap) the copy
// rhs_p(:, :, nzp+2) = rhs_p(:, :, 2); with z walls no copy.  Points left alone keep the input the caller passed,
// which the staging buffer still holds.
template <typename T>
__global__ void __launch_bounds__(256) k_pack_rhs_p_bc(Dims d, int n1, int n2, int n3, int xwrap, int zwrap,
                                                       const T *__restrict__ f, double *__restrict__ out) {
    pdl_enter();
    long long n = (long long)n1 * n2 * n3;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        int i = (int)(p % n1);
        const long long q = p / n1;
        const int j = (int)(q % n2);
        int k = (int)(q / n2);
        if (k < d.Nz && i >= d.Nx) {
            if (!xwrap) continue;
            i %= d.Nx;
        }
        if (k >= d.Nz) {
            if (!zwrap) {
                // a z wall leaves the plane nzg alone, except for the x copy rhs_p(nxg-1) = rhs_p(2), which covers
                // every z plane: the input at i = 0, which nothing writes at this k
                if (xwrap && i == d.Nx) out[p] = out[p - d.Nx];
                continue;
            }
            if (k > d.Nz) continue;
            k = 0;
            if (i >= d.Nx) {
                if (!xwrap) continue;
                i %= d.Nx;
            }
        }
        out[p] = (double)f[((long long)k * d.Ny + j) * d.Nx + i];
    }
}

// ---- spanwise walls alone (z walls, periodic x and y; src/projection.f90:136-143,219-250,310-316) -------------------
// The operator is the channel's with y and z exchanged, so the context stores the field as [y][z][x] (Dims: Ny = the
// nz - 1 wall-bounded z cells, Nz = the nyp periodic y rows) and runs the channel's chain unchanged: x FFT, FFT along
// the periodic axis, one tridiagonal solve per (kx, ky) along the wall axis, and the inverses.  rhs_p (x, y, z) ->
// the swapped field:
template <typename T>
__global__ void __launch_bounds__(256) k_unpack_rhs_p_swap(Dims d, int n1, int n2, const double *__restrict__ in,
                                                           T *__restrict__ f) {
    pdl_enter();
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < d.cells; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % d.Nx);
        const long long q = p / d.Nx;
        const int kz = (int)(q % d.Ny), jy = (int)(q / d.Ny);
        f[p] = (T)in[((long long)kz * n2 + jy) * n1 + i];
    }
}
// ... and back into rhs_p's shape with the reference's copies: x (rhs_p(nxg-1) = rhs_p(2); the plane nxg as the next
// wrap, as k_pack_rhs_p writes it), then y (rhs_p(:, nyg-1, :) = rhs_p(:, 2, :)), both over every z plane; the wall
// plane nzg is otherwise left as passed.  On that plane each copy reads a point that no thread writes.
template <typename T>
__global__ void __launch_bounds__(256) k_pack_rhs_p_swap(Dims d, int n1, int n2, int n3, const T *__restrict__ f,
                                                         double *__restrict__ out) {
    pdl_enter();
    const long long n = (long long)n1 * n2 * n3;
    const int nyp = d.Nz;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % n1);
        const long long q = p / n1;
        const int j = (int)(q % n2), k = (int)(q / n2);
        if (k < d.Ny) {
            const int ii = i % d.Nx, jj = j % nyp;
            out[p] = (double)f[((long long)jj * d.Ny + k) * d.Nx + ii];
        } else {
            const int si = i == d.Nx ? 0 : i, sj = j == nyp ? 0 : j;
            if (si != i || sj != j) out[p] = out[((long long)k * n2 + sj) * n1 + si];
        }
    }
}

// ---- the 4-wall duct (z walls with y walls; src/projection.f90:172-217, GPU src/poisson_gpu.f90:498-589) ----------
// The z-eigenmode transform: out[m][col] = sum_k M[k][m] in[k][col] over the spectrum's columns col = j Nxc + kx
// (z is the slowest index, so each k is one contiguous row of Ny Nxc complex values).  Forward, M[k][m] =
// Qz(k,m) sqrt(w_k) (projection onto the orthonormal eigenbasis of S = W^(1/2) Dzz W^(-1/2) after scaling by the
// square root of the cell width); inverse, M[m][k] = Qz(k,m) / sqrt(w_k), times nzp so that the inverse x kernel's
// division by nxp nzp leaves the 1/nxp of a solve in physical z.  A block takes ZEIG_COLS columns and
// zeig_modes<T>() outputs m, with its slice of M in shared memory; each thread walks its column down k (coalesced
// rows), so the rows are read Nz / zeig_modes times, from L2.
constexpr int ZEIG_NMAX = 512, ZEIG_COLS = 128;
template <typename T> __host__ __device__ constexpr int zeig_modes() { return sizeof(T) == 4 ? 16 : 8; }   // outputs m per block
template <typename T>
__global__ void __launch_bounds__(ZEIG_COLS) k_zeig(Dims d, const typename cplx_t<T>::type *__restrict__ in,
                                                    typename cplx_t<T>::type *__restrict__ out, const T *__restrict__ M) {
    pdl_enter();
    constexpr int RM = zeig_modes<T>();
    __shared__ __align__(16) T ms[ZEIG_NMAX * RM];
    const int n = d.Nz, m0 = blockIdx.y * RM;
    const long long cols = (long long)d.Ny * d.Nxc;
    for (int e = threadIdx.x; e < n * RM; e += blockDim.x) {
        const int k = e / RM, q = e - k * RM;
        ms[e] = m0 + q < n ? M[(size_t)k * n + m0 + q] : T(0);
    }
    __syncthreads();
    const long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= cols) return;
    T ar[RM], ai[RM];
#pragma unroll
    for (int q = 0; q < RM; ++q) { ar[q] = T(0); ai[q] = T(0); }
    for (int k = 0; k < n; ++k) {
        const typename cplx_t<T>::type v = in[(size_t)k * cols + col];
        T mk[RM];
#pragma unroll
        for (int q = 0; q < RM; q += 16 / sizeof(T)) {   // the row's coefficients as 16-byte broadcast loads
            typedef typename std::conditional<sizeof(T) == 4, float4, double2>::type V;
            const V w = *reinterpret_cast<const V *>(ms + k * RM + q);
            const T *ws = reinterpret_cast<const T *>(&w);
#pragma unroll
            for (int u = 0; u < (int)(16 / sizeof(T)); ++u) mk[q + u] = ws[u];
        }
#pragma unroll
        for (int q = 0; q < RM; ++q) {
            ar[q] = fma(mk[q], v.x, ar[q]);
            ai[q] = fma(mk[q], v.y, ai[q]);
        }
    }
#pragma unroll
    for (int q = 0; q < RM; ++q)
        if (m0 + q < n) out[(size_t)(m0 + q) * cols + col] = mkc<T>(ar[q], ai[q]);
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
    pdl_enter();
    typedef typename cplx_t<T>::type C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Dims &d = a.d;
    const int Nx = d.Nx, M = Nx / 2, Nxc = d.Nxc;
    C *b0 = (C *)smem_raw, *b1 = b0 + lx * M;
    const int nlines_tot = d.Ny * d.Nz;
    const int line0 = blockIdx.x * lx;
    const int nl = min(lx, nlines_tot - line0);
    for (int e = threadIdx.x; e < nl * M; e += blockDim.x) {
        int ll = (int)fdiv((unsigned)e, a.fM), kx = e - ll * M;
        const C *row = spec + (line0 + ll) * Nxc;
        C X = row[kx], Xm = row[M - kx];
        if (kx == 0) { X.y = T(0); Xm.y = T(0); }
        // E2 = X + conj(Xm), D2 = X - conj(Xm), O2 = D2 * conj(W^k)
        T E2r = X.x + Xm.x, E2i = X.y - Xm.y;
        T D2r = X.x - Xm.x, D2i = X.y + Xm.y;
        C w = __ldg(twr + kx);
        T O2r = D2r * w.x + D2i * w.y, O2i = D2i * w.x - D2r * w.y;
        C Z; Z.x = E2r - O2i; Z.y = E2i + O2r;
        b0[ll * M + kx] = Z;
    }
    __syncthreads();
    C *res = fft_lines<T, true, false>(b0, b1, nl, M, 1, p, tw);
    const T *rr = (const T *)res;
    for (int e = threadIdx.x; e < nl * Nx; e += blockDim.x) {
        T v = rr[e];
        T o;
        if (sizeof(T) == 8) o = (T)((double)v / a.norm);
        else o = v * (T)(1.0 / a.norm);
        phi[line0 * Nx + e] = o;
    }
}

// ---- 5. project_velocity (src/projection.f90:551-604) and the stage-3 pressure save --------------------------
// With uo != NULL the stage buffers hold the increment du (FP32-mixed stage 3) and u* = uo + du is formed here,
// rounded exactly as the stage kernel would have rounded it.
template <typename T>
__global__ void __launch_bounds__(256) k_correct(PoissonArgs<T> a, const T *__restrict__ phi, const T *__restrict__ us,
                                                 const T *__restrict__ vs, const T *__restrict__ ws, T *__restrict__ U,
                                                 T *__restrict__ V, T *__restrict__ W, T *__restrict__ P,
                                                 const T *__restrict__ uo, const T *__restrict__ vo, const T *__restrict__ wo) {
    pdl_enter();
    typedef Arith<T> A;
    const Dims &d = a.d;
    const int Nx = d.Nx, Ny = d.Ny, Nz = d.Nz, plane = Nx * Ny;
    int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= Nx || j >= Ny) return;
    int p = k * plane + j * Nx + i;
    T pc = __ldg(phi + p);
    T pxp = __ldg(phi + (i == Nx - 1 ? p - (Nx - 1) : p + 1));
    T pzp = __ldg(phi + (k == Nz - 1 ? p - (Nz - 1) * plane : p + plane));
    T su = us[p], sw = ws[p];
    if (uo) { su = uo[p] + su; sw = wo[p] + sw; }
    U[p] = su - (pxp - pc) * a.inv_dx;
    W[p] = sw - (pzp - pc) * A::inv(a.mz.df, a.mz.idf, k);
    if (j < d.NyV) {
        T pyp = __ldg(phi + (j == Ny - 1 ? p - (Ny - 1) * Nx : p + Nx));
        T sv = vs[p];
        if (uo) sv = vo[p] + sv;
        V[p] = sv - (pyp - pc) * A::inv(a.my.df, a.my.idf, j);
    }
    if (P) {
        const double pdiv = a.dtp ? *a.dtp * (3.0 / 4.0) : a.pdiv;
        if (sizeof(T) == 8) P[p] = (T)((double)pc / pdiv);
        else P[p] = pc * (T)(1.0 / pdiv);
    }
}

// Same correction, four consecutive x cells per thread with 16-byte (FP32) / 2x16-byte (FP64) accesses; needs
// Nx % 4 == 0.  One block row covers 64 x 4 cells of one (j,k) line pair.
template <typename T> struct Vec4;
template <> struct Vec4<float> { typedef float4 type; };
template <> struct Vec4<double> { typedef double4 type; };

template <typename T, class BC>
__device__ __forceinline__ void k_correct4_body(const BC &bc, const PoissonArgs<T> &a, const T *__restrict__ phi, const T *__restrict__ us,
                                                  const T *__restrict__ vs, const T *__restrict__ ws, T *__restrict__ U,
                                                  T *__restrict__ V, T *__restrict__ W, T *__restrict__ P,
                                                  const T *__restrict__ uo, const T *__restrict__ vo, const T *__restrict__ wo) {
    typedef typename Vec4<T>::type V4;
    typedef Arith<T> A;
    const Dims &d = a.d;
    const int Nx = d.Nx, Ny = d.Ny, Nz = d.Nz, plane = Nx * Ny, nq = Nx >> 2;
    const int iq = bc.idx().x * blockDim.x + threadIdx.x;
    const int j = bc.idx().y * blockDim.y + threadIdx.y, k = bc.idx().z;
    if (iq >= nq || j >= Ny) return;
    const int i = iq << 2;
    const int p = k * plane + j * Nx + i;
    const V4 pc = *reinterpret_cast<const V4 *>(phi + p);
    const T pnext = __ldg(phi + (i + 4 == Nx ? p + 4 - Nx : p + 4));
    const V4 pz = *reinterpret_cast<const V4 *>(phi + (k == Nz - 1 ? p - (Nz - 1) * plane : p + plane));
    const T idx = a.inv_dx, idz = A::inv(a.mz.df, a.mz.idf, k);
    V4 u = *reinterpret_cast<const V4 *>(us + p), w = *reinterpret_cast<const V4 *>(ws + p);
    if (uo) {   // increment form: u* = uo + du, rounded as the stage kernel rounds it
        const V4 bu = *reinterpret_cast<const V4 *>(uo + p), bw = *reinterpret_cast<const V4 *>(wo + p);
        u.x = bu.x + u.x; u.y = bu.y + u.y; u.z = bu.z + u.z; u.w = bu.w + u.w;
        w.x = bw.x + w.x; w.y = bw.y + w.y; w.z = bw.z + w.z; w.w = bw.w + w.w;
    }
    u.x = u.x - (pc.y - pc.x) * idx; u.y = u.y - (pc.z - pc.y) * idx;
    u.z = u.z - (pc.w - pc.z) * idx; u.w = u.w - (pnext - pc.w) * idx;
    w.x = w.x - (pz.x - pc.x) * idz; w.y = w.y - (pz.y - pc.y) * idz;
    w.z = w.z - (pz.z - pc.z) * idz; w.w = w.w - (pz.w - pc.w) * idz;
    *reinterpret_cast<V4 *>(U + p) = u;
    *reinterpret_cast<V4 *>(W + p) = w;
    if (j < d.NyV) {
        const V4 py = *reinterpret_cast<const V4 *>(phi + (j == Ny - 1 ? p - (Ny - 1) * Nx : p + Nx));
        const T idy = A::inv(a.my.df, a.my.idf, j);
        V4 v = *reinterpret_cast<const V4 *>(vs + p);
        if (vo) {
            const V4 bv = *reinterpret_cast<const V4 *>(vo + p);
            v.x = bv.x + v.x; v.y = bv.y + v.y; v.z = bv.z + v.z; v.w = bv.w + v.w;
        }
        v.x = v.x - (py.x - pc.x) * idy; v.y = v.y - (py.y - pc.y) * idy;
        v.z = v.z - (py.z - pc.z) * idy; v.w = v.w - (py.w - pc.w) * idy;
        *reinterpret_cast<V4 *>(V + p) = v;
    }
    if (P) {
        V4 o;
        const double pdiv = a.dtp ? *a.dtp * (3.0 / 4.0) : a.pdiv;
        if (sizeof(T) == 8) {
            o.x = (T)((double)pc.x / pdiv); o.y = (T)((double)pc.y / pdiv);
            o.z = (T)((double)pc.z / pdiv); o.w = (T)((double)pc.w / pdiv);
        } else {
            const T r = (T)(1.0 / pdiv);
            o.x = pc.x * r; o.y = pc.y * r; o.z = pc.z * r; o.w = pc.w * r;
        }
        *reinterpret_cast<V4 *>(P + p) = o;
    }
}
template <typename T>
__global__ void __launch_bounds__(256) k_correct4(PoissonArgs<T> a, const T *__restrict__ phi, const T *__restrict__ us,
                                                  const T *__restrict__ vs, const T *__restrict__ ws, T *__restrict__ U,
                                                  T *__restrict__ V, T *__restrict__ W, T *__restrict__ P,
                                                  const T *__restrict__ uo, const T *__restrict__ vo, const T *__restrict__ wo) {
    pdl_enter();
    k_correct4_body<T>(HwBlock(), a, phi, us, vs, ws, U, V, W, P, uo, vo, wo);
}

}  // namespace dfdm
