// kernels_fft2l.cuh -- the Poisson transforms for lengths with a two-level split (fft_reg.cuh).
//
// Same operations, inputs, outputs and rounding points as the Stockham kernels of kernels_poisson.cuh
// (k_fwd_x, k_col_fft, k_inv_x): only the transform itself is organised differently.  Step 1 of the z transforms
// and of the inverse x transform reads its operands straight from global memory (the inverse x kernel forms the
// packed half-length spectrum there), and their step 2 writes straight to global memory, so a line crosses shared
// memory once.  The forward x transform first forms the divergence pairs in shared memory with coalesced loads,
// and its real-to-complex unpacking pairs elements k and M-k through shared memory once more.
#pragma once

#include "fft_reg.cuh"
#include "kernels_poisson.cuh"

namespace dfdm {

template <typename T> struct Vec2;
template <> struct Vec2<float> { typedef float2 type; };
template <> struct Vec2<double> { typedef double2 type; };

// ---- div u* (or a real field) + forward real-to-complex x transform, line length Nx = 2M ----------------------
// Phase A forms the packed half-length line z_n = x_2n + i x_2n+1 in shared memory with consecutive threads on
// consecutive pairs (coalesced 8-byte loads of the velocity pairs); the two register steps follow.
template <typename T, bool FROM_DIV, int M, class BC>
__device__ __forceinline__ void k_fwd_x2_body(const BC &bc, const PoissonArgs<T> &a, int lx, const T *__restrict__ U, const T *__restrict__ V,
                                                const T *__restrict__ W, const T *__restrict__ src,
                                                typename cplx_t<T>::type *__restrict__ spec,
                                                const typename cplx_t<T>::type *__restrict__ tw,
                                                const typename cplx_t<T>::type *__restrict__ twr) {
    typedef typename cplx_t<T>::type C;
    typedef typename Vec2<T>::type T2;
    typedef Arith<T> A;
    constexpr int N1 = Split<M>::N1, N2 = Split<M>::N2, Nx = 2 * M;
    constexpr int LDA = RowLayout<M>::LDA, LDT = RowLayout<M>::LDT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *bt = (C *)smem_raw, *ba = bt + lx * LDT;
    const Dims &d = a.d;
    const int Ny = d.Ny, Nz = d.Nz, plane = Nx * Ny;
    // blocks run roughly in index order: the first take the highest lines (top z planes), which the stage kernel
    // wrote last and which are the likeliest to still be in L2
    const int line0 = (bc.dim().x - 1 - bc.idx().x) * lx;
    const int nl = min(lx, Ny * Nz - line0);
    constexpr int ITEMS = RowLines<T, M>::value * M;   // lx == RowLines<T, M>::value, blockDim.x == 256
    constexpr int PER = (ITEMS + 255) / 256, UNR = sizeof(T) == 4 ? 4 : 2;   // items per thread; items loaded together
    const int lim = nl * M;
#pragma unroll 1
    for (int b0 = 0; b0 < PER; b0 += UNR) {
        // all loads of UNR items first (predicated, no early exit), then their arithmetic
        T2 ru[UNR], rv[UNR], rvm[UNR], rw[UNR], rwm[UNR];
        T rum[UNR], riy[UNR], riz[UNR];
#pragma unroll
        for (int q = 0; q < UNR; ++q) {
            const int e = (b0 + q) * 256 + threadIdx.x;
            if (b0 + q < PER && e < lim) {
                const int ll = e / M, n = e - ll * M;
                const int line = line0 + ll;
                if (FROM_DIV) {
                    const int k = (int)fdiv((unsigned)line, a.fNy), j = line - k * Ny;
                    const int ob = k * plane + j * Nx, i = 2 * n, o = ob + i;
                    const int dkm = (k == 0) ? (Nz - 1) * plane : -plane;
                    const int djm = (j > 0) ? -Nx : (Ny - 1) * Nx;
                    const bool vzero = (j == 0) && !d.yper;
                    riy[q] = A::inv(a.my.dc, a.my.idc, j);
                    riz[q] = A::inv(a.mz.dc, a.mz.idc, k);
                    ru[q] = *reinterpret_cast<const T2 *>(U + o);
                    rum[q] = __ldg(U + (i == 0 ? ob + Nx - 1 : o - 1));
                    rv[q] = *reinterpret_cast<const T2 *>(V + o);
                    if (vzero) { rvm[q].x = T(0); rvm[q].y = T(0); }
                    else rvm[q] = *reinterpret_cast<const T2 *>(V + o + djm);
                    rw[q] = *reinterpret_cast<const T2 *>(W + o);
                    rwm[q] = *reinterpret_cast<const T2 *>(W + o + dkm);
                } else {
                    ru[q] = *reinterpret_cast<const T2 *>(src + (size_t)line * Nx + 2 * n);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < UNR; ++q) {
            const int e = (b0 + q) * 256 + threadIdx.x;
            if (b0 + q < PER && e < lim) {
                const int ll = e / M, n = e - ll * M;
                C z;
                if (FROM_DIV) {
                    const T2 u = ru[q], v = rv[q], vm = rvm[q], w = rw[q], wm = rwm[q];
                    z.x = (u.x - rum[q]) * a.inv_dx + (v.x - vm.x) * riy[q] + (w.x - wm.x) * riz[q];
                    z.y = (u.y - u.x) * a.inv_dx + (v.y - vm.y) * riy[q] + (w.y - wm.y) * riz[q];
                } else {
                    z.x = ru[q].x;
                    z.y = ru[q].y;
                }
                ba[ll * LDA + n] = z;
            }
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nl * N2; b += blockDim.x) {
        const int ll = b / N2, n2 = b - ll * N2;
        C v[N1];
        const C *al = ba + ll * LDA + n2;
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) v[n1] = al[n1 * N2];
        row_step1<T, false, M>(v, bt + ll * LDT, n2, tw);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nl * N1; b += blockDim.x) {
        const int ll = b / N1, k1 = b - ll * N1;
        C v[N2];
        const C *tl = bt + ll * LDT + k1 * (N2 + 1);
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) v[n2] = tl[n2];
        Codelet<T, false, N2>::run(v);
        C *al = ba + ll * LDA;
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) al[k1 + N1 * k2] = v[k2];
    }
    __syncthreads();
    const int Nxc = d.Nxc;
    for (int e = threadIdx.x; e < nl * (M + 1); e += blockDim.x) {
        const int ll = e / (M + 1), kx = e - ll * (M + 1);
        const C *res = ba + ll * LDA;
        C Zk = res[kx == M ? 0 : kx];
        C Zm = res[kx == 0 ? 0 : M - kx];
        T Er = T(0.5) * (Zk.x + Zm.x), Ei = T(0.5) * (Zk.y - Zm.y);
        T Dr = T(0.5) * (Zk.x - Zm.x), Di = T(0.5) * (Zk.y + Zm.y);
        T Or = Di, Oi = -Dr;
        C w = __ldg(twr + kx);
        C X;
        X.x = Er + (w.x * Or - w.y * Oi);
        X.y = Ei + (w.x * Oi + w.y * Or);
        spec[(size_t)(line0 + ll) * Nxc + kx] = X;
    }
}
template <typename T, bool FROM_DIV, int M>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2) k_fwd_x2(PoissonArgs<T> a, int lx, const T *__restrict__ U, const T *__restrict__ V,
                                                const T *__restrict__ W, const T *__restrict__ src,
                                                typename cplx_t<T>::type *__restrict__ spec,
                                                const typename cplx_t<T>::type *__restrict__ tw,
                                                const typename cplx_t<T>::type *__restrict__ twr) {
    pdl_enter();
    k_fwd_x2_body<T, FROM_DIV, M>(HwBlock(), a, lx, U, V, W, src, spec, tw, twr);
}

// ---- inverse complex-to-real x transform, writes phi = x / (nxp*nzp) -----------------------------------------
template <typename T, int M, class BC>
__device__ __forceinline__ void k_inv_x2_body(const BC &bc, const PoissonArgs<T> &a, int lx, const typename cplx_t<T>::type *__restrict__ spec,
                                                T *__restrict__ phi, const typename cplx_t<T>::type *__restrict__ tw,
                                                const typename cplx_t<T>::type *__restrict__ twr) {
    typedef typename cplx_t<T>::type C;
    typedef typename Vec2<T>::type T2;
    constexpr int N1 = Split<M>::N1, N2 = Split<M>::N2, Nx = 2 * M;
    constexpr int LDT = RowLayout<M>::LDT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *bt = (C *)smem_raw;
    const Dims &d = a.d;
    const int Nxc = d.Nxc;
    const int line0 = bc.idx().x * lx;
    const int nl = min(lx, d.Ny * d.Nz - line0);
    for (int b = threadIdx.x; b < nl * N2; b += blockDim.x) {
        const int ll = b / N2, n2 = b - ll * N2;
        const C *row = spec + (size_t)(line0 + ll) * Nxc;
        C v[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) {
            const int kx = n1 * N2 + n2;
            C X = row[kx], Xm = row[M - kx];
            if (kx == 0) { X.y = T(0); Xm.y = T(0); }
            T E2r = X.x + Xm.x, E2i = X.y - Xm.y;
            T D2r = X.x - Xm.x, D2i = X.y + Xm.y;
            C w = __ldg(twr + kx);
            T O2r = D2r * w.x + D2i * w.y, O2i = D2i * w.x - D2r * w.y;
            v[n1].x = E2r - O2i;
            v[n1].y = E2i + O2r;
        }
        row_step1<T, true, M>(v, bt + ll * LDT, n2, tw);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nl * N1; b += blockDim.x) {
        const int ll = b / N1, k1 = b - ll * N1;
        C v[N2];
        const C *tl = bt + ll * LDT + k1 * (N2 + 1);
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) v[n2] = tl[n2];
        Codelet<T, true, N2>::run(v);
        T2 *out = reinterpret_cast<T2 *>(phi + (size_t)(line0 + ll) * Nx);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
            T2 o;
            if (sizeof(T) == 8) { o.x = (T)((double)v[k2].x / a.norm); o.y = (T)((double)v[k2].y / a.norm); }
            else { o.x = v[k2].x * (T)(1.0 / a.norm); o.y = v[k2].y * (T)(1.0 / a.norm); }
            out[k1 + N1 * k2] = o;
        }
    }
}
template <typename T, int M>
__global__ void __launch_bounds__(256) k_inv_x2(PoissonArgs<T> a, int lx, const typename cplx_t<T>::type *__restrict__ spec,
                                                T *__restrict__ phi, const typename cplx_t<T>::type *__restrict__ tw,
                                                const typename cplx_t<T>::type *__restrict__ twr) {
    pdl_enter();
    k_inv_x2_body<T, M>(HwBlock(), a, lx, spec, phi, tw, twr);
}

// ---- z transforms (MODE 0 forward, 1 inverse) and the periodic-y solve (MODE 2) on tiles of NL kx columns ----
// MODE 2: forward FFT along y, division by kxx+kyy+kzz with the (0,0,0) mode set to zero, inverse FFT, division
// by nyp (src/projection.f90:246-273).
template <typename T, int MODE, int NL, int L>
__global__ void __launch_bounds__(256) k_col2(Dims d, typename cplx_t<T>::type *__restrict__ spec,
                                              const typename cplx_t<T>::type *__restrict__ tw,
                                              const double *__restrict__ kxx, const double *__restrict__ kyy,
                                              const double *__restrict__ kzz) {
    pdl_enter();
#define DFDM_BLOCK_IDX blockIdx
#include "k_col2_body.inc"
#undef DFDM_BLOCK_IDX
}

}  // namespace dfdm
