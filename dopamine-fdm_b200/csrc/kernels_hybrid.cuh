// kernels_hybrid.cuh -- advection_scheme = 2: the upwind-biased dissipation of src/adv_hybrid.f90.
//
// The skew-symmetric central convection of the stage kernels is kept and beta |u_c| D is added as a conservative flux
// difference, D the third difference / 12 (order 3) or minus the fifth difference / 60 (order 5) of the advected
// velocity across the face, with the face's convecting velocity u_c.  With no immersed body beta = adv_beta0
// everywhere.  One thread per cell computes the three components into out[0..cells), [cells..2 cells),
// [2 cells..3 cells); the stage kernels add them to their right-hand sides.
//
// Index conventions: device cell (i, j, k) is the reference's (i+2, j+2, k+2).  x and z are periodic (the padded
// copies of pad_field_dev, src/halo_pad.f90:185-240); in y the reference reads rows 1..nyg (U, W) or 1..ny (V) with
// clamped indices and reduces the order next to the ends (adv_ord_y), whatever the y boundary type.  Row values
// follow the ghost rules of apply_boundary_conditions: with walls, U and W mirror (-u of the first interior row)
// and V is zero on the wall faces; with periodic y every row wraps.
#pragma once

#include "dfdm_common.cuh"

namespace dfdm {

template <typename T> struct HybArgs {
    Dims d;
    T beta, inv_dx;
    Metric1D<T> my, mz;   // idc: 1/(face spacing around a centre); idf: 1/(centre spacing around a face)
    const T *ub;          // streamwise base profile by row (zeros in FP64)
};

template <int ORD> struct HybW;
template <> struct HybW<3> {
    template <typename T> static __device__ __forceinline__ T sum(T a, T b, T c, T d, T e, T f) {
        (void)a; (void)f;
        return (T(-1) * b + T(3) * c + T(-3) * d + T(1) * e) / T(12);
    }
};
template <> struct HybW<5> {
    template <typename T> static __device__ __forceinline__ T sum(T a, T b, T c, T d, T e, T f) {
        return (T(1) * a + T(-5) * b + T(10) * c + T(-10) * d + T(5) * e + T(-1) * f) / T(60);
    }
};

// adv_ord_y (src/adv_hybrid.f90:120-133): the order usable for the face between rows m and m+1 of 1..n
__device__ __forceinline__ int hyb_ord_y(int m, int n, int ord) {
    if (ord == 5 && m - 2 >= 1 && m + 3 <= n) return 5;
    if (m - 1 >= 1 && m + 2 <= n) return 3;
    return 0;
}

template <typename T>
__device__ __forceinline__ T hyb_wsum(int o, T a, T b, T c, T d, T e, T f) {
    if (o == 5) return HybW<5>::sum(a, b, c, d, e, f);
    if (o == 3) return HybW<3>::sum(a, b, c, d, e, f);
    return T(0);
}

template <typename T, int ORD>
__global__ void __launch_bounds__(256) k_adv_hybrid(HybArgs<T> h, const T *__restrict__ U, const T *__restrict__ V,
                                                    const T *__restrict__ W, T *__restrict__ out) {
    const Dims &d = h.d;
    const int Nx = d.Nx, Ny = d.Ny, Nz = d.Nz;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, k = blockIdx.z;
    if (i >= Nx || j >= Ny) return;
    const int nyg = d.yper ? Ny + 3 : Ny + 2, ny = d.yper ? Ny + 2 : Ny + 1;   // the reference's row counts
    // device row of reference row J for a y-centred field, with the wall mirror sign
    auto crow = [&](int J, T &sgn) -> int {
        sgn = T(1);
        if (d.yper) return wrap(J - 2, Ny);
        if (J <= 1) { sgn = T(-1); return 0; }
        if (J >= Ny + 2) { sgn = T(-1); return Ny - 1; }
        return J - 2;
    };
    auto at = [&](const T *F, int x, int r, int z) -> T {
        return __ldg(F + ((size_t)wrap(z, Nz) * Ny + r) * Nx + wrap(x, Nx));
    };
    // total U and W at reference row J (device x, z), the base profile added back and the ghost rules applied
    auto Ut = [&](int x, int J, int z) -> T {
        T s;
        const int r = crow(J, s);
        return s * (at(U, x, r, z) + h.ub[r]);
    };
    auto Wt = [&](int x, int J, int z) -> T {
        T s;
        const int r = crow(J, s);
        return s * at(W, x, r, z);
    };
    // V at reference face row J (1..ny): zero on the wall faces
    auto Vf = [&](int x, int J, int z) -> T {
        if (d.yper) return at(V, x, wrap(J - 2, Ny), z);
        if (J <= 1 || J >= Ny + 1) return T(0);
        return at(V, x, J - 2, z);
    };
    const int J = j + 2;
    const T beta = h.beta, idx = h.inv_dx;
    const size_t p = ((size_t)k * Ny + j) * Nx + i;

    // ---- u (adv_add_u, :136-176): stored deviations in x and z (the profile cancels), totals in y ----
    {
        const T dyj = h.my.idc[j], dzk = h.mz.idc[k];
        const T ubj = h.ub[j];
        T r = T(0);
#pragma unroll
        for (int m = 0; m <= 1; ++m) {
            const T sg = T(2 * m - 1);
            const int ii = i - 1 + m, jj = J - 1 + m, kk = k - 1 + m;
            T uc = T(0.5) * ((at(U, ii, j, k) + ubj) + (at(U, ii + 1, j, k) + ubj));
            T s = HybW<ORD>::sum(at(U, ii - 2, j, k), at(U, ii - 1, j, k), at(U, ii, j, k), at(U, ii + 1, j, k),
                                 at(U, ii + 2, j, k), at(U, ii + 3, j, k));
            r = r - sg * (beta * fabs(uc) * s) * idx;
            uc = T(0.5) * (Vf(i, jj, k) + Vf(i + 1, jj, k));
            s = hyb_wsum(hyb_ord_y(jj, nyg, ORD), Ut(i, max(jj - 2, 1), k), Ut(i, max(jj - 1, 1), k), Ut(i, jj, k),
                         Ut(i, jj + 1, k), Ut(i, min(jj + 2, nyg), k), Ut(i, min(jj + 3, nyg), k));
            r = r - sg * (beta * fabs(uc) * s) * dyj;
            uc = T(0.5) * (at(W, i, j, kk) + at(W, i + 1, j, kk));
            s = HybW<ORD>::sum(at(U, i, j, kk - 2), at(U, i, j, kk - 1), at(U, i, j, kk), at(U, i, j, kk + 1),
                               at(U, i, j, kk + 2), at(U, i, j, kk + 3));
            r = r - sg * (beta * fabs(uc) * s) * dzk;
        }
        out[p] = r;
    }
    // ---- v (adv_add_v, :179-219) ----
    if (j < d.NyV) {
        const T dyj = h.my.idf[j], dzk = h.mz.idc[k];
        T r = T(0);
#pragma unroll
        for (int m = 0; m <= 1; ++m) {
            const T sg = T(2 * m - 1);
            const int ii = i - 1 + m, jj = J - 1 + m, kk = k - 1 + m;
            T uc = T(0.5) * (Ut(ii, J, k) + Ut(ii, J + 1, k));
            T s = HybW<ORD>::sum(at(V, ii - 2, j, k), at(V, ii - 1, j, k), at(V, ii, j, k), at(V, ii + 1, j, k),
                                 at(V, ii + 2, j, k), at(V, ii + 3, j, k));
            r = r - sg * (beta * fabs(uc) * s) * idx;
            uc = T(0.5) * (Vf(i, jj, k) + Vf(i, jj + 1, k));
            s = hyb_wsum(hyb_ord_y(jj, ny, ORD), Vf(i, max(jj - 2, 1), k), Vf(i, max(jj - 1, 1), k), Vf(i, jj, k),
                         Vf(i, jj + 1, k), Vf(i, min(jj + 2, ny), k), Vf(i, min(jj + 3, ny), k));
            r = r - sg * (beta * fabs(uc) * s) * dyj;
            uc = T(0.5) * (Wt(i, J, kk) + Wt(i, J + 1, kk));
            s = HybW<ORD>::sum(at(V, i, j, kk - 2), at(V, i, j, kk - 1), at(V, i, j, kk), at(V, i, j, kk + 1),
                               at(V, i, j, kk + 2), at(V, i, j, kk + 3));
            r = r - sg * (beta * fabs(uc) * s) * dzk;
        }
        out[d.cells + p] = r;
    } else {
        out[d.cells + p] = T(0);
    }
    // ---- w (adv_add_w, :222-262) ----
    {
        const T dyj = h.my.idc[j], dzk = h.mz.idf[k];
        T r = T(0);
#pragma unroll
        for (int m = 0; m <= 1; ++m) {
            const T sg = T(2 * m - 1);
            const int ii = i - 1 + m, jj = J - 1 + m, kk = k - 1 + m;
            T uc = T(0.5) * (Ut(ii, J, k) + Ut(ii, J, k + 1));
            T s = HybW<ORD>::sum(at(W, ii - 2, j, k), at(W, ii - 1, j, k), at(W, ii, j, k), at(W, ii + 1, j, k),
                                 at(W, ii + 2, j, k), at(W, ii + 3, j, k));
            r = r - sg * (beta * fabs(uc) * s) * idx;
            uc = T(0.5) * (Vf(i, jj, k) + Vf(i, jj, k + 1));
            s = hyb_wsum(hyb_ord_y(jj, nyg, ORD), Wt(i, max(jj - 2, 1), k), Wt(i, max(jj - 1, 1), k), Wt(i, jj, k),
                         Wt(i, jj + 1, k), Wt(i, min(jj + 2, nyg), k), Wt(i, min(jj + 3, nyg), k));
            r = r - sg * (beta * fabs(uc) * s) * dyj;
            uc = T(0.5) * (at(W, i, j, kk) + at(W, i, j, kk + 1));
            s = HybW<ORD>::sum(at(W, i, j, kk - 2), at(W, i, j, kk - 1), at(W, i, j, kk), at(W, i, j, kk + 1),
                               at(W, i, j, kk + 2), at(W, i, j, kk + 3));
            r = r - sg * (beta * fabs(uc) * s) * dzk;
        }
        out[2 * d.cells + p] = r;
    }
}

}  // namespace dfdm
