// kernels_hybrid.cuh -- advection_scheme = 2: the upwind-biased dissipation of src/adv_hybrid.f90.
//
// The skew-symmetric central convection of the stage kernels is kept and beta |u_c| D is added as a conservative flux
// difference, D the third difference / 12 (order 3) or minus the fifth difference / 60 (order 5) of the advected
// velocity across the face, with the face's convecting velocity u_c.  With no immersed body beta = adv_beta0
// everywhere.  k_adv_hybrid_tiled computes the three components into out[0..cells), [cells..2 cells),
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

// the stencil weights of adv_wsel (src/adv_hybrid.f90:88-103), divided as the reference divides them (in double),
// applied to s(-2:3) = a..f as sum(w*s); the zero weights of order 3 are skipped
template <int ORD> struct HybW;
template <> struct HybW<3> {
    template <typename T> static __device__ __forceinline__ T sum(T a, T b, T c, T d, T e, T f) {
        (void)a; (void)f;
        return T(-1.0 / 12.0) * b + T(3.0 / 12.0) * c + T(-3.0 / 12.0) * d + T(1.0 / 12.0) * e;
    }
};
template <> struct HybW<5> {
    template <typename T> static __device__ __forceinline__ T sum(T a, T b, T c, T d, T e, T f) {
        return T(1.0 / 60.0) * a + T(-5.0 / 60.0) * b + T(10.0 / 60.0) * c + T(-10.0 / 60.0) * d + T(5.0 / 60.0) * e +
               T(-1.0 / 60.0) * f;
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

// A block owns a 32 x 8 column of cells and marches through KC z-planes; the
// planes k-3 .. k+3 of U, V, W, each a (32+6) x (8+6) tile with a 3-cell halo in x and y, rotate through eight
// shared planes filled by cp.async four planes ahead.  After a plane's copies land, each thread turns the
// elements it copied into the values the reference reads: U (plus the base profile) and W mirrored and V zero on
// wall rows, rows beyond a wall holding the clamped row's value (Max(jj-2,1), Min(jj+3,nyg)), periodic rows
// wrapped.  Totals throughout (the x and z differences then carry the base profile's rounding: the terms are small).
template <typename T, int ORD, int KC>
__global__ void __launch_bounds__(256) k_adv_hybrid_tiled(HybArgs<T> h, const T *__restrict__ U, const T *__restrict__ V,
                                                          const T *__restrict__ W, T *__restrict__ out) {
    constexpr int TX = 32, TY = 8, H = 3, PX = TX + 2 * H, PY = TY + 2 * H, PS = PX * PY, NT = TX * TY;
    constexpr int NP = 8, PER = (PS + NT - 1) / NT;
    extern __shared__ __align__(16) unsigned char hyb_smem[];
    T *sm = reinterpret_cast<T *>(hyb_smem);   // [3][NP][PS]
    const Dims &d = h.d;
    const int Nx = d.Nx, Ny = d.Ny, Nz = d.Nz, plane = Nx * Ny;
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY, k0 = blockIdx.z * KC, kend = min(k0 + KC, Nz);
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int i = i0 + tx, j = j0 + ty;
    const bool active = i < Nx && j < Ny;
    // this thread's plane elements: global offset (row, column), the row's sign for U/W (-1: mirror), V zero,
    // and the base profile of the row
    int off[PER];
    T sg[PER], ubq[PER];
    bool vz[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int e = threadIdx.x + q * NT;
        off[q] = -1; sg[q] = T(1); ubq[q] = T(0); vz[q] = false;
        if (e < PS) {
            const int jj = e / PX, ii = e - jj * PX;
            int gi = i0 - H + ii;
            gi = gi < 0 ? gi + Nx : gi;
            while (gi >= Nx) gi -= Nx;
            const int gj = j0 - H + jj;   // device row; the reference's J = gj + 2
            int g;
            if (d.yper) {
                g = gj % Ny; if (g < 0) g += Ny;
            } else if (gj < 0) {
                g = 0; sg[q] = T(-1); vz[q] = true;                 // J <= 1: the bottom ghost (V: the wall face)
            } else if (gj >= Ny) {
                g = Ny - 1; sg[q] = T(-1); vz[q] = true;            // J >= nyg: the top ghost
            } else {
                g = gj;
                vz[q] = gj >= Ny - 1;                               // V row Ny-1 (J = ny) is the top wall face
            }
            off[q] = g * Nx + gi;
            ubq[q] = h.ub[g];
        }
    }
    auto slot = [&](int k) { return (k - k0 + H) & (NP - 1); };
    auto issue = [&](int k) {
        const int kw = k < 0 ? k + Nz : (k >= Nz ? k - Nz : k), sl = slot(k);
        const size_t kb = (size_t)kw * plane;
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            if (off[q] < 0) continue;
            const int e = threadIdx.x + q * NT;
            cp_async<sizeof(T)>(&sm[(0 * NP + sl) * PS + e], U + kb + off[q]);
            cp_async<sizeof(T)>(&sm[(1 * NP + sl) * PS + e], V + kb + off[q]);
            cp_async<sizeof(T)>(&sm[(2 * NP + sl) * PS + e], W + kb + off[q]);
        }
    };
    auto fix = [&](int k) {
        const int sl = slot(k);
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            if (off[q] < 0) continue;
            const int e = threadIdx.x + q * NT;
            T &u = sm[(0 * NP + sl) * PS + e], &v = sm[(1 * NP + sl) * PS + e], &w = sm[(2 * NP + sl) * PS + e];
            u = sg[q] * (u + ubq[q]);
            w = sg[q] * w;
            if (vz[q]) v = T(0);
        }
    };
    const int nyg = d.yper ? Ny + 3 : Ny + 2, ny = d.yper ? Ny + 2 : Ny + 1;
    const int J = j + 2;
    const T beta = h.beta, idx = h.inv_dx;
    const T dyU = h.my.idc[min(j, Ny - 1)], dyV = h.my.idf[min(j, Ny - 1)];
    for (int k = k0 - H; k <= k0 + H; ++k) issue(k);
    cp_async_commit();
    cp_async_wait_all();
    for (int k = k0 - H; k <= k0 + H; ++k) fix(k);
    __syncthreads();
    for (int k = k0; k < kend; ++k) {
        const bool more = k + 1 < kend;
        if (more) issue(k + H + 1);
        cp_async_commit();
        if (active) {
            // value of field f at this thread's cell offset by (dx, dy, dz)
            auto S = [&](int f, int dx, int dy, int dz) -> T {
                return sm[(f * NP + slot(k + dz)) * PS + (ty + H + dy) * PX + (tx + H + dx)];
            };
            // the clamped y rows of the reference, as offsets from this thread's row (J = j + 2)
            auto yo = [&](int Jr, int n) -> int { return max(1, min(n, Jr)) - J; };
            const T dzU = h.mz.idc[k], dzW = h.mz.idf[k];
            const size_t p = ((size_t)k * Ny + j) * Nx + i;
            // ---- u ----
            T r = T(0);
#pragma unroll
            for (int m = 0; m <= 1; ++m) {
                const T sgm = T(2 * m - 1);
                const int a = m - 1;   // ii - i, jj - J, kk - k
                T uc = T(0.5) * (S(0, a, 0, 0) + S(0, a + 1, 0, 0));
                T s = HybW<ORD>::sum(S(0, a - 2, 0, 0), S(0, a - 1, 0, 0), S(0, a, 0, 0), S(0, a + 1, 0, 0),
                                     S(0, a + 2, 0, 0), S(0, a + 3, 0, 0));
                r = r - sgm * (beta * fabs(uc) * s) * idx;
                const int jj = J + a;
                uc = T(0.5) * (S(1, 0, a, 0) + S(1, 1, a, 0));
                s = hyb_wsum(hyb_ord_y(jj, nyg, ORD), S(0, 0, yo(jj - 2, nyg), 0), S(0, 0, yo(jj - 1, nyg), 0),
                             S(0, 0, a, 0), S(0, 0, a + 1, 0), S(0, 0, yo(jj + 2, nyg), 0), S(0, 0, yo(jj + 3, nyg), 0));
                r = r - sgm * (beta * fabs(uc) * s) * dyU;
                uc = T(0.5) * (S(2, 0, 0, a) + S(2, 1, 0, a));
                s = HybW<ORD>::sum(S(0, 0, 0, a - 2), S(0, 0, 0, a - 1), S(0, 0, 0, a), S(0, 0, 0, a + 1),
                                   S(0, 0, 0, a + 2), S(0, 0, 0, a + 3));
                r = r - sgm * (beta * fabs(uc) * s) * dzU;
            }
            out[p] = r;
            // ---- v ----
            r = T(0);
            if (j < d.NyV) {
#pragma unroll
                for (int m = 0; m <= 1; ++m) {
                    const T sgm = T(2 * m - 1);
                    const int a = m - 1;
                    T uc = T(0.5) * (S(0, a, 0, 0) + S(0, a, 1, 0));
                    T s = HybW<ORD>::sum(S(1, a - 2, 0, 0), S(1, a - 1, 0, 0), S(1, a, 0, 0), S(1, a + 1, 0, 0),
                                         S(1, a + 2, 0, 0), S(1, a + 3, 0, 0));
                    r = r - sgm * (beta * fabs(uc) * s) * idx;
                    const int jj = J + a;
                    uc = T(0.5) * (S(1, 0, a, 0) + S(1, 0, a + 1, 0));
                    s = hyb_wsum(hyb_ord_y(jj, ny, ORD), S(1, 0, yo(jj - 2, ny), 0), S(1, 0, yo(jj - 1, ny), 0),
                                 S(1, 0, a, 0), S(1, 0, a + 1, 0), S(1, 0, yo(jj + 2, ny), 0), S(1, 0, yo(jj + 3, ny), 0));
                    r = r - sgm * (beta * fabs(uc) * s) * dyV;
                    uc = T(0.5) * (S(2, 0, 0, a) + S(2, 0, 1, a));
                    s = HybW<ORD>::sum(S(1, 0, 0, a - 2), S(1, 0, 0, a - 1), S(1, 0, 0, a), S(1, 0, 0, a + 1),
                                       S(1, 0, 0, a + 2), S(1, 0, 0, a + 3));
                    r = r - sgm * (beta * fabs(uc) * s) * dzU;
                }
            }
            out[d.cells + p] = r;
            // ---- w ----
            r = T(0);
#pragma unroll
            for (int m = 0; m <= 1; ++m) {
                const T sgm = T(2 * m - 1);
                const int a = m - 1;
                T uc = T(0.5) * (S(0, a, 0, 0) + S(0, a, 0, 1));
                T s = HybW<ORD>::sum(S(2, a - 2, 0, 0), S(2, a - 1, 0, 0), S(2, a, 0, 0), S(2, a + 1, 0, 0),
                                     S(2, a + 2, 0, 0), S(2, a + 3, 0, 0));
                r = r - sgm * (beta * fabs(uc) * s) * idx;
                const int jj = J + a;
                uc = T(0.5) * (S(1, 0, a, 0) + S(1, 0, a, 1));
                s = hyb_wsum(hyb_ord_y(jj, nyg, ORD), S(2, 0, yo(jj - 2, nyg), 0), S(2, 0, yo(jj - 1, nyg), 0),
                             S(2, 0, a, 0), S(2, 0, a + 1, 0), S(2, 0, yo(jj + 2, nyg), 0), S(2, 0, yo(jj + 3, nyg), 0));
                r = r - sgm * (beta * fabs(uc) * s) * dyU;
                uc = T(0.5) * (S(2, 0, 0, a) + S(2, 0, 0, a + 1));
                s = HybW<ORD>::sum(S(2, 0, 0, a - 2), S(2, 0, 0, a - 1), S(2, 0, 0, a), S(2, 0, 0, a + 1),
                                   S(2, 0, 0, a + 2), S(2, 0, 0, a + 3));
                r = r - sgm * (beta * fabs(uc) * s) * dzW;
            }
            out[2 * d.cells + p] = r;
        }
        cp_async_wait_all();
        if (more) fix(k + H + 1);
        __syncthreads();
    }
}

}  // namespace dfdm
