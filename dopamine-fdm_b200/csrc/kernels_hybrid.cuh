// kernels_hybrid.cuh -- advection_scheme = 2: the upwind-biased dissipation of src/adv_hybrid.f90.
//
// The skew-symmetric central convection of the stage kernels is kept and beta |u_c| D is added as a conservative flux
// difference, D the third difference / 12 (order 3) or minus the fifth difference / 60 (order 5) of the advected
// velocity across the face, with the face's convecting velocity u_c.  With no immersed body beta = adv_beta0
// everywhere.  k_adv_hybrid_faces computes the three components into out[0..cells), [cells..2 cells),
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

// Shared memory of k_adv_hybrid_faces: the ring of 8 planes of U, V, W, each a 40 x (8 + 2H) tile (a 4-cell x halo,
// so that tile rows start on 16-byte boundaries; H = 2 rows for order 3, 3 for order 5), then the x faces [3][8][33]
// and the y faces [3][9][32] of the current plane.
template <typename T, int ORD> constexpr size_t hyb_faces_smem_bytes() {
    return ((size_t)3 * 8 * 40 * (8 + 2 * (ORD == 5 ? 3 : 2)) + 3 * 8 * 33 + 3 * 9 * 32) * sizeof(T);
}

// A block owns a 32 x 8 column of cells and marches through kc z-planes; the planes of U, V, W rotate through eight
// shared tiles filled by cp.async H+1 planes ahead (y halo H = 2 rows for order 3, 3 for order 5; x halo 4 cells).
// After a plane's copies land, each thread turns the vectors it copied into the values the reference reads: U (plus
// the base profile) and W mirrored and V zero on wall rows, rows beyond a wall holding the clamped row's value
// (Max(jj-2,1), Min(jj+3,nyg)), periodic rows wrapped.  Totals throughout (the x and z differences then carry the
// base profile's rounding: the terms are small).
// Each face flux is evaluated once.  The flux through a face, beta |u_c| D (without the cell's metric), depends
// only on the face, so a cell's two faces per direction are shared with its neighbours:
//   x: each thread evaluates the face on its left; y: each thread the face below its row; the tile's right-hand x
//      faces and its top y faces are spread over warps 0..5, one face per thread;
//   z: each thread the face above its cell, carried in registers to the next plane as the face below; the cell's
//      own column of each field (the z stencil) is a register queue that takes one new plane per step.
// x and y faces pass through shared memory (a barrier between their stores and the reads).  The cell then assembles
//   r = -(-1)Fx(-) dx' - (-1)Fy(-) dy' - (-1)Fz(-) dz' - Fx(+) dx' - Fy(+) dy' - Fz(+) dz'
// in the order of adv_dflux (src/adv_hybrid.f90:136-210): the lower faces, then the upper faces, x, y, z.  y rows
// are clamped to the reference's ranges by absolute row.
template <typename T, int ORD, int VW>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? (ORD == 5 ? 3 : 4) : (ORD == 5 ? 1 : 2))
    k_adv_hybrid_faces(HybArgs<T> h, int kc, const T *__restrict__ U, const T *__restrict__ V, const T *__restrict__ W,
                       T *__restrict__ out) {
    pdl_enter();
    constexpr int TX = 32, TY = 8, H = ORD == 5 ? 3 : 2, HX = 4, PX = TX + 2 * HX, PY = TY + 2 * H, PS = PX * PY;
    constexpr int NT = TX * TY, NP = 8;
    // the loader copies VW consecutive x cells at a time (VW = 4 in FP32 when Nx % 4 == 0, else 2): every vector
    // starts at a column that is a multiple of VW, so it never straddles the periodic seam
    constexpr int VB = VW * (int)sizeof(T), RV = PX / VW, NV = PY * RV, PER = (NV + NT - 1) / NT;
    static_assert(VB == 8 || VB == 16, "8- or 16-byte copies");
    struct alignas(VB) Vec { T v[VW]; };
    constexpr int FXP = TX + 1;   // pitch of the x-face rows
    extern __shared__ __align__(16) unsigned char hyb_smem[];
    T *sm = reinterpret_cast<T *>(hyb_smem);   // [3][NP][PS]
    T *fx = sm + 3 * NP * PS;                  // [3][TY][TX + 1]: face between columns c-1 and c at [row][c]
    T *fy = fx + 3 * TY * FXP;                 // [3][TY + 1][TX]: face between rows r-1 and r at [r][col]
    const Dims &d = h.d;
    const int Nx = d.Nx, Ny = d.Ny, Nz = d.Nz, plane = Nx * Ny;
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY, k0 = blockIdx.z * kc, kend = min(k0 + kc, Nz);
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int i = i0 + tx, j = j0 + ty;
    const bool active = i < Nx && j < Ny;
    int off[PER];
    T sg[PER], ubq[PER];
    bool vz[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int e = threadIdx.x + q * NT;
        off[q] = -1; sg[q] = T(1); ubq[q] = T(0); vz[q] = false;
        if (e < NV) {
            const int jj = e / RV, vc = e - jj * RV;
            int gi = i0 - HX + vc * VW;
            gi = gi < 0 ? gi + Nx : gi;
            while (gi >= Nx) gi -= Nx;
            const int gj = j0 - H + jj;
            int g;
            if (d.yper) {
                g = gj % Ny; if (g < 0) g += Ny;
            } else if (gj < 0) {
                g = 0; sg[q] = T(-1); vz[q] = true;
            } else if (gj >= Ny) {
                g = Ny - 1; sg[q] = T(-1); vz[q] = true;
            } else {
                g = gj;
                vz[q] = gj >= Ny - 1;
            }
            off[q] = g * Nx + gi;
            ubq[q] = h.ub[g];
        }
    }
    auto issue = [&](int k) {
        const int kw = k < 0 ? k + Nz : (k >= Nz ? k - Nz : k), sl = (k - k0 + H) & (NP - 1);
        const int kb = kw * plane;   // 3 x cells < 2^31 (checked at context creation)
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            if (off[q] < 0) continue;
            const int e = (threadIdx.x + q * NT) * VW;
            cp_async<VB>(&sm[(0 * NP + sl) * PS + e], U + kb + off[q]);
            cp_async<VB>(&sm[(1 * NP + sl) * PS + e], V + kb + off[q]);
            cp_async<VB>(&sm[(2 * NP + sl) * PS + e], W + kb + off[q]);
        }
    };
    auto fix = [&](int k) {
        const int sl = (k - k0 + H) & (NP - 1);
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            if (off[q] < 0) continue;
            const int e = (threadIdx.x + q * NT) * VW;
            Vec *pu = reinterpret_cast<Vec *>(&sm[(0 * NP + sl) * PS + e]);
            Vec *pv = reinterpret_cast<Vec *>(&sm[(1 * NP + sl) * PS + e]);
            Vec *pw = reinterpret_cast<Vec *>(&sm[(2 * NP + sl) * PS + e]);
            Vec u = *pu, w = *pw;
#pragma unroll
            for (int m = 0; m < VW; ++m) { u.v[m] = sg[q] * (u.v[m] + ubq[q]); w.v[m] = sg[q] * w.v[m]; }
            *pu = u; *pw = w;
            if (vz[q]) {
                Vec z;
#pragma unroll
                for (int m = 0; m < VW; ++m) z.v[m] = T(0);
                *pv = z;
            }
        }
    };
    // field f at tile row r, column c (0-based within the tile, -H .. TY+H-1 / -HX .. TX+HX-1), plane kk
    auto A = [&](int f, int r, int c, int kk) -> T {
        return sm[(f * NP + ((kk - k0 + H) & (NP - 1))) * PS + (r + H) * PX + (c + HX)];
    };
    const int nyg = d.yper ? Ny + 3 : Ny + 2, ny = d.yper ? Ny + 2 : Ny + 1;
    // beta * |0.5 (a + b)| = (0.5 beta) |a + b| exactly (scaling by a power of two)
    const T bh = T(0.5) * h.beta;
    // the tile row of the reference's (clamped) row Jr: device row Jr - 2
    auto yrow = [&](int Jr, int n) -> int { return max(1, min(n, Jr)) - 2 - j0; };
    // y-face rows: the face between tile rows r-1 and r is the reference's face jj = J(r) - 1 (adv_ord_y, the
    // clamped stencil rows jj-2 .. jj+3 for U and W (n = nyg) and for V (n = ny))
    struct YRows { int o, m2, m1, p2, p3; };
    auto yrows = [&](int r, int n) -> YRows {
        const int jj = j0 + r + 2 - 1;
        return YRows{hyb_ord_y(jj, n, ORD), yrow(jj - 2, n), yrow(jj - 1, n), yrow(jj + 2, n), yrow(jj + 3, n)};
    };
    auto xface = [&](int comp, int r, int c, int kk) -> T {   // between columns c-1 and c
        T uc;
        if (comp == 0) uc = A(0, r, c - 1, kk) + A(0, r, c, kk);
        else if (comp == 1) uc = A(0, r, c - 1, kk) + A(0, r + 1, c - 1, kk);
        else uc = A(0, r, c - 1, kk) + A(0, r, c - 1, kk + 1);
        T s;
        if constexpr (ORD == 5)
            s = HybW<5>::sum(A(comp, r, c - 3, kk), A(comp, r, c - 2, kk), A(comp, r, c - 1, kk), A(comp, r, c, kk),
                             A(comp, r, c + 1, kk), A(comp, r, c + 2, kk));
        else   // order 3 reads s(-1:2) only
            s = HybW<3>::sum(T(0), A(comp, r, c - 2, kk), A(comp, r, c - 1, kk), A(comp, r, c, kk),
                             A(comp, r, c + 1, kk), T(0));
        return bh * fabs(uc) * s;
    };
    auto yface = [&](int comp, int r, int c, int kk, const YRows &y) -> T {   // between rows r-1 and r
        T uc;
        if (comp == 0) uc = A(1, r - 1, c, kk) + A(1, r - 1, c + 1, kk);
        else if (comp == 1) uc = A(1, r - 1, c, kk) + A(1, r, c, kk);
        else uc = A(1, r - 1, c, kk) + A(1, r - 1, c, kk + 1);
        T s;
        if constexpr (ORD == 5)
            s = hyb_wsum(y.o, A(comp, y.m2, c, kk), A(comp, y.m1, c, kk), A(comp, r - 1, c, kk), A(comp, r, c, kk),
                         A(comp, y.p2, c, kk), A(comp, y.p3, c, kk));
        else
            s = hyb_wsum(y.o, T(0), A(comp, y.m1, c, kk), A(comp, r - 1, c, kk), A(comp, r, c, kk),
                         A(comp, y.p2, c, kk), T(0));
        return bh * fabs(uc) * s;
    };
    // this cell's own column of each field in registers: q[f][m] is plane k - (NQ/2 - 1) + m, the planes of the
    // stencil of the face between k and k+1; each plane adds one shared-memory read per field
    constexpr int NQ = ORD == 5 ? 6 : 4, QC = NQ / 2 - 1;   // q[f][QC] is plane k
    T q[3][NQ] = {};   // filled from shared memory once the first planes have landed
    auto zface = [&](int comp, int kk) -> T {   // between planes kk and kk+1, from the queue of plane kk
        T uc;
        if (comp == 0) uc = q[2][QC] + A(2, ty, tx + 1, kk);
        else if (comp == 1) uc = q[2][QC] + A(2, ty + 1, tx, kk);
        else uc = q[2][QC] + q[2][QC + 1];
        T s;
        if constexpr (ORD == 5) s = HybW<5>::sum(q[comp][0], q[comp][1], q[comp][2], q[comp][3], q[comp][4], q[comp][5]);
        else s = HybW<3>::sum(T(0), q[comp][0], q[comp][1], q[comp][2], q[comp][3], T(0));
        return bh * fabs(uc) * s;
    };
    const YRows yg = yrows(ty, nyg), yv = yrows(ty, ny);          // this thread's face below its row
    const YRows ygt = yrows(TY, nyg), yvt = yrows(TY, ny);        // warp TY-1: the faces above the tile
    const T idx = h.inv_dx;
    const T dyU = h.my.idc[min(j, Ny - 1)], dyV = h.my.idf[min(j, Ny - 1)];
    for (int k = k0 - H; k <= k0 + H; ++k) issue(k);
    cp_async_commit();
    cp_async_wait_all();
    for (int k = k0 - H; k <= k0 + H; ++k) fix(k);
    __syncthreads();
    T zb[3];   // the face below this cell (between planes k-1 and k)
#pragma unroll
    for (int f = 0; f < 3; ++f)
#pragma unroll
        for (int m = 0; m < NQ; ++m) q[f][m] = A(f, ty, tx, k0 - 1 - QC + m);
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) zb[comp] = zface(comp, k0 - 1);
    for (int k = k0; k < kend; ++k) {
        const bool more = k + 1 < kend;
        if (more) issue(k + H + 1);
        cp_async_commit();
#pragma unroll
        for (int f = 0; f < 3; ++f) {
#pragma unroll
            for (int m = 0; m + 1 < NQ; ++m) q[f][m] = q[f][m + 1];
            q[f][NQ - 1] = A(f, ty, tx, k + NQ - 1 - QC);
        }
        // every face value first (no shared store between the stencil reads), then the stores
        T xb[3], yb[3], za[3];
#pragma unroll
        for (int comp = 0; comp < 3; ++comp) {
            xb[comp] = xface(comp, ty, tx, k);
            yb[comp] = yface(comp, ty, tx, k, comp == 1 ? yv : yg);
            za[comp] = zface(comp, k);
        }
        // the tile's edge faces, one per thread of warps 0..5: warp c < 3 the y faces above the tile of component c,
        // lanes 0..7 of warp 3 + c the right-hand x faces of the tile's rows (row = lane) of component c
        T ex = T(0);
        if (ty < 3) ex = yface(ty, TY, tx, k, ty == 1 ? yvt : ygt);
        else if (ty < 6 && tx < TY) ex = xface(ty - 3, tx, TX, k);
#pragma unroll
        for (int comp = 0; comp < 3; ++comp) {
            fx[(comp * TY + ty) * FXP + tx] = xb[comp];
            fy[(comp * (TY + 1) + ty) * TX + tx] = yb[comp];
        }
        if (ty < 3) fy[(ty * (TY + 1) + TY) * TX + tx] = ex;
        else if (ty < 6 && tx < TY) fx[((ty - 3) * TY + tx) * FXP + TX] = ex;
        __syncthreads();
        if (active) {
            const T dzU = h.mz.idc[k], dzW = h.mz.idf[k];
            const int p = (k * Ny + j) * Nx + i;
#pragma unroll
            for (int comp = 0; comp < 3; ++comp) {
                const T dy = comp == 1 ? dyV : dyU, dz = comp == 2 ? dzW : dzU;
                const T xa = fx[(comp * TY + ty) * FXP + tx + 1], ya = fy[(comp * (TY + 1) + ty + 1) * TX + tx];
                T r = T(0);
                r = r - T(-1) * xb[comp] * idx;
                r = r - T(-1) * yb[comp] * dy;
                r = r - T(-1) * zb[comp] * dz;
                r = r - T(1) * xa * idx;
                r = r - T(1) * ya * dy;
                r = r - T(1) * za[comp] * dz;
                if (comp == 1 && j >= d.NyV) r = T(0);   // v rows beyond the last interior face
                out[comp * (int)d.cells + p] = r;
            }
        }
#pragma unroll
        for (int comp = 0; comp < 3; ++comp) zb[comp] = za[comp];
        cp_async_wait_all();
        if (more) fix(k + H + 1);
        __syncthreads();
    }
}

}  // namespace dfdm
