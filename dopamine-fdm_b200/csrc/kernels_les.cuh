// kernels_les.cuh -- the LES stage kernel with the eddy viscosity recomputed in the tile.
//
// compute_time_step_RK3 evaluates the eddy viscosity from the velocity each stage starts from: at the step start
// (stage 1) and after the projections of stages 1 and 2 (src/time_integration.f90:144,361,493).  That velocity is
// exactly what the stage kernel loads, so instead of a separate full-grid pass that writes nu_t and a stage kernel
// that reads it back, this kernel computes nu_t (nut_at: compute_vreman pass 1, src/sgs_model.f90:118-223, AMD or
// Vreman with the wall-model override) from its own shared-memory velocity tiles, on the tile and a one-cell halo,
// and the right-hand sides read it from shared memory.  The values are the separate pass's bit for bit: the same
// function on the same loaded (and, with CORR, corrected) velocity.
//
// Tiles: 32 x 8 cells per block marching through a z-chunk, one cell per thread.  The velocity planes carry a
// two-cell halo in x and y (nu_t at the tile's halo centres needs their neighbours) and rotate through five slots:
// at plane k the block holds velocity planes k-1 .. k+2 and the copy of plane k+3 is in flight.  nu_t of plane k+1
// is computed at the start of iteration k into a three-plane ring (planes k-1, k, k+1 for the stencil); its wall
// ghosts are zero and its periodic halo values come from the wrapped velocity, as sgs_fill_ghosts (:458-531) sets
// them.  CORR applies the previous stage's projection in the loader, as k_tiled does; phi travels two planes
// ahead of the velocity (seven slots), so the phi a plane's correction reads has passed a barrier before it.
// With nut_out (stage 3) each thread also stores its cell's nu_t, the value the separate pass leaves after a step.
#pragma once

#include "kernels_step.cuh"

namespace dfdm {

namespace les {
constexpr int TX = 32, TY = 8, H = 2;
constexpr int PX = TX + 2 * H, PY = TY + 2 * H, PS = PX * PY;   // velocity / nu_t plane: 36 x 12
constexpr int PXP = PX + 1, PSP = PXP * (PY + 1);                // phi plane: one more column and row
constexpr int NV = 5, NN = 3, NP = 7;                            // velocity, nu_t and phi ring slots
constexpr int NT = TX * TY;
template <typename T> constexpr size_t smem_bytes(bool corr) {
    return sizeof(T) * ((size_t)3 * NV * PS + (size_t)NN * PS + (corr ? (size_t)NP * PSP : 0));
}
}  // namespace les

template <typename T, bool WM, bool CORR>
__global__ void __launch_bounds__(les::NT, 2) k_les(StepArgs<T> a, const T *__restrict__ U, const T *__restrict__ V,
                                                    const T *__restrict__ W, const double *__restrict__ tau_x,
                                                    const double *__restrict__ tau_z, StageCoef sc, int kc,
                                                    T *__restrict__ uo, T *__restrict__ vo, T *__restrict__ wo,
                                                    T *__restrict__ f1u, T *__restrict__ f1v, T *__restrict__ f1w,
                                                    T *__restrict__ us, T *__restrict__ vs, T *__restrict__ wsf,
                                                    T *__restrict__ nut_out) {
    pdl_enter();
    using namespace les;
    constexpr int PER = (PS + NT - 1) / NT, PERP = (PSP + NT - 1) / NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *smv = reinterpret_cast<T *>(smem_raw);   // [3][NV][PS] velocity
    T *smn = smv + 3 * NV * PS;                 // [NN][PS] nu_t
    T *smp = smn + NN * PS;                     // [NP][PSP] phi (CORR)
    auto vel = [&](int f, int slot) { return smv + (f * NV + slot) * PS; };
    const Dims &d = a.d;
    const int Nx = d.Nx, Ny = d.Ny, Nz = d.Nz;
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
    const int k0 = blockIdx.z * kc, kend = min(k0 + kc, Nz);
    const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
    const int i = i0 + tx, j = j0 + ty;
    const bool active = i < Nx && j < Ny;
    const int plane = Nx * Ny;
    auto wrapz = [&](int k) { return k < 0 ? k + Nz : (k >= Nz ? k - Nz : k); };
    auto vslot = [&](int p) { return (p - (k0 - 2)) % NV; };   // velocity plane p (p >= k0-2)
    auto nslot = [&](int p) { return (p - (k0 - 1)) % NN; };   // nu_t plane p (p >= k0-1)
    auto pslot = [&](int p) { return (p - (k0 - 2)) % NP; };   // phi plane p (p >= k0-2)

    // this thread's share of a velocity plane: offset within a plane (or -1) and the wall rule
    int off[PER];
    bool ghost[PER];
    int pix[CORR ? PER : 1];
    T iyq[CORR ? PER : 1];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int e = threadIdx.x + q * NT;
        off[q] = -1; ghost[q] = false;
        if (e < PS) {
            const int jj = e / PX, ii = e - jj * PX;
            int gi = i0 - H + ii;
            gi = gi < 0 ? gi + Nx : gi;
            while (gi >= Nx) gi -= Nx;
            const int gj = j0 - H + jj;
            int g;
            if (d.yper) {
                g = gj;
                while (g < 0) g += Ny;
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
    int offp[CORR ? PERP : 1];
    if constexpr (CORR) {
#pragma unroll
        for (int q = 0; q < PERP; ++q) {
            const int e = threadIdx.x + q * NT;
            offp[q] = -1;
            if (e < PSP) {
                const int jj = e / PXP, ii = e - jj * PXP;
                int gi = i0 - H + ii;
                gi = gi < 0 ? gi + Nx : gi;
                while (gi >= Nx) gi -= Nx;
                const int gj = j0 - H + jj;
                int g;
                if (d.yper) { g = gj; while (g < 0) g += Ny; while (g >= Ny) g -= Ny; }
                else g = gj < 0 ? 0 : (gj >= Ny ? Ny - 1 : gj);
                offp[q] = g * Nx + gi;
            }
        }
    }
    auto issue = [&](int p) {   // velocity plane p (and, CORR, phi plane p+2)
        const int kb = wrapz(p) * plane, s = vslot(p);
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            if (off[q] < 0) continue;
            const int o = kb + off[q], e = threadIdx.x + q * NT;
            cp_async<sizeof(T)>(vel(0, s) + e, U + o);
            cp_async<sizeof(T)>(vel(2, s) + e, W + o);
            if (!ghost[q]) cp_async<sizeof(T)>(vel(1, s) + e, V + o);
        }
        if constexpr (CORR) {
            const int kp = wrapz(p + 2) * plane, sp = pslot(p + 2);
#pragma unroll
            for (int q = 0; q < PERP; ++q)
                if (offp[q] >= 0) cp_async<sizeof(T)>(smp + sp * PSP + threadIdx.x + q * NT, a.phi + kp + offp[q]);
        }
    };
    auto issue_phi = [&](int p) {   // phi plane p alone (the first two planes of the chunk's ring)
        if constexpr (CORR) {
            const int kp = wrapz(p) * plane, sp = pslot(p);
#pragma unroll
            for (int q = 0; q < PERP; ++q)
                if (offp[q] >= 0) cp_async<sizeof(T)>(smp + sp * PSP + threadIdx.x + q * NT, a.phi + kp + offp[q]);
        }
    };
    auto fix = [&](int p) {   // after the copies of plane p (and, CORR, phi p and p+1) have landed
        const int s = vslot(p);
        if constexpr (CORR) {   // project_velocity of the previous stage (k_correct's arithmetic)
            const T *p0 = smp + pslot(p) * PSP, *p1 = smp + pslot(p + 1) * PSP;
            const T iz = Arith<T>::inv(a.mz.df, a.mz.idf, wrapz(p));
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                if (off[q] < 0) continue;
                const int e = threadIdx.x + q * NT;
                const T pc = p0[pix[q]], pxp = p0[pix[q] + 1], pzp = p1[pix[q]];
                vel(0, s)[e] = vel(0, s)[e] - (pxp - pc) * a.inv_dx;
                vel(2, s)[e] = vel(2, s)[e] - (pzp - pc) * iz;
                if (iyq[q] != T(0)) vel(1, s)[e] = vel(1, s)[e] - (p0[pix[q] + PXP] - pc) * iyq[q];
            }
        }
#pragma unroll
        for (int q = 0; q < PER; ++q) {   // wall ghost rows
            if (off[q] < 0 || !ghost[q]) continue;
            const int e = threadIdx.x + q * NT;
            vel(0, s)[e] = -vel(0, s)[e];
            vel(2, s)[e] = -vel(2, s)[e];
            vel(1, s)[e] = T(0);
        }
    };
    // base profile of row g (with the wall mirror of the ghost rows)
    auto ub_row = [&](int g) -> T {
        if (d.yper) { while (g < 0) g += Ny; while (g >= Ny) g -= Ny; return __ldg(a.ub + g); }
        if (g < 0) return -__ldg(a.ub + 0);
        if (g >= Ny) return -__ldg(a.ub + Ny - 1);
        return __ldg(a.ub + g);
    };
    // nu_t of plane p on the tile and its one-cell halo: centres x = i0-1 .. i0+TX, y = j0-1 .. j0+TY
    auto eddy = [&](int p) {
        const int pw = wrapz(p);
        T *dst = smn + nslot(p) * PS;
        for (int e = threadIdx.x; e < (TX + 2) * (TY + 2); e += NT) {
            const int jj = e / (TX + 2), ii = e - jj * (TX + 2);
            int g = j0 - 1 + jj;
            const int loc = (jj + 1) * PX + ii + 1;
            T nu = T(0);
            bool wall_ghost = !d.yper && (g < 0 || g >= Ny);
            if (!wall_ghost) {
                if (d.yper) { while (g < 0) g += Ny; while (g >= Ny) g -= Ny; }
                TileQ<T, PX> q;
                q.c = loc;
                q.ub[0] = ub_row(g - 1); q.ub[1] = ub_row(g); q.ub[2] = ub_row(g + 1);
                q.u[0] = vel(0, vslot(p - 1)); q.u[1] = vel(0, vslot(p)); q.u[2] = vel(0, vslot(p + 1));
                q.v[0] = vel(1, vslot(p - 1)); q.v[1] = vel(1, vslot(p)); q.v[2] = vel(1, vslot(p + 1));
                q.w[0] = vel(2, vslot(p - 1)); q.w[1] = vel(2, vslot(p)); q.w[2] = vel(2, vslot(p + 1));
                q.n[0] = q.n[1] = q.n[2] = nullptr;
                int gi = i0 - 1 + ii;
                gi = gi < 0 ? gi + Nx : gi;
                while (gi >= Nx) gi -= Nx;
                nu = nut_at<T>(a, q, gi, g, pw);
            }
            dst[loc] = nu;
        }
    };

    T ubr[3];
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj) ubr[dj + 1] = ub_row(min(j, Ny - 1) + dj);
    AxisLocal<T> Y;
    Y.load(a.my, min(j, Ny - 1));

    // velocity planes k0-2 .. k0+2 (and phi k0-2 .. k0+4), fixed; nu_t of planes k0-1 and k0
    issue_phi(k0 - 2);
    issue_phi(k0 - 1);
    for (int p = k0 - 2; p <= k0 + 2; ++p) issue(p);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();   // phi and ghost-row sources copied by other threads
    for (int p = k0 - 2; p <= k0 + 2; ++p) fix(p);
    __syncthreads();
    eddy(k0 - 1);
    eddy(k0);
    __syncthreads();   // nu_t of plane k0-1 read velocity plane k0-2, whose slot the first iteration refills
    const int cloc = (ty + H) * PX + tx + H;
    for (int k = k0; k < kend; ++k) {
        // plane k+3 goes into the slot of plane k-2, whose last reader (the stencil of plane k-1) is done
        const bool more = k + 3 <= kend + 1;
        if (more) issue(k + 3);
        cp_async_commit();
        eddy(k + 1);   // from velocity planes k .. k+2
        __syncthreads();
        if (active) {
            TileQ<T, PX> q;
            q.c = cloc;
            q.ub[0] = ubr[0]; q.ub[1] = ubr[1]; q.ub[2] = ubr[2];
            q.u[0] = vel(0, vslot(k - 1)); q.u[1] = vel(0, vslot(k)); q.u[2] = vel(0, vslot(k + 1));
            q.v[0] = vel(1, vslot(k - 1)); q.v[1] = vel(1, vslot(k)); q.v[2] = vel(1, vslot(k + 1));
            q.w[0] = vel(2, vslot(k - 1)); q.w[1] = vel(2, vslot(k)); q.w[2] = vel(2, vslot(k + 1));
            q.n[0] = smn + nslot(k - 1) * PS; q.n[1] = smn + nslot(k) * PS; q.n[2] = smn + nslot(k + 1) * PS;
            stage_cell<T, true, WM, false>(a, q, Y, tau_x, tau_z, sc, i, j, k, uo, vo, wo, f1u, f1v, f1w, us, vs, wsf,
                                           nullptr);
            if (nut_out) nut_out[k * plane + j * Nx + i] = q.N(0, 0, 0);   // stage 3: the step's last nu_t, kept
        }
        cp_async_wait_all();   // this thread's copies of plane k+3; phi k+3 and k+4 passed earlier barriers
        if (more) fix(k + 3);
        __syncthreads();
    }
}

}  // namespace dfdm
