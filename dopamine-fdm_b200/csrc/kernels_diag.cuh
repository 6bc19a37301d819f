// kernels_diag.cuh -- reductions (FP64 compensated sums), the constant-flux shift and the ghosted state transfers.
#pragma once

#include "dfdm_common.cuh"

namespace dfdm {

// Kahan-compensated accumulator in double.
struct Kahan {
    double s, c;
    __device__ __forceinline__ void init() { s = 0.0; c = 0.0; }
    __device__ __forceinline__ void add(double x) {
        double y = x - c;
        double t = s + y;
        c = (t - s) - y;
        s = t;
    }
};

// Block reduction of two compensated sums; thread 0 writes the block's pair to out[2*blk] (blk: the block's index in
// its own grid, which in a grouped launch is not blockIdx.x).
__device__ __forceinline__ void block_sum2(double a, double b, double *out, int blk) {
    __shared__ double sa[32], sb[32];
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { sa[wid] = a; sb[wid] = b; }
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x + 31) >> 5;
        a = lane < nw ? sa[lane] : 0.0;
        b = lane < nw ? sb[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
        }
        if (lane == 0) { out[2 * blk] = a; out[2 * blk + 1] = b; }
    }
}

// Block maximum of two non-negative doubles, then one atomicMax of each bit pattern per block (non-negative
// doubles order as their bit patterns); one atomic pair per block keeps the two addresses uncontended.
__device__ __forceinline__ void block_max2_atomic(double a, double b, unsigned long long *out) {
    __shared__ double sa[32], sb[32];
    for (int o = 16; o > 0; o >>= 1) {
        a = fmax(a, __shfl_down_sync(0xffffffffu, a, o));
        b = fmax(b, __shfl_down_sync(0xffffffffu, b, o));
    }
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { sa[wid] = a; sb[wid] = b; }
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x + 31) >> 5;
        a = lane < nw ? sa[lane] : 0.0;
        b = lane < nw ? sb[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            a = fmax(a, __shfl_down_sync(0xffffffffu, a, o));
            b = fmax(b, __shfl_down_sync(0xffffffffu, b, o));
        }
        if (lane == 0) {
            atomicMax(out, (unsigned long long)__double_as_longlong(a));
            atomicMax(out + 1, (unsigned long long)__double_as_longlong(b));
        }
    }
}

// 16-byte row chunks: NV = 16 / sizeof(T) consecutive cells in one load (rows start 16-byte aligned when Nx*sizeof(T)
// is a multiple of 16: the fields are 256-byte aligned)
template <typename T> struct Chunk {
    static constexpr int NV = 16 / sizeof(T);
    T x[NV];
    __device__ __forceinline__ void load(const T *p) {
        const uint4 v = __ldg(reinterpret_cast<const uint4 *>(p));
        if constexpr (sizeof(T) == 4) {
            x[0] = __uint_as_float(v.x); x[1] = __uint_as_float(v.y); x[2] = __uint_as_float(v.z); x[3] = __uint_as_float(v.w);
        } else {
            x[0] = __hiloint2double((int)v.y, (int)v.x); x[1] = __hiloint2double((int)v.w, (int)v.z);
        }
    }
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int c = 0; c < NV; ++c) x[c] = T(0);
    }
};

// compute_bulk_velocity (src/monitor.f90:463-523): sum of 0.5 (U_i + U_{i-1}) dy_j dz_k over the independent cells
// and of the weights dy_j dz_k, one partial pair per block (deterministic, no atomics).  Over a periodic x-row the
// face averages telescope, sum_i 0.5 (U_i + U_{i-1}) = sum_i U_i, so a row contributes dy_j dz_k (sum_i u_i + Nx ub_j)
// (u the stored field, ub the base profile).  A warp walks whole x-rows (row = k*Ny + j): the row's metrics are
// loaded once, with no per-cell index division, and a lane reads its cells in 16-byte chunks (VEC: Nx a multiple of
// the chunk; otherwise one cell at a time).
template <typename T, bool VEC, class BC>
__device__ __forceinline__ void k_bulk_partial_body(const BC &bc, const Dims &d, const T *__restrict__ U, const double *__restrict__ dyc,
                                                      const double *__restrict__ dzc, const double *__restrict__ ubd,
                                                      double *__restrict__ part) {
    typedef Chunk<T> Ch;
    Kahan s, w; s.init(); w.init();
    const int rows = d.Ny * d.Nz, Nx = d.Nx, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int row = bc.idx().x * wpb + (threadIdx.x >> 5); row < rows; row += bc.dim().x * wpb) {
        const int k = row / d.Ny, j = row - k * d.Ny;
        const double a = dyc[j] * dzc[k], ub = ubd[j];
        const T *Ur = U + (size_t)row * Nx;
        double t = 0.0;
        int n = 0;
        if constexpr (VEC) {
            const int nq = Nx / Ch::NV;
            constexpr int CH = 2;   // chunks per lane loaded before any is summed
            for (int q0 = lane; q0 < nq; q0 += 32 * CH) {
                Ch u[CH];
#pragma unroll
                for (int m = 0; m < CH; ++m)
                    if (q0 + 32 * m < nq) u[m].load(Ur + (size_t)(q0 + 32 * m) * Ch::NV); else u[m].zero();
#pragma unroll
                for (int m = 0; m < CH; ++m) {
#pragma unroll
                    for (int c = 0; c < Ch::NV; ++c) t += (double)u[m].x[c];
                    if (q0 + 32 * m < nq) n += Ch::NV;
                }
            }
        } else {
            for (int i = lane; i < Nx; i += 32) { t += (double)Ur[i]; ++n; }
        }
        s.add((t + n * ub) * a);
        w.add(n * a);
    }
    block_sum2(s.s, w.s, part, bc.idx().x);
}
template <typename T, bool VEC>
__global__ void __launch_bounds__(256) k_bulk_partial(Dims d, const T *__restrict__ U, const double *__restrict__ dyc,
                                                      const double *__restrict__ dzc, const double *__restrict__ ubd,
                                                      double *__restrict__ part) {
    pdl_enter();
    k_bulk_partial_body<T, VEC>(HwBlock(), d, U, dyc, dzc, ubd, part);
}

// Final pass over the block partials (one block): compensated per-thread sums in a fixed order, then a fixed tree;
// writes Ub and the shift Ub_target - Ub.
template <class BC>
__device__ __forceinline__ void k_bulk_final_body(const BC &bc, int nparts, const double *__restrict__ part, double Ub_target,
                                                    double *__restrict__ out) {
    __shared__ double tot[2];
    Kahan s, w; s.init(); w.init();
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) { s.add(part[2 * b]); w.add(part[2 * b + 1]); }
    block_sum2(s.s, w.s, tot, 0);   // one block: tot[0], tot[1]
    __syncthreads();
    if (threadIdx.x == 0) {
        const double Ub = tot[0] / fmax(tot[1], 1e-14);
        out[0] = Ub;
        out[1] = Ub_target - Ub;
    }
}
__global__ void __launch_bounds__(256) k_bulk_final(int nparts, const double *__restrict__ part, double Ub_target,
                                                    double *__restrict__ out) {
    pdl_enter();
    k_bulk_final_body(HwBlock(), nparts, part, Ub_target, out);
}

// U += (Ub_target - Ub) on every independent U face (src/time_integration.f90:581-583); four faces per thread
// when the cell count allows 16-byte (FP32) accesses.
template <typename T, class BC>
__device__ __forceinline__ void k_shift_body(const BC &bc, const Dims &d, T *__restrict__ U, const double *__restrict__ dU) {
    const T s = (T)dU[1];
    const long long stride = (long long)bc.dim().x * blockDim.x;
    const long long first = (long long)bc.idx().x * blockDim.x + threadIdx.x;
    if constexpr (sizeof(T) == 4) {
        if ((d.cells & 3) == 0) {
            float4 *U4 = reinterpret_cast<float4 *>(U);
            for (long long p = first; p < d.cells / 4; p += stride) {
                float4 x = U4[p];
                x.x = x.x + s; x.y = x.y + s; x.z = x.z + s; x.w = x.w + s;
                U4[p] = x;
            }
            return;
        }
    }
    for (long long p = first; p < d.cells; p += stride) U[p] = U[p] + s;
}
template <typename T>
__global__ void __launch_bounds__(256) k_shift(Dims d, T *__restrict__ U, const double *__restrict__ dU) {
    pdl_enter();
    k_shift_body<T>(HwBlock(), d, U, dU);
}

// check_divergence (src/projection.f90:607-639), max |U| over the U faces and the NaN / |u| > 1e8 guard of
// output_monitor (src/monitor.f90:32-58) in one pass: out[0] = max |div u|, out[1] = max |U| (bit patterns, atomicMax
// per block), flag |= 1 when the guard trips.  div u = (U_i - U_{i-1})/dx_i + (V_j - V_{j-1})/dy_j +
// (W_k - W_{k-1})/dz_k in double, divided as the reference divides; U is the stored field plus the base profile.
// A warp walks whole x-rows (row = k*Ny + j), four cells per lane loaded before any is used.
template <typename T>
__global__ void __launch_bounds__(256) k_monitor_rows(Dims d, const T *__restrict__ U, const T *__restrict__ V,
                                                      const T *__restrict__ W, const double *__restrict__ ubd,
                                                      const double *__restrict__ dxc, const double *__restrict__ dyc,
                                                      const double *__restrict__ dzc, unsigned long long *__restrict__ out,
                                                      int *__restrict__ flag) {
    pdl_enter();
    double mdiv = 0.0, mu = 0.0;
    int bad = 0;
    const int rows = d.Ny * d.Nz, Nx = d.Nx, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int row = blockIdx.x * wpb + (threadIdx.x >> 5); row < rows; row += gridDim.x * wpb) {
        const int k = row / d.Ny, j = row - k * d.Ny;
        const double ub = ubd[j], dy = dyc[j], dz = dzc[k];
        const T *Ur = U + (size_t)row * Nx, *Vr = V + (size_t)row * Nx, *Wr = W + (size_t)row * Nx;
        const int jm = j - 1 < 0 ? (d.yper ? d.Ny - 1 : -1) : j - 1;
        const T *Vm = jm < 0 ? nullptr : V + ((size_t)k * d.Ny + jm) * Nx;
        const T *Wm = W + ((size_t)(k == 0 ? d.Nz - 1 : k - 1) * d.Ny + j) * Nx;
        constexpr int CH = 4;
        for (int i0 = lane; i0 < Nx; i0 += 32 * CH) {
            T u0[CH], um[CH], v0[CH], vm[CH], w0[CH], wm[CH];
#pragma unroll
            for (int m = 0; m < CH; ++m) {
                const int i = i0 + 32 * m;
                if (i < Nx) {
                    u0[m] = Ur[i]; um[m] = Ur[i == 0 ? Nx - 1 : i - 1];
                    v0[m] = Vr[i]; vm[m] = Vm ? Vm[i] : T(0);
                    w0[m] = Wr[i]; wm[m] = Wm[i];
                }
            }
#pragma unroll
            for (int m = 0; m < CH; ++m) {
                const int i = i0 + 32 * m;
                if (i < Nx) {
                    const double du = (double)u0[m] - (double)um[m], dv = (double)v0[m] - (double)vm[m];
                    const double dw = (double)w0[m] - (double)wm[m];
                    mdiv = fmax(mdiv, fabs(du / dxc[i] + dv / dy + dw / dz));
                    const double ut = (double)u0[m] + ub;
                    mu = fmax(mu, fabs(ut));
                    if (!(fabs(ut) <= 1e8) || !(fabs((double)v0[m]) <= 1e8) || !(fabs((double)w0[m]) <= 1e8)) bad = 1;
                }
            }
        }
    }
    block_max2_atomic(mdiv, mu, out);
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

// wall_diag_sums (src/wallmodel.f90:700-723): the sums of the wall model's u_tau (tx, planes (wall, k, i)) over the
// reference's columns i = 2..nx-1, k = 2..nzg-1 into out[0], out[1].  Those are the Nx*Nz independent columns plus
// the periodic duplicate k = nzg-1 of the first z-plane, so plane k = 0 counts twice and the column count is
// Nx*(Nz+1).  One block, compensated per-thread sums then a fixed tree.
__global__ void __launch_bounds__(256) k_wall_diag(int Nx, int Nz, const double *__restrict__ tx,
                                                   double *__restrict__ out) {
    pdl_enter();
    Kahan s, w; s.init(); w.init();
    const int plane = Nx * Nz;
    for (int q = threadIdx.x; q < plane + Nx; q += blockDim.x) {
        const int p = q < plane ? q : q - plane;
        s.add(tx[p]);
        w.add(tx[plane + p]);
    }
    block_sum2(s.s, w.s, out, 0);   // one block
}

// The monitor values (the layout of dfdm_monitor): t, dt, mean U, max |U|, max |div u|, CFL conv, CFL visc, mean
// u_tau of the lower and upper wall, NaN flag.  dtt = {dt of the step, t, dt before landing, landing targets} when
// the time step lives on the device, else null and the host's t and dt are used.  One thread.
__global__ void k_monitor_final(const unsigned long long *__restrict__ bits, const int *__restrict__ flag,
                                const double *__restrict__ bulk, const double *__restrict__ wsum, int ncol,
                                const double *__restrict__ dtt, double t_host, double dt_host, double *__restrict__ out) {
    pdl_enter();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double dt = dtt ? dtt[2] : dt_host, t = dtt ? dtt[1] : t_host;
    out[0] = t;
    out[1] = dt;
    out[2] = bulk[0];
    out[3] = __longlong_as_double((long long)bits[3]);
    out[4] = __longlong_as_double((long long)bits[2]);
    out[5] = __longlong_as_double((long long)bits[0]) * dt;
    out[6] = __longlong_as_double((long long)bits[1]) * dt;
    out[7] = wsum ? wsum[0] / (double)ncol : 0.0;
    out[8] = wsum ? wsum[1] / (double)ncol : 0.0;
    out[9] = *flag ? 1.0 : 0.0;
}

// compute_cfl (src/monitor.f90:304-424) without its IBM, buoyancy, rotation and actuator terms: the maxima over the
// centres of |u_c|/dx + |v_c|/dy_j + |w_c|/dz_k (face velocities averaged to the centre) and of
// (nu + nu_t) 2 (1/dx^2 + 1/dy_j^2 + 1/dz_k^2), as exact integer maxima of their bit patterns.  The convective term
// is computed in the storage type (double in the FP64 form, float in the FP32-mixed form, whose velocities carry
// float rounding already) as |u_i + u_{i-1} + 2 ub| (dx^-1/2) + ..., the halving moved onto the metric (exact); the
// viscous term is in double from the row maximum of nu_t (exact: the term grows monotonically with nu_t).  A warp
// walks whole x-rows (row = k*Ny + j) with no per-cell index division; a lane reads 16-byte chunks of cells and takes
// U_{i-1} of its first cell from the lane before (the warp's last lane carries it to the next batch); without VEC
// (Nx not a multiple of the chunk) one cell at a time.
template <typename T, bool VEC>
__global__ void __launch_bounds__(256) k_cfl(Dims d, const T *__restrict__ U, const T *__restrict__ V,
                                             const T *__restrict__ W, const T *__restrict__ NU,
                                             const double *__restrict__ ubd, double inv_dx, const double *__restrict__ dyc,
                                             const double *__restrict__ dzc, double nu, unsigned long long *__restrict__ out) {
    pdl_enter();
    typedef Chunk<T> Ch;
    constexpr int NV = Ch::NV;
    double mv = 0.0;
    T mc = T(0);
    const double idx2 = inv_dx * inv_dx;
    const T hx = (T)(0.5 * inv_dx);
    const int rows = d.Ny * d.Nz, Nx = d.Nx, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int row = blockIdx.x * wpb + (threadIdx.x >> 5); row < rows; row += gridDim.x * wpb) {
        const int k = row / d.Ny, j = row - k * d.Ny;
        const double idy = 1.0 / fmax(dyc[j], 1e-14), idz = 1.0 / fmax(dzc[k], 1e-14);
        const T ub2 = (T)(2.0 * ubd[j]), hy = (T)(0.5 * idy), hz = (T)(0.5 * idz);
        const T *Ur = U + (size_t)row * Nx, *Vr = V + (size_t)row * Nx, *Wr = W + (size_t)row * Nx;
        // V at j-1 (periodic wrap, or the zero wall value below the first row) and W at k-1 (periodic)
        const int jm = j - 1 < 0 ? (d.yper ? d.Ny - 1 : -1) : j - 1;
        const T *Vm = jm < 0 ? nullptr : V + ((size_t)k * d.Ny + jm) * Nx;
        const T *Wm = W + ((size_t)(k == 0 ? d.Nz - 1 : k - 1) * d.Ny + j) * Nx;
        const T *Nr = NU ? NU + (size_t)row * Nx : nullptr;
        T nmax = T(0);
        auto cell = [&](T u0, T um, T v0, T vm, T w0, T wm, T nt) {
            mc = max(mc, fabs(u0 + um + ub2) * hx + fabs(v0 + vm) * hy + fabs(w0 + wm) * hz);
            nmax = max(nmax, nt);
        };
        if constexpr (VEC) {
            const int nq = Nx / NV;
            constexpr int CH = 2;                        // chunks per lane loaded before any is used
            T carry = Ur[Nx - 1];                        // U_{i-1} of the row's first cell (periodic)
            for (int q0 = 0; q0 < nq; q0 += 32 * CH) {   // warp-uniform: every lane takes part in the shuffles
                Ch u[CH], v[CH], vm[CH], w[CH], wm[CH], n[CH];
#pragma unroll
                for (int m = 0; m < CH; ++m) {
                    const int q = q0 + lane + 32 * m;
                    if (q < nq) {
                        const size_t o = (size_t)q * NV;
                        u[m].load(Ur + o); v[m].load(Vr + o); w[m].load(Wr + o); wm[m].load(Wm + o);
                        if (Vm) vm[m].load(Vm + o); else vm[m].zero();
                        if (Nr) n[m].load(Nr + o); else n[m].zero();
                    } else {
                        u[m].zero(); v[m].zero(); vm[m].zero(); w[m].zero(); wm[m].zero(); n[m].zero();
                    }
                }
#pragma unroll
                for (int m = 0; m < CH; ++m) {
                    const T up = __shfl_up_sync(0xffffffffu, u[m].x[NV - 1], 1);
                    const T um0 = lane == 0 ? carry : up;
                    carry = __shfl_sync(0xffffffffu, u[m].x[NV - 1], 31);
                    if (q0 + lane + 32 * m < nq) {
                        cell(u[m].x[0], um0, v[m].x[0], vm[m].x[0], w[m].x[0], wm[m].x[0], n[m].x[0]);
#pragma unroll
                        for (int c = 1; c < NV; ++c)
                            cell(u[m].x[c], u[m].x[c - 1], v[m].x[c], vm[m].x[c], w[m].x[c], wm[m].x[c], n[m].x[c]);
                    }
                }
            }
        } else {
            for (int i = lane; i < Nx; i += 32)
                cell(Ur[i], Ur[i == 0 ? Nx - 1 : i - 1], Vr[i], Vm ? Vm[i] : T(0), Wr[i], Wm[i], Nr ? Nr[i] : T(0));
        }
        mv = fmax(mv, (nu + (double)nmax) * 2.0 * (idx2 + idy * idy + idz * idz));
    }
    block_max2_atomic((double)mc, mv, out);
}

// select_dt (src/monitor.f90:429-444) and landing_dt (:450-458) on the device, one thread.  dtt = {dt of the
// step, t, dt before landing, landing targets [3..7]}: the adaptive dt from the CFL maxima (bit patterns of
// non-negative doubles per unit dt), kept in dtt[2] as the dt between steps; then, for each target in select_dt's
// order (tsave_next, chunk_tsave_next, slice_tnext, line_tnext, sim_end_time; NaN: none), a remainder below 2 dt
// is taken in one step and one between dt and 2 dt in two halves.  A target within 1e-10 of t counts as reached.
// The step's dt goes to dtt[0] and t advances.
__global__ void k_select_dt(const unsigned long long *__restrict__ cfl, double *__restrict__ dtt, int adaptive,
                            double cfl_target, double cfl_safety, double dt_min, double dt_max) {
    pdl_enter();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double dt = dtt[2];
    if (adaptive) {
        const double conv = __longlong_as_double((long long)cfl[0]) * dt;
        const double visc = __longlong_as_double((long long)cfl[1]) * dt;
        const double now = fmax(conv, visc);
        if (now > 0.0) dt = fmax(dt_min, fmin(dt_max, dt * cfl_target / now * cfl_safety));
    }
    dtt[2] = dt;
    for (int q = 0; q < 5; ++q) {
        const double rem = dtt[3 + q] - dtt[1];   // NaN: no target
        if (rem > 1e-10 && rem < 2.0 * dt) dt = rem > dt ? 0.5 * rem : rem;
    }
    dtt[0] = dt;
    dtt[1] += dt;
}

// Volume-weighted kinetic energy 0.5 <u.u> with face velocities averaged to the centres (compensated sums).
template <typename T>
__global__ void __launch_bounds__(256) k_ke_partial(Dims d, const T *__restrict__ U, const T *__restrict__ V,
                                                    const T *__restrict__ W, double dx, const double *__restrict__ dyc,
                                                    const double *__restrict__ dzc, const double *__restrict__ ubd,
                                                    double *__restrict__ part) {
    pdl_enter();
    Kahan s, w; s.init(); w.init();
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < d.cells; p += (long long)gridDim.x * blockDim.x) {
        int i = (int)(p % d.Nx);
        long long q = p / d.Nx;
        int j = (int)(q % d.Ny), k = (int)(q / d.Ny);
        double vol = dyc[j] * dzc[k] * dx;
        double uc = 0.5 * (((double)U[p] + ubd[j]) + ((double)U[idx3(d, wrap(i - 1, d.Nx), j, k)] + ubd[j]));
        double vc = 0.5 * ((double)ld_yf(V, d, i, j, k) + (double)ld_yf(V, d, i, j - 1, k));
        double wc = 0.5 * ((double)W[p] + (double)W[idx3(d, i, j, wrap(k - 1, d.Nz))]);
        s.add(0.5 * (uc * uc + vc * vc + wc * wc) * vol);
        w.add(vol);
    }
    block_sum2(s.s, w.s, part, blockIdx.x);
}

__global__ void k_ratio_final(int nparts, const double *__restrict__ part, double *__restrict__ out) {
    pdl_enter();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Kahan s, w; s.init(); w.init();
    for (int b = 0; b < nparts; ++b) { s.add(part[2 * b]); w.add(part[2 * b + 1]); }
    out[0] = s.s / w.s;
}


// ---- state transfer ---------------------------------------------------------------------------------------------
// Field kinds of the ghosted reference arrays.
enum FieldKind { FK_U = 0, FK_V = 1, FK_W = 2, FK_P = 3, FK_NUT = 4 };

// Device index and sign of one ghosted reference element (Fortran 1-based (I,J,K)).  Mirrors the ghost rules of
// apply_boundary_conditions (velocities), finish_pressure_ghosts (P) and sgs_fill_ghosts (nu_t); sign 0 means the
// element is zero.
__device__ __forceinline__ long long map_ghost(const Dims &d, int kind, int I, int J, int K, int &sign, int &jdev) {
    sign = 1;
    int i = I - 2, j = J - 2, k = K - 2;
    i = ((i % d.Nx) + d.Nx) % d.Nx;   // x periodic for every field (faces and centres alike)
    k = ((k % d.Nz) + d.Nz) % d.Nz;   // z periodic
    if (d.yper) {
        if (kind == FK_P) {
            if (j < 0 || j >= d.Ny) j = 0;          // P(1) = P(2), P(nyg-1) = P(2), P(nyg) = P(nyg-1)
        } else {
            j = ((j % d.Ny) + d.Ny) % d.Ny;
        }
    } else if (kind == FK_V) {
        if (j < 0 || j >= d.Ny - 1) { sign = 0; j = 0; }   // wall faces (index kept valid, never read)
    } else if (kind == FK_P) {
        if (j < 0) j = 0;
        if (j >= d.Ny) j = d.Ny - 1;
    } else if (kind == FK_NUT) {
        if (j < 0 || j >= d.Ny) { sign = 0; j = 0; }
    } else {   // U, W: no-slip mirror
        if (j < 0) { j = 0; sign = -1; }
        if (j >= d.Ny) { j = d.Ny - 1; sign = -1; }
    }
    jdev = j;
    return idx3(d, i, j, k);
}

// Expand a device field into its ghosted FP64 reference array (n1 x n2 x n3, Fortran order).
template <typename T>
__global__ void __launch_bounds__(256) k_pack(Dims d, int kind, int n1, int n2, int n3, const T *__restrict__ f,
                                              const double *__restrict__ ubd, double *__restrict__ out) {
    pdl_enter();
    long long n = (long long)n1 * n2 * n3;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        int I = (int)(p % n1) + 1;
        long long q = p / n1;
        int J = (int)(q % n2) + 1, K = (int)(q / n2) + 1;
        int sg, jd;
        long long s = map_ghost(d, kind, I, J, K, sg, jd);
        double v = 0.0;
        if (sg != 0) {
            v = (double)f[s];
            if (kind == FK_U) v += ubd[jd];
            if (sg < 0) v = -v;
        }
        out[p] = v;
    }
}

// Extract the independent cells of a ghosted FP64 reference array (n1 x n2 x n3) into a device field.
template <typename T>
__global__ void __launch_bounds__(256) k_unpack(Dims d, int kind, int n1, int n2, const double *__restrict__ in,
                                                const double *__restrict__ ubd, T *__restrict__ f) {
    pdl_enter();
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < d.cells; p += (long long)gridDim.x * blockDim.x) {
        int i = (int)(p % d.Nx);
        long long q = p / d.Nx;
        int j = (int)(q % d.Ny), k = (int)(q / d.Ny);
        T v;
        if (kind == FK_V && !d.yper && j == d.Ny - 1) v = T(0);   // top wall face
        else {
            double x = in[((long long)(k + 1) * n2 + (j + 1)) * n1 + (i + 1)];
            if (kind == FK_U) x -= ubd[j];
            v = (T)x;
        }
        f[p] = v;
    }
}

// rhs arrays in the reference's interior shapes (2:n1+1, 2:n2+1, 2:n3+1): device element (i,j,k) -> (i,j,k)
// for i < Nx etc.; the duplicated last periodic cell repeats index 0.
template <typename T>
__global__ void __launch_bounds__(256) k_pack_interior(Dims d, int n1, int n2, int n3, const T *__restrict__ f,
                                                       double *__restrict__ out) {
    pdl_enter();
    long long n = (long long)n1 * n2 * n3;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        int i = (int)(p % n1);
        long long q = p / n1;
        int j = (int)(q % n2), k = (int)(q / n2);
        i = i % d.Nx; k = k % d.Nz; if (d.yper) j = j % d.Ny;
        out[p] = (double)f[idx3(d, i, j, k)];
    }
}

// Wall-stress planes to the reference's tau_x (nx,2,nzg) [is_z = 0] or tau_z (nxg,2,nz) [is_z = 1] shapes.
// Interior rows map to the device planes; the duplicated periodic row repeats row 0 and the ghost rows copy the
// nearest computed row, as compute_flat_wall_eqwm does (src/wallmodel.f90:515-522, :571-578).
__global__ void k_pack_tau(Dims d, int is_z, int n1, int n3, const double *__restrict__ t, double *__restrict__ out) {
    pdl_enter();
    long long n = (long long)n1 * 2 * n3;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        int i = (int)(p % n1) - 1;
        long long q = p / n1;
        int iw = (int)(q % 2), k = (int)(q / 2) - 1;
        if (!is_z) {   // U faces in x (clamp), centres in z (wrap the duplicate and the ghosts to row 0)
            i = min(max(i, 0), d.Nx - 1);
            if (k < 0 || k >= d.Nz) k = 0;
        } else {       // centres in x (wrap), faces in z (clamp)
            if (i < 0 || i >= d.Nx) i = 0;
            k = min(max(k, 0), d.Nz - 1);
        }
        out[p] = t[((long long)iw * d.Nz + k) * d.Nx + i];
    }
}

// Real field in the rhs_p shape (2:nxg, 2:nyg-1, 2:nzg) -> independent centres.
template <typename T>
__global__ void __launch_bounds__(256) k_unpack_rhs_p(Dims d, int n1, int n2, const double *__restrict__ in, T *__restrict__ f) {
    pdl_enter();
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < d.cells; p += (long long)gridDim.x * blockDim.x) {
        int i = (int)(p % d.Nx);
        long long q = p / d.Nx;
        int j = (int)(q % d.Ny), k = (int)(q / d.Ny);
        f[p] = (T)in[((long long)k * n2 + j) * n1 + i];
    }
}

// Independent centres -> rhs_p shape with apply_periodic_xz_pressure's copies (rhs_p(nxg-1) = rhs_p(2),
// rhs_p(:,:,nzg-1) = rhs_p(:,:,2), periodic y: rhs_p(:,nyg-1,:) = rhs_p(:,2,:)); the outermost planes (nxg, nzg)
// that the reference leaves unset at one rank are written as copies of the next wrap.
template <typename T>
__global__ void __launch_bounds__(256) k_pack_rhs_p(Dims d, int n1, int n2, int n3, const T *__restrict__ f, double *__restrict__ out) {
    pdl_enter();
    long long n = (long long)n1 * n2 * n3;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        int i = (int)(p % n1);
        long long q = p / n1;
        int j = (int)(q % n2), k = (int)(q / n2);
        i = i % d.Nx; k = k % d.Nz; if (d.yper) j = j % d.Ny;
        out[p] = (double)f[idx3(d, i, j, k)];
    }
}

}  // namespace dfdm
