// kernels_tma.cuh -- the packed FP32 stage kernel with its z-plane tiles moved by the Tensor Memory Accelerator.
//
// The arithmetic is k_tiled2's (stage_pair, packed FP32x2 pairs, 64 x 8 cells per block marching through a z-chunk);
// only the way the planes reach shared memory differs.  Each plane of each input field arrives as one 3-D TMA box
// (cp.async.bulk.tensor, 72 x 10 x 1 floats starting at x = i0-4, y = j0-1; 72 x 11 for the potential phi of the
// fused correction) whose completion is counted on an mbarrier, instead of per-element cp.async copies.  One thread
// issues the boxes of plane k+4 while the block evaluates plane k, into a ring of six plane slots per field, so four
// planes are in flight.  All boxes read this GPU's own fields (the tensor maps cover the context's own buffers) and
// none uses cluster multicast.
//
// Boundary rules that a box cannot express:
//   * y walls: rows outside 0..Ny-1 arrive zero-filled.  That is already the wall value of V and nu_t; U and W are
//     mirrored with a sign flip, written by the thread that owns the first / last interior row.
//   * periodic x: the first tile's columns x = -2, -1 and the last tile's x = Nx .. Nx+2 arrive zero-filled; two
//     4-wide patch boxes (x = Nx-4 and x = 0) bring the wrapped values, which the fix pass copies in.
// The fix pass is element-local: each thread writes only its own elements, reading their loaded values, the patch
// boxes and phi, which nothing writes, so it needs no barrier of its own.  With the fused correction (CORR) it also
// applies the previous stage's projection, u = u* - grad(phi), with k_correct's arithmetic.
//
// Eligibility (checked on the host): FP32, walls in y, Nx a multiple of 4 (TMA needs 16-byte row strides and
// 16-byte aligned x coordinates).  Every mbarrier wait is bounded: a wait that gives up sets the context's error flag,
// waits (bounded again) for the block's copies still in flight and returns, and the host reports DFDM_ERR_TIMEOUT.
#pragma once

#include <cuda.h>

#include "kernels_step.cuh"

namespace dfdm {

// The tensor maps of one launch: main boxes and x-wrap patch boxes of U, V, W (and nu_t), and of phi.
struct TmaMaps {
    CUtensorMap f[4];    // 72 x 10 x 1 boxes of the input fields u, v, w, nu_t
    CUtensorMap fp[4];   // 4 x 10 x 1 patch boxes of the same fields
    CUtensorMap phi;     // 72 x 11 x 1 box of phi (CORR)
    CUtensorMap phip;    // 4 x 11 x 1 patch box of phi
};

namespace tma {
constexpr int BX = 72, BY = 10, BYP = 11, PW = 4;
constexpr int SLOTS = 6, AHEAD = 4;
constexpr int FSLOT = 2944;              // bytes of a field slot: 72*10*4 = 2880 rounded up to 128
constexpr int PSLOT = 3200;              // phi slot: 72*11*4 = 3168 rounded up to 128
constexpr int QSLOT = 256;               // a patch box (4*10*4 or 4*11*4 bytes) rounded up to 128
constexpr unsigned WAIT_LIMIT = 1u << 22;   // polls of a bounded mbarrier wait (the copies land in microseconds)

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// true when the phase with this parity completed; false after WAIT_LIMIT polls
__device__ __forceinline__ bool mbar_wait(uint64_t *b, unsigned parity) {
    for (unsigned it = 0; it < WAIT_LIMIT; ++it)
        if (mbar_try_wait(b, parity)) return true;
    return false;
}
// untiled bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned), completing on the same barrier
__device__ __forceinline__ void load_bulk(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void load_box(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n"
        ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
}  // namespace tma

template <bool LES, bool CORR> struct TmaSmem {
    static constexpr int NF = LES ? 4 : 3;
    alignas(128) unsigned char f[NF][tma::SLOTS][tma::FSLOT];
    alignas(128) unsigned char fp[NF][tma::SLOTS][2][tma::QSLOT];
    alignas(128) unsigned char p[CORR ? tma::SLOTS : 1][CORR ? tma::PSLOT : 128];
    alignas(128) unsigned char pp[CORR ? tma::SLOTS : 1][2][CORR ? tma::QSLOT : 128];
    alignas(8) uint64_t full[tma::SLOTS];
    alignas(16) float zm[tma::SLOTS][8];   // the z metrics of each slot's plane (32-byte bulk copies)
};

template <bool LES, bool WM, bool HYB, bool CORR>
__global__ void __launch_bounds__(256, 2) k_tma2(StepArgs<float> a, const __grid_constant__ TmaMaps tm,
                                                 const double *__restrict__ tau_x, const double *__restrict__ tau_z,
                                                 StageCoef sc, int kc, float *__restrict__ uo, float *__restrict__ vo,
                                                 float *__restrict__ wo, float *__restrict__ f1u, float *__restrict__ f1v,
                                                 float *__restrict__ f1w, float *__restrict__ us, float *__restrict__ vs,
                                                 float *__restrict__ wsf, float *__restrict__ rhs_only,
                                                 int *__restrict__ err) {
    pdl_enter();
    using namespace tma;
    constexpr int NF = LES ? 4 : 3, PX = BX;
    constexpr int NPAIR = 34;   // pairs at tile columns 2..69 (x = i0-2 .. i0+65): every column a stencil reads
    extern __shared__ __align__(128) unsigned char smem_raw[];
    TmaSmem<LES, CORR> &S = *reinterpret_cast<TmaSmem<LES, CORR> *>(smem_raw);
    const Dims &d = a.d;
    const int Nx = d.Nx, Ny = d.Ny, Nz = d.Nz;
    const int i0 = blockIdx.x * 64, j0 = blockIdx.y * 8;
    const int k0 = blockIdx.z * kc, kend = min(k0 + kc, Nz);
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int i = i0 + 2 * tx, j = j0 + ty;
    const bool active = i < Nx && j < Ny;
    // tile columns c hold x = i0 - 4 + c; x < 0 and x >= Nx come from the patch boxes.  Cells read x up to
    // i0 + 65 and the correction phi up to i0 + 66.
    const bool wrapl = i0 == 0, wrapr = i0 + 66 >= Nx;
    const bool lo_row = j0 == 0, hi_row = j0 + 8 >= Ny;   // a wall ghost row (y = -1 / y = Ny) lies in the box
    const bool edge = wrapl || wrapr || lo_row || hi_row;
    const int npatch = (wrapl ? 1 : 0) + (wrapr ? 1 : 0);
    // bytes one plane brings: every field's main box and its patches, (CORR) phi of the same plane, and the plane's
    // eight z metrics
    const unsigned tx_bytes = NF * (BX * BY * 4 + npatch * PW * BY * 4) +
                              (CORR ? BX * BYP * 4 + npatch * PW * BYP * 4 : 0) + 32;
    // planes k0-1 .. kend are evaluated or read as neighbours; CORR also needs phi(kend+1) for the fix of kend
    const int plast = kend + (CORR ? 1 : 0);

    auto slot_of = [&](int p) { return (p - (k0 - 1)) % SLOTS; };
    auto par_of = [&](int p) { return (unsigned)(((p - (k0 - 1)) / SLOTS) & 1); };
    // the boxes of plane p into slot_of(p): thread 0 only
    auto issue = [&](int p) {
        const int s = slot_of(p);
        uint64_t *bar = &S.full[s];
        const int pw = p < 0 ? p + Nz : (p >= Nz ? p - Nz : p);
        fence_proxy_async();   // the slot was last read and written through the generic proxy
        mbar_expect_tx(bar, tx_bytes);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            load_box(S.f[f][s], &tm.f[f], i0 - 4, j0 - 1, pw, bar);
            if (wrapl) load_box(S.fp[f][s][0], &tm.fp[f], Nx - 4, j0 - 1, pw, bar);
            if (wrapr) load_box(S.fp[f][s][1], &tm.fp[f], 0, j0 - 1, pw, bar);
        }
        if constexpr (CORR) {
            load_box(S.p[s], &tm.phi, i0 - 4, j0 - 1, pw, bar);
            if (wrapl) load_box(S.pp[s][0], &tm.phip, Nx - 4, j0 - 1, pw, bar);
            if (wrapr) load_box(S.pp[s][1], &tm.phip, 0, j0 - 1, pw, bar);
        }
        load_bulk(S.zm[s], a.zm8 + 8 * pw, 32, bar);
    };
    bool ok = true;
    auto wait_plane = [&](int p) {
        if (ok && !mbar_wait(&S.full[slot_of(p)], par_of(p))) {
            ok = false;
            atomicExch(err, 1);
        }
    };
    // loaded value at tile column c (even: a pair), row r of a box with row pitch BX, or of its patch box
    auto raw2 = [&](const unsigned char *tile, const unsigned char *pl, const unsigned char *pr, int c, int r) {
        const int xg = i0 - 4 + c;
        if (wrapl && xg < 0) return *reinterpret_cast<const float2 *>(pl + 4 * (r * PW + c));
        if (wrapr && xg >= Nx) return *reinterpret_cast<const float2 *>(pr + 4 * (r * PW + (xg - Nx)));
        return *reinterpret_cast<const float2 *>(tile + 4 * (r * BX + c));
    };
    auto raw1 = [&](const unsigned char *tile, const unsigned char *pl, const unsigned char *pr, int c, int r) {
        const int xg = i0 - 4 + c;
        if (wrapl && xg < 0) return *reinterpret_cast<const float *>(pl + 4 * (r * PW + c));
        if (wrapr && xg >= Nx) return *reinterpret_cast<const float *>(pr + 4 * (r * PW + (xg - Nx)));
        return *reinterpret_cast<const float *>(tile + 4 * (r * BX + c));
    };
    // the fix pass of plane p: wrapped columns, wall ghost rows and (CORR) the previous stage's projection
    auto fix = [&](int p) {
        if (!CORR && !edge) return;
        const int s = slot_of(p);
        const int pw = p < 0 ? p + Nz : (p >= Nz ? p - Nz : p);
        const int s1 = slot_of(p + 1);   // CORR: phi(p+1) for the w correction
        const float iz = CORR ? Arith<float>::inv(a.mz.df, a.mz.idf, pw) : 0.0f;
        for (int e = threadIdx.x; e < NPAIR * BY; e += 256) {
            const int r = e / NPAIR, c = 2 + 2 * (e - r * NPAIR);
            const int yg = j0 - 1 + r;
            if (yg < 0 || yg >= Ny) continue;   // wall ghost rows: written by the owner of the mirrored row
            const int xg = i0 - 4 + c;          // even, like Nx: a pair lies wholly on one side of x = 0 and x = Nx
            if (xg >= Nx + 2) continue;         // beyond the wrapped halo: read by no active cell
            const bool wc = (wrapl && xg < 0) || (wrapr && xg >= Nx);
            const bool mlo = lo_row && yg == 0, mhi = hi_row && yg == Ny - 1;
            if (!CORR && !wc && !mlo && !mhi) continue;
            float2 u = raw2(S.f[0][s], S.fp[0][s][0], S.fp[0][s][1], c, r);
            float2 v = raw2(S.f[1][s], S.fp[1][s][0], S.fp[1][s][1], c, r);
            float2 w = raw2(S.f[2][s], S.fp[2][s][0], S.fp[2][s][1], c, r);
            if constexpr (CORR) {
                // project_velocity of the previous stage with k_correct's arithmetic
                const unsigned char *P0 = S.p[s], *P0l = S.pp[s][0], *P0r = S.pp[s][1];
                const float2 pc = raw2(P0, P0l, P0r, c, r);
                const float pn = raw1(P0, P0l, P0r, c + 2, r);
                const float2 pz = raw2(S.p[s1], S.pp[s1][0], S.pp[s1][1], c, r);
                u.x = u.x - (pc.y - pc.x) * a.inv_dx; u.y = u.y - (pn - pc.y) * a.inv_dx;
                w.x = w.x - (pz.x - pc.x) * iz; w.y = w.y - (pz.y - pc.y) * iz;
                if (yg < d.NyV) {
                    const float iy = Arith<float>::inv(a.my.df, a.my.idf, yg);
                    const float2 py = raw2(P0, P0l, P0r, c, r + 1);
                    v.x = v.x - (py.x - pc.x) * iy; v.y = v.y - (py.y - pc.y) * iy;
                }
            }
            const int o = 4 * (r * BX + c);
            *reinterpret_cast<float2 *>(S.f[0][s] + o) = u;
            *reinterpret_cast<float2 *>(S.f[1][s] + o) = v;
            *reinterpret_cast<float2 *>(S.f[2][s] + o) = w;
            if (LES && wc)
                *reinterpret_cast<float2 *>(S.f[NF - 1][s] + o) = raw2(S.f[NF - 1][s], S.fp[NF - 1][s][0], S.fp[NF - 1][s][1], c, r);
            // no-slip mirror of U and W into the ghost row (V and nu_t keep the zero the box brought)
            if (mlo) {
                *reinterpret_cast<float2 *>(S.f[0][s] + o - 4 * BX) = make_float2(-u.x, -u.y);
                *reinterpret_cast<float2 *>(S.f[2][s] + o - 4 * BX) = make_float2(-w.x, -w.y);
            }
            if (mhi && r + 1 < BY) {
                *reinterpret_cast<float2 *>(S.f[0][s] + o + 4 * BX) = make_float2(-u.x, -u.y);
                *reinterpret_cast<float2 *>(S.f[2][s] + o + 4 * BX) = make_float2(-w.x, -w.y);
            }
        }
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < SLOTS; ++s) mbar_init(&S.full[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int p = k0 - 1; p <= min(k0 - 1 + AHEAD, plast); ++p) issue(p);

    F2 ubr[3];
#pragma unroll
    for (int dj = -1; dj <= 1; ++dj) {
        int gj = min(j, Ny - 1) + dj;
        float sgn = 1.0f;
        if (gj < 0 || gj >= Ny) { gj = gj < 0 ? 0 : Ny - 1; sgn = -1.0f; }
        ubr[dj + 1] = F2(sgn * __ldg(a.ub + gj));
    }
    AxisLocal<F2> Y;
    Y.load(a.my, min(j, Ny - 1));

    // planes k0-1, k0, k0+1 fixed before the first evaluation (CORR: their fix reads phi up to plane k0+2)
    for (int p = k0 - 1; p <= k0 + (CORR ? 2 : 1); ++p) wait_plane(p);
    if (ok) { fix(k0 - 1); fix(k0); fix(k0 + 1); }
    ok = __syncthreads_and(ok);
    const int cloc = (ty + 1) * PX + 4 + 2 * tx;
    for (int k = k0; k < kend && ok; ++k) {
        // plane k+AHEAD goes into the slot of plane k+AHEAD-SLOTS = k-2, last read before the previous barrier
        if (threadIdx.x == 0 && k + AHEAD <= plast) issue(k + AHEAD);
        if (active) {
            const int sm_ = slot_of(k - 1), s0 = slot_of(k), sp = slot_of(k + 1);
            TileQ2<PX> q;
            q.c = cloc;
            q.ub[0] = ubr[0]; q.ub[1] = ubr[1]; q.ub[2] = ubr[2];
            q.u[0] = (const float *)S.f[0][sm_]; q.u[1] = (const float *)S.f[0][s0]; q.u[2] = (const float *)S.f[0][sp];
            q.v[0] = (const float *)S.f[1][sm_]; q.v[1] = (const float *)S.f[1][s0]; q.v[2] = (const float *)S.f[1][sp];
            q.w[0] = (const float *)S.f[2][sm_]; q.w[1] = (const float *)S.f[2][s0]; q.w[2] = (const float *)S.f[2][sp];
            q.n[0] = (const float *)S.f[NF - 1][sm_]; q.n[1] = (const float *)S.f[NF - 1][s0];
            q.n[2] = (const float *)S.f[NF - 1][sp];
            stage_pair<LES, WM, HYB>(a, q, Y, S.zm[s0], tau_x, tau_z, sc, i, j, k, uo, vo, wo, f1u, f1v, f1w, us, vs,
                                     wsf, rhs_only);
        }
        if (k + 2 <= kend) {
            wait_plane(k + 2);
            if (CORR) wait_plane(k + 3);
            if (ok) fix(k + 2);
        }
        ok = __syncthreads_and(ok);
    }
    if (!ok) {
        // a wait gave up: let every issued copy land (bounded again) before the block's shared memory is released
        const int pmax = min(plast, kend + AHEAD);
        for (int p = k0 - 1; p <= pmax; ++p) (void)mbar_wait(&S.full[slot_of(p)], par_of(p));
    }
}

}  // namespace dfdm
