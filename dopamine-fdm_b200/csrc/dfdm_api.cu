// dfdm_api.cu -- the C ABI (include/dfdm.h): context set-up, the RK3 step driver, state transfer and the unit
// entry points that mirror the reference's Fortran subroutines.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <limits>
#include <map>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "dfdm.h"
#include "dfdm_common.cuh"
#include "fft_smem.cuh"
#include "kernels_diag.cuh"
#include "kernels_fft2l.cuh"
#include "kernels_poisson.cuh"
#include "kernels_step.cuh"
#include "kernels_hybrid.cuh"
#include "kernels_tma.cuh"
#include "kernels_les.cuh"
#include "tridiag_eigen.h"
#include "kernels_group.cuh"

using namespace dfdm;

namespace {

thread_local std::string g_err;
thread_local long long g_launches = 0;   // kernels enqueued by this thread (read back into the context)

struct TuneEntry {
    int variant;
    double ms[3];
};
std::mutex g_tune_mu;
std::map<std::array<int, 6>, TuneEntry> g_tune;   // stage-kernel choice per (device, Nx, Ny, Nz, LES, wall model)

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

#define CK(call)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) {                                                                       \
            return fail(e_ == cudaErrorMemoryAllocation ? DFDM_ERR_NOMEM : DFDM_ERR_CUDA,              \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                          \
        }                                                                                              \
    } while (0)

#define CKL()                                                                                          \
    do {                                                                                               \
        cudaError_t e_ = cudaGetLastError();                                                           \
        if (e_ != cudaSuccess) return fail(DFDM_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
        ++g_launches;                                                                                  \
    } while (0)

const double PI = 4.0 * std::atan(1.0);   // pi = 4d0*datan(1d0)

// cuTensorMapEncodeTiled through the runtime's driver entry point, so the library loads where no driver is present
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    });
    return fn;
}
const int MAX_NY = 1024;                  // longest y line of the shared-memory y transform

}  // namespace

// ----------------------------------------------------------------------------------------------------------------
struct dfdm_ctx {
    dfdm_params prm;
    int prec = DFDM_FP64;
    size_t ts = 8;                 // sizeof storage type
    int nx = 0, ny = 0, nz = 0, nxg = 0, nyg = 0, nzg = 0;
    int yper = 0;
    Dims d{};
    // host metrics (1-based, as the reference's arrays)
    std::vector<double> x, y, z, xg, yg, zg;
    double dx = 0, dz = 0, Ly = 0;
    int nwl = 0, wm_filter_mode = 0, wm = 0, les = 0;
    double dPdx = 0, dPdz = 0;
    // device memory
    std::vector<void *> allocs;
    char *arena = nullptr;            // one allocation holding every buffer that dfdm_create makes
    size_t arena_size = 0, arena_off = 0;
    bool in_create = false;
    void *u = nullptr, *v = nullptr, *w = nullptr, *uo = nullptr, *vo = nullptr, *wo = nullptr;
    void *f1u = nullptr, *f1v = nullptr, *f1w = nullptr, *us = nullptr, *vs = nullptr, *wsf = nullptr;
    // Fused corrections (DNS or filtered wall model, no hybrid scheme: the stage kernel is the only reader of the
    // corrected velocity at stages 2 and 3): the stage-1 and stage-2 corrections run inside the next stage kernel's
    // loader instead of k_correct, U keeps the step-start velocity until the stage-3 correction (so it also serves
    // as uo), and u* alternates between us/vs/wsf and us2/vs2/ws2 so that a stage kernel reads the previous u*
    // while it writes its own.
    void *us2 = nullptr, *vs2 = nullptr, *ws2 = nullptr;
    bool fuse_ok = false, fused = false;
    void *nut = nullptr, *p = nullptr, *phi = nullptr, *spec = nullptr, *rhs3 = nullptr;
    void *my_t = nullptr, *mz_t = nullptr;      // 6 metric arrays each, storage type
    void *zm8 = nullptr;                        // FP32: the z metrics of each plane in load8 order (StepArgs::zm8)
    double *d_wfac = nullptr;                   // LES + wall model: wall factors of the eddy viscosity (k_wall_sgs)
    double *my_d = nullptr, *mz_d = nullptr;    // same in double
    void *tw_x = nullptr, *twr_x = nullptr, *tw_z = nullptr, *tw_y = nullptr;
    FFTPlan plan_x{}, plan_z{}, plan_y{};
    double *d_kxx = nullptr, *d_kzz = nullptr, *d_kyy = nullptr, *d_lo = nullptr, *d_di = nullptr, *d_up = nullptr;
    double *d_rpiv = nullptr;                   // 1/D(r) of every (kx,kz) tridiagonal system, layout (kz, r, kx)
    double *d_dxc = nullptr, *d_dyc = nullptr, *d_dzc = nullptr;
    void *d_ub = nullptr;                       // streamwise base profile (storage type), zero in FP64
    bool ub_set = false;
    double *d_ubd = nullptr;                    // the same in double
    WallState wsd{};
    double *red_part = nullptr, *red_out = nullptr;
    int red_blocks = 0;
    int cfl_blocks = 1;
    // monitor block: [0],[1] CFL maxima, [2] max |div u|, [3] max |U| (bit patterns), [4] guard flag (int),
    // [5],[6] wall u_tau sums (double), [8..17] the dfdm_monitor values
    unsigned long long *d_mon = nullptr;
    unsigned long long *d_cfl = nullptr;        // convective and viscous CFL maxima (bit patterns)
    // device time step: with the adaptive time step (cfl_adaptive = 1) or an output-landing target, dt and t live on
    // the device in d_dtt = {dt of the step, t, dt before landing, landing targets[5]}, set by k_select_dt at every
    // step start, so a run of steps (or its graph) needs no host round trip
    double *d_dtt = nullptr;
    bool adaptive = false, landing = false;
    double cfl_target = 0.5, cfl_safety = 0.9, dt_min = 1e-10, dt_max = 1e10;
    // landing targets in select_dt's order: tsave_next, chunk_tsave_next, slice_tnext, line_tnext, sim_end_time
    double t_land[5] = {NAN, NAN, NAN, NAN, NAN};
    void *adv = nullptr;   // advection_scheme = 2: the dissipative terms, 3 fields of the storage type
    bool dev_dt() const { return adaptive || landing; }
    double *staging = nullptr;
    size_t staging_n = 0;
    // launch geometry
    int lx = 8, tzx = 8;
    int kc_stage = 8, kc_sgs = 8;               // z-planes per block of the tiled kernels
    int kc_stage2 = 8;                          // the same for the packed FP32 stage kernel
    int kc_les = 8;                             // the same for the LES stage kernel with in-tile eddy viscosity
    // LES: the stage kernels compute the eddy viscosity in their tiles (k_les) instead of reading it from a
    // separate pass (dfdm_set_sgs_in_tile; the pass is the default)
    bool sgs_tile = false;
    int kc_hyb = 32;                            // the same for the hybrid-scheme kernel
    int stage_variant = 0;                      // FP32 stage kernel in use: 0 one cell per thread, 1 packed pairs,
                                                // 2 packed pairs with TMA plane tiles
    double stage_ms[3] = {-1.0, -1.0, -1.0};    // autotuner timings of the variants (ms per launch), -1 = not timed
    // TMA stage kernel (variant 2): eligible with FP32, walls in y and Nx a multiple of 4.  Tensor maps of each input
    // buffer (main box and x-wrap patch box), encoded on first use; a host-mapped flag that a bounded mbarrier wait
    // sets when it gives up.
    bool tma_ok = false;
    int kc_tma = 8;
    std::map<std::pair<const void *, int>, std::array<CUtensorMap, 2>> tmaps;
    int *h_err = nullptr, *d_err = nullptr;
    size_t smem_x = 0, smem_z = 0, smem_y = 0;
    // two-level register transforms (fft_reg.cuh) where the length has a split; Stockham otherwise
    bool x2 = false, z2 = false, y2 = false;
    bool ys3 = false;                           // walls in y: the staged-column y solve (k_ysolve3) fits
    // inflow/outflow x (x_bc_type = 1): a context for the DCT-IV pressure solve only (dfdm_solve_poisson); Nx = nx - 1
    // cells, every x mode kx = 0..Nx-1 in the spectrum, d_dct the Nx x Nx DCT-IV matrix
    bool xdct = false;
    void *d_dct = nullptr;   // the DCT-IV matrix, in the context's precision
    // the 4-wall duct (z_bc_type = 1 with walls in y): a context for its pressure solve only; Nz = nz - 1 cells, the
    // z-eigenmode transforms (forward, inverse) in the context's precision, and a second spectrum for them
    bool duct = false;
    void *d_zf = nullptr, *d_zi = nullptr, *spec2 = nullptr;
    // spanwise walls alone (z_bc_type = 1 with periodic y): a context for that pressure solve only, holding the field
    // with y and z exchanged (Ny = nz - 1 wall-bounded cells, Nz = ny - 2 periodic rows) so that the channel's
    // transforms and y solve serve it
    bool zwall = false;
    int lx2 = 1, lxi2 = 1, thr_z2 = 256, thr_y2 = 256;   // x lines per block: forward, inverse
    size_t smem_x2 = 0, smem_xi2 = 0, smem_z2 = 0, smem_y2 = 0;
    cudaStream_t own_stream = nullptr, stream = nullptr;
    // asynchronous state transfer (dfdm_set_state_async / dfdm_get_state_async): one copy stream per direction, one
    // FP64 staging buffer per field and direction, and events that keep a buffer from being refilled before its
    // last reader is done.  Made on first use, outside the footprint.
    cudaStream_t cin = nullptr, cout = nullptr;
    double *stage_in[4] = {nullptr, nullptr, nullptr, nullptr}, *stage_out[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t ev_in[4] = {}, ev_unpacked[4] = {}, ev_packed[4] = {}, ev_out[4] = {};
    double t = 0.0;
    bool wmf_seeded = false;
    // graphs
    bool graphs = false;
    cudaGraphExec_t gexec = nullptr;
    cudaGraph_t graph = nullptr;
    bool unit_projection = false;    // dfdm_compute_projection_step: u* is the resident state, not an increment
    bool projected = false;          // the resident velocity is a full step's output (no set_state since)
    long long launches = 0;          // kernels enqueued (host-side count)
    long long graph_launches = 0;    // kernels in the captured step graph
};

namespace {

template <typename T> struct Impl;

int dalloc(dfdm_ctx *c, void **p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (c->in_create) {   // carve from the context's arena (256-byte aligned)
        const size_t need = (bytes + 255) & ~(size_t)255;
        if (c->arena_off + need > c->arena_size) {
            *p = nullptr;
            return fail(DFDM_ERR_NOMEM, "context arena exhausted (" + std::to_string(c->arena_off + need) + " > " +
                                            std::to_string(c->arena_size) + " bytes)");
        }
        *p = c->arena + c->arena_off;
        c->arena_off += need;
        CK(cudaMemsetAsync(*p, 0, bytes, c->stream));
        return DFDM_OK;
    }
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(DFDM_ERR_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
    }
    c->allocs.push_back(*p);
    CK(cudaMemsetAsync(*p, 0, bytes, c->stream));
    return DFDM_OK;
}

void centres_of(const std::vector<double> &f, int n, std::vector<double> &c) {
    // src/initialization.f90:250-270 (f and c 1-based)
    int nm = n - 1;
    std::vector<double> m(nm + 1);
    for (int i = 1; i <= nm; ++i) m[i] = 0.5 * (f[i] + f[i + 1]);
    c.assign(nm + 3, 0.0);
    for (int i = 1; i <= nm; ++i) c[i + 1] = m[i];
    c[1] = m[1] - 2.0 * (m[1] - f[1]);
    c[nm + 2] = m[nm] + 2.0 * (f[n] - m[nm]);
}

// Metric arrays of one direction, offset by one (index -1 valid), 6 arrays of length N+3 each:
//   [0] dc, [1] df, [2] w0, [3] w1, [4] 1/dc, [5] 1/df  -- see Metric1D
void build_metric(const std::vector<double> &f, const std::vector<double> &g, int nf, int N, std::vector<double> &out) {
    const int L = N + 3;
    out.assign(6 * (size_t)L, 0.0);
    int ng = nf + 1;
    for (int jp = -1; jp <= N + 1; ++jp) {
        int j = jp + 2;   // reference index
        size_t o = (size_t)(jp + 1);
        if (j - 1 >= 1 && j <= nf) out[0 * L + o] = f[j] - f[j - 1];
        if (j + 1 <= ng && j >= 1) out[1 * L + o] = g[j + 1] - g[j];
        if (j >= 1 && j <= nf && j + 1 <= ng) {
            double w0 = (g[j + 1] - f[j]) / (g[j + 1] - g[j]);
            out[2 * L + o] = w0;
            out[3 * L + o] = 1.0 - w0;
        }
        if (out[0 * L + o] != 0.0) out[4 * L + o] = 1.0 / out[0 * L + o];
        if (out[1 * L + o] != 0.0) out[5 * L + o] = 1.0 / out[1 * L + o];
    }
}

template <typename T> Metric1D<T> metric_view(void *base, int N) {
    const int L = N + 3;
    T *b = (T *)base;
    Metric1D<T> m;
    m.dc = b + 0 * L + 1; m.df = b + 1 * L + 1; m.w0 = b + 2 * L + 1; m.w1 = b + 3 * L + 1;
    m.idc = b + 4 * L + 1; m.idf = b + 5 * L + 1;
    return m;
}

template <typename T> int upload_as(dfdm_ctx *c, void **dst, const std::vector<double> &h) {
    std::vector<T> tmp(h.size());
    for (size_t i = 0; i < h.size(); ++i) tmp[i] = (T)h[i];
    int rc = dalloc(c, dst, tmp.size() * sizeof(T));
    if (rc) return rc;
    CK(cudaMemcpyAsync(*dst, tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DFDM_OK;
}

template <typename T> int upload_twiddles(dfdm_ctx *c, void **dst, int n, int count) {
    std::vector<double> h(2 * (size_t)count);
    for (int k = 0; k < count; ++k) {
        double a = -2.0 * PI * (double)k / (double)n;
        h[2 * k] = std::cos(a);
        h[2 * k + 1] = std::sin(a);
    }
    return upload_as<T>(c, dst, h);
}

template <typename T> StepArgs<T> step_args(dfdm_ctx *c) {
    StepArgs<T> a;
    a.d = c->d;
    a.my = metric_view<T>(c->my_t, c->d.Ny);
    a.mz = metric_view<T>(c->mz_t, c->d.Nz);
    a.myd = metric_view<double>(c->my_d, c->d.Ny);
    a.mzd = metric_view<double>(c->mz_d, c->d.Nz);
    double inv_dx = 1.0 / c->dx;
    a.nu = (T)c->prm.nu;
    a.inv_dx = (T)inv_dx;
    a.inv_dx2 = (T)(inv_dx * inv_dx);
    a.dx2 = (T)(c->dx * c->dx);
    a.dPdx = (T)c->dPdx;
    a.dPdz = (T)c->dPdz;
    a.w_adv = (T)((c->prm.advection_scheme == 1) ? 0.0 : 0.5);
    a.nwl = c->nwl;
    a.wm = c->wm;
    a.sgs_model = c->prm.sgs_model;
    a.C_amd = (T)c->prm.C_amd;
    a.c_V = (T)(2.5 * c->prm.Cs_vreman * c->prm.Cs_vreman);
    a.nu_d = c->prm.nu;
    a.Ly = c->Ly;
    a.yg2 = c->yg[2];
    a.ygtop = c->Ly - c->yg[c->nyg - 1];
    a.ub = (const T *)c->d_ub;
    a.ubd = c->d_ubd;
    a.adv = (const T *)c->adv;
    a.phi = (const T *)c->phi;
    a.zm8 = (const float *)c->zm8;
    a.wfac = c->d_wfac;
    return a;
}

template <typename T> PoissonArgs<T> poisson_args(dfdm_ctx *c) {
    PoissonArgs<T> a;
    a.d = c->d;
    a.my = metric_view<T>(c->my_t, c->d.Ny);
    a.mz = metric_view<T>(c->mz_t, c->d.Nz);
    a.inv_dx = (T)(1.0 / c->dx);
    a.norm = (double)((long long)c->d.Nx * (long long)c->d.Nz);
    a.pdiv = c->prm.dt * (3.0 / 4.0);
    a.dtp = c->dev_dt() ? c->d_dtt : nullptr;
    a.fNx = make_fastdiv((unsigned)c->d.Nx);
    a.fNy = make_fastdiv((unsigned)c->d.Ny);
    a.fM = make_fastdiv((unsigned)(c->d.Nx / 2));
    a.fM1 = make_fastdiv((unsigned)(c->d.Nx / 2 + 1));
    return a;
}

dim3 cell_grid(const Dims &d) { return dim3((d.Nx + 31) / 32, (d.Ny + 7) / 8, d.Nz); }
const dim3 CELL_BLOCK(32, 8, 1);
constexpr int TILE_X = 32, TILE_Y = 8;   // (i,j) tile of the 2.5-D blocked kernels
const int TILE_X2 = 64;   // x cells per block of the packed FP32 stage kernel (32 threads x 2 cells)
dim3 tile_grid(const Dims &d, int kc, int tx = TILE_X) { return dim3((d.Nx + tx - 1) / tx, (d.Ny + TILE_Y - 1) / TILE_Y, (d.Nz + kc - 1) / kc); }
// z-planes per block: enough blocks for about four waves at the measured occupancy, at most 32 planes
// z-planes per block of the 2.5-D tiled kernels.  A block of a (tx x ty) column runs kc planes after loading `halo`
// extra planes; blocks_per_sm of them share an SM.  The chunking minimises (kc + halo) x g, g the waves the launch
// takes: full waves of blocks_per_sm x nsm blocks, then a last wave as long as its most loaded SM (its blocks over
// blocks_per_sm) but never shorter than 0.6 of a wave (a lone block hides little latency).  Measured at 256 x 192 x
// 256 cells: the packed stage kernel and the order-3 hybrid kernel are fastest with 3 chunks of 86 planes (one
// wave), the order-5 hybrid kernel (3 blocks per SM) with 6 chunks of 43; the earlier fixed four-wave target (13
// chunks of 20 planes, 4.2 waves) cost about 1.5 % of a step.
int choose_kc(const Dims &d, int blocks_per_sm, int nsm, int tx = TILE_X, int ty = TILE_Y, int halo = 2) {
    const long long cols = (long long)((d.Nx + tx - 1) / tx) * ((d.Ny + ty - 1) / ty);
    const int bps = std::max(1, blocks_per_sm), sms = std::max(1, nsm);
    const long long cap = (long long)bps * sms;
    double best = -1.0;
    int best_kc = d.Nz;
    for (int chunks = 1; chunks <= d.Nz; ++chunks) {
        const int kc = (d.Nz + chunks - 1) / chunks;
        if (kc < 2 && d.Nz >= 2) break;
        const long long blocks = cols * ((d.Nz + kc - 1) / kc), rem = blocks % cap;
        double g = (double)(blocks / cap);
        if (rem) g += std::max(0.6, (double)((rem + sms - 1) / sms) / bps);
        const double cost = g * (kc + halo);
        if (best < 0.0 || cost < best - 1e-9) { best = cost; best_kc = kc; }
    }
    return std::max(1, best_kc);
}

int reduce_grid(const Dims &d);

template <typename T> struct Impl {
    typedef typename cplx_t<T>::type C;
    static constexpr int CT = (sizeof(T) == 8) ? 4 : 8;    // kx columns per block of the column transforms (64 B rows)
    static constexpr int NL = (sizeof(T) == 8) ? 8 : 16;   // kx columns per block of the two-level column transforms
    static T *f(void *p) { return (T *)p; }
    // threads of a two-level column block: one work item per thread in the longer step
    static int col_threads(int n1, int n2) { return std::min(256, ((NL * std::max(n1, n2) + 31) / 32) * 32); }

    static int setup_fft2l(dfdm_ctx *c) {
        const Dims &d = c->d;
        int rc = DFDM_OK;
        auto setattr = [&](const void *fn, size_t bytes) {
            if (rc) return;
            cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
            if (e != cudaSuccess) rc = fail(DFDM_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
        };
        c->x2 = with_fft2l(d.Nx / 2, [&](auto n) {
            constexpr int N = decltype(n)::value;
            const size_t perline = (size_t)(RowLayout<N>::LDA + RowLayout<N>::LDT) * sizeof(C);
            c->lx2 = RowLines<T, N>::value;   // the forward kernel's loop bound assumes exactly this
            c->smem_x2 = (size_t)c->lx2 * perline;
            c->lxi2 = (int)std::max<size_t>(1, std::min<size_t>(64, 73728 / perline));   // measured best for the inverse
            c->smem_xi2 = (size_t)c->lxi2 * RowLayout<N>::LDT * sizeof(C);
            setattr((const void *)k_fwd_x2<T, true, N>, c->smem_x2);
            setattr((const void *)k_fwd_x2<T, false, N>, c->smem_x2);
            setattr((const void *)k_inv_x2<T, N>, c->smem_xi2);
        });
        c->z2 = with_fft2l(d.Nz, [&](auto n) {
            constexpr int N = decltype(n)::value;
            c->smem_z2 = (size_t)N * NL * sizeof(C);
            c->thr_z2 = col_threads(Split<N>::N1, Split<N>::N2);
            setattr((const void *)k_col2<T, 0, NL, N>, c->smem_z2);
            setattr((const void *)k_col2<T, 1, NL, N>, c->smem_z2);
        });
        c->y2 = d.yper && with_fft2l(d.Ny, [&](auto n) {
            constexpr int N = decltype(n)::value;
            c->smem_y2 = (size_t)2 * N * NL * sizeof(C);
            c->thr_y2 = col_threads(Split<N>::N1, Split<N>::N2);
            setattr((const void *)k_col2<T, 2, NL, N>, c->smem_y2);
        });
        return rc;
    }

    // div u* (from_div) or the real field src, and the forward real-to-complex x transform into the spectrum
    static int fwd_x(dfdm_ctx *c, bool from_div, const T *src) {
        const Dims &d = c->d;
        cudaStream_t st = c->stream;
        const long long lines = (long long)d.Ny * d.Nz;
        if (c->x2) {
            const int nb = (int)((lines + c->lx2 - 1) / c->lx2);
            with_fft2l(d.Nx / 2, [&](auto n) {
                constexpr int N = decltype(n)::value;
                if (from_div)
                    k_fwd_x2<T, true, N><<<nb, 256, c->smem_x2, st>>>(poisson_args<T>(c), c->lx2, f(c->us), f(c->vs), f(c->wsf),
                                                                       nullptr, (C *)c->spec, (const C *)c->tw_x, (const C *)c->twr_x);
                else
                    k_fwd_x2<T, false, N><<<nb, 256, c->smem_x2, st>>>(poisson_args<T>(c), c->lx2, nullptr, nullptr, nullptr,
                                                                        src, (C *)c->spec, (const C *)c->tw_x, (const C *)c->twr_x);
            });
        } else {
            const int nb = (int)((lines + c->lx - 1) / c->lx);
            if (from_div)
                k_fwd_x<T, true><<<nb, 256, c->smem_x, st>>>(poisson_args<T>(c), c->lx, f(c->us), f(c->vs), f(c->wsf), nullptr,
                                                             (C *)c->spec, c->plan_x, (const C *)c->tw_x, (const C *)c->twr_x);
            else
                k_fwd_x<T, false><<<nb, 256, c->smem_x, st>>>(poisson_args<T>(c), c->lx, nullptr, nullptr, nullptr, src,
                                                              (C *)c->spec, c->plan_x, (const C *)c->tw_x, (const C *)c->twr_x);
        }
        CKL();
        return DFDM_OK;
    }


    // the transforms of a DCT-IV Poisson context: z (two-level or Stockham) and the y solve
    static int setup_poisson_only(dfdm_ctx *c) {
        const Dims &d = c->d;
        int optin = 0, dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        c->tzx = CT;
        c->smem_z = 2 * (size_t)d.Nz * c->tzx * sizeof(C);
        if (c->smem_z > (size_t)optin) return fail(DFDM_ERR_UNSUPPORTED, "grid too large for the shared-memory transforms");
        for (const void *fn : {(const void *)k_col_fft<T, 0, CT>, (const void *)k_col_fft<T, 1, CT>})
            CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        int rc = DFDM_OK;
        c->z2 = with_fft2l(d.Nz, [&](auto n) {
            constexpr int N = decltype(n)::value;
            c->smem_z2 = (size_t)N * NL * sizeof(C);
            c->thr_z2 = col_threads(Split<N>::N1, Split<N>::N2);
            for (const void *fn : {(const void *)k_col2<T, 0, NL, N>, (const void *)k_col2<T, 1, NL, N>})
                if (!rc && cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->smem_z2) != cudaSuccess)
                    rc = fail(DFDM_ERR_CUDA, "cudaFuncSetAttribute failed");
        });
        if (rc) return rc;
        return setup_ys3(c, optin);
    }
    // the staged-column y solve where three of its blocks fit on an SM (as setup_kernels decides it)
    static int setup_ys3(dfdm_ctx *c, int optin) {
        const Dims &d = c->d;
        c->ys3 = false;
        if (ysolve3_smem<T>(d.Ny) <= (size_t)optin) {
            CK(cudaFuncSetAttribute(k_ysolve3<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
            int ys_occ = 0;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ys_occ, k_ysolve3<T>, YS_COLS, (int)ysolve3_smem<T>(d.Ny)));
            c->ys3 = ys_occ >= 3;
        }
        return DFDM_OK;
    }
    // the transforms of a duct Poisson context: x (two-level or Stockham) and the y solve
    static int setup_duct_only(dfdm_ctx *c) {
        const Dims &d = c->d;
        int optin = 0, dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        const int M = d.Nx / 2;
        c->lx = std::max(1, std::min(64, 1024 / std::max(1, M)));
        c->smem_x = 2 * (size_t)c->lx * M * sizeof(C);
        if (c->smem_x > (size_t)optin) return fail(DFDM_ERR_UNSUPPORTED, "grid too large for the shared-memory transforms");
        CK(cudaFuncSetAttribute(k_fwd_x<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        CK(cudaFuncSetAttribute(k_inv_x<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        if (c->zwall) {   // the periodic axis, transformed by the z kernels
            c->tzx = CT;
            c->smem_z = 2 * (size_t)d.Nz * c->tzx * sizeof(C);
            if (c->smem_z > (size_t)optin) return fail(DFDM_ERR_UNSUPPORTED, "grid too large for the shared-memory transforms");
            for (const void *fn : {(const void *)k_col_fft<T, 0, CT>, (const void *)k_col_fft<T, 1, CT>})
                CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        }
        if (int rc = setup_ys3(c, optin)) return rc;
        return setup_fft2l(c);
    }
    // dfdm_solve_poisson on a spanwise-wall context: the channel's chain on the field with y and z exchanged
    static int solve_zwall(dfdm_ctx *c, int n1, int n2, int n3) {
        const Dims &d = c->d;
        const size_t n = (size_t)n1 * n2 * n3;
        cudaStream_t st = c->stream;
        k_unpack_rhs_p_swap<T><<<reduce_grid(d), 256, 0, st>>>(d, n1, n2, c->staging, f(c->phi));
        CKL();
        if (int rc = fwd_x(c, false, f(c->phi))) return rc;
        for (int which : {3, 4, 5, 6})
            if (int rc = launch(c, which, 1)) return rc;
        k_pack_rhs_p_swap<T><<<(int)std::min<size_t>((n + 255) / 256, 148 * 8), 256, 0, st>>>(d, n1, n2, n3, f(c->phi),
                                                                                             c->staging);
        CKL();
        return DFDM_OK;
    }
    // dfdm_solve_poisson on a duct context: staging (rhs_p) -> phi -> x FFT -> z eigenmodes -> y solve per (kx, mode)
    // -> z^-1 -> x FFT^-1 -> staging.  The eigenmode transforms run out of place; the y solve works on whichever
    // buffer is the context's spectrum, so the two are swapped around it.
    static int solve_duct(dfdm_ctx *c, int n1, int n2, int n3) {
        const Dims &d = c->d;
        const size_t n = (size_t)n1 * n2 * n3;
        cudaStream_t st = c->stream;
        k_unpack_rhs_p<T><<<reduce_grid(d), 256, 0, st>>>(d, n1, n2, c->staging, f(c->phi));
        CKL();
        // x: the FFT, or with inflow/outflow x the DCT-IV (the duct of the reference's CPU build)
        const int nbd = (d.Ny * d.Nz + DCT_LINES - 1) / DCT_LINES, ntd = (d.Nx + 31) / 32 * 32;
        if (c->xdct) {
            k_dct_x<T><<<nbd, ntd, 0, st>>>(d, f(c->phi), f(c->d_dct), (C *)c->spec);
            CKL();
        } else if (int rc = fwd_x(c, false, f(c->phi))) {
            return rc;
        }
        const long long cols = (long long)d.Ny * d.Nxc;
        const dim3 g((unsigned)((cols + ZEIG_COLS - 1) / ZEIG_COLS), (unsigned)((d.Nz + zeig_modes<T>() - 1) / zeig_modes<T>()));
        k_zeig<T><<<g, ZEIG_COLS, 0, st>>>(d, (const C *)c->spec, (C *)c->spec2, f(c->d_zf));
        CKL();
        {
            struct Swap {
                dfdm_ctx *c;
                explicit Swap(dfdm_ctx *cc) : c(cc) { std::swap(c->spec, c->spec2); }
                ~Swap() { std::swap(c->spec, c->spec2); }
            } swapped(c);
            if (int rc = launch(c, 4, 1)) return rc;
            k_zeig<T><<<g, ZEIG_COLS, 0, st>>>(d, (const C *)c->spec, (C *)c->spec2, f(c->d_zi));
            CKL();
        }
        if (c->xdct) {
            const T inv_norm = (T)(1.0 / (2.0 * (double)d.Nx * (double)d.Nz));   // the nzp cancels the inverse matrix's
            k_idct_x<T><<<nbd, ntd, 0, st>>>(d, (const C *)c->spec, f(c->d_dct), inv_norm, f(c->phi));
            CKL();
        } else if (int rc = launch(c, 6, 1)) {
            return rc;
        }
        k_pack_rhs_p_bc<T><<<(int)std::min<size_t>((n + 255) / 256, 148 * 8), 256, 0, st>>>(d, n1, n2, n3, c->xdct ? 0 : 1,
                                                                                           0, f(c->phi), c->staging);
        CKL();
        return DFDM_OK;
    }
    // dfdm_solve_poisson on a DCT-IV context: staging (rhs_p) -> phi -> DCT-IV x -> z -> y solve -> z^-1 -> DCT-IV x
    // -> phi / (2 nxp nzp) -> staging
    static int solve_dct(dfdm_ctx *c, int n1, int n2, int n3) {
        const Dims &d = c->d;
        const size_t n = (size_t)n1 * n2 * n3;
        k_unpack_rhs_p<T><<<reduce_grid(d), 256, 0, c->stream>>>(d, n1, n2, c->staging, f(c->phi));
        CKL();
        const int nb = (d.Ny * d.Nz + DCT_LINES - 1) / DCT_LINES, nt = (d.Nx + 31) / 32 * 32;
        k_dct_x<T><<<nb, nt, 0, c->stream>>>(d, f(c->phi), f(c->d_dct), (C *)c->spec);
        CKL();
        for (int which : {3, 4, 5})
            if (int rc = launch(c, which, 1)) return rc;
        const T inv_norm = (T)(1.0 / (2.0 * (double)d.Nx * (double)d.Nz));
        k_idct_x<T><<<nb, nt, 0, c->stream>>>(d, (const C *)c->spec, f(c->d_dct), inv_norm, f(c->phi));
        CKL();
        k_pack_rhs_p_bc<T><<<(int)std::min<size_t>((n + 255) / 256, 148 * 8), 256, 0, c->stream>>>(d, n1, n2, n3, 0, 1,
                                                                                                   f(c->phi), c->staging);
        CKL();
        return DFDM_OK;
    }

    static int setup_kernels(dfdm_ctx *c) {
        const Dims &d = c->d;
        const int M = d.Nx / 2;
        c->lx = std::max(1, std::min(64, 1024 / std::max(1, M)));
        c->smem_x = 2 * (size_t)c->lx * M * sizeof(C);
        c->tzx = CT;
        c->smem_z = 2 * (size_t)d.Nz * c->tzx * sizeof(C);
        c->smem_y = 2 * (size_t)d.Ny * c->tzx * sizeof(C);
        size_t maxs = std::max(c->smem_x, std::max(c->smem_z, c->smem_y));
        if (maxs > 227 * 1024) return fail(DFDM_ERR_UNSUPPORTED, "grid too large for the shared-memory transforms");
        // The dynamic shared-memory cap is an attribute of the kernel for the whole process, not of a launch: for
        // kernels whose shared memory depends on the grid it is set to the device's opt-in maximum, so that a
        // context of a smaller grid cannot lower it under a larger context's launches (or its captured graphs).
        int optin = 0, dev0 = 0;
        CK(cudaGetDevice(&dev0));
        CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev0));
        CK(cudaFuncSetAttribute(k_fwd_x<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        CK(cudaFuncSetAttribute(k_fwd_x<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        CK(cudaFuncSetAttribute(k_inv_x<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        CK(cudaFuncSetAttribute(k_col_fft<T, 0, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        CK(cudaFuncSetAttribute(k_col_fft<T, 1, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        CK(cudaFuncSetAttribute(k_col_fft<T, 2, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
        // the staged-column y solve where at least three of its blocks fit on an SM: with fewer, too few columns
        // sweep at a time (measured at Ny = 192, FP32: 101 us against 42 us for k_ysolve2; at Ny = 96 and 64 it
        // is 15-30 % faster than k_ysolve2)
        c->ys3 = false;
        if (!d.yper && ysolve3_smem<T>(d.Ny) <= (size_t)optin) {
            const int ysm = (int)ysolve3_smem<T>(d.Ny);
            CK(cudaFuncSetAttribute(k_ysolve3<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
            int ys_occ = 0;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ys_occ, k_ysolve3<T>, YS_COLS, ysm));
            c->ys3 = ys_occ >= 3;
        }
        int dev = 0, nsm = 148, occ = 1;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        const void *stage_fn;
        if constexpr (sizeof(T) == 8)
            stage_fn = c->les ? (const void *)k_tiled<T, true, true, TILE_X, TILE_Y, 0>
                              : (const void *)k_tiled<T, false, true, TILE_X, TILE_Y, 0>;
        else
            stage_fn = c->les ? (c->wm ? (const void *)k_tiled<T, true, true, TILE_X, TILE_Y, 0>
                                       : (const void *)k_tiled<T, true, false, TILE_X, TILE_Y, 0>)
                              : (c->wm ? (const void *)k_tiled<T, false, true, TILE_X, TILE_Y, 0>
                                       : (const void *)k_tiled<T, false, false, TILE_X, TILE_Y, 0>);
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, stage_fn, TILE_X * TILE_Y, 0));
        c->kc_stage = choose_kc(d, occ, nsm);
        if constexpr (sizeof(T) == 4) {
            const void *fn2 = c->les ? (c->wm ? (const void *)k_tiled2<true, true> : (const void *)k_tiled2<true, false>)
                                     : (c->wm ? (const void *)k_tiled2<false, true> : (const void *)k_tiled2<false, false>);
            int occ2 = 1;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, fn2, 256, 0));
            c->kc_stage2 = choose_kc(d, occ2, nsm, TILE_X2);
            if (int rc = setup_tma(c, nsm)) return rc;
        }
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tiled<T, false, false, TILE_X, TILE_Y, 1>, TILE_X * TILE_Y, 0));
        c->kc_sgs = choose_kc(d, occ, nsm);
        if (c->les) {
            const int b0 = (int)les::smem_bytes<T>(false), b1 = (int)les::smem_bytes<T>(true);
            CK(cudaFuncSetAttribute(k_les<T, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b0));
            CK(cudaFuncSetAttribute(k_les<T, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b1));
            CK(cudaFuncSetAttribute(k_les<T, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b0));
            CK(cudaFuncSetAttribute(k_les<T, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b1));
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_les<T, true, true>, les::NT, b1));
            c->kc_les = choose_kc(d, std::max(1, occ), nsm, les::TX, les::TY, 4);
            // measured on the Re_tau 395 LES grid (96 x 64 x 96, one B200): the separate pass plus the stage kernel
            // take 0.254 ms per FP32 step against 0.326 ms in the tile, so the pass is the default and fused
            // corrections (which need the in-tile form) start off
            c->sgs_tile = false;
            c->fused = false;
        }
        // the CFL maxima: one wave of resident blocks, at most one warp per x-row
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cfl<T, true>, 256, 0));
        c->cfl_blocks = (int)std::max(1LL, std::min((long long)std::max(1, occ) * nsm, ((long long)d.Ny * d.Nz + 7) / 8));
        if (c->prm.advection_scheme == 2) {
            const bool quads = sizeof(T) == 4 && d.Nx % 4 == 0;
            const void *fn = nullptr;
            auto attr = [&](const void *k, size_t bytes) {
                CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
                return DFDM_OK;
            };
            if (int rc = attr((const void *)k_adv_hybrid_faces<T, 3, 2>, hyb_faces_smem_bytes<T, 3>())) return rc;
            if (int rc = attr((const void *)k_adv_hybrid_faces<T, 5, 2>, hyb_faces_smem_bytes<T, 5>())) return rc;
            if (int rc = attr((const void *)k_adv_hybrid_faces<T, 3, 16 / sizeof(T)>, hyb_faces_smem_bytes<T, 3>())) return rc;
            if (int rc = attr((const void *)k_adv_hybrid_faces<T, 5, 16 / sizeof(T)>, hyb_faces_smem_bytes<T, 5>())) return rc;
            const bool o5 = c->prm.adv_order == 5;
            fn = o5 ? (quads ? (const void *)k_adv_hybrid_faces<T, 5, 16 / sizeof(T)> : (const void *)k_adv_hybrid_faces<T, 5, 2>)
                    : (quads ? (const void *)k_adv_hybrid_faces<T, 3, 16 / sizeof(T)> : (const void *)k_adv_hybrid_faces<T, 3, 2>);
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 256, o5 ? hyb_faces_smem_bytes<T, 5>() : hyb_faces_smem_bytes<T, 3>()));
            c->kc_hyb = choose_kc(d, occ, nsm, 32, 8, o5 ? 6 : 4);
        }
        return setup_fft2l(c);
    }

    // The TMA stage kernel (variant 2): eligible with walls in y and Nx a multiple of 4 (16-byte row strides and box
    // origins), when the driver's tensor-map encoder is reachable.  Every instantiation a step can launch gets its
    // dynamic shared memory; the error flag lives in host-mapped pinned memory.
    template <bool LES, bool WM, bool HYB, bool CORR> static int tma_attr() {
        if constexpr (sizeof(T) == 4) {
            CK(cudaFuncSetAttribute(k_tma2<LES, WM, HYB, CORR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sizeof(TmaSmem<LES, CORR>)));
        }
        return DFDM_OK;
    }
    static int setup_tma(dfdm_ctx *c, int nsm) {
        const Dims &d = c->d;
        c->tma_ok = false;
        if (d.yper || d.Nx % 4 != 0 || !encode_tiled()) return DFDM_OK;
        int rc = DFDM_OK;
        for (int les = 0; les < 2 && !rc; ++les)
            for (int wm = 0; wm < 2 && !rc; ++wm)
                for (int hyb = 0; hyb < 2 && !rc; ++hyb) {
                    if (les) rc = wm ? (hyb ? tma_attr<true, true, true, false>() : tma_attr<true, true, false, false>())
                                     : (hyb ? tma_attr<true, false, true, false>() : tma_attr<true, false, false, false>());
                    else rc = wm ? (hyb ? tma_attr<false, true, true, false>() : tma_attr<false, true, false, false>())
                                 : (hyb ? tma_attr<false, false, true, false>() : tma_attr<false, false, false, false>());
                }
        if (!rc) rc = tma_attr<false, true, false, true>();
        if (!rc) rc = tma_attr<false, false, false, true>();
        if (rc) return rc;
        int occ = 1;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_tma2<false, false, false, true>, 256,
                                                         sizeof(TmaSmem<false, true>)));
        c->kc_tma = choose_kc(d, std::max(1, occ), nsm, TILE_X2);
        if (!c->h_err) {
            void *h = nullptr, *dp = nullptr;
            CK(cudaHostAlloc(&h, sizeof(int), cudaHostAllocMapped));
            *(volatile int *)h = 0;
            if (cudaHostGetDevicePointer(&dp, h, 0) != cudaSuccess) {
                cudaFreeHost(h);
                return fail(DFDM_ERR_CUDA, "cudaHostGetDevicePointer of the stage kernel's error flag failed");
            }
            c->h_err = (int *)h;
            c->d_err = (int *)dp;
        }
        c->tma_ok = true;
        return DFDM_OK;
    }
    // the main box (72 x rows x 1) and the x-wrap patch box (4 x rows x 1) of a field buffer, encoded once
    static int tensor_maps(dfdm_ctx *c, const void *buf, int rows, CUtensorMap *main_box, CUtensorMap *patch_box) {
        auto key = std::make_pair(buf, rows);
        auto it = c->tmaps.find(key);
        if (it == c->tmaps.end()) {
            const Dims &d = c->d;
            std::array<CUtensorMap, 2> m;
            const cuuint64_t dims[3] = {(cuuint64_t)d.Nx, (cuuint64_t)d.Ny, (cuuint64_t)d.Nz};
            const cuuint64_t strides[2] = {(cuuint64_t)d.Nx * sizeof(float), (cuuint64_t)d.Nx * d.Ny * sizeof(float)};
            const cuuint32_t estr[3] = {1, 1, 1};
            for (int b = 0; b < 2; ++b) {
                const cuuint32_t box[3] = {b == 0 ? (cuuint32_t)tma::BX : (cuuint32_t)tma::PW, (cuuint32_t)rows, 1};
                CUresult r = encode_tiled()(&m[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void *>(buf), dims,
                                            strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
                if (r != CUDA_SUCCESS) return fail(DFDM_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
            }
            it = c->tmaps.emplace(key, m).first;
        }
        *main_box = it->second[0];
        *patch_box = it->second[1];
        return DFDM_OK;
    }


    // is the output of a full step (so div uo vanishes up to the rounding of its storage).  Solving for div(du)
    // alone keeps that rounding noise, amplified by dx/dt, out of the saved pressure P = phi/(dt*3/4); the
    // correction forms u = uo + du - grad(phi).  Right after set_state (a field that need not be solenoidal), in
    // the unit entry points and in the FP64 form, u* = uo + du is projected as the reference does.
    static bool incr_form(const dfdm_ctx *c, int s) {
        return sizeof(T) == 4 && s == 3 && c->projected && !c->unit_projection;
    }

    // CORR: the input planes are the previous stage's u* (us2/vs2/ws2 after the swap in step_enqueue), corrected in
    // the loader; with fused corrections the step-start velocity U doubles as uo
    template <bool LES, bool WM, bool HYB, bool CORR> static int stage_launch(dfdm_ctx *c, const StageCoef &sc, T *rhs_only) {
        const Dims &d = c->d;
        const T *iu = CORR ? f(c->us2) : f(c->u), *iv = CORR ? f(c->vs2) : f(c->v), *iw = CORR ? f(c->ws2) : f(c->w);
        T *uo = c->fused && !rhs_only ? f(c->u) : f(c->uo), *vo = c->fused && !rhs_only ? f(c->v) : f(c->vo);
        T *wo = c->fused && !rhs_only ? f(c->w) : f(c->wo);
        if constexpr (sizeof(T) == 4) {
            if (c->stage_variant == 2 && c->tma_ok) {
                TmaMaps tm;
                std::memset(&tm, 0, sizeof(tm));
                const void *in[4] = {iu, iv, iw, LES ? c->nut : iu};
                for (int q = 0; q < 4; ++q)
                    if (int rc = tensor_maps(c, in[q], tma::BY, &tm.f[q], &tm.fp[q])) return rc;
                if (CORR)
                    if (int rc = tensor_maps(c, c->phi, tma::BYP, &tm.phi, &tm.phip)) return rc;
                k_tma2<LES, WM, HYB, CORR><<<tile_grid(d, c->kc_tma, TILE_X2), 256, sizeof(TmaSmem<LES, CORR>), c->stream>>>(
                    step_args<T>(c), tm, c->wsd.tau_x, c->wsd.tau_z, sc, c->kc_tma, uo, vo, wo, f(c->f1u), f(c->f1v),
                    f(c->f1w), f(c->us), f(c->vs), f(c->wsf), rhs_only, c->d_err);
                return DFDM_OK;
            }
            if (c->stage_variant == 1) {
                k_tiled2<LES, WM, 8, HYB, CORR><<<tile_grid(d, c->kc_stage2, TILE_X2), 256, 0, c->stream>>>(step_args<T>(c),
                    iu, iv, iw, LES ? f(c->nut) : nullptr, c->wsd.tau_x, c->wsd.tau_z, sc, c->kc_stage2,
                    uo, vo, wo, f(c->f1u), f(c->f1v), f(c->f1w), f(c->us), f(c->vs), f(c->wsf), rhs_only);
                return DFDM_OK;
            }
        }
        k_tiled<T, LES, WM, TILE_X, TILE_Y, HYB ? 2 : 0, CORR><<<tile_grid(d, c->kc_stage), TILE_X * TILE_Y, 0, c->stream>>>(
            step_args<T>(c), iu, iv, iw, LES ? f(c->nut) : nullptr, c->wsd.tau_x, c->wsd.tau_z, sc,
            c->kc_stage, uo, vo, wo, f(c->f1u), f(c->f1v), f(c->f1w), f(c->us), f(c->vs), f(c->wsf),
            rhs_only, nullptr);
        return DFDM_OK;
    }
    // the eddy viscosity's wall factors (wall model only) from the velocity it is about to be computed from
    template <bool CORR> static int wall_factors(dfdm_ctx *c, const T *u, const T *w) {
        if (!c->d_wfac) return DFDM_OK;
        const Dims &d = c->d;
        k_wall_sgs<T, CORR><<<dim3((d.Nx + 127) / 128, d.Nz), 128, 0, c->stream>>>(step_args<T>(c), u, w,
                                                                                   CORR ? f(c->phi) : nullptr, c->d_wfac);
        CKL();
        return DFDM_OK;
    }
    // LES stage with the eddy viscosity computed in the tile (stage 3 also stores it in nu_t)
    template <bool WM, bool CORR> static int les_launch(dfdm_ctx *c, const StageCoef &sc) {
        const Dims &d = c->d;
        const T *iu = CORR ? f(c->us2) : f(c->u), *iv = CORR ? f(c->vs2) : f(c->v), *iw = CORR ? f(c->ws2) : f(c->w);
        if (int rc = wall_factors<CORR>(c, iu, iw)) return rc;
        T *uo = c->fused ? f(c->u) : f(c->uo), *vo = c->fused ? f(c->v) : f(c->vo), *wo = c->fused ? f(c->w) : f(c->wo);
        k_les<T, WM, CORR><<<tile_grid(d, c->kc_les), les::NT, les::smem_bytes<T>(CORR), c->stream>>>(
            step_args<T>(c), iu, iv, iw, c->wsd.tau_x, c->wsd.tau_z, sc, c->kc_les, uo, vo, wo, f(c->f1u), f(c->f1v),
            f(c->f1w), f(c->us), f(c->vs), f(c->wsf), sc.stage == 3 ? f(c->nut) : nullptr);
        return DFDM_OK;
    }
    template <bool CORR> static int les_dispatch(dfdm_ctx *c, const StageCoef &sc) {
        if constexpr (sizeof(T) == 8) return les_launch<true, CORR>(c, sc);   // FP64 keeps the runtime flag
        else return c->wm ? les_launch<true, CORR>(c, sc) : les_launch<false, CORR>(c, sc);
    }
    template <bool HYB> static int stage_dispatch(dfdm_ctx *c, const StageCoef &sc, T *rhs_only) {
        if constexpr (sizeof(T) == 8) {   // FP64 keeps the runtime wall-model flag
            return c->les ? stage_launch<true, true, HYB, false>(c, sc, rhs_only) : stage_launch<false, true, HYB, false>(c, sc, rhs_only);
        } else {
            if (c->les) {
                if (c->wm) return stage_launch<true, true, HYB, false>(c, sc, rhs_only); else return stage_launch<true, false, HYB, false>(c, sc, rhs_only);
            } else {
                if (c->wm) return stage_launch<false, true, HYB, false>(c, sc, rhs_only); else return stage_launch<false, false, HYB, false>(c, sc, rhs_only);
            }
        }
    }
    // stages 2 and 3 with the fused correction (no hybrid scheme: fuse_eligible; LES goes through les_dispatch)
    static int stage_dispatch_corr(dfdm_ctx *c, const StageCoef &sc) {
        if constexpr (sizeof(T) == 8) return stage_launch<false, true, false, true>(c, sc, nullptr);
        else if (c->wm) return stage_launch<false, true, false, true>(c, sc, nullptr);
        else return stage_launch<false, false, false, true>(c, sc, nullptr);
    }

    static int stage_kernel(dfdm_ctx *c, const StageCoef &sc, T *rhs_only) {
        if (c->les && c->sgs_tile && !rhs_only && !c->adv) {
            if (int rc = les_dispatch<false>(c, sc)) return rc;
            CKL();
            return DFDM_OK;
        }
        if (int rc = c->adv ? stage_dispatch<true>(c, sc, rhs_only) : stage_dispatch<false>(c, sc, rhs_only)) return rc;
        CKL();
        return DFDM_OK;
    }

    // Autotuner of the FP32 stage kernel: times the variants on this grid (a stage-2 launch, 2 warm-up + 5 timed;
    // the TMA variant where the grid allows it) and keeps the fastest.  The choice is cached per device, grid shape and model flags for the process, so a
    // serving loop that opens many contexts of one shape pays the timing once.
    static int tune_stage(dfdm_ctx *c, bool force) {
        if constexpr (sizeof(T) == 8) { (void)force; c->stage_variant = 0; return DFDM_OK; }
        int dev = 0;
        CK(cudaGetDevice(&dev));
        const std::array<int, 6> key = {dev, c->d.Nx, c->d.Ny, c->d.Nz, c->les, c->wm};
        // held through the timing: contexts of one shape created at the same time all take the first one's choice,
        // so every context of a shape in the process runs the same kernel (the variants round differently)
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end() && !force) {
            c->stage_variant = it->second.variant;
            for (int v = 0; v < 3; ++v) c->stage_ms[v] = it->second.ms[v];
            return DFDM_OK;
        }
        StageCoef sc{2, 0.0, c->prm.dt, 0.25, 5.0 / 12.0, 0};
        // the variants are those of the stage kernel that reads a stored eddy viscosity (k_les has one form)
        struct Restore { dfdm_ctx *c; bool v; ~Restore() { c->sgs_tile = v; } } restore{c, c->sgs_tile};
        c->sgs_tile = false;
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        int rc = DFDM_OK;
        for (int v = 0; v < (c->tma_ok ? 3 : 2) && !rc; ++v) {
            c->stage_variant = v;
            for (int r = 0; r < 2 && !rc; ++r) rc = stage_kernel(c, sc, nullptr);
            if (rc) break;
            cudaEventRecord(e0, c->stream);
            for (int r = 0; r < 5 && !rc; ++r) rc = stage_kernel(c, sc, nullptr);
            cudaEventRecord(e1, c->stream);
            if (cudaEventSynchronize(e1) != cudaSuccess) rc = fail(DFDM_ERR_CUDA, "stage-kernel tuning failed");
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            c->stage_ms[v] = ms / 5.0;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (rc) return rc;
        c->stage_variant = 0;
        for (int v = 1; v < 3; ++v)
            if (c->stage_ms[v] > 0.0 && c->stage_ms[v] < c->stage_ms[c->stage_variant]) c->stage_variant = v;
        g_tune[key] = TuneEntry{c->stage_variant, {c->stage_ms[0], c->stage_ms[1], c->stage_ms[2]}};
        return DFDM_OK;
    }

    // ---- one kernel family of one stage ----
    static int launch(dfdm_ctx *c, int which, int s) {
        const Dims &d = c->d;
        cudaStream_t st = c->stream;
        switch (which) {
        case 0: {   // SGS
            if (!c->les) return DFDM_OK;
            StageCoef sc{1, 0.0, 0.0, 0.0, 0.0, 0};
            if (int rc = wall_factors<false>(c, f(c->u), f(c->w))) return rc;
            k_tiled<T, false, false, TILE_X, TILE_Y, 1><<<tile_grid(d, c->kc_sgs), TILE_X * TILE_Y, 0, st>>>(
                step_args<T>(c), f(c->u), f(c->v), f(c->w), nullptr, nullptr, nullptr, sc, c->kc_sgs, nullptr, nullptr,
                nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, f(c->nut));
            CKL();
            return DFDM_OK;
        }
        case 8: {   // wall model (filter update at stage 1)
            if (!c->wm) return DFDM_OK;
            dim3 g((d.Nx + 127) / 128, d.Nz);
            int filt = c->wm_filter_mode == 1;
            if (s == 1 && filt) {
                k_wm_filter<T><<<g, 128, 0, st>>>(step_args<T>(c), c->wsd, f(c->u), f(c->w), c->wmf_seeded ? 0 : 1,
                                                 c->prm.dt, c->dev_dt() ? c->d_dtt : nullptr, c->prm.wm_filter_Tf_fac);
                CKL();
                c->wmf_seeded = true;
            }
            if (s == 1 || !filt) {   // with the filter the stress only changes with the filter (once per step)
                k_wall_model<T><<<g, 128, 0, st>>>(step_args<T>(c), c->wsd, f(c->u), f(c->w), filt);
                CKL();
            }
            return DFDM_OK;
        }
        case 1: {   // fused RHS + RK update
            StageCoef sc;
            sc.stage = s;
            sc.dt_a11 = c->prm.dt * (8.0 / 15.0);
            sc.dt = c->prm.dt;
            sc.c1 = 1.0 / 4.0;
            sc.c2 = (s == 2) ? 5.0 / 12.0 : 3.0 / 4.0;
            sc.incr = incr_form(c, s);
            sc.dtp = c->dev_dt() ? c->d_dtt : nullptr;
            sc.no_uo = c->fused ? 1 : 0;
            if (c->fused && s >= 2) {
                if (int rc = c->les ? les_dispatch<true>(c, sc) : stage_dispatch_corr(c, sc)) return rc;
                CKL();
                return DFDM_OK;
            }
            return stage_kernel(c, sc, nullptr);
        }
        case 2:   // div + forward x
            return fwd_x(c, true, nullptr);
        case 3: case 5: {   // z transforms
            if (c->z2) {
                dim3 g((d.Nxc + NL - 1) / NL, d.Ny);
                with_fft2l(d.Nz, [&](auto n) {
                    constexpr int N = decltype(n)::value;
                    if (which == 3)
                        k_col2<T, 0, NL, N><<<g, c->thr_z2, c->smem_z2, st>>>(d, (C *)c->spec, (const C *)c->tw_z, c->d_kxx,
                                                                              c->d_kyy, c->d_kzz);
                    else
                        k_col2<T, 1, NL, N><<<g, c->thr_z2, c->smem_z2, st>>>(d, (C *)c->spec, (const C *)c->tw_z, c->d_kxx,
                                                                              c->d_kyy, c->d_kzz);
                });
            } else {
                dim3 g((d.Nxc + c->tzx - 1) / c->tzx, d.Ny);
                if (which == 3)
                    k_col_fft<T, 0, CT><<<g, 256, c->smem_z, st>>>(d, (C *)c->spec, c->plan_z, (const C *)c->tw_z, c->d_kxx, c->d_kyy, c->d_kzz);
                else
                    k_col_fft<T, 1, CT><<<g, 256, c->smem_z, st>>>(d, (C *)c->spec, c->plan_z, (const C *)c->tw_z, c->d_kxx, c->d_kyy, c->d_kzz);
            }
            CKL();
            return DFDM_OK;
        }
        case 4: {   // y solve
            if (d.yper && c->y2) {
                dim3 g((d.Nxc + NL - 1) / NL, d.Nz);
                with_fft2l(d.Ny, [&](auto n) {
                    constexpr int N = decltype(n)::value;
                    k_col2<T, 2, NL, N><<<g, c->thr_y2, c->smem_y2, st>>>(d, (C *)c->spec, (const C *)c->tw_y, c->d_kxx,
                                                                          c->d_kyy, c->d_kzz);
                });
            } else if (d.yper) {
                dim3 g((d.Nxc + c->tzx - 1) / c->tzx, d.Nz);
                k_col_fft<T, 2, CT><<<g, 256, c->smem_y, st>>>(d, (C *)c->spec, c->plan_y, (const C *)c->tw_y, c->d_kxx, c->d_kyy, c->d_kzz);
            } else if (c->ys3) {
                const int ncol = d.Nxc * d.Nz;
                k_ysolve3<T><<<(ncol + YS_COLS - 1) / YS_COLS, YS_COLS, ysolve3_smem<T>(d.Ny), st>>>(
                    d, (C *)c->spec, c->d_rpiv, c->d_lo, c->d_up);
            } else {
                dim3 g((d.Nxc + 63) / 64, d.Nz);
                k_ysolve2<T, sizeof(T) == 4 ? 16 : 8><<<g, 64, 2 * d.Ny * sizeof(double), st>>>(d, (C *)c->spec, c->d_rpiv, c->d_lo, c->d_up);
            }
            CKL();
            return DFDM_OK;
        }
        case 6: {   // inverse x
            long long lines = (long long)d.Ny * d.Nz;
            if (c->x2) {
                int nb = (int)((lines + c->lxi2 - 1) / c->lxi2);
                with_fft2l(d.Nx / 2, [&](auto n) {
                    constexpr int N = decltype(n)::value;
                    k_inv_x2<T, N><<<nb, 256, c->smem_xi2, st>>>(poisson_args<T>(c), c->lxi2, (const C *)c->spec, f(c->phi),
                                                                  (const C *)c->tw_x, (const C *)c->twr_x);
                });
            } else {
                int nb = (int)((lines + c->lx - 1) / c->lx);
                k_inv_x<T><<<nb, 256, c->smem_x, st>>>(poisson_args<T>(c), c->lx, (const C *)c->spec, f(c->phi), c->plan_x,
                                                       (const C *)c->tw_x, (const C *)c->twr_x);
            }
            CKL();
            return DFDM_OK;
        }
        case 7: {   // correction (+ P at stage 3)
            bool inc = incr_form(c, s);
            void *pu = c->fused ? c->u : c->uo, *pv = c->fused ? c->v : c->vo, *pw = c->fused ? c->w : c->wo;
            if (d.Nx % 4 == 0) {
                dim3 g((d.Nx / 4 + 63) / 64, (d.Ny + 3) / 4, d.Nz);
                k_correct4<T><<<g, dim3(64, 4, 1), 0, st>>>(poisson_args<T>(c), f(c->phi), f(c->us), f(c->vs), f(c->wsf),
                                                            f(c->u), f(c->v), f(c->w), s == 3 ? f(c->p) : nullptr,
                                                            inc ? f(pu) : nullptr, inc ? f(pv) : nullptr,
                                                            inc ? f(pw) : nullptr);
            } else {
                k_correct<T><<<cell_grid(d), CELL_BLOCK, 0, st>>>(poisson_args<T>(c), f(c->phi), f(c->us), f(c->vs), f(c->wsf),
                                                                  f(c->u), f(c->v), f(c->w), s == 3 ? f(c->p) : nullptr,
                                                                  inc ? f(pu) : nullptr, inc ? f(pv) : nullptr,
                                                                  inc ? f(pw) : nullptr);
            }
            CKL();
            return DFDM_OK;
        }
        case 9: {   // constant-flux shift
            if (c->prm.flow_forcing_mode != 1) return DFDM_OK;
            bulk_partial(c);
            CKL();
            k_bulk_final<<<1, 256, 0, st>>>(c->red_blocks, c->red_part, c->prm.Ub_target, c->red_out);
            CKL();
            k_shift<T><<<c->red_blocks, 256, 0, st>>>(d, f(c->u), c->red_out);
            CKL();
            return DFDM_OK;
        }
        case 10:   // CFL maxima (the step-start part of the adaptive time step)
            return cfl_maxima(c);
        case 11: {   // advection_scheme = 2: the dissipative terms of the coming stage kernel
            if (!c->adv) return DFDM_OK;
            HybArgs<T> h;
            h.d = d;
            h.beta = (T)c->prm.adv_beta0;
            h.inv_dx = (T)(1.0 / c->dx);
            h.my = metric_view<T>(c->my_t, d.Ny);
            h.mz = metric_view<T>(c->mz_t, d.Nz);
            h.ub = (const T *)c->d_ub;
            const int kc = c->kc_hyb;
            const dim3 g((d.Nx + 31) / 32, (d.Ny + 7) / 8, (d.Nz + kc - 1) / kc);
            // 16-byte row copies in FP32 when Nx % 4 == 0, else 8-byte pairs (Nx is even)
            const bool quads = sizeof(T) == 4 && d.Nx % 4 == 0;
            const size_t sb = c->prm.adv_order == 5 ? hyb_faces_smem_bytes<T, 5>() : hyb_faces_smem_bytes<T, 3>();
            if (c->prm.adv_order == 5) {
                if (quads) k_adv_hybrid_faces<T, 5, 16 / sizeof(T)><<<g, 256, sb, st>>>(h, kc, f(c->u), f(c->v), f(c->w), f(c->adv));
                else k_adv_hybrid_faces<T, 5, 2><<<g, 256, sb, st>>>(h, kc, f(c->u), f(c->v), f(c->w), f(c->adv));
            } else {
                if (quads) k_adv_hybrid_faces<T, 3, 16 / sizeof(T)><<<g, 256, sb, st>>>(h, kc, f(c->u), f(c->v), f(c->w), f(c->adv));
                else k_adv_hybrid_faces<T, 3, 2><<<g, 256, sb, st>>>(h, kc, f(c->u), f(c->v), f(c->w), f(c->adv));
            }
            CKL();
            return DFDM_OK;
        }
        }
        return fail(DFDM_ERR_INVALID, "unknown kernel family");
    }

    static int poisson_chain(dfdm_ctx *c, int s) {
        int rc;
        for (int k = 2; k <= 7; ++k) {
            if (k == 7 && c->fused && s < 3 && !c->unit_projection) break;   // the next stage kernel applies it
            if ((rc = launch(c, k, s))) return rc;
        }
        return DFDM_OK;
    }

    // rows of 16-byte chunks (Nx * sizeof(T) a multiple of 16): the row reductions load whole chunks
    static bool row_chunks(const dfdm_ctx *c) { return c->d.Nx % (16 / (int)sizeof(T)) == 0; }
    static void bulk_partial(dfdm_ctx *c) {
        auto fn = row_chunks(c) ? k_bulk_partial<T, true> : k_bulk_partial<T, false>;
        fn<<<c->red_blocks, 256, 0, c->stream>>>(c->d, f(c->u), c->d_dyc, c->d_dzc, c->d_ubd, c->red_part);
    }
    // the CFL maxima of the resident state into d_cfl (zeroed first)
    static int cfl_maxima(dfdm_ctx *c) {
        CK(cudaMemsetAsync(c->d_cfl, 0, 2 * sizeof(unsigned long long), c->stream));
        auto fn = row_chunks(c) ? k_cfl<T, true> : k_cfl<T, false>;
        fn<<<c->cfl_blocks, 256, 0, c->stream>>>(c->d, f(c->u), f(c->v), f(c->w), c->les ? f(c->nut) : nullptr,
                                                        c->d_ubd, 1.0 / c->dx, c->d_dyc, c->d_dzc, c->prm.nu, c->d_cfl);
        CKL();
        return DFDM_OK;
    }
    // max |div u|, max |U| and the finite guard into d_mon[2], [3], [4] (zeroed first)
    static int monitor_rows(dfdm_ctx *c) {
        CK(cudaMemsetAsync(c->d_mon + 2, 0, 3 * sizeof(unsigned long long), c->stream));
        k_monitor_rows<T><<<c->cfl_blocks, 256, 0, c->stream>>>(c->d, f(c->u), f(c->v), f(c->w), c->d_ubd, c->d_dxc,
                                                                 c->d_dyc, c->d_dzc, c->d_mon + 2, (int *)(c->d_mon + 4));
        CKL();
        return DFDM_OK;
    }
    // output_monitor: every value into d_mon[8..17] (the dfdm_monitor layout), no host synchronisation
    static int monitor(dfdm_ctx *c) {
        CK(cudaMemsetAsync(c->d_mon, 0, 2 * sizeof(unsigned long long), c->stream));
        auto fn = row_chunks(c) ? k_cfl<T, true> : k_cfl<T, false>;
        fn<<<c->cfl_blocks, 256, 0, c->stream>>>(c->d, f(c->u), f(c->v), f(c->w), c->les ? f(c->nut) : nullptr,
                                                 c->d_ubd, 1.0 / c->dx, c->d_dyc, c->d_dzc, c->prm.nu, c->d_mon);
        CKL();
        if (int rc = monitor_rows(c)) return rc;
        bulk_partial(c);
        CKL();
        k_bulk_final<<<1, 256, 0, c->stream>>>(c->red_blocks, c->red_part, 0.0, c->red_out);
        CKL();
        const int ncol = c->d.Nx * (c->d.Nz + 1);   // the reference's (nx-2)*(nzg-2) columns
        double *wsum = c->wm ? (double *)(c->d_mon + 5) : nullptr;
        if (wsum) {
            k_wall_diag<<<1, 256, 0, c->stream>>>(c->d.Nx, c->d.Nz, c->wsd.tx, wsum);
            CKL();
        }
        k_monitor_final<<<1, 32, 0, c->stream>>>(c->d_mon, (const int *)(c->d_mon + 4), c->red_out, wsum, ncol,
                                                 c->dev_dt() ? c->d_dtt : nullptr, c->t, c->prm.dt,
                                                 (double *)(c->d_mon + 8));
        CKL();
        return DFDM_OK;
    }
    static int select_dt(dfdm_ctx *c) {
        if (c->adaptive)
            if (int rc = cfl_maxima(c)) return rc;
        k_select_dt<<<1, 32, 0, c->stream>>>(c->d_cfl, c->d_dtt, c->adaptive ? 1 : 0, c->cfl_target, c->cfl_safety,
                                             c->dt_min, c->dt_max);
        CKL();
        return DFDM_OK;
    }

    // compute_time_step_RK3, single-phase flag set (src/time_integration.f90:120-713)
    static int step_enqueue(dfdm_ctx *c) {
        int rc;
        for (int s = 1; s <= 3; ++s) {
            // SGS (step start, then stages 2 and 3); with the eddy viscosity in the stage tiles only the adaptive
            // step's start-of-step CFL needs the field
            if ((!c->sgs_tile || (s == 1 && c->dev_dt())) && (rc = launch(c, 0, s))) return rc;
            if (s == 1 && c->dev_dt() && (rc = select_dt(c))) return rc;   // dt from the start-of-step CFL, after nu_t
            if ((rc = launch(c, 8, s))) return rc;   // wall model
            if ((rc = launch(c, 11, s))) return rc;  // hybrid-scheme dissipation (advection_scheme = 2)
            if (c->fused && s >= 2) {   // the previous u* becomes this stage kernel's input; it writes the other set
                std::swap(c->us, c->us2); std::swap(c->vs, c->vs2); std::swap(c->wsf, c->ws2);
            }
            if ((rc = launch(c, 1, s))) return rc;   // RHS + RK update
            if ((rc = poisson_chain(c, s))) return rc;
        }
        return launch(c, 9, 3);
    }
};

template <typename F> int dispatch(dfdm_ctx *c, F fn) {
    if (c->prec == DFDM_FP64) return fn(Impl<double>());
    return fn(Impl<float>());
}

int check_any(dfdm_ctx *c) {
    if (!c) return fail(DFDM_ERR_INVALID, "null context");
    return DFDM_OK;
}
int check_ctx(dfdm_ctx *c) {
    if (!c) return fail(DFDM_ERR_INVALID, "null context");
    if (c->xdct)
        return fail(DFDM_ERR_UNSUPPORTED, "a context of an inflow/outflow-x grid (x_bc_type = 1) serves dfdm_solve_poisson "
                                          "only: the step's stencils need periodic x");
    if (c->duct || c->zwall)
        return fail(DFDM_ERR_UNSUPPORTED, "a context of a grid with z walls (z_bc_type = 1) serves dfdm_solve_poisson only: "
                                          "the step's stencils need periodic z");
    return DFDM_OK;
}

int ensure_staging(dfdm_ctx *c, size_t n) {
    if (c->staging_n >= n) return DFDM_OK;
    if (c->staging) {
        cudaStreamSynchronize(c->stream);
        cudaFree(c->staging);
        c->allocs.erase(std::remove(c->allocs.begin(), c->allocs.end(), (void *)c->staging), c->allocs.end());
        c->staging = nullptr;
        c->staging_n = 0;
    }
    void *p = nullptr;
    int rc = dalloc(c, &p, n * sizeof(double));
    if (rc) return rc;
    c->staging = (double *)p;
    c->staging_n = n;
    return DFDM_OK;
}

int reduce_grid(const Dims &d) {
    long long b = (d.cells + 255) / 256;
    return (int)std::max(1LL, std::min(b, 148LL * 8));
}

void destroy_graph(dfdm_ctx *c) {
    if (c->gexec) { cudaGraphExecDestroy(c->gexec); c->gexec = nullptr; }
    if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
}

int validate(const dfdm_grid *g, const dfdm_params *p) {
    if (!g || !p) return fail(DFDM_ERR_INVALID, "null grid or params");
    if (!g->x || !g->y || !g->z) return fail(DFDM_ERR_INVALID, "grid face arrays must not be NULL");
    if (g->nx % 2 || g->nz % 2) return fail(DFDM_ERR_INVALID, "Error: nx and nz must be even");
    if (g->nx < 6 || g->nz < 6 || g->ny < 4) return fail(DFDM_ERR_INVALID, "grid too small (nx, nz >= 6, ny >= 4)");
    if ((g->x_bc_type != 0 && g->x_bc_type != 1) || (g->z_bc_type != 0 && g->z_bc_type != 1))
        return fail(DFDM_ERR_UNSUPPORTED, "x_bc_type must be 0 (periodic) or 1 (inflow/outflow) and z_bc_type 0 (periodic) "
                                          "or 1 (walls)");
    if (g->z_bc_type == 1) {   // the 4-wall duct's Poisson path (src/initialization.f90:98-100)
        if (g->x_bc_type != 0 && g->y_bc_type != 1)   // inflow/outflow x with z walls: the duct only (CPU build)
            return fail(DFDM_ERR_UNSUPPORTED, "spanwise walls with inflow/outflow x are not built: z_bc_type=1 with "
                                              "x_bc_type=1 needs y walls (the 4-wall duct)");
        if (g->y_bc_type == 1 && g->nz - 1 > ZEIG_NMAX)
            return fail(DFDM_ERR_UNSUPPORTED, "4-wall duct: at most " + std::to_string(ZEIG_NMAX) + " z cells (nz <= " +
                                                  std::to_string(ZEIG_NMAX + 1) + ")");
        if (g->y_bc_type == 0 && g->nz - 1 > MAX_NY)   // spanwise walls: z is solved by the y-solve kernels
            return fail(DFDM_ERR_UNSUPPORTED, "spanwise walls: at most " + std::to_string(MAX_NY) + " z cells");
    }
    if (g->x_bc_type == 1) {   // the DCT-IV Poisson path (src/initialization.f90:95-99: walls in y, periodic z)
        if (g->y_bc_type != 1)
            return fail(DFDM_ERR_INVALID, "ERROR: GPU_POISSON with y_bc_type=0 (periodic y) requires x_bc_type=0 too");
        if (g->nx - 1 > DCT_NMAX)
            return fail(DFDM_ERR_UNSUPPORTED, "inflow/outflow x: at most " + std::to_string(DCT_NMAX) + " x cells (nx <= " +
                                                  std::to_string(DCT_NMAX + 1) + ")");
    }
    if (g->y_bc_type != 0 && g->y_bc_type != 1) return fail(DFDM_ERR_INVALID, "y_bc_type must be 0 or 1");
    if (g->y_bc_type == 1 && (g->bc_face_ylo != 1 || g->bc_face_yhi != 1))
        return fail(DFDM_ERR_UNSUPPORTED, "only no-slip y walls (bc_face_ylo = bc_face_yhi = 1) are supported");
    if (p->sgs_model < 0 || p->sgs_model > 2) return fail(DFDM_ERR_INVALID, "ERROR: sgs_model must be 0 (DNS), 1 (Vreman) or 2 (AMD)");
    if (p->flat_wall_model_flag < 0 || p->flat_wall_model_flag > 1)
        return fail(DFDM_ERR_UNSUPPORTED, "flat_wall_model_flag must be 0 or 1 (the rough-wall law is off the path)");
    if (p->flat_wall_model_flag == 1 && g->y_bc_type != 1) return fail(DFDM_ERR_INVALID, "the flat-wall model needs y walls");
    if (p->advection_scheme < 0 || p->advection_scheme > 2)
        return fail(DFDM_ERR_INVALID, "ERROR: advection_scheme must be 0 (skew-symmetric), 1 (divergence-form central) or 2 "
                                      "(skew-symmetric + upwind-biased dissipation)");
    if (p->advection_scheme == 2) {
        if (p->adv_order != 3 && p->adv_order != 5) return fail(DFDM_ERR_INVALID, "ERROR: adv_order must be 3 or 5");
        if (!(p->adv_beta0 >= 0.0)) return fail(DFDM_ERR_INVALID, "ERROR: adv_beta0 and adv_beta_ibm must be >= 0");
    }
    if (!(p->dt > 0.0)) return fail(DFDM_ERR_INVALID, "ERROR: &NUMERICS dt must be > 0");
    if (!(p->nu >= 0.0)) return fail(DFDM_ERR_INVALID, "ERROR: &PHYSICS nu must be set");
    if (p->precision != DFDM_FP64 && p->precision != DFDM_FP32_MIXED) return fail(DFDM_ERR_INVALID, "unknown precision");
    if (p->wm_filter_mode == 1 && (p->flat_wall_model_flag == 0 || !(p->wm_filter_Tf_fac > 0.0)))
        return fail(DFDM_ERR_INVALID, "ERROR: wm_filter_mode=1 needs flat_wall_model_flag>0 and wm_filter_Tf_fac>0");
    FFTPlan tmp;
    int Nx = g->nx - 2, Nz = g->nz - 2;
    int Ny = g->y_bc_type == 0 ? g->ny - 2 : g->ny - 1;
    if ((g->x_bc_type == 0 && !make_fft_plan(Nx / 2, tmp)) || (g->z_bc_type == 0 && !make_fft_plan(Nz, tmp)) ||
        (g->y_bc_type == 0 && !make_fft_plan(Ny, tmp)))
        return fail(DFDM_ERR_UNSUPPORTED, "transform lengths must factor into 2, 3 and 5");
    if (Ny > MAX_NY) return fail(DFDM_ERR_UNSUPPORTED, "ny too large for the y solve");
    if ((double)Nx * Ny * Nz * 3.0 >= 2147483647.0)
        return fail(DFDM_ERR_UNSUPPORTED, "grid too large for one context (32-bit cell indexing)");
    for (int i = 1; i < g->nx; ++i) if (!(g->x[i] > g->x[i - 1])) return fail(DFDM_ERR_INVALID, "x faces must increase");
    for (int i = 1; i < g->ny; ++i) if (!(g->y[i] > g->y[i - 1])) return fail(DFDM_ERR_INVALID, "y faces must increase");
    for (int i = 1; i < g->nz; ++i) if (!(g->z[i] > g->z[i - 1])) return fail(DFDM_ERR_INVALID, "z faces must increase");
    return DFDM_OK;
}

// The fused-correction step applies (see dfdm_ctx::fused): no SGS model, the wall model only with its temporal
// filter (automatic with periodic z), and not the hybrid advection scheme.
// The fused correction needs the stage kernel to be the only reader of the corrected velocity: no hybrid scheme,
// the wall model only with its filter (its stage 2-3 inputs are the filtered planes), and LES only through the
// in-tile eddy viscosity (no separate pass reading u).
bool fuse_eligible(const dfdm_params *p) {
    return (p->flat_wall_model_flag == 0 || p->wm_filter_mode != 0) && p->advection_scheme != 2;
}

// Bytes of the buffers dfdm_create carves from the context's arena (every sub-allocation 256-byte aligned).
size_t arena_bytes(const dfdm_grid *g, const dfdm_params *p) {
    size_t ts = p->precision == DFDM_FP64 ? 8 : 4;
    if (g->x_bc_type == 1 && g->z_bc_type == 1) {   // the inflow/outflow duct: the DCT and the duct's buffers together
        size_t Nx = g->nx - 1, Nz = g->nz - 1, Ny = g->ny - 1;
        return Nx * Ny * Nz * ts + Nx * Ny * Nz * (4 * ts + 8) + Nx * Nx * 8 + 2 * Nz * Nz * ts + (1 << 20);
    }
    if (g->x_bc_type == 1) {   // the DCT-IV Poisson context: phi, the spectrum, the pivot table, the DCT matrix
        size_t Nx = g->nx - 1, Nz = g->nz - 2, Ny = g->ny - 1;
        return Nx * Ny * Nz * (ts + 2 * ts + 8) + Nx * Nx * 8 + (1 << 20);
    }
    if (g->z_bc_type == 1 && g->y_bc_type == 0) {   // spanwise walls: phi, the spectrum, the pivot table
        size_t Nx = g->nx - 2, Nw = g->nz - 1, Np = g->ny - 2, Nxc = Nx / 2 + 1;
        return Nx * Nw * Np * ts + Nxc * Nw * Np * (2 * ts + 8) + (1 << 20);
    }
    if (g->z_bc_type == 1) {   // the duct's Poisson context: phi, two spectra, the pivot table, two eigenmode matrices
        size_t Nx = g->nx - 2, Nz = g->nz - 1, Ny = g->ny - 1, Nxc = Nx / 2 + 1;
        return Nx * Ny * Nz * ts + Nxc * Ny * Nz * (4 * ts + 8) + 2 * Nz * Nz * ts + (1 << 20);
    }
    size_t Nx = g->nx - 2, Nz = g->nz - 2, Ny = g->y_bc_type == 0 ? g->ny - 2 : g->ny - 1;
    size_t cells = Nx * Ny * Nz, spec = (Nx / 2 + 1) * Ny * Nz;
    size_t n = cells * ts * (3 /*u*/ + 3 /*uo*/ + 3 /*F1*/ + 3 /*u**/ + 1 /*P*/ + 1 /*phi*/ + (p->sgs_model ? 1 : 0) +
                             (p->advection_scheme == 2 ? 3 /*hybrid-scheme terms*/ : 0) +
                             (fuse_eligible(p) ? 3 /*second u* set*/ : 0));
    n += spec * 2 * ts;
    if (g->y_bc_type != 0) n += (Nx / 2 + 1) * Ny * Nz * 8;   // pivot table of the y solves
    n += 9 * Nx * Nz * 2 * 8;   // wall planes (and the eddy viscosity's wall factors)
    n += 1 << 20;               // metrics, twiddles, reductions, alignment
    return n;
}
// FP64 staging of the ghosted host arrays (set_state / get_state and the unit entry points), allocated on first use.
size_t staging_bytes(const dfdm_grid *g) { return ((size_t)g->nx + 1) * ((size_t)g->ny + 1) * ((size_t)g->nz + 1) * 8; }

size_t footprint(const dfdm_grid *g, const dfdm_params *p) { return arena_bytes(g, p) + staging_bytes(g); }

}  // namespace

// ================================================================================================================
extern "C" {

const char *dfdm_last_error(void) { return g_err.c_str(); }
const char *dfdm_version(void) { return "dfdm-b200 0.1 (sm_100a)"; }

void dfdm_default_params(dfdm_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->nu = -1.0;
    p->dt = 0.0;
    p->sgs_model = 2;            // src/global.f90:305
    p->Cs_vreman = 0.17;         // :306
    p->C_amd = 1.0 / 3.0;        // :307
    p->flat_wall_model_flag = 0; // :312
    p->advection_scheme = 0;
    p->adv_order = 3;
    p->adv_beta0 = 0.05;
    p->adv_wall_layers = -1;
    p->wm_filter_mode = -1;
    p->wm_filter_Tf_fac = 1.0;
    p->flow_forcing_mode = 0;
    p->precision = DFDM_FP64;
}

int dfdm_footprint_bytes(const dfdm_grid *grid, const dfdm_params *params, size_t *bytes) {
    g_err.clear();
    int rc = validate(grid, params);
    if (rc) return rc;
    if (!bytes) return fail(DFDM_ERR_INVALID, "null output");
    *bytes = footprint(grid, params);
    return DFDM_OK;
}

// A context for one of the pressure solves whose step is not built, served by dfdm_solve_poisson alone (and the
// stream and lifetime calls):
//  - inflow/outflow x (x_bc_type = 1, walls in y, periodic z): the DCT-IV wavenumbers in x, kxx(i) =
//    2 (cos(pi (2i+1) / (2 nxp)) - 1) / dx^2 (src/initialization.f90:455-457), no null-mode fix (the DCT-IV modes have
//    none, src/projection.f90:292), the z transforms and the N x N DCT-IV matrix;
//  - the 4-wall duct (z_bc_type = 1 with walls in y, periodic x): the x transforms, Dzz (src/initialization.f90:
//    543-572) and the eigenbasis of S = W^(1/2) Dzz W^(-1/2) (:579-608), whose eigenvalues lambda_z(m) stand in for kzz;
//    the null mode pinned where kx = 0 meets the zero eigenvalue (src/projection.f90:200-207);
// with, for both, the y operator Dyy and the pivot table of every (kx, z mode) system.
static int create_poisson_only(const dfdm_grid *g, const dfdm_params *prm, dfdm_ctx **out) {
    dfdm_ctx *c = new dfdm_ctx();
    c->xdct = g->x_bc_type == 1;
    c->duct = g->z_bc_type == 1 && g->y_bc_type == 1;
    c->zwall = g->z_bc_type == 1 && g->y_bc_type == 0;
    c->prm = *prm;
    c->prec = prm->precision;
    c->ts = c->prec == DFDM_FP64 ? 8 : 4;
    c->nx = g->nx; c->ny = g->ny; c->nz = g->nz;
    c->nxg = g->nx + 1; c->nyg = g->ny + 1; c->nzg = g->nz + 1;
    c->yper = 0;
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return fail(DFDM_ERR_CUDA, "cudaStreamCreate failed");
    }
    c->stream = c->own_stream;
    auto bail = [&](int code) { dfdm_destroy(c); return code; };
    int rc;
    c->x.assign(c->nx + 1, 0.0); c->y.assign(c->ny + 1, 0.0); c->z.assign(c->nz + 1, 0.0);
    for (int i = 1; i <= c->nx; ++i) c->x[i] = g->x[i - 1];
    for (int j = 1; j <= c->ny; ++j) c->y[j] = g->y[j - 1];
    for (int k = 1; k <= c->nz; ++k) c->z[k] = g->z[k - 1];
    centres_of(c->x, c->nx, c->xg); centres_of(c->y, c->ny, c->yg); centres_of(c->z, c->nz, c->zg);
    double dxmin = 1e300, dzmin = 1e300;
    for (int i = 1; i <= c->nxg - 1; ++i) dxmin = std::min(dxmin, c->xg[i + 1] - c->xg[i]);
    for (int k = 1; k <= c->nzg - 1; ++k) dzmin = std::min(dzmin, c->zg[k + 1] - c->zg[k]);
    c->dx = dxmin; c->dz = dzmin;
    Dims &d = c->d;
    d.Nx = c->xdct ? c->nx - 1 : c->nx - 2;
    d.Nz = c->duct ? c->nz - 1 : c->zwall ? c->ny - 2 : c->nz - 2;
    d.Ny = c->zwall ? c->nz - 1 : c->ny - 1;
    d.NyV = d.Ny - 1;
    d.Nxc = c->xdct ? d.Nx : d.Nx / 2 + 1;
    d.yper = 0;
    d.plane = (long long)d.Nx * d.Ny;
    d.cells = d.plane * d.Nz;
    c->arena_size = arena_bytes(g, prm);
    {
        cudaError_t e = cudaMalloc((void **)&c->arena, c->arena_size);
        if (e != cudaSuccess) {
            cudaGetLastError();
            c->arena = nullptr;
            return bail(fail(DFDM_ERR_NOMEM, std::string("cudaMalloc of the context arena failed: ") + cudaGetErrorString(e)));
        }
        c->allocs.push_back(c->arena);
    }
    c->in_create = true;
    const size_t spec_bytes = (size_t)d.Nxc * d.Ny * d.Nz * 2 * c->ts;
    if ((rc = dalloc(c, &c->phi, (size_t)d.cells * c->ts))) return bail(rc);
    if ((rc = dalloc(c, &c->spec, spec_bytes))) return bail(rc);
    if (c->duct && (rc = dalloc(c, &c->spec2, spec_bytes))) return bail(rc);
    const int nxp = d.Nx, nzp = d.Nz;
    std::vector<double> kxx(d.Nxc), kzz(d.Nz, 0.0), kyy(1, 0.0);
    if (c->xdct) {
        for (int i = 0; i < d.Nxc; ++i)
            kxx[i] = 2.0 * (std::cos(PI * (double)(2 * i + 1) / (2.0 * (double)nxp)) - 1.0) / std::pow(c->dx, 2.0);
    } else {
        const int cx = (int)std::ceil((double)nxp / 2.0);
        for (int i = 0; i < d.Nxc; ++i) {
            const double ii = (i <= cx) ? (double)i : (double)(-nxp + i);
            kxx[i] = 2.0 * (std::cos(2.0 * PI * ii / (double)nxp) - 1.0) / std::pow(c->dx, 2.0);
        }
    }
    // the second-difference operator of a wall-bounded direction (Dyy, src/initialization.f90:507-535; Dzz the same
    // on the z grid, :543-572): rows 2..n+1 of faces f and centres fg as (lower, diagonal, upper), 0-based
    auto wall_operator = [](const std::vector<double> &f, const std::vector<double> &fg, int ng, std::vector<double> &lo,
                            std::vector<double> &di, std::vector<double> &up) {
        const int n = ng - 2;
        lo.assign(n, 0.0); di.assign(n, 0.0); up.assign(n, 0.0);
        auto abc = [&](int j, double &a, double &b, double &cc) {
            a = 1.0 / (f[j] - f[j - 1]) / (fg[j + 1] - fg[j]);
            b = 1.0 / (f[j] - f[j - 1]) * (-1.0 / (fg[j + 1] - fg[j]) - 1.0 / (fg[j] - fg[j - 1]));
            cc = 1.0 / (f[j] - f[j - 1]) / (fg[j] - fg[j - 1]);
        };
        for (int j = 3; j <= ng - 2; ++j) {
            double a, b, cc; abc(j, a, b, cc);
            up[j - 2] = a; lo[j - 2] = cc; di[j - 2] = b;
        }
        double a, b, cc;
        abc(2, a, b, cc); di[0] = b + cc; up[0] = a;
        abc(ng - 1, a, b, cc); di[ng - 3] = a + b; lo[ng - 3] = cc;
    };
    std::vector<double> lo, di, up;
    if (c->zwall) wall_operator(c->z, c->zg, c->nzg, lo, di, up);   // the wall axis is z
    else wall_operator(c->y, c->yg, c->nyg, lo, di, up);
    std::vector<double> lambda_z, Qz, sqrt_w;
    if (c->duct) {
        std::vector<double> zlo, zdi, zup;
        wall_operator(c->z, c->zg, c->nzg, zlo, zdi, zup);
        std::vector<double> w(nzp), off(std::max(0, nzp - 1));
        sqrt_w.resize(nzp);
        for (int k = 0; k < nzp; ++k) { w[k] = c->z[k + 2] - c->z[k + 1]; sqrt_w[k] = std::sqrt(w[k]); }
        for (int k = 0; k + 1 < nzp; ++k) off[k] = 1.0 / ((c->zg[k + 3] - c->zg[k + 2]) * std::sqrt(w[k] * w[k + 1]));
        lambda_z = zdi;   // S's diagonal is Dzz's
        if (!tridiag_eigen(lambda_z, off, Qz))
            return bail(fail(DFDM_ERR_INVALID, "ERROR: the spanwise (z) wall operator could not be diagonalised (4-wall duct)"));
    } else {
        // the periodic axis: z, or with spanwise walls y (kyy, src/initialization.f90:436-447: uniform y, dy = y(2) - y(1))
        const double h = c->zwall ? c->y[2] - c->y[1] : c->dz;
        const int cz = (int)std::ceil((double)nzp / 2.0);
        for (int k = 0; k < nzp; ++k) {
            const double kk = (k <= cz) ? (double)k : (double)(-nzp + k);
            kzz[k] = 2.0 * (std::cos(2.0 * PI * kk / (double)nzp) - 1.0) / std::pow(h, 2.0);
        }
    }
    void *tmp = nullptr;
    if ((rc = upload_as<double>(c, &tmp, kxx))) return bail(rc);
    c->d_kxx = (double *)tmp;
    if ((rc = upload_as<double>(c, &tmp, c->duct ? lambda_z : kzz))) return bail(rc);
    c->d_kzz = (double *)tmp;
    if ((rc = upload_as<double>(c, &tmp, kyy))) return bail(rc);
    c->d_kyy = (double *)tmp;
    if ((rc = upload_as<double>(c, &tmp, lo))) return bail(rc);
    c->d_lo = (double *)tmp;
    if ((rc = upload_as<double>(c, &tmp, di))) return bail(rc);
    c->d_di = (double *)tmp;
    if ((rc = upload_as<double>(c, &tmp, up))) return bail(rc);
    c->d_up = (double *)tmp;
    {
        double lmax = 0.0;
        for (double l : lambda_z) lmax = std::max(lmax, std::fabs(l));
        std::vector<double> rpiv((size_t)d.Nxc * d.Ny * d.Nz);
        for (int kz = 0; kz < d.Nz; ++kz)
            for (int kx = 0; kx < d.Nxc; ++kx) {
                const double lz = c->duct ? lambda_z[kz] : kzz[kz];
                const double lam = kxx[kx] + lz;
                double D = di[0] + lam;
                // the duct's null mode: kx = 0 with the zero eigenvalue, found by magnitude (src/projection.f90:206)
                if (c->duct && !c->xdct && kx == 0 && std::fabs(lz) < 1e-8 * lmax) D = 3.0 / 2.0 * D;
                // spanwise walls: the (kx, ky) = (0, 0) system, as the y-wall branch pins its own (src/projection.f90:242)
                if (c->zwall && kx == 0 && kz == 0) D = 3.0 / 2.0 * D;
                const size_t b = (size_t)kz * d.Ny * d.Nxc + kx;
                rpiv[b] = 1.0 / D;
                for (int r = 1; r < d.Ny; ++r) {
                    const double m = lo[r] / D;
                    D = (di[r] + lam) - m * up[r - 1];
                    if (D == 0.0) return bail(fail(DFDM_ERR_INVALID, "singular pressure operator"));
                    rpiv[b + (size_t)r * d.Nxc] = 1.0 / D;
                }
            }
        if ((rc = upload_as<double>(c, &tmp, rpiv))) return bail(rc);
        c->d_rpiv = (double *)tmp;
    }
    auto upload_t = [&](void **dst, const std::vector<double> &v) {
        return c->prec == DFDM_FP64 ? upload_as<double>(c, dst, v) : upload_as<float>(c, dst, v);
    };
    auto tws = [&](void **dst, int n, int count) {
        return c->prec == DFDM_FP64 ? upload_twiddles<double>(c, dst, n, count) : upload_twiddles<float>(c, dst, n, count);
    };
    // the x transform: the DCT-IV matrix, C[k][n] = 2 cos(pi (2n+1)(2k+1) / (4 nxp)) with the angle reduced exactly
    // modulo 2 pi (8 nxp quarter-steps); or the real-to-complex FFT, whose kernels take the metric views of the full
    // step (zeroed here, and never read by the transforms)
    if (c->xdct) {
        const long P = 8L * nxp;
        std::vector<double> cs((size_t)P), C((size_t)(nxp * nxp));
        for (long m = 0; m < P; ++m) cs[(size_t)m] = std::cos(PI * (double)m / (4.0 * (double)nxp));
        for (long k = 0; k < nxp; ++k)
            for (long n = 0; n < nxp; ++n) C[(size_t)(k * nxp + n)] = 2.0 * cs[(size_t)(((2 * n + 1) * (2 * k + 1)) % P)];
        if ((rc = upload_t(&c->d_dct, C))) return bail(rc);
    } else {
        make_fft_plan(d.Nx / 2, c->plan_x);
        if ((rc = tws(&c->tw_x, d.Nx / 2, d.Nx / 2))) return bail(rc);
        if ((rc = tws(&c->twr_x, d.Nx, d.Nx / 2 + 1))) return bail(rc);
        std::vector<double> my((size_t)6 * (d.Ny + 3), 0.0), mz((size_t)6 * (d.Nz + 3), 0.0);
        if ((rc = upload_t(&c->my_t, my))) return bail(rc);
        if ((rc = upload_t(&c->mz_t, mz))) return bail(rc);
    }
    // the z transform: the duct's eigenmode matrices, [source index][destination index], forward Qz(k,m) sqrt(w_k),
    // inverse Qz(k,m) / sqrt(w_k) times nzp, which the inverse x transform's division by nxp nzp (2 nxp nzp for the
    // DCT-IV) takes back out; or the FFT of the periodic axis (z, or y with spanwise walls)
    if (c->duct) {
        std::vector<double> zf((size_t)nzp * nzp), zi((size_t)nzp * nzp);
        for (int k = 0; k < nzp; ++k)
            for (int m = 0; m < nzp; ++m) {
                zf[(size_t)k * nzp + m] = Qz[(size_t)k * nzp + m] * sqrt_w[k];
                zi[(size_t)m * nzp + k] = Qz[(size_t)k * nzp + m] / sqrt_w[k] * (double)nzp;
            }
        if ((rc = upload_t(&c->d_zf, zf))) return bail(rc);
        if ((rc = upload_t(&c->d_zi, zi))) return bail(rc);
    } else {
        make_fft_plan(d.Nz, c->plan_z);
        if ((rc = tws(&c->tw_z, d.Nz, d.Nz))) return bail(rc);
    }
    c->in_create = false;
    rc = dispatch(c, [&](auto impl) {
        return c->xdct ? decltype(impl)::setup_poisson_only(c) : decltype(impl)::setup_duct_only(c);
    });
    if (rc) return bail(rc);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(fail(DFDM_ERR_CUDA, "set-up synchronisation failed"));
    *out = c;
    return DFDM_OK;
}

int dfdm_create(const dfdm_grid *g, const dfdm_params *prm, dfdm_ctx **out) {
    g_err.clear();
    if (!out) return fail(DFDM_ERR_INVALID, "null output pointer");
    *out = nullptr;
    int rc = validate(g, prm);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(DFDM_ERR_CUDA, "no CUDA device: the dfdm library has no CPU fallback");
    }
    if (g->x_bc_type == 1 || g->z_bc_type == 1) return create_poisson_only(g, prm, out);
    dfdm_ctx *c = new dfdm_ctx();
    c->prm = *prm;
    c->prec = prm->precision;
    c->ts = c->prec == DFDM_FP64 ? 8 : 4;
    c->nx = g->nx; c->ny = g->ny; c->nz = g->nz;
    c->nxg = g->nx + 1; c->nyg = g->ny + 1; c->nzg = g->nz + 1;
    c->yper = g->y_bc_type == 0;
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return fail(DFDM_ERR_CUDA, "cudaStreamCreate failed");
    }
    c->stream = c->own_stream;
    auto bail = [&](int code) { dfdm_destroy(c); return code; };

    // ---- grid (src/initialization.f90:243-345) ----
    c->x.assign(c->nx + 1, 0.0); c->y.assign(c->ny + 1, 0.0); c->z.assign(c->nz + 1, 0.0);
    for (int i = 1; i <= c->nx; ++i) c->x[i] = g->x[i - 1];
    for (int j = 1; j <= c->ny; ++j) c->y[j] = g->y[j - 1];
    for (int k = 1; k <= c->nz; ++k) c->z[k] = g->z[k - 1];
    centres_of(c->x, c->nx, c->xg); centres_of(c->y, c->ny, c->yg); centres_of(c->z, c->nz, c->zg);
    double dxmin = 1e300, dzmin = 1e300;
    for (int i = 1; i <= c->nxg - 1; ++i) dxmin = std::min(dxmin, c->xg[i + 1] - c->xg[i]);
    for (int k = 1; k <= c->nzg - 1; ++k) dzmin = std::min(dzmin, c->zg[k + 1] - c->zg[k]);
    c->dx = dxmin; c->dz = dzmin;
    c->Ly = c->y[c->ny] - c->y[1];
    Dims &d = c->d;
    d.Nx = c->nx - 2; d.Nz = c->nz - 2;
    d.Ny = c->yper ? c->ny - 2 : c->ny - 1;
    d.NyV = c->yper ? d.Ny : d.Ny - 1;
    d.Nxc = d.Nx / 2 + 1;
    d.yper = c->yper;
    d.plane = (long long)d.Nx * d.Ny;
    d.cells = d.plane * d.Nz;
    // automatic defaults (src/input_output.f90:938-940, :967-970)
    c->nwl = prm->adv_wall_layers;
    if (c->nwl < 0) { c->nwl = 0; if (prm->flat_wall_model_flag > 0 && prm->advection_scheme != 1) c->nwl = 8; }
    c->wm_filter_mode = prm->wm_filter_mode;
    if (c->wm_filter_mode < 0) { c->wm_filter_mode = 0; if (prm->flat_wall_model_flag > 0) c->wm_filter_mode = 1; }
    c->wm = (!c->yper && prm->flat_wall_model_flag > 0) ? 1 : 0;
    c->les = prm->sgs_model != 0;
    // dPdx = 0 under constant flux (src/time_integration.f90:212-216); steady forcing otherwise
    c->dPdx = prm->flow_forcing_mode == 1 ? 0.0 : prm->dPdx;
    c->dPdz = prm->dPdz;

    // ---- one arena for every buffer made here ----
    c->arena_size = arena_bytes(g, prm);
    {
        cudaError_t e = cudaMalloc((void **)&c->arena, c->arena_size);
        if (e != cudaSuccess) {
            cudaGetLastError();
            c->arena = nullptr;
            return bail(fail(DFDM_ERR_NOMEM, "cudaMalloc of the " + std::to_string(c->arena_size) +
                                                 "-byte context arena failed: " + cudaGetErrorString(e)));
        }
        c->allocs.push_back(c->arena);
    }
    c->in_create = true;

    // ---- fields ----
    const size_t F = (size_t)d.cells * c->ts;
    void **fields[] = {&c->u, &c->v, &c->w, &c->uo, &c->vo, &c->wo, &c->f1u, &c->f1v, &c->f1w,
                       &c->us, &c->vs, &c->wsf, &c->p, &c->phi};
    for (void **fp : fields)
        if ((rc = dalloc(c, fp, F))) return bail(rc);
    if (fuse_eligible(prm)) {
        void **alt[] = {&c->us2, &c->vs2, &c->ws2};
        for (void **fp : alt)
            if ((rc = dalloc(c, fp, F))) return bail(rc);
        c->fuse_ok = c->fused = true;
    }
    if ((rc = dalloc(c, &c->nut, c->les ? F : c->ts))) return bail(rc);
    if ((rc = dalloc(c, &c->spec, (size_t)d.Nxc * d.Ny * d.Nz * 2 * c->ts))) return bail(rc);

    // ---- metrics ----
    std::vector<double> my, mz;
    build_metric(c->y, c->yg, c->ny, d.Ny, my);
    build_metric(c->z, c->zg, c->nz, d.Nz, mz);
    void *tmp = nullptr;
    if ((rc = upload_as<double>(c, &tmp, my))) return bail(rc);
    c->my_d = (double *)tmp;
    if ((rc = upload_as<double>(c, &tmp, mz))) return bail(rc);
    c->mz_d = (double *)tmp;
    if (c->prec == DFDM_FP64) { c->my_t = c->my_d; c->mz_t = c->mz_d; }
    else {
        if ((rc = upload_as<float>(c, &c->my_t, my))) return bail(rc);
        if ((rc = upload_as<float>(c, &c->mz_t, mz))) return bail(rc);
        // per plane k: w0(k-1), w1(k-1), w0(k), w1(k), idc(k), idc(k+1), idf(k-1), idf(k) of metric_view's layout
        // (AxisLocal<F2>::metric_src), the same FP32 values as mz_t
        const int L = d.Nz + 3;
        std::vector<double> z8((size_t)d.Nz * 8);
        for (int k = 0; k < d.Nz; ++k) {
            const int src[8][2] = {{2, k - 1}, {3, k - 1}, {2, k}, {3, k}, {4, k}, {4, k + 1}, {5, k - 1}, {5, k}};
            for (int t = 0; t < 8; ++t) z8[(size_t)k * 8 + t] = mz[(size_t)src[t][0] * L + 1 + src[t][1]];
        }
        if ((rc = upload_as<float>(c, &c->zm8, z8))) return bail(rc);
    }
    std::vector<double> dxc(d.Nx), dyc(d.Ny), dzc(d.Nz);
    for (int i = 0; i < d.Nx; ++i) dxc[i] = c->x[i + 2] - c->x[i + 1];
    for (int j = 0; j < d.Ny; ++j) dyc[j] = c->y[j + 2] - c->y[j + 1];
    for (int k = 0; k < d.Nz; ++k) dzc[k] = c->z[k + 2] - c->z[k + 1];
    if ((rc = upload_as<double>(c, &tmp, dxc))) return bail(rc);
    c->d_dxc = (double *)tmp;
    if ((rc = upload_as<double>(c, &tmp, dyc))) return bail(rc);
    c->d_dyc = (double *)tmp;
    if ((rc = upload_as<double>(c, &tmp, dzc))) return bail(rc);
    c->d_dzc = (double *)tmp;
    if ((rc = dalloc(c, &c->d_ub, (size_t)d.Ny * c->ts))) return bail(rc);
    if ((rc = dalloc(c, &tmp, (size_t)d.Ny * sizeof(double)))) return bail(rc);
    c->d_ubd = (double *)tmp;

    // ---- modified wavenumbers (src/initialization.f90:417-434, :480-489) and Dyy (:507-535) ----
    int nxp = d.Nx, nzp = d.Nz;
    std::vector<double> kxx(d.Nxc), kzz(d.Nz), kyy(std::max(1, d.Ny));
    int cx = (int)std::ceil((double)nxp / 2.0), cz = (int)std::ceil((double)nzp / 2.0);
    for (int i = 0; i < d.Nxc; ++i) {
        double ii = (i <= cx) ? (double)i : (double)(-nxp + i);
        kxx[i] = 2.0 * (std::cos(2.0 * PI * ii / (double)nxp) - 1.0) / std::pow(c->dx, 2.0);
    }
    for (int k = 0; k < nzp; ++k) {
        double kk = (k <= cz) ? (double)k : (double)(-nzp + k);
        kzz[k] = 2.0 * (std::cos(2.0 * PI * kk / (double)nzp) - 1.0) / std::pow(c->dz, 2.0);
    }
    if (c->yper) {
        int nyp = d.Ny;
        double dy = c->y[2] - c->y[1];
        int cy = (int)std::ceil((double)nyp / 2.0);
        for (int j = 0; j < nyp; ++j) {
            double jj = (j <= cy) ? (double)j : (double)(-nyp + j);
            kyy[j] = 2.0 * (std::cos(2.0 * PI * jj / (double)nyp) - 1.0) / std::pow(dy, 2.0);
        }
    }
    std::vector<double> lo(d.Ny, 0.0), di(d.Ny, 0.0), up(d.Ny, 0.0);
    if (!c->yper) {
        const std::vector<double> &y = c->y, &yg = c->yg;
        int nyg = c->nyg;
        auto abc = [&](int j, double &a, double &b, double &cc) {
            a = 1.0 / (y[j] - y[j - 1]) / (yg[j + 1] - yg[j]);
            b = 1.0 / (y[j] - y[j - 1]) * (-1.0 / (yg[j + 1] - yg[j]) - 1.0 / (yg[j] - yg[j - 1]));
            cc = 1.0 / (y[j] - y[j - 1]) / (yg[j] - yg[j - 1]);
        };
        for (int j = 3; j <= nyg - 2; ++j) {
            double a, b, cc; abc(j, a, b, cc);
            up[j - 2] = a; lo[j - 2] = cc; di[j - 2] = b;
        }
        double a, b, cc;
        abc(2, a, b, cc); di[0] = b + cc; up[0] = a;
        abc(nyg - 1, a, b, cc); di[nyg - 3] = a + b; lo[nyg - 3] = cc;
    }
    if ((rc = upload_as<double>(c, &tmp, kxx))) return bail(rc);
    c->d_kxx = (double *)tmp;
    if ((rc = upload_as<double>(c, &tmp, kzz))) return bail(rc);
    c->d_kzz = (double *)tmp;
    if ((rc = upload_as<double>(c, &tmp, kyy))) return bail(rc);
    c->d_kyy = (double *)tmp;
    if ((rc = upload_as<double>(c, &tmp, lo))) return bail(rc);
    c->d_lo = (double *)tmp;
    if ((rc = upload_as<double>(c, &tmp, di))) return bail(rc);
    c->d_di = (double *)tmp;
    if ((rc = upload_as<double>(c, &tmp, up))) return bail(rc);
    c->d_up = (double *)tmp;
    if (!c->yper) {
        // pivots of the no-interchange zgtsv elimination of every (kx,kz) system (src/projection.f90:284-295)
        std::vector<double> rpiv((size_t)d.Nxc * d.Ny * d.Nz);
        for (int kz = 0; kz < d.Nz; ++kz)
            for (int kx = 0; kx < d.Nxc; ++kx) {
                double lam = kxx[kx] + kzz[kz];
                double D = di[0] + lam;
                if (kx == 0 && kz == 0) D = 3.0 / 2.0 * D;
                size_t b = (size_t)kz * d.Ny * d.Nxc + kx;
                rpiv[b] = 1.0 / D;
                for (int r = 1; r < d.Ny; ++r) {
                    double m = lo[r] / D;
                    D = (di[r] + lam) - m * up[r - 1];
                    if (D == 0.0) return bail(fail(DFDM_ERR_INVALID, "singular pressure operator"));
                    rpiv[b + (size_t)r * d.Nxc] = 1.0 / D;
                }
            }
        if ((rc = upload_as<double>(c, &tmp, rpiv))) return bail(rc);
        c->d_rpiv = (double *)tmp;
    }

    // ---- FFT plans and twiddles ----
    make_fft_plan(d.Nx / 2, c->plan_x);
    make_fft_plan(d.Nz, c->plan_z);
    if (c->yper) make_fft_plan(d.Ny, c->plan_y);
    auto tws = [&](void **dst, int n, int count) {
        return c->prec == DFDM_FP64 ? upload_twiddles<double>(c, dst, n, count) : upload_twiddles<float>(c, dst, n, count);
    };
    if ((rc = tws(&c->tw_x, d.Nx / 2, d.Nx / 2))) return bail(rc);
    if ((rc = tws(&c->twr_x, d.Nx, d.Nx / 2 + 1))) return bail(rc);
    if ((rc = tws(&c->tw_z, d.Nz, d.Nz))) return bail(rc);
    if ((rc = tws(&c->tw_y, c->yper ? d.Ny : 1, c->yper ? d.Ny : 1))) return bail(rc);

    // ---- wall model planes ----
    size_t wp = (size_t)2 * d.Nz * d.Nx * sizeof(double);
    double **wsp[] = {&c->wsd.tau_x, &c->wsd.tau_z, &c->wsd.ux, &c->wsd.wx, &c->wsd.tx, &c->wsd.uz, &c->wsd.wz, &c->wsd.tz};
    for (double **pp : wsp)
        if ((rc = dalloc(c, (void **)pp, wp))) return bail(rc);
    if (c->les && c->wm) {   // the first-cell gradient factors of the eddy viscosity's wall override (k_wall_sgs)
        if ((rc = dalloc(c, &tmp, wp))) return bail(rc);
        c->d_wfac = (double *)tmp;
    }

    // ---- reductions ----
    c->red_blocks = reduce_grid(d);
    if ((rc = dalloc(c, &tmp, (size_t)2 * c->red_blocks * sizeof(double)))) return bail(rc);
    c->red_part = (double *)tmp;
    if ((rc = dalloc(c, &tmp, 4 * sizeof(double)))) return bail(rc);
    c->red_out = (double *)tmp;
    if ((rc = dalloc(c, &tmp, 32 * sizeof(unsigned long long)))) return bail(rc);
    c->d_mon = (unsigned long long *)tmp;
    if ((rc = dalloc(c, &tmp, 2 * sizeof(unsigned long long)))) return bail(rc);
    c->d_cfl = (unsigned long long *)tmp;
    if ((rc = dalloc(c, &tmp, 8 * sizeof(double)))) return bail(rc);
    c->d_dtt = (double *)tmp;
    if (prm->advection_scheme == 2) {   // the dissipative terms of the hybrid scheme
        if ((rc = dalloc(c, &c->adv, (size_t)3 * d.cells * c->ts))) return bail(rc);
        CK(cudaMemsetAsync(c->adv, 0, (size_t)3 * d.cells * c->ts, c->stream));
    }
    c->in_create = false;   // later buffers (host staging, the unit RHS output) are separate allocations

    rc = dispatch(c, [&](auto impl) { return decltype(impl)::setup_kernels(c); });
    if (rc) return bail(rc);
    rc = dispatch(c, [&](auto impl) { return decltype(impl)::tune_stage(c, false); });   // on the zeroed fields
    if (rc) return bail(rc);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(fail(DFDM_ERR_CUDA, "set-up synchronisation failed"));
    *out = c;
    return DFDM_OK;
}

int dfdm_destroy(dfdm_ctx *c) {
    if (!c) return DFDM_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->cin) cudaStreamSynchronize(c->cin);
    if (c->cout) cudaStreamSynchronize(c->cout);
    for (int q = 0; q < 4; ++q) {
        cudaEvent_t *evs[4] = {&c->ev_in[q], &c->ev_unpacked[q], &c->ev_packed[q], &c->ev_out[q]};
        for (cudaEvent_t *e : evs)
            if (*e) cudaEventDestroy(*e);
    }
    if (c->cin) cudaStreamDestroy(c->cin);
    if (c->cout) cudaStreamDestroy(c->cout);
    destroy_graph(c);
    for (void *p : c->allocs) cudaFree(p);
    c->allocs.clear();
    if (c->h_err) cudaFreeHost(c->h_err);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return DFDM_OK;
}

int dfdm_get_stream(dfdm_ctx *c, void **s) {
    if (int rc = check_any(c)) return rc;
    if (!s) return fail(DFDM_ERR_INVALID, "null output");
    *s = (void *)c->stream;
    return DFDM_OK;
}

int dfdm_set_stream(dfdm_ctx *c, void *s) {
    if (int rc = check_any(c)) return rc;
    CK(cudaStreamSynchronize(c->stream));
    c->stream = s ? (cudaStream_t)s : c->own_stream;
    destroy_graph(c);
    return DFDM_OK;
}

}  // extern "C"

// the flag a bounded wait of the TMA stage kernel sets when it gives up (read after the stream has drained)
static int check_err_flag(dfdm_ctx *c) {
    if (c->h_err && *(volatile int *)c->h_err) {
        *(volatile int *)c->h_err = 0;
        return fail(DFDM_ERR_TIMEOUT, "a bounded wait of the stage kernel gave up: its tile copies did not arrive");
    }
    return DFDM_OK;
}

extern "C" {

int dfdm_synchronize(dfdm_ctx *c) {
    if (int rc = check_any(c)) return rc;
    CK(cudaStreamSynchronize(c->stream));
    if (c->cin) CK(cudaStreamSynchronize(c->cin));
    if (c->cout) CK(cudaStreamSynchronize(c->cout));
    return check_err_flag(c);
}

// copy streams, staging buffers and events of the asynchronous transfers, made together on first use: the context
// publishes them only when all exist, and a failure part-way frees what it made (so a retry starts clean)
static int ensure_async(dfdm_ctx *c) {
    if (c->cin) return DFDM_OK;
    const size_t n = (size_t)(c->nxg) * c->nyg * c->nzg;   // the largest ghosted shape
    void *buf[8] = {};
    cudaEvent_t ev[16] = {};
    cudaStream_t sin = nullptr, sout = nullptr;
    auto unwind = [&](int rc) {
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
        if (sin) cudaStreamDestroy(sin);
        if (sout) cudaStreamDestroy(sout);
        for (void *b : buf) {
            if (!b) continue;
            auto it = std::find(c->allocs.begin(), c->allocs.end(), b);
            if (it != c->allocs.end()) c->allocs.erase(it);
            cudaFree(b);
        }
        return rc;
    };
    for (int q = 0; q < 8; ++q)
        if (int rc = dalloc(c, &buf[q], n * sizeof(double))) return unwind(rc);
    for (int q = 0; q < 16; ++q)
        if (cudaEventCreateWithFlags(&ev[q], cudaEventDisableTiming) != cudaSuccess)
            return unwind(fail(DFDM_ERR_CUDA, "cudaEventCreateWithFlags of the transfer events failed"));
    if (cudaStreamCreateWithFlags(&sin, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&sout, cudaStreamNonBlocking) != cudaSuccess)
        return unwind(fail(DFDM_ERR_CUDA, "cudaStreamCreateWithFlags of the copy streams failed"));
    // a first wait on an event that was never recorded is a no-op: record them once on the compute stream
    for (int q = 0; q < 4; ++q)
        if (cudaEventRecord(ev[4 * q + 1], c->stream) != cudaSuccess || cudaEventRecord(ev[4 * q + 3], c->stream) != cudaSuccess)
            return unwind(fail(DFDM_ERR_CUDA, "cudaEventRecord of the transfer events failed"));
    for (int q = 0; q < 4; ++q) {
        c->stage_in[q] = (double *)buf[2 * q];
        c->stage_out[q] = (double *)buf[2 * q + 1];
        c->ev_in[q] = ev[4 * q];
        c->ev_unpacked[q] = ev[4 * q + 1];
        c->ev_packed[q] = ev[4 * q + 2];
        c->ev_out[q] = ev[4 * q + 3];
    }
    c->cout = sout;
    c->cin = sin;
    return DFDM_OK;
}

// ---- state transfer ----
static int put_field(dfdm_ctx *c, int kind, void *dst, const double *src, int n1, int n2, int n3) {
    size_t n = (size_t)n1 * n2 * n3;
    int rc = ensure_staging(c, n);
    if (rc) return rc;
    CK(cudaMemcpyAsync(c->staging, src, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    int gb = reduce_grid(c->d);
    if (c->prec == DFDM_FP64) k_unpack<double><<<gb, 256, 0, c->stream>>>(c->d, kind, n1, n2, c->staging, c->d_ubd, (double *)dst);
    else k_unpack<float><<<gb, 256, 0, c->stream>>>(c->d, kind, n1, n2, c->staging, c->d_ubd, (float *)dst);
    CKL();
    return DFDM_OK;
}

static int get_field(dfdm_ctx *c, int kind, const void *srcf, double *dst, int n1, int n2, int n3) {
    size_t n = (size_t)n1 * n2 * n3;
    int rc = ensure_staging(c, n);
    if (rc) return rc;
    int gb = (int)std::min<size_t>((n + 255) / 256, 148 * 8);
    if (c->prec == DFDM_FP64) k_pack<double><<<gb, 256, 0, c->stream>>>(c->d, kind, n1, n2, n3, (const double *)srcf, c->d_ubd, c->staging);
    else k_pack<float><<<gb, 256, 0, c->stream>>>(c->d, kind, n1, n2, n3, (const float *)srcf, c->d_ubd, c->staging);
    CKL();
    CK(cudaMemcpyAsync(dst, c->staging, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return DFDM_OK;
}

int dfdm_set_state(dfdm_ctx *c, const double *U, const double *V, const double *W, const double *P) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (!U || !V || !W) return fail(DFDM_ERR_INVALID, "U, V and W must not be NULL");
    int rc;
    if (c->prec == DFDM_FP32_MIXED && !c->ub_set) {
        // streamwise base profile, fixed by the first set_state of the context: the x-z mean of the given U at
        // every centre row, rounded to FP32, so that the stored deviation U - ub carries rounding noise of the
        // fluctuation's size, not of the mean flow's
        const Dims &d = c->d;
        std::vector<double> ubd(d.Ny);
        std::vector<float> ubf(d.Ny);
        for (int j = 0; j < d.Ny; ++j) {
            double acc = 0.0;
            for (int k = 0; k < d.Nz; ++k)
                for (int i = 0; i < d.Nx; ++i)
                    acc += U[(size_t)(i + 1) + (size_t)c->nx * ((size_t)(j + 1) + (size_t)c->nyg * (size_t)(k + 1))];
            ubf[j] = (float)(acc / ((double)d.Nx * d.Nz));
            ubd[j] = (double)ubf[j];
        }
        CK(cudaMemcpyAsync(c->d_ub, ubf.data(), d.Ny * sizeof(float), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->d_ubd, ubd.data(), d.Ny * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        c->ub_set = true;
    }
    if ((rc = put_field(c, FK_U, c->u, U, c->nx, c->nyg, c->nzg))) return rc;
    if ((rc = put_field(c, FK_V, c->v, V, c->nxg, c->ny, c->nzg))) return rc;
    if ((rc = put_field(c, FK_W, c->w, W, c->nxg, c->nyg, c->nz))) return rc;
    if (P && (rc = put_field(c, FK_P, c->p, P, c->nxg, c->nyg, c->nzg))) return rc;
    c->projected = false;
    CK(cudaStreamSynchronize(c->stream));
    return DFDM_OK;
}

int dfdm_get_state(dfdm_ctx *c, double *U, double *V, double *W, double *P) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    int rc;
    if (U) { if ((rc = get_field(c, FK_U, c->u, U, c->nx, c->nyg, c->nzg))) return rc; CK(cudaStreamSynchronize(c->stream)); }
    if (V) { if ((rc = get_field(c, FK_V, c->v, V, c->nxg, c->ny, c->nzg))) return rc; CK(cudaStreamSynchronize(c->stream)); }
    if (W) { if ((rc = get_field(c, FK_W, c->w, W, c->nxg, c->nyg, c->nz))) return rc; CK(cudaStreamSynchronize(c->stream)); }
    if (P) { if ((rc = get_field(c, FK_P, c->p, P, c->nxg, c->nyg, c->nzg))) return rc; CK(cudaStreamSynchronize(c->stream)); }
    return DFDM_OK;
}

int dfdm_set_state_async(dfdm_ctx *c, const double *U, const double *V, const double *W, const double *P) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (!U || !V || !W) return fail(DFDM_ERR_INVALID, "U, V and W must not be NULL");
    if (c->prec == DFDM_FP32_MIXED && !c->ub_set)   // the first state fixes the base profile (host work): synchronous
        return dfdm_set_state(c, U, V, W, P);
    if (int rc = ensure_async(c)) return rc;
    struct { const double *h; int kind; void *dst; int n1, n2, n3; } f[4] = {
        {U, FK_U, c->u, c->nx, c->nyg, c->nzg}, {V, FK_V, c->v, c->nxg, c->ny, c->nzg},
        {W, FK_W, c->w, c->nxg, c->nyg, c->nz}, {P, FK_P, c->p, c->nxg, c->nyg, c->nzg}};
    const int gb = reduce_grid(c->d);
    for (int q = 0; q < 4; ++q) {
        if (!f[q].h) continue;
        const size_t n = (size_t)f[q].n1 * f[q].n2 * f[q].n3;
        CK(cudaStreamWaitEvent(c->cin, c->ev_unpacked[q], 0));   // the buffer's previous contents are unpacked
        CK(cudaMemcpyAsync(c->stage_in[q], f[q].h, n * sizeof(double), cudaMemcpyHostToDevice, c->cin));
        CK(cudaEventRecord(c->ev_in[q], c->cin));
        CK(cudaStreamWaitEvent(c->stream, c->ev_in[q], 0));
        if (c->prec == DFDM_FP64)
            k_unpack<double><<<gb, 256, 0, c->stream>>>(c->d, f[q].kind, f[q].n1, f[q].n2, c->stage_in[q], c->d_ubd, (double *)f[q].dst);
        else
            k_unpack<float><<<gb, 256, 0, c->stream>>>(c->d, f[q].kind, f[q].n1, f[q].n2, c->stage_in[q], c->d_ubd, (float *)f[q].dst);
        CKL();
        CK(cudaEventRecord(c->ev_unpacked[q], c->stream));
    }
    c->projected = false;
    return DFDM_OK;
}

int dfdm_get_state_async(dfdm_ctx *c, double *U, double *V, double *W, double *P) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (int rc = ensure_async(c)) return rc;
    struct { double *h; int kind; const void *src; int n1, n2, n3; } f[4] = {
        {U, FK_U, c->u, c->nx, c->nyg, c->nzg}, {V, FK_V, c->v, c->nxg, c->ny, c->nzg},
        {W, FK_W, c->w, c->nxg, c->nyg, c->nz}, {P, FK_P, c->p, c->nxg, c->nyg, c->nzg}};
    for (int q = 0; q < 4; ++q) {
        if (!f[q].h) continue;
        const size_t n = (size_t)f[q].n1 * f[q].n2 * f[q].n3;
        const int gb = (int)std::min<size_t>((n + 255) / 256, 148 * 8);
        CK(cudaStreamWaitEvent(c->stream, c->ev_out[q], 0));   // the buffer's previous contents are downloaded
        if (c->prec == DFDM_FP64)
            k_pack<double><<<gb, 256, 0, c->stream>>>(c->d, f[q].kind, f[q].n1, f[q].n2, f[q].n3, (const double *)f[q].src, c->d_ubd, c->stage_out[q]);
        else
            k_pack<float><<<gb, 256, 0, c->stream>>>(c->d, f[q].kind, f[q].n1, f[q].n2, f[q].n3, (const float *)f[q].src, c->d_ubd, c->stage_out[q]);
        CKL();
        CK(cudaEventRecord(c->ev_packed[q], c->stream));
        CK(cudaStreamWaitEvent(c->cout, c->ev_packed[q], 0));
        CK(cudaMemcpyAsync(f[q].h, c->stage_out[q], n * sizeof(double), cudaMemcpyDeviceToHost, c->cout));
        CK(cudaEventRecord(c->ev_out[q], c->cout));
    }
    return DFDM_OK;
}

int dfdm_get_nu_t(dfdm_ctx *c, double *nu_t) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (!nu_t) return fail(DFDM_ERR_INVALID, "null output");
    if (!c->les) { std::memset(nu_t, 0, sizeof(double) * (size_t)c->nxg * c->nyg * c->nzg); return DFDM_OK; }
    int rc = get_field(c, FK_NUT, c->nut, nu_t, c->nxg, c->nyg, c->nzg);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    return DFDM_OK;
}

int dfdm_set_nu_t(dfdm_ctx *c, const double *nu_t) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (!c->les) return fail(DFDM_ERR_INVALID, "nu_t is only stored for LES (sgs_model > 0)");
    int rc = put_field(c, FK_NUT, c->nut, nu_t, c->nxg, c->nyg, c->nzg);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    return DFDM_OK;
}

// the device time step: d_dtt = {dt of the last step, t, dt before landing, landing targets[5]} to the host (c->t;
// the dt before landing into *dt) and back (with c->t_land)
static int pull_dtt(dfdm_ctx *c, double *dt) {
    double v[8] = {c->prm.dt, c->t, c->prm.dt, NAN, NAN, NAN, NAN, NAN};
    if (c->dev_dt()) {
        CK(cudaMemcpyAsync(v, c->d_dtt, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        c->t = v[1];
    }
    if (dt) *dt = v[2];
    return DFDM_OK;
}
static int push_dtt(dfdm_ctx *c, double dt) {
    double v[8] = {dt, c->t, dt, 0, 0, 0, 0, 0};
    for (int q = 0; q < 5; ++q) v[3 + q] = c->t_land[q];
    CK(cudaMemcpyAsync(c->d_dtt, v, sizeof(v), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DFDM_OK;
}

int dfdm_set_time(dfdm_ctx *c, double t) {
    if (int rc = check_ctx(c)) return rc;
    if (!c->dev_dt()) { c->t = t; return DFDM_OK; }
    double dt = 0.0;
    if (int rc = pull_dtt(c, &dt)) return rc;
    c->t = t;
    return push_dtt(c, dt);
}

int dfdm_get_time(dfdm_ctx *c, double *t) {
    if (int rc = check_ctx(c)) return rc;
    if (int rc = pull_dtt(c, nullptr)) return rc;
    if (t) *t = c->t;
    return DFDM_OK;
}

int dfdm_get_dt(dfdm_ctx *c, double *dt) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (!dt) return fail(DFDM_ERR_INVALID, "null output");
    return pull_dtt(c, dt);
}

int dfdm_set_adaptive_dt(dfdm_ctx *c, int enable, double cfl_target, double cfl_safety, double dt_min, double dt_max) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (enable) {
        if (!(cfl_target > 0.0) || !(cfl_safety > 0.0)) return fail(DFDM_ERR_INVALID, "cfl_target and cfl_safety must be > 0");
        if (!(dt_min > 0.0) || !(dt_max >= dt_min)) return fail(DFDM_ERR_INVALID, "need 0 < dt_min <= dt_max");
    }
    double dt = c->prm.dt;
    if (int rc = pull_dtt(c, &dt)) return rc;   // the current time (and dt, when it was on the device already)
    CK(cudaStreamSynchronize(c->stream));
    destroy_graph(c);   // the captured kernels read dt from the host value or from d_dtt
    if (!enable) {
        c->adaptive = false;   // back to the fixed dt of the parameters
        return c->landing ? push_dtt(c, c->prm.dt) : DFDM_OK;
    }
    c->cfl_target = cfl_target; c->cfl_safety = cfl_safety; c->dt_min = dt_min; c->dt_max = dt_max;
    c->adaptive = true;
    return push_dtt(c, dt);
}

// the landing targets of the coming steps (NaN: a slot without a target)
static int set_landings(dfdm_ctx *c, const double tl[5]) {
    double dt = c->prm.dt;
    if (int rc = pull_dtt(c, &dt)) return rc;
    const bool was = c->dev_dt();
    c->landing = false;
    for (int q = 0; q < 5; ++q) {
        c->t_land[q] = tl[q];
        c->landing = c->landing || !std::isnan(tl[q]);
    }
    if (was != c->dev_dt()) destroy_graph(c);   // new targets alone keep the graph: they are read from d_dtt
    return c->dev_dt() ? push_dtt(c, dt) : DFDM_OK;
}

int dfdm_set_landing_time(dfdm_ctx *c, int enable, double t_land) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (enable && !std::isfinite(t_land)) return fail(DFDM_ERR_INVALID, "the landing time must be finite");
    const double tl[5] = {enable ? t_land : NAN, NAN, NAN, NAN, NAN};
    return set_landings(c, tl);
}

int dfdm_set_landing_times(dfdm_ctx *c, int n, const double *t_land) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (n < 0 || n > 5) return fail(DFDM_ERR_INVALID, "between 0 and 5 landing targets");
    if (n > 0 && !t_land) return fail(DFDM_ERR_INVALID, "null landing targets");
    double tl[5] = {NAN, NAN, NAN, NAN, NAN};
    for (int q = 0; q < n; ++q) {
        if (std::isinf(t_land[q])) return fail(DFDM_ERR_INVALID, "a landing time must be finite (NaN: no target)");
        tl[q] = t_land[q];
    }
    return set_landings(c, tl);
}

// ---- the step ----
// Programmatic dependent launch in the captured steps: every kernel-to-kernel edge of the graph becomes a
// programmatic edge (the destination may be scheduled once every block of the source has started, and waits in
// pdl_enter for the source's completion).  An edge the runtime does not accept as programmatic stays as it was.
static int make_programmatic(cudaGraph_t g) {
    size_t n = 0;
    if (cudaGraphGetEdges_v2(g, nullptr, nullptr, nullptr, &n) != cudaSuccess) { cudaGetLastError(); return DFDM_OK; }
    std::vector<cudaGraphNode_t> from(n), to(n);
    std::vector<cudaGraphEdgeData> ed(n);
    if (n == 0 || cudaGraphGetEdges_v2(g, from.data(), to.data(), ed.data(), &n) != cudaSuccess) {
        cudaGetLastError();
        return DFDM_OK;
    }
    for (size_t i = 0; i < n; ++i) {
        cudaGraphNodeType a, b;
        if (cudaGraphNodeGetType(from[i], &a) != cudaSuccess || cudaGraphNodeGetType(to[i], &b) != cudaSuccess) continue;
        if (a != cudaGraphNodeTypeKernel || b != cudaGraphNodeTypeKernel || ed[i].type != cudaGraphDependencyTypeDefault)
            continue;
        cudaGraphEdgeData pe;
        std::memset(&pe, 0, sizeof(pe));
        pe.type = cudaGraphDependencyTypeProgrammatic;
        pe.from_port = cudaGraphKernelNodePortProgrammatic;
        CK(cudaGraphRemoveDependencies_v2(g, &from[i], &to[i], &ed[i], 1));
        if (cudaGraphAddDependencies_v2(g, &from[i], &to[i], &pe, 1) != cudaSuccess) {
            cudaGetLastError();
            CK(cudaGraphAddDependencies_v2(g, &from[i], &to[i], &ed[i], 1));
        }
    }
    return DFDM_OK;
}

static int step_n(dfdm_ctx *c, int nsteps) {
    for (int n = 0; n < nsteps; ++n) {
        double to = c->t;
        // the captured step is the steady one: filter seeded and (FP32-mixed) increment form at stage 3
        bool can_graph = c->graphs && c->projected && (c->wm_filter_mode != 1 || !c->wm || c->wmf_seeded);
        if (can_graph) {
            if (!c->gexec) {
                CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
                long long before = g_launches;
                int rc = dispatch(c, [&](auto impl) { return decltype(impl)::step_enqueue(c); });
                c->graph_launches = g_launches - before;
                g_launches = before;
                cudaGraph_t g = nullptr;
                cudaError_t e = cudaStreamEndCapture(c->stream, &g);
                if (rc) { if (g) cudaGraphDestroy(g); return rc; }
                if (e != cudaSuccess) return fail(DFDM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
                c->graph = g;
                if (int rp = make_programmatic(c->graph)) return rp;
                CK(cudaGraphInstantiate(&c->gexec, c->graph, 0));
            }
            CK(cudaGraphLaunch(c->gexec, c->stream));
            c->launches += c->graph_launches;
        } else {
            long long before = g_launches;
            int rc = dispatch(c, [&](auto impl) { return decltype(impl)::step_enqueue(c); });
            c->launches += g_launches - before;
            if (rc) return rc;
        }
        if (!c->dev_dt()) c->t = to + 1.0 * c->prm.dt;   // t = to + rk_t(3)*dt (device dt: k_select_dt advances t)
        c->projected = true;
    }
    return DFDM_OK;
}

int dfdm_compute_time_step_rk3_async(dfdm_ctx *c, int nsteps) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (nsteps < 0) return fail(DFDM_ERR_INVALID, "nsteps must be >= 0");
    return step_n(c, nsteps);
}

int dfdm_compute_time_step_rk3(dfdm_ctx *c, int nsteps, double *t) {
    int rc = dfdm_compute_time_step_rk3_async(c, nsteps);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    if (int rc1 = check_err_flag(c)) return rc1;
    if (int rc2 = pull_dtt(c, nullptr)) return rc2;
    if (t) *t = c->t;
    return DFDM_OK;
}

int dfdm_enable_graphs(dfdm_ctx *c, int enable) {
    if (int rc = check_ctx(c)) return rc;
    CK(cudaStreamSynchronize(c->stream));
    c->graphs = enable != 0;
    if (!c->graphs) destroy_graph(c);
    return DFDM_OK;
}

// ---- unit entry points ----
int dfdm_compute_sgs_model(dfdm_ctx *c) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    int rc = dispatch(c, [&](auto impl) { return decltype(impl)::launch(c, 0, 1); });
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    return DFDM_OK;
}

int dfdm_compute_wall_model(dfdm_ctx *c, int update_filter, double *tau_x, double *tau_z) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (c->wm) {
        int rc = dispatch(c, [&](auto impl) { return decltype(impl)::launch(c, 8, update_filter ? 1 : 2); });
        if (rc) return rc;
    }
    const Dims &d = c->d;
    size_t nx_n = (size_t)c->nx * 2 * c->nzg, nz_n = (size_t)c->nxg * 2 * c->nz;
    int rc = ensure_staging(c, std::max(nx_n, nz_n));
    if (rc) return rc;
    if (tau_x) {
        k_pack_tau<<<64, 256, 0, c->stream>>>(d, 0, c->nx, c->nzg, c->wsd.tau_x, c->staging);
        CKL();
        CK(cudaMemcpyAsync(tau_x, c->staging, nx_n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    if (tau_z) {
        k_pack_tau<<<64, 256, 0, c->stream>>>(d, 1, c->nxg, c->nz, c->wsd.tau_z, c->staging);
        CKL();
        CK(cudaMemcpyAsync(tau_z, c->staging, nz_n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    return DFDM_OK;
}

int dfdm_compute_rhs(dfdm_ctx *c, double *rhs_u, double *rhs_v, double *rhs_w) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    const Dims &d = c->d;
    if (!c->rhs3) {
        int rc = dalloc(c, &c->rhs3, (size_t)3 * d.cells * c->ts);
        if (rc) return rc;
    }
    int rc = dispatch(c, [&](auto impl) {
        typedef decltype(impl) I;
        StageCoef sc{1, 0.0, 0.0, 0.0, 0.0, 0};
        if (int rc2 = I::launch(c, 11, 1)) return rc2;   // the hybrid scheme's dissipation of the resident state
        return I::stage_kernel(c, sc, I::f(c->rhs3));
    });
    if (rc) return rc;
    struct { double *dst; int n1, n2, n3; } outs[3] = {
        {rhs_u, c->nx - 2, c->nyg - 2, c->nzg - 2},
        {rhs_v, c->nxg - 2, c->ny - 2, c->nzg - 2},
        {rhs_w, c->nxg - 2, c->nyg - 2, c->nz - 2}};
    for (int q = 0; q < 3; ++q) {
        if (!outs[q].dst) continue;
        size_t n = (size_t)outs[q].n1 * outs[q].n2 * outs[q].n3;
        if ((rc = ensure_staging(c, n))) return rc;
        int gb = (int)std::min<size_t>((n + 255) / 256, 148 * 8);
        if (c->prec == DFDM_FP64)
            k_pack_interior<double><<<gb, 256, 0, c->stream>>>(d, outs[q].n1, outs[q].n2, outs[q].n3, (const double *)c->rhs3 + q * d.cells, c->staging);
        else
            k_pack_interior<float><<<gb, 256, 0, c->stream>>>(d, outs[q].n1, outs[q].n2, outs[q].n3, (const float *)c->rhs3 + q * d.cells, c->staging);
        CKL();
        CK(cudaMemcpyAsync(outs[q].dst, c->staging, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return DFDM_OK;
}

int dfdm_apply_boundary_conditions(dfdm_ctx *c, int after_projection) {
    (void)after_projection;
    return check_ctx(c);
}

int dfdm_compute_projection_step(dfdm_ctx *c, int save_p) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    size_t F = (size_t)c->d.cells * c->ts;
    CK(cudaMemcpyAsync(c->us, c->u, F, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->vs, c->v, F, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->wsf, c->w, F, cudaMemcpyDeviceToDevice, c->stream));
    c->unit_projection = true;
    int rc = dispatch(c, [&](auto impl) { return decltype(impl)::poisson_chain(c, save_p ? 3 : 1); });
    c->unit_projection = false;
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
    return DFDM_OK;
}

int dfdm_solve_poisson(dfdm_ctx *c, const double *rhs_in, double *phi_out) {
    g_err.clear();
    if (int rc = check_any(c)) return rc;
    if (!rhs_in || !phi_out) return fail(DFDM_ERR_INVALID, "null array");
    const Dims &d = c->d;
    int n1 = c->nxg - 1, n2 = c->nyg - 2, n3 = c->nzg - 1;
    size_t n = (size_t)n1 * n2 * n3;
    int rc = ensure_staging(c, n);
    if (rc) return rc;
    CK(cudaMemcpyAsync(c->staging, rhs_in, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (c->xdct || c->duct || c->zwall) {
        long long before = g_launches;
        rc = dispatch(c, [&](auto impl) {
            typedef decltype(impl) I;
            return c->duct ? I::solve_duct(c, n1, n2, n3) : c->zwall ? I::solve_zwall(c, n1, n2, n3) : I::solve_dct(c, n1, n2, n3);
        });
        c->launches += g_launches - before;
        if (rc) return rc;
        CK(cudaMemcpyAsync(phi_out, c->staging, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return DFDM_OK;
    }
    rc = dispatch(c, [&](auto impl) {
        typedef decltype(impl) I;
        typedef typename std::remove_pointer<decltype(I::f(nullptr))>::type T;
        typedef typename cplx_t<T>::type C;
        int gb = reduce_grid(d);
        k_unpack_rhs_p<T><<<gb, 256, 0, c->stream>>>(d, n1, n2, c->staging, I::f(c->phi));
        CKL();
        int r2;
        if ((r2 = I::fwd_x(c, false, I::f(c->phi)))) return r2;
        if ((r2 = I::launch(c, 3, 1))) return r2;
        if ((r2 = I::launch(c, 4, 1))) return r2;
        if ((r2 = I::launch(c, 5, 1))) return r2;
        if ((r2 = I::launch(c, 6, 1))) return r2;
        int gb2 = (int)std::min<size_t>((n + 255) / 256, 148 * 8);
        k_pack_rhs_p<T><<<gb2, 256, 0, c->stream>>>(d, n1, n2, n3, I::f(c->phi), c->staging);
        CKL();
        return DFDM_OK;
    });
    if (rc) return rc;
    CK(cudaMemcpyAsync(phi_out, c->staging, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DFDM_OK;
}

}  // extern "C"

// Staging array of dfdm_solve_poisson_noalloc. It is reserved once per device when the module is loaded there, so
// the entry point itself never allocates; every call on a device shares it.
static __device__ __align__(256) double g_noalloc_scratch[DFDM_NOALLOC_MAX_POINTS];

namespace {
const int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
double *g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

// Address of the staging array on the current device. It is looked up again on every call made outside a stream
// capture, so a module reloaded after cudaDeviceReset is found at its new address; a call inside a capture uses the
// address of the last call outside one (the first call on a device must therefore precede any capture).
int noalloc_scratch(cudaStream_t stream, double **out) {
    int dev = -1;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(DFDM_ERR_UNSUPPORTED, "device ordinal beyond 63");
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(stream, &cap));
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev] || cap == cudaStreamCaptureStatusNone) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return fail(DFDM_ERR_CUDA, std::string("cudaGetSymbolAddress of the staging array: ") + cudaGetErrorString(e));
        }
        g_noalloc_ptr[dev] = (double *)p;
    }
    *out = g_noalloc_ptr[dev];
    return DFDM_OK;
}
}  // namespace

extern "C" {

int dfdm_solve_poisson_noalloc(dfdm_ctx *c, const double *rhs_in, double *phi_out) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (!rhs_in || !phi_out) return fail(DFDM_ERR_INVALID, "null array");
    const Dims &d = c->d;
    int n1 = c->nxg - 1, n2 = c->nyg - 2, n3 = c->nzg - 1;
    size_t n = (size_t)n1 * n2 * n3;
    if (n > (size_t)DFDM_NOALLOC_MAX_POINTS)
        return fail(DFDM_ERR_INVALID, "rhs_p has " + std::to_string(n) + " points; dfdm_solve_poisson_noalloc takes at most " +
                                          std::to_string(DFDM_NOALLOC_MAX_POINTS) + " (use dfdm_solve_poisson)");
    double *scratch = nullptr;
    if (int rc = noalloc_scratch(c->stream, &scratch)) return rc;
    // The host copy fills scratch[0, n) before the unpack kernel reads it, and the pack kernel rewrites
    // scratch[0, n) before the copy back: nothing has to start at zero.
    CK(cudaMemcpyAsync(scratch, rhs_in, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    long long before = g_launches;
    int rc = dispatch(c, [&](auto impl) {
        typedef decltype(impl) I;
        typedef typename std::remove_pointer<decltype(I::f(nullptr))>::type T;
        typedef typename cplx_t<T>::type C;
        int gb = reduce_grid(d);
        k_unpack_rhs_p<T><<<gb, 256, 0, c->stream>>>(d, n1, n2, scratch, I::f(c->phi));
        CKL();
        int r2;
        if ((r2 = I::fwd_x(c, false, I::f(c->phi)))) return r2;
        if ((r2 = I::launch(c, 3, 1))) return r2;
        if ((r2 = I::launch(c, 4, 1))) return r2;
        if ((r2 = I::launch(c, 5, 1))) return r2;
        if ((r2 = I::launch(c, 6, 1))) return r2;
        int gb2 = (int)std::min<size_t>((n + 255) / 256, 148 * 8);
        k_pack_rhs_p<T><<<gb2, 256, 0, c->stream>>>(d, n1, n2, n3, I::f(c->phi), scratch);
        CKL();
        return DFDM_OK;
    });
    c->launches += g_launches - before;
    if (rc) return rc;
    CK(cudaMemcpyAsync(phi_out, scratch, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DFDM_OK;
}

}  // extern "C"

namespace {
// ---- the reference's restart format (one rank, a stream of int32 and float64 words) ----
// The staggered restart and its .wmf are opened without convert= (src/input_output.f90:1272,1842,1996,2019), so
// they take the build's default byte order, which every compiler branch of the reference's CMakeLists.txt sets to
// big-endian (:210 gfortran -fconvert=big-endian, Intel -convert big_endian, NVHPC -Mbyteswapio). Only the
// box-snapshot magic probe (:1235) and the box snapshot itself (:1723) are explicitly little-endian.
const int32_t SNAP_MAGIC = -4242;
static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "the snapshot code assumes a little-endian host");

inline int32_t bswap(int32_t v) { return (int32_t)__builtin_bswap32((uint32_t)v); }
inline double bswap(double v) {
    uint64_t u;
    std::memcpy(&u, &v, 8);
    u = __builtin_bswap64(u);
    std::memcpy(&v, &u, 8);
    return v;
}
// write n words, byte-swapped when `swap` (a big-endian file), through a bounded buffer
template <class T> bool put_words(FILE *f, const T *p, size_t n, bool swap) {
    if (!swap) return fwrite(p, sizeof(T), n, f) == n;
    std::vector<T> buf(std::min(n, (size_t)65536));
    for (size_t o = 0; o < n; o += buf.size()) {
        const size_t m = std::min(buf.size(), n - o);
        for (size_t i = 0; i < m; ++i) buf[i] = bswap(p[o + i]);
        if (fwrite(buf.data(), sizeof(T), m, f) != m) return false;
    }
    return true;
}
template <class T> bool get_words(FILE *f, T *p, size_t n, bool swap) {
    if (fread(p, sizeof(T), n, f) != n) return false;
    if (swap) for (size_t i = 0; i < n; ++i) p[i] = bswap(p[i]);
    return true;
}
bool put_block(FILE *f, const double *a, int n1, int n2, int n3, bool swap) {
    const int32_t h[3] = {n1, n2, n3};
    const size_t n = (size_t)n1 * n2 * n3;
    return put_words(f, h, 3, swap) && put_words(f, a, n, swap);
}
int get_block(FILE *f, std::vector<double> &a, int n1, int n2, int n3, const char *what, bool swap) {
    int32_t h[3];
    if (!get_words(f, h, 3, swap)) return fail(DFDM_ERR_INVALID, std::string("restart file ends before ") + what);
    if (h[0] != n1 || h[1] != n2 || h[2] != n3)
        return fail(DFDM_ERR_INVALID, std::string("restart file field block size mismatch for ") + what + ": found " +
                                          std::to_string(h[0]) + " " + std::to_string(h[1]) + " " + std::to_string(h[2]) +
                                          " expected " + std::to_string(n1) + " " + std::to_string(n2) + " " + std::to_string(n3));
    a.resize((size_t)n1 * n2 * n3);
    if (!get_words(f, a.data(), a.size(), swap))
        return fail(DFDM_ERR_INVALID, std::string("restart file ends inside the ") + what + " block");
    return DFDM_OK;
}
// Byte order of a restart or .wmf file from its first word, which is nx in both: big-endian when the word read
// big-endian is nx, little-endian when the word read little-endian is. Returns 1 (big), 0 (little) or -1 (neither).
int detect_order(int32_t first_le, int nx) {
    if (bswap(first_le) == nx) return 1;
    if (first_le == nx) return 0;
    return -1;
}
// the six mesh arrays of the header: faces x, y, z (1-based host copies) and their centres
std::vector<std::vector<double>> mesh_arrays(const dfdm_ctx *c) {
    std::vector<std::vector<double>> m;
    const std::vector<double> *f[3] = {&c->x, &c->y, &c->z};
    const int n[3] = {c->nx, c->ny, c->nz};
    for (int a = 0; a < 3; ++a) m.emplace_back(f[a]->begin() + 1, f[a]->begin() + 1 + n[a]);
    for (int a = 0; a < 3; ++a) {
        std::vector<double> xm(n[a] - 1);
        for (int i = 0; i < n[a] - 1; ++i) xm[i] = 0.5 * ((*f[a])[i + 1] + (*f[a])[i + 2]);
        m.push_back(xm);
    }
    return m;
}
// filter planes between the device layout (iw*Nz + k)*Nx + i and the reference shapes (nx,2,nzg) / (nxg,2,nz)
// with the x/z ghost planes zero (write_distributed_field_block with interior_only)
void wmf_to_ref(const dfdm_ctx *c, const std::vector<double> &dev, bool xface, std::vector<double> &ref) {
    const Dims &d = c->d;
    const int n1 = xface ? c->nx : c->nxg, n3 = xface ? c->nzg : c->nz;
    ref.assign((size_t)n1 * 2 * n3, 0.0);
    for (int k = 2; k <= n3 - 1; ++k)
        for (int iw = 0; iw < 2; ++iw)
            for (int i = 2; i <= n1 - 1; ++i) {
                const int di = (i - 2) % d.Nx, dk = (k - 2) % d.Nz;
                ref[(size_t)(i - 1) + (size_t)n1 * (iw + 2 * (size_t)(k - 1))] = dev[((size_t)iw * d.Nz + dk) * d.Nx + di];
            }
}
void wmf_from_ref(const dfdm_ctx *c, const std::vector<double> &ref, bool xface, std::vector<double> &dev) {
    const Dims &d = c->d;
    const int n1 = xface ? c->nx : c->nxg;
    dev.assign((size_t)2 * d.Nz * d.Nx, 0.0);
    for (int iw = 0; iw < 2; ++iw)
        for (int k = 0; k < d.Nz; ++k)
            for (int i = 0; i < d.Nx; ++i)
                dev[((size_t)iw * d.Nz + k) * d.Nx + i] = ref[(size_t)(i + 1) + (size_t)n1 * (iw + 2 * (size_t)(k + 1))];
}
struct FileCloser {
    FILE *f;
    ~FileCloser() { if (f) fclose(f); }
};
}  // namespace

extern "C" {

int dfdm_write_snapshot(dfdm_ctx *c, const char *path) { return dfdm_write_snapshot_ex(c, path, DFDM_BIG_ENDIAN); }

int dfdm_write_snapshot_ex(dfdm_ctx *c, const char *path, int byte_order) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (!path) return fail(DFDM_ERR_INVALID, "null path");
    if (byte_order != DFDM_BIG_ENDIAN && byte_order != DFDM_LITTLE_ENDIAN)
        return fail(DFDM_ERR_INVALID, "byte_order must be DFDM_BIG_ENDIAN or DFDM_LITTLE_ENDIAN");
    const bool sw = byte_order == DFDM_BIG_ENDIAN;
    const size_t nU = (size_t)c->nx * c->nyg * c->nzg, nV = (size_t)c->nxg * c->ny * c->nzg;
    const size_t nW = (size_t)c->nxg * c->nyg * c->nz, nP = (size_t)c->nxg * c->nyg * c->nzg;
    std::vector<double> U(nU), V(nV), W(nW), P(nP), NU;
    int rc = dfdm_get_state(c, U.data(), V.data(), W.data(), P.data());
    if (rc) return rc;
    if (c->les) {
        NU.resize(nP);
        if ((rc = dfdm_get_nu_t(c, NU.data()))) return rc;
    }
    FileCloser fc{fopen(path, "wb")};
    if (!fc.f) return fail(DFDM_ERR_INVALID, std::string("cannot open ") + path + " for writing");
    bool ok = true;
    for (const std::vector<double> &m : mesh_arrays(c)) {
        const int32_t n = (int32_t)m.size();
        ok = ok && put_words(fc.f, &n, 1, sw) && put_words(fc.f, m.data(), m.size(), sw);
    }
    ok = ok && put_block(fc.f, U.data(), c->nx, c->nyg, c->nzg, sw) && put_block(fc.f, V.data(), c->nxg, c->ny, c->nzg, sw) &&
         put_block(fc.f, W.data(), c->nxg, c->nyg, c->nz, sw) && put_block(fc.f, P.data(), c->nxg, c->nyg, c->nzg, sw);
    if (c->les) ok = ok && put_block(fc.f, NU.data(), c->nxg, c->nyg, c->nzg, sw);
    if (!ok || fclose(fc.f) != 0) { fc.f = nullptr; return fail(DFDM_ERR_INVALID, std::string("write to ") + path + " failed"); }
    fc.f = nullptr;
    if (!(c->wm && c->wm_filter_mode == 1 && c->wmf_seeded)) return DFDM_OK;
    // write_wm_filter_state
    const size_t np = (size_t)2 * c->d.Nz * c->d.Nx;
    double *planes[6] = {c->wsd.ux, c->wsd.wx, c->wsd.tx, c->wsd.uz, c->wsd.wz, c->wsd.tz};
    FileCloser fw{fopen((std::string(path) + ".wmf").c_str(), "wb")};
    if (!fw.f) return fail(DFDM_ERR_INVALID, std::string("cannot open ") + path + ".wmf for writing");
    std::vector<double> dev(np), ref;
    for (int q = 0; q < 6; ++q) {
        CK(cudaMemcpyAsync(dev.data(), planes[q], np * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        const bool xf = q < 3;
        wmf_to_ref(c, dev, xf, ref);
        ok = ok && put_block(fw.f, ref.data(), xf ? c->nx : c->nxg, 2, xf ? c->nzg : c->nz, sw);
    }
    if (!ok || fclose(fw.f) != 0) { fw.f = nullptr; return fail(DFDM_ERR_INVALID, std::string("write to ") + path + ".wmf failed"); }
    fw.f = nullptr;
    return DFDM_OK;
}

// write_box_snapshot (src/input_output.f90:1699-1767) of a one-rank run: field_box (:1586-1598) gives each field's
// stagger flags st and global range gl:gh over the face box f1:f2 (a staggered direction holds faces f1..f2, a centred
// one cells f1..f2-1); fill_box_block (:1623-1659) maps global index g to the ghosted array index g + 1 - st, and with
// location 1 averages each velocity to the cell centres over the two faces of its own direction.
int dfdm_write_box_snapshot(dfdm_ctx *c, const char *path, const int32_t f1[3], const int32_t f2[3], int location,
                            int32_t step) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (!path || !f1 || !f2) return fail(DFDM_ERR_INVALID, "null argument");
    if (location != 0 && location != 1)
        return fail(DFDM_ERR_INVALID, "snapshot_location must be 0 (staggered) or 1 (cell-centred)");
    const int nf3[3] = {c->nx, c->ny, c->nz};
    for (int a = 0; a < 3; ++a)
        if (!(f1[a] >= 1 && f2[a] <= nf3[a] && f1[a] < f2[a]))
            return fail(DFDM_ERR_INVALID, "chunk box is empty or outside the domain in direction " + std::to_string(a + 1));
    const size_t nU = (size_t)c->nx * c->nyg * c->nzg, nV = (size_t)c->nxg * c->ny * c->nzg;
    const size_t nW = (size_t)c->nxg * c->nyg * c->nz, nP = (size_t)c->nxg * c->nyg * c->nzg;
    std::vector<double> U(nU), V(nV), W(nW), P(nP), NU;
    int rc = dfdm_get_state(c, U.data(), V.data(), W.data(), P.data());
    if (rc) return rc;
    if (c->les) {   // sgs_model /= 0
        NU.resize(nP);
        if ((rc = dfdm_get_nu_t(c, NU.data()))) return rc;
    }
    double t = 0.0;
    if ((rc = dfdm_get_time(c, &t))) return rc;
    struct Field { const char *name; const double *a; int ic, n1, n2; };
    std::vector<Field> fields = {{"U", U.data(), 1, c->nx, c->nyg}, {"V", V.data(), 2, c->nxg, c->ny},
                                 {"W", W.data(), 3, c->nxg, c->nyg}, {"P", P.data(), 0, c->nxg, c->nyg}};
    if (c->les) fields.push_back({"nu_t", NU.data(), 0, c->nxg, c->nyg});
    auto box = [&](int ic, int32_t st[3], int32_t gl[3], int32_t gh[3]) {
        for (int a = 0; a < 3; ++a) st[a] = (location == 0 && ic == a + 1) ? 1 : 0;
        for (int a = 0; a < 3; ++a) { gl[a] = f1[a]; gh[a] = f2[a] - 1 + st[a]; }
    };
    FileCloser fc{fopen(path, "wb")};
    if (!fc.f) return fail(DFDM_ERR_INVALID, std::string("cannot open ") + path + " for writing");
    bool ok = true;
    auto put = [&](const void *p, size_t sz, size_t n) { ok = ok && fwrite(p, sz, n, fc.f) == n; };
    const int32_t head[4] = {SNAP_MAGIC, (int32_t)location, step, (int32_t)fields.size()};
    put(head, sizeof(int32_t), 4);
    put(&t, sizeof(double), 1);
    put(f1, sizeof(int32_t), 3);
    put(f2, sizeof(int32_t), 3);
    const std::vector<std::vector<double>> mesh = mesh_arrays(c);   // x, y, z, xm, ym, zm
    for (int a = 0; a < 3; ++a) {
        put(mesh[a].data() + (f1[a] - 1), sizeof(double), (size_t)(f2[a] - f1[a] + 1));
        put(mesh[3 + a].data() + (f1[a] - 1), sizeof(double), (size_t)(f2[a] - f1[a]));
    }
    for (const Field &fl : fields) {
        char name[8];
        std::memset(name, ' ', sizeof(name));
        std::memcpy(name, fl.name, std::strlen(fl.name));
        int32_t st[3], gl[3], gh[3];
        box(fl.ic, st, gl, gh);
        put(name, 1, 8);
        put(st, sizeof(int32_t), 3);
        put(gl, sizeof(int32_t), 3);
        put(gh, sizeof(int32_t), 3);
    }
    for (const Field &fl : fields) {
        int32_t st[3], gl[3], gh[3];
        box(fl.ic, st, gl, gh);
        const bool centred = location == 1 && fl.ic > 0;
        std::vector<double> buf;
        buf.reserve((size_t)(gh[0] - gl[0] + 1) * (gh[1] - gl[1] + 1) * (gh[2] - gl[2] + 1));
        auto at = [&](int i, int j, int k) {   // 1-based ghosted indices
            return fl.a[((size_t)(k - 1) * fl.n2 + (j - 1)) * fl.n1 + (i - 1)];
        };
        for (int k = gl[2]; k <= gh[2]; ++k)
            for (int j = gl[1]; j <= gh[1]; ++j)
                for (int i = gl[0]; i <= gh[0]; ++i) {
                    const int ia = i + 1 - st[0], ja = j + 1 - st[1], ka = k + 1 - st[2];
                    double v;
                    if (centred && fl.ic == 1) v = 0.5 * (at(ia - 1, ja, ka) + at(ia, ja, ka));
                    else if (centred && fl.ic == 2) v = 0.5 * (at(ia, ja - 1, ka) + at(ia, ja, ka));
                    else if (centred && fl.ic == 3) v = 0.5 * (at(ia, ja, ka - 1) + at(ia, ja, ka));
                    else v = at(ia, ja, ka);
                    buf.push_back(v);
                }
        put(buf.data(), sizeof(double), buf.size());
    }
    if (!ok || fclose(fc.f) != 0) { fc.f = nullptr; return fail(DFDM_ERR_INVALID, std::string("write to ") + path + " failed"); }
    fc.f = nullptr;
    return DFDM_OK;
}

int dfdm_read_snapshot(dfdm_ctx *c, const char *path) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (!path) return fail(DFDM_ERR_INVALID, "null path");
    FileCloser fc{fopen(path, "rb")};
    if (!fc.f) return fail(DFDM_ERR_INVALID, std::string("cannot open restart file ") + path);
    int32_t first = 0;
    if (fread(&first, sizeof(first), 1, fc.f) != 1) return fail(DFDM_ERR_INVALID, "restart file is empty");
    if (first == SNAP_MAGIC)   // the magic probe reads little-endian (src/input_output.f90:1235)
        return fail(DFDM_ERR_INVALID, "the file is a cell-centred/chunked box snapshot and cannot be used for restart");
    // size check of read_input_data: the mesh, then U, V, W and P
    const std::vector<std::vector<double>> mesh = mesh_arrays(c);
    long long expect = 6 * 4;
    for (const auto &m : mesh) expect += 8LL * (long long)m.size();
    expect += 4 * 12 + 8LL * ((long long)c->nx * c->nyg * c->nzg + (long long)c->nxg * c->ny * c->nzg +
                              (long long)c->nxg * c->nyg * c->nz + (long long)c->nxg * c->nyg * c->nzg);
    fseek(fc.f, 0, SEEK_END);
    const long long have = ftell(fc.f);
    if (have < expect)
        return fail(DFDM_ERR_INVALID, "restart file is smaller than expected for this grid: " + std::to_string(have) +
                                          " < " + std::to_string(expect) + " bytes");
    const int order = detect_order(first, c->nx);
    if (order < 0)
        return fail(DFDM_ERR_INVALID, "restart file nx = " + std::to_string(bswap(first)) + " (big-endian) or " +
                                          std::to_string(first) + " (little-endian) but the grid gives " + std::to_string(c->nx));
    const bool sw = order == 1;
    fseek(fc.f, 0, SEEK_SET);
    const char *names[6] = {"nx", "ny", "nz", "nxm", "nym", "nzm"};
    for (int a = 0; a < 6; ++a) {
        int32_t n = 0;
        if (!get_words(fc.f, &n, 1, sw)) return fail(DFDM_ERR_INVALID, "restart file header truncated");
        if (n != (int32_t)mesh[a].size())
            return fail(DFDM_ERR_INVALID, std::string("restart file ") + names[a] + " = " + std::to_string(n) +
                                              " but the grid gives " + std::to_string(mesh[a].size()));
        std::vector<double> f(n);
        if (!get_words(fc.f, f.data(), (size_t)n, sw)) return fail(DFDM_ERR_INVALID, "restart file header truncated");
        double scale = 1.0;
        for (double v : mesh[a]) scale = std::max(scale, std::fabs(v));
        for (int i = 0; i < n; ++i)
            if (std::fabs(f[i] - mesh[a][i]) > 1e-12 * scale)
                return fail(DFDM_ERR_INVALID, std::string("restart file coordinates (") + names[a] + ") differ from the grid");
    }
    std::vector<double> U, V, W, P;
    int rc;
    if ((rc = get_block(fc.f, U, c->nx, c->nyg, c->nzg, "U", sw))) return rc;
    if ((rc = get_block(fc.f, V, c->nxg, c->ny, c->nzg, "V", sw))) return rc;
    if ((rc = get_block(fc.f, W, c->nxg, c->nyg, c->nz, "W", sw))) return rc;
    if ((rc = get_block(fc.f, P, c->nxg, c->nyg, c->nzg, "P", sw))) return rc;
    if ((rc = dfdm_set_state(c, U.data(), V.data(), W.data(), P.data()))) return rc;
    c->wmf_seeded = false;
    if (!(c->wm && c->wm_filter_mode == 1)) return DFDM_OK;
    FileCloser fw{fopen((std::string(path) + ".wmf").c_str(), "rb")};
    if (!fw.f) return DFDM_OK;   // no filter file: the filter re-seeds on the next step
    // the .wmf comes from the same build as the restart: the restart's byte order
    const size_t np = (size_t)2 * c->d.Nz * c->d.Nx;
    double *planes[6] = {c->wsd.ux, c->wsd.wx, c->wsd.tx, c->wsd.uz, c->wsd.wz, c->wsd.tz};
    const char *wn[6] = {"wmf_ux", "wmf_wx", "wmf_tx", "wmf_uz", "wmf_wz", "wmf_tz"};
    std::vector<double> ref, dev;
    for (int q = 0; q < 6; ++q) {
        const bool xf = q < 3;
        if ((rc = get_block(fw.f, ref, xf ? c->nx : c->nxg, 2, xf ? c->nzg : c->nz, wn[q], sw))) return rc;
        wmf_from_ref(c, ref, xf, dev);
        CK(cudaMemcpyAsync(planes[q], dev.data(), np * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    c->wmf_seeded = true;
    return DFDM_OK;
}

int dfdm_compute_bulk_velocity(dfdm_ctx *c, double *Ub) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (!Ub) return fail(DFDM_ERR_INVALID, "null output");
    int rc = dispatch(c, [&](auto impl) {
        typedef decltype(impl) I;
        I::bulk_partial(c);
        CKL();
        k_bulk_final<<<1, 256, 0, c->stream>>>(c->red_blocks, c->red_part, 0.0, c->red_out);
        CKL();
        return DFDM_OK;
    });
    if (rc) return rc;
    CK(cudaMemcpyAsync(Ub, c->red_out, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DFDM_OK;
}

int dfdm_check_divergence(dfdm_ctx *c, double *max_div) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (!max_div) return fail(DFDM_ERR_INVALID, "null output");
    int rc = dispatch(c, [&](auto impl) { return decltype(impl)::monitor_rows(c); });
    if (rc) return rc;
    unsigned long long bits = 0;
    CK(cudaMemcpyAsync(&bits, c->d_mon + 2, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::memcpy(max_div, &bits, sizeof(double));
    return DFDM_OK;
}

int dfdm_output_monitor_async(dfdm_ctx *c, dfdm_monitor *out) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (!out) return fail(DFDM_ERR_INVALID, "null output");
    static_assert(sizeof(dfdm_monitor) == 10 * sizeof(double), "dfdm_monitor is ten doubles");
    long long before = g_launches;
    int rc = dispatch(c, [&](auto impl) { return decltype(impl)::monitor(c); });
    c->launches += g_launches - before;
    if (rc) return rc;
    CK(cudaMemcpyAsync(out, c->d_mon + 8, sizeof(dfdm_monitor), cudaMemcpyDefault, c->stream));
    return DFDM_OK;
}

int dfdm_output_monitor(dfdm_ctx *c, dfdm_monitor *out) {
    if (!out) return fail(DFDM_ERR_INVALID, "null output");
    dfdm_monitor m;
    if (int rc = dfdm_output_monitor_async(c, &m)) return rc;
    CK(cudaStreamSynchronize(c->stream));
    *out = m;
    if (m.nan_flag != 0.0) return fail(DFDM_ERR_NOT_FINITE, "NaN, Inf or |u| > 1e8 in the velocity field");
    return DFDM_OK;
}

int dfdm_compute_cfl(dfdm_ctx *c, double *cfl_conv, double *cfl_visc) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (!cfl_conv || !cfl_visc) return fail(DFDM_ERR_INVALID, "null output");
    int rc = dispatch(c, [&](auto impl) { return decltype(impl)::cfl_maxima(c); });
    if (rc) return rc;
    unsigned long long bits[2] = {0, 0};
    CK(cudaMemcpyAsync(bits, c->d_cfl, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    double m[2], dt = c->prm.dt;
    std::memcpy(m, bits, sizeof(m));
    if ((rc = pull_dtt(c, &dt))) return rc;   // the CFL numbers of the current dt
    *cfl_conv = m[0] * dt;
    *cfl_visc = m[1] * dt;
    return DFDM_OK;
}

int dfdm_kinetic_energy(dfdm_ctx *c, double *ke) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (!ke) return fail(DFDM_ERR_INVALID, "null output");
    int rc = dispatch(c, [&](auto impl) {
        typedef decltype(impl) I;
        typedef typename std::remove_pointer<decltype(I::f(nullptr))>::type T;
        k_ke_partial<T><<<c->red_blocks, 256, 0, c->stream>>>(c->d, I::f(c->u), I::f(c->v), I::f(c->w), c->dx, c->d_dyc,
                                                              c->d_dzc, c->d_ubd, c->red_part);
        CKL();
        k_ratio_final<<<1, 32, 0, c->stream>>>(c->red_blocks, c->red_part, c->red_out + 2);
        CKL();
        return DFDM_OK;
    });
    if (rc) return rc;
    CK(cudaMemcpyAsync(ke, c->red_out + 2, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return DFDM_OK;
}

int dfdm_check_finite(dfdm_ctx *c) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    int rc = dispatch(c, [&](auto impl) { return decltype(impl)::monitor_rows(c); });
    if (rc) return rc;
    int flag = 0;
    CK(cudaMemcpyAsync(&flag, c->d_mon + 4, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (flag) return fail(DFDM_ERR_NOT_FINITE, "NaN, Inf or |U| > 1e8 in the velocity field");
    return DFDM_OK;
}

int dfdm_pad_field(dfdm_ctx *c, int field, int extra_planes, double *out) {
    (void)field; (void)extra_planes; (void)out;
    if (int rc = check_ctx(c)) return rc;
    return fail(DFDM_ERR_UNSUPPORTED,
                "pad_field_dev serves the hybrid advection scheme, the immersed boundary and the particles; "
                "none of them is on the single-phase path");
}

int dfdm_launch_kernel_async(dfdm_ctx *c, int which, int rk_stage) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (which < 0 || which > 11 || rk_stage < 1 || rk_stage > 3) return fail(DFDM_ERR_INVALID, "bad kernel id or stage");
    long long before = g_launches;
    int rc = dispatch(c, [&](auto impl) { return decltype(impl)::launch(c, which, rk_stage); });
    c->launches += g_launches - before;
    return rc;
}

int dfdm_set_fused_correction(dfdm_ctx *c, int enable) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (enable && !c->fuse_ok)
        return fail(DFDM_ERR_UNSUPPORTED, "fused corrections need a DNS or filtered-wall-model case without the hybrid scheme");
    if (enable && c->les && !c->sgs_tile)
        return fail(DFDM_ERR_UNSUPPORTED, "fused corrections in LES need the eddy viscosity computed in the stage tiles");
    CK(cudaStreamSynchronize(c->stream));
    destroy_graph(c);   // the captured step holds the other launch sequence
    c->fused = enable != 0;
    return DFDM_OK;
}

int dfdm_set_sgs_in_tile(dfdm_ctx *c, int enable) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (!c->les) return fail(DFDM_ERR_UNSUPPORTED, "the eddy viscosity is only computed for LES (sgs_model > 0)");
    CK(cudaStreamSynchronize(c->stream));
    destroy_graph(c);   // the captured step holds the other launch sequence
    c->sgs_tile = enable != 0;
    // the separate pass reads the corrected velocity from U; the in-tile form takes the fused corrections with it
    c->fused = c->sgs_tile && c->fuse_ok;
    return DFDM_OK;
}

int dfdm_get_sgs_in_tile(dfdm_ctx *c, int *enabled) {
    if (int rc = check_ctx(c)) return rc;
    if (!enabled) return fail(DFDM_ERR_INVALID, "null output");
    *enabled = c->sgs_tile ? 1 : 0;
    return DFDM_OK;
}

int dfdm_get_fused_correction(dfdm_ctx *c, int *enabled) {
    if (int rc = check_ctx(c)) return rc;
    if (!enabled) return fail(DFDM_ERR_INVALID, "null output");
    *enabled = c->fused ? 1 : 0;
    return DFDM_OK;
}

int dfdm_set_stage_variant(dfdm_ctx *c, int variant) {
    g_err.clear();
    if (int rc = check_ctx(c)) return rc;
    if (variant < -1 || variant > 2) return fail(DFDM_ERR_INVALID, "stage variant must be -1, 0, 1 or 2");
    if (variant >= 1 && c->prec == DFDM_FP64) return fail(DFDM_ERR_UNSUPPORTED, "the packed stage kernels are FP32 only");
    if (variant == 2 && !c->tma_ok)
        return fail(DFDM_ERR_UNSUPPORTED, "the TMA stage kernel needs walls in y and Nx a multiple of 4");
    CK(cudaStreamSynchronize(c->stream));
    destroy_graph(c);   // the captured step holds the previous kernel
    if (variant >= 0) { c->stage_variant = variant; return DFDM_OK; }
    return dispatch(c, [&](auto impl) { return decltype(impl)::tune_stage(c, true); });
}

int dfdm_get_stage_variant(dfdm_ctx *c, int *variant, double *ms_one, double *ms_pairs) {
    if (int rc = check_ctx(c)) return rc;
    if (variant) *variant = c->stage_variant;
    if (ms_one) *ms_one = c->stage_ms[0];
    if (ms_pairs) *ms_pairs = c->stage_ms[1];
    return DFDM_OK;
}

int dfdm_get_stage_timing(dfdm_ctx *c, int variant, double *ms) {
    if (int rc = check_ctx(c)) return rc;
    if (variant < 0 || variant > 2) return fail(DFDM_ERR_INVALID, "stage variant must be 0, 1 or 2");
    if (!ms) return fail(DFDM_ERR_INVALID, "null output");
    *ms = c->stage_ms[variant];
    return DFDM_OK;
}

int dfdm_launch_count(dfdm_ctx *c, long long *count) {
    if (int rc = check_any(c)) return rc;
    if (!count) return fail(DFDM_ERR_INVALID, "null output");
    *count = c->launches;
    return DFDM_OK;
}

int dfdm_kernel_bytes(dfdm_ctx *c, int which, double *bytes) {
    if (int rc = check_ctx(c)) return rc;
    if (!bytes) return fail(DFDM_ERR_INVALID, "null output");
    const Dims &d = c->d;
    double cell = (double)d.cells * (double)c->ts;
    double spec = (double)d.Nxc * d.Ny * d.Nz * 2.0 * (double)c->ts;
    double b = 0.0;
    switch (which) {
    case 0: b = c->les ? 4.0 * cell : 0.0; break;                 // read U,V,W; write nu_t
    case 1: b = 12.0 * cell + (c->les ? cell : 0.0) + (c->fused ? cell : 0.0); break;   // stage 1: 3 in, 9 out; stages 2/3:
                                                                  // 9 in, 3 out (fused corrections: + phi)
    case 2: b = 3.0 * cell + spec; break;                         // read u*, write spectrum
    case 3: case 4: case 5: b = 2.0 * spec; break;                // read + write spectrum
    case 6: b = spec + cell; break;                               // read spectrum, write phi
    case 7: b = 7.0 * cell; break;                                // read phi, u*; write u (+P at stage 3)
    case 9: b = c->prm.flow_forcing_mode == 1 ? 3.0 * cell : 0.0; break;   // bulk sum reads U; the shift reads + writes U
    case 10: b = 3.0 * cell + (c->les ? cell : 0.0); break;       // read U, V, W (+ nu_t)
    case 11: b = c->adv ? 6.0 * cell : 0.0; break;                // read U, V, W; write the three terms
    default: return fail(DFDM_ERR_INVALID, "bad kernel id");
    }
    *bytes = b;
    return DFDM_OK;
}

}  // extern "C"

// ================================================================================================================
// Serving groups: the steady steps of several FP32-mixed contexts advanced together, one grouped launch per kernel
// family (and transform length) for all of them.  See kernels_group.cuh.
// tile shape of a member's grouped stage launches: z-planes per block, and whether resident blocks walk the tiles
struct GroupTile {
    int kc;
    bool walk;
};

struct dfdm_group {
    std::vector<dfdm_ctx *> cs;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    bool own_stream = false;               // created by dfdm_group_create (stream argument NULL)
    // at most this many cells per graph branch (0: one branch per class).  Measured on one B200 (FP32, graphed
    // steps, cell-steps/s against per-context graphs on one stream each): 16 x 32^3 1.27x, 64 x 32^3 1.79x,
    // 16 x 48^3 1.02x, 16 x 64^3 0.96x, 8 x 96^3 0.98x, a 32^3-128^3 mix 0.98x; one branch per class gave 0.92x at
    // 16 x 64^3 and 1.5x at 64 x 32^3.
    long long branch_cells = 512 * 1024;
    std::map<const dfdm_ctx *, GroupTile> tile;   // tuned tile shape of the members' grouped stage launches
    int walk_cap[2] = {0, 0};              // resident blocks of the walking stage kernels (form 0, 1) on the device
    bool tuned = false;
    GroupTile forced{-1, false};           // dfdm_group_set_stage_tiles (kc < 0: tuned)
    cudaEvent_t ev = nullptr;              // orders the members' own streams with the group's launches
    // the branch streams and fork/join events of the step's capture, released once the capture has ended
    std::vector<cudaStream_t> cap_streams;
    std::vector<cudaEvent_t> cap_events;
    long long launches = 0, graph_launches = 0;
};

namespace {

// the per-job block counts and the launches of one family, GROUP_MAX jobs at a time
template <class Job, class L> int launch_groups(const std::vector<Job> &jobs, L &&launch) {
    for (size_t o = 0; o < jobs.size(); o += GROUP_MAX) {
        GroupTable<Job> t;
        const int n = (int)std::min<size_t>(GROUP_MAX, jobs.size() - o);
        t.njobs = n;
        int tot = 0;
        for (int q = 0; q < n; ++q) {
            t.start[q] = tot;
            t.jobs[q] = jobs[o + q];
            tot += (int)(jobs[o + q].grid.x * jobs[o + q].grid.y * jobs[o + q].grid.z);
        }
        for (int q = n; q <= GROUP_MAX; ++q) t.start[q] = tot;
        launch(t, tot);
        CKL();
    }
    return DFDM_OK;
}

// can this context step inside a group?  (FP32-mixed DNS with fused corrections, fixed dt, two-level transforms,
// first step taken)
int group_eligible(const dfdm_ctx *c) {
    if (c->prec != DFDM_FP32_MIXED) return fail(DFDM_ERR_UNSUPPORTED, "serving groups take FP32-mixed contexts");
    if (c->les || c->wm || c->adv) return fail(DFDM_ERR_UNSUPPORTED, "serving groups take DNS contexts (no SGS, wall model or hybrid scheme)");
    if (!c->fused) return fail(DFDM_ERR_UNSUPPORTED, "serving groups need the fused corrections");
    if (c->dev_dt()) return fail(DFDM_ERR_UNSUPPORTED, "serving groups take a fixed time step");
    if (!c->x2 || !c->z2 || (c->yper && !c->y2)) return fail(DFDM_ERR_UNSUPPORTED, "serving groups need two-level transform lengths");
    if (c->d.Nx % 4 != 0) return fail(DFDM_ERR_UNSUPPORTED, "serving groups need Nx a multiple of 4");
    if (!c->yper && ysolve3_smem<float>(c->d.Ny) > 227 * 1024)
        return fail(DFDM_ERR_UNSUPPORTED, "serving groups need Ny <= 440 with walls");
    if (!c->projected) return fail(DFDM_ERR_INVALID, "take a context's first step before it joins a group");
    return DFDM_OK;
}

// one step of the cases `cs` on stream st (the launch sequence of step_enqueue, family by family across the cases)
// the grouped stage launch of one form (0 one cell per thread, 1 packed pairs) and RK stage kind (corr: stages 2, 3):
// one block per tile, or (walk) at most walk_cap[v] resident blocks walking the tiles
int launch_stage_jobs(const std::vector<StageJob> &jobs, int v, bool corr, bool walk, const int *walk_cap, cudaStream_t st) {
    return launch_groups(jobs, [&](const GroupTable<StageJob> &t, int nb) {
        const int g = walk ? std::max(1, std::min(nb, walk_cap[v])) : nb;
        if (v == 1) {
            if (walk) { if (corr) kg_stage2_walk<true><<<g, 256, 0, st>>>(t); else kg_stage2_walk<false><<<g, 256, 0, st>>>(t); }
            else { if (corr) kg_stage2<true><<<g, 256, 0, st>>>(t); else kg_stage2<false><<<g, 256, 0, st>>>(t); }
        } else {
            if (walk) { if (corr) kg_stage1_walk<true><<<g, 256, 0, st>>>(t); else kg_stage1_walk<false><<<g, 256, 0, st>>>(t); }
            else { if (corr) kg_stage1<true><<<g, 256, 0, st>>>(t); else kg_stage1<false><<<g, 256, 0, st>>>(t); }
        }
    });
}

// the stage form a member runs in a group: variant 2 is variant 1's arithmetic (the per-case launch falls back to
// variant 0 without TMA)
int group_stage_form(const dfdm_ctx *c) { return (c->stage_variant == 1 || (c->stage_variant == 2 && c->tma_ok)) ? 1 : 0; }

// one member's stage-kernel job of RK stage s (the pointers as they stand; with s >= 2 after the u* swap), kc planes per
// block
StageJob group_stage_job(dfdm_ctx *c, int s, int kc) {
    typedef Impl<float> I;
    const bool corr = s >= 2;
    StageJob J;
    const int v = group_stage_form(c);
    J.kc = kc;
    J.grid = v ? tile_grid(c->d, J.kc, TILE_X2) : tile_grid(c->d, J.kc);
    J.a = step_args<float>(c);
    J.U = corr ? (const float *)c->us2 : (const float *)c->u;
    J.V = corr ? (const float *)c->vs2 : (const float *)c->v;
    J.W = corr ? (const float *)c->ws2 : (const float *)c->w;
    J.tau_x = c->wsd.tau_x; J.tau_z = c->wsd.tau_z;
    StageCoef sc;
    sc.stage = s;
    sc.dt_a11 = c->prm.dt * (8.0 / 15.0);
    sc.dt = c->prm.dt;
    sc.c1 = 1.0 / 4.0;
    sc.c2 = (s == 2) ? 5.0 / 12.0 : 3.0 / 4.0;
    sc.incr = I::incr_form(c, s);
    sc.dtp = nullptr;
    sc.no_uo = 1;
    J.sc = sc;
    J.uo = (float *)c->u; J.vo = (float *)c->v; J.wo = (float *)c->w;   // fused: U is the RK base state
    J.f1u = (float *)c->f1u; J.f1v = (float *)c->f1v; J.f1w = (float *)c->f1w;
    J.us = (float *)c->us; J.vs = (float *)c->vs; J.wsf = (float *)c->wsf;
    J.nu = nullptr; J.rhs_only = nullptr; J.nut_out = nullptr;
    return J;
}

// one step of the cases `cs` (one branch) on stream st (the launch sequence of step_enqueue, family by family across
// the cases); tile: the stage launches' z-planes per block of each member and whether they walk the tiles with
// resident blocks (absent: the member's own kc, one block per tile); walk_cap: resident blocks of the walking kernels
int members_step_enqueue(const std::vector<dfdm_ctx *> &cs, cudaStream_t st,
                         const std::map<const dfdm_ctx *, GroupTile> &tile, const int *walk_cap) {
    typedef Impl<float> I;
    typedef float2 C;
    constexpr int NL = I::NL;
    for (int s = 1; s <= 3; ++s) {
        // ---- stage kernels ----
        std::vector<StageJob> stage[2];   // [variant 0 one cell, variant 1 packed]
        const bool corr = s >= 2;
        for (dfdm_ctx *c : cs) {
            if (corr) { std::swap(c->us, c->us2); std::swap(c->vs, c->vs2); std::swap(c->wsf, c->ws2); }
            const int v = group_stage_form(c);
            auto it = tile.find(c);
            stage[v].push_back(group_stage_job(c, s, it != tile.end() ? it->second.kc : (v ? c->kc_stage2 : c->kc_stage)));
        }
        auto it0 = tile.find(cs[0]);
        const bool walk = it0 != tile.end() && it0->second.walk;
        int rc;
        for (int v = 1; v >= 0; --v)
            if ((rc = launch_stage_jobs(stage[v], v, corr, walk, walk_cap, st))) return rc;
        // ---- div u* + forward x, per length ----
        std::map<int, std::vector<FwdXJob>> fx;
        std::map<int, size_t> fx_smem;
        for (dfdm_ctx *c : cs) {
            FwdXJob J;
            const long long lines = (long long)c->d.Ny * c->d.Nz;
            J.grid = dim3((unsigned)((lines + c->lx2 - 1) / c->lx2), 1, 1);
            J.a = poisson_args<float>(c); J.lx = c->lx2;
            J.U = (const float *)c->us; J.V = (const float *)c->vs; J.W = (const float *)c->wsf; J.src = nullptr;
            J.spec = (C *)c->spec; J.tw = (const C *)c->tw_x; J.twr = (const C *)c->twr_x;
            fx[c->d.Nx / 2].push_back(J);
            fx_smem[c->d.Nx / 2] = c->smem_x2;
        }
        for (auto &kv : fx) {
            with_fft2l(kv.first, [&](auto n) {
                constexpr int M = decltype(n)::value;
                rc = launch_groups(kv.second, [&](const GroupTable<FwdXJob> &t, int nb) { kg_fwd_x<M><<<nb, 256, fx_smem[M], st>>>(t); });
            });
            if (rc) return rc;
        }
        // ---- z transforms and the y solve, per length ----
        auto col_family = [&](int mode) -> int {
            std::map<int, std::vector<ColJob>> jobs;
            std::map<int, std::pair<int, size_t>> cfg;   // threads, shared bytes
            for (dfdm_ctx *c : cs) {
                if (mode == 2 && !c->yper) continue;
                ColJob J;
                const int L = mode == 2 ? c->d.Ny : c->d.Nz;
                J.grid = dim3((unsigned)((c->d.Nxc + NL - 1) / NL), (unsigned)(mode == 2 ? c->d.Nz : c->d.Ny), 1);
                J.d = c->d; J.spec = (C *)c->spec; J.tw = (const C *)(mode == 2 ? c->tw_y : c->tw_z);
                J.kxx = c->d_kxx; J.kyy = c->d_kyy; J.kzz = c->d_kzz;
                jobs[L].push_back(J);
                cfg[L] = mode == 2 ? std::make_pair(c->thr_y2, c->smem_y2) : std::make_pair(c->thr_z2, c->smem_z2);
            }
            int r = DFDM_OK;
            for (auto &kv : jobs) {
                const int thr = cfg[kv.first].first;
                const size_t sm = cfg[kv.first].second;
                with_fft2l(kv.first, [&](auto n) {
                    constexpr int L = decltype(n)::value;
                    if (mode == 0) r = launch_groups(kv.second, [&](const GroupTable<ColJob> &t, int nb) { kg_col<0, L><<<nb, thr, sm, st>>>(t); });
                    else if (mode == 1) r = launch_groups(kv.second, [&](const GroupTable<ColJob> &t, int nb) { kg_col<1, L><<<nb, thr, sm, st>>>(t); });
                    else r = launch_groups(kv.second, [&](const GroupTable<ColJob> &t, int nb) { kg_col<2, L><<<nb, thr, sm, st>>>(t); });
                });
                if (r) return r;
            }
            return r;
        };
        if ((rc = col_family(0))) return rc;
        {
            std::vector<YJob> yj;
            size_t ysm = 0;
            for (dfdm_ctx *c : cs) {
                if (c->yper) continue;
                YJob J;
                J.grid = dim3((unsigned)((c->d.Nxc * c->d.Nz + YS_COLS - 1) / YS_COLS), 1, 1);
                J.d = c->d; J.spec = (C *)c->spec; J.rpiv = c->d_rpiv; J.lo = c->d_lo; J.up = c->d_up;
                yj.push_back(J);
                ysm = std::max(ysm, ysolve3_smem<float>(c->d.Ny));
            }
            if ((rc = launch_groups(yj, [&](const GroupTable<YJob> &t, int nb) { kg_ysolve<<<nb, YS_COLS, ysm, st>>>(t); }))) return rc;
        }
        if ((rc = col_family(2))) return rc;
        if ((rc = col_family(1))) return rc;
        // ---- inverse x, per length ----
        std::map<int, std::vector<InvXJob>> ix;
        std::map<int, size_t> ix_smem;
        for (dfdm_ctx *c : cs) {
            InvXJob J;
            const long long lines = (long long)c->d.Ny * c->d.Nz;
            J.grid = dim3((unsigned)((lines + c->lxi2 - 1) / c->lxi2), 1, 1);
            J.a = poisson_args<float>(c); J.lx = c->lxi2;
            J.spec = (const C *)c->spec; J.phi = (float *)c->phi; J.tw = (const C *)c->tw_x; J.twr = (const C *)c->twr_x;
            ix[c->d.Nx / 2].push_back(J);
            ix_smem[c->d.Nx / 2] = c->smem_xi2;
        }
        for (auto &kv : ix) {
            with_fft2l(kv.first, [&](auto n) {
                constexpr int M = decltype(n)::value;
                rc = launch_groups(kv.second, [&](const GroupTable<InvXJob> &t, int nb) { kg_inv_x<M><<<nb, 256, ix_smem[M], st>>>(t); });
            });
            if (rc) return rc;
        }
        // ---- stage 3: the correction (+ P); stages 1 and 2 are corrected in the next stage kernel's loader ----
        if (s == 3) {
            std::vector<CorrJob> cj;
            for (dfdm_ctx *c : cs) {
                const bool inc = I::incr_form(c, 3);
                CorrJob J;
                const Dims &d = c->d;
                J.grid = dim3((unsigned)((d.Nx / 4 + 63) / 64), (unsigned)((d.Ny + 3) / 4), (unsigned)d.Nz);
                J.a = poisson_args<float>(c);
                J.phi = (const float *)c->phi; J.us = (const float *)c->us; J.vs = (const float *)c->vs; J.ws = (const float *)c->wsf;
                J.U = (float *)c->u; J.V = (float *)c->v; J.W = (float *)c->w; J.P = (float *)c->p;
                J.uo = inc ? (const float *)c->u : nullptr; J.vo = inc ? (const float *)c->v : nullptr;
                J.wo = inc ? (const float *)c->w : nullptr;
                cj.push_back(J);
            }
            if ((rc = launch_groups(cj, [&](const GroupTable<CorrJob> &t, int nb) { kg_correct4<<<nb, dim3(64, 4, 1), 0, st>>>(t); }))) return rc;
        }
    }
    // ---- constant-flux shift of the channel cases ----
    std::vector<BulkJob> bj;
    std::vector<FinalJob> fj;
    std::vector<ShiftJob> sj;
    for (dfdm_ctx *c : cs) {
        if (c->prm.flow_forcing_mode != 1) continue;
        BulkJob B;
        B.grid = dim3((unsigned)c->red_blocks, 1, 1);
        B.d = c->d; B.U = (const float *)c->u; B.dyc = c->d_dyc; B.dzc = c->d_dzc; B.ubd = c->d_ubd; B.part = c->red_part;
        bj.push_back(B);
        FinalJob F;
        F.grid = dim3(1, 1, 1);
        F.nparts = c->red_blocks; F.part = c->red_part; F.Ub_target = c->prm.Ub_target; F.out = c->red_out;
        fj.push_back(F);
        ShiftJob S;
        S.grid = dim3((unsigned)c->red_blocks, 1, 1);
        S.d = c->d; S.U = (float *)c->u; S.dU = c->red_out;
        sj.push_back(S);
    }
    int rc;
    if ((rc = launch_groups(bj, [&](const GroupTable<BulkJob> &t, int nb) { kg_bulk_partial<<<nb, 256, 0, st>>>(t); }))) return rc;
    if ((rc = launch_groups(fj, [&](const GroupTable<FinalJob> &t, int nb) { kg_bulk_final<<<nb, 256, 0, st>>>(t); }))) return rc;
    if ((rc = launch_groups(sj, [&](const GroupTable<ShiftJob> &t, int nb) { kg_shift<<<nb, 256, 0, st>>>(t); }))) return rc;
    return DFDM_OK;
}

// the members split into branches: shape classes (stage form, Nx, Nz, periodic Ny), each cut into runs of consecutive
// members of at most branch_cells cells
std::vector<std::vector<dfdm_ctx *>> group_branches(const dfdm_group *g) {
    std::map<std::array<int, 4>, std::vector<dfdm_ctx *>> classes;
    for (dfdm_ctx *c : g->cs) classes[{group_stage_form(c), c->d.Nx, c->d.Nz, c->yper ? c->d.Ny : -1}].push_back(c);
    std::vector<std::vector<dfdm_ctx *>> branches;
    for (auto &kv : classes) {
        std::vector<dfdm_ctx *> cur;
        long long cells = 0;
        for (dfdm_ctx *c : kv.second) {
            const long long n = (long long)c->d.Nx * c->d.Ny * c->d.Nz;
            if (!cur.empty() && g->branch_cells > 0 && cells + n > g->branch_cells) {
                branches.push_back(cur);
                cur.clear();
                cells = 0;
            }
            cur.push_back(c);
            cells += n;
        }
        branches.push_back(cur);
    }
    return branches;
}

// Tile shapes of the grouped stage launches.  A member's own z-chunk (kc) fills the GPU with that case alone; in a
// group the tiles of all members of a branch share the device, and longer chunks re-read fewer halo planes.  For each
// branch the candidates are the members' own kc, the chunking the same wave model (choose_kc) picks for the branch's
// tiles together, and one chunk per column, each with one block per tile or with resident blocks walking the tiles;
// each is timed with stage-1 launches of the branch (2 + 3 launches, CUDA events on the group's stream) and the
// fastest kept.  The stage kernel's arithmetic does not depend on kc, so neither
// do the results.  Stage-1 launches write only F1 and u*, which every step's stage 1 rewrites before reading, so the
// timing leaves the members' state untouched.  The choice is cached per device, branch shape and member count.
std::mutex g_group_tile_mu;
std::map<std::array<long long, 7>, GroupTile> g_group_tile;

int group_tune(dfdm_group *g) {
    g->tile.clear();
    if (g->forced.kc >= 0) {   // set by the caller: 0 keeps each member's own kc
        for (dfdm_ctx *c : g->cs) {
            const int own = group_stage_form(c) ? c->kc_stage2 : c->kc_stage;
            g->tile[c] = GroupTile{g->forced.kc > 0 ? std::min(g->forced.kc, c->d.Nz) : own, g->forced.walk};
        }
    }
    int dev = 0, nsm = 148;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    for (int v = 0; v < 2; ++v) {
        int occ = 1;
        const void *fn = v ? (const void *)kg_stage2_walk<true> : (const void *)kg_stage1_walk<true>;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 256, 0) != cudaSuccess) occ = 1;
        g->walk_cap[v] = std::max(1, occ) * nsm;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    int rc = DFDM_OK;
    for (auto &members : group_branches(g)) {
        if (g->forced.kc >= 0) break;
        dfdm_ctx *c0 = members[0];
        const int v = group_stage_form(c0);
        const Dims &d = c0->d;
        const std::array<long long, 7> key = {dev, v, d.Nx, d.Ny, d.Nz, c0->yper, (long long)members.size()};
        GroupTile choice{-1, false};
        {
            std::lock_guard<std::mutex> lk(g_group_tile_mu);
            auto it = g_group_tile.find(key);
            if (it != g_group_tile.end()) choice = it->second;
        }
        if (choice.kc < 0) {
            int occ = 1;
            const void *fn = v ? (const void *)kg_stage2<false> : (const void *)kg_stage1<false>;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 256, 0) != cudaSuccess) occ = 1;
            const int tx = v ? TILE_X2 : TILE_X;
            // the wave model over the branch's tiles: as choose_kc with every member's columns side by side
            Dims dd = d;
            dd.Ny = d.Ny * (int)members.size();
            const int own = v ? c0->kc_stage2 : c0->kc_stage;
            const int kcs[3] = {own, choose_kc(dd, occ, nsm, tx), d.Nz};
            double best = 1e30;
            for (int q = 0; q < 6 && !rc; ++q) {
                const int kc = kcs[q % 3];
                const bool walk = q >= 3;
                bool seen = false;
                for (int r = 0; r < q % 3; ++r) seen = seen || kcs[r] == kc;
                if (seen) continue;
                std::vector<StageJob> jobs;
                for (dfdm_ctx *c : members) jobs.push_back(group_stage_job(c, 1, kc));
                for (int r = 0; r < 2 && !rc; ++r) rc = launch_stage_jobs(jobs, v, false, walk, g->walk_cap, g->stream);
                if (rc) break;
                cudaEventRecord(e0, g->stream);
                for (int r = 0; r < 3 && !rc; ++r) rc = launch_stage_jobs(jobs, v, false, walk, g->walk_cap, g->stream);
                cudaEventRecord(e1, g->stream);
                if (cudaEventSynchronize(e1) != cudaSuccess) { rc = fail(DFDM_ERR_CUDA, "group tuning failed"); break; }
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms < best) { best = ms; choice = GroupTile{kc, walk}; }
            }
            if (rc) break;
            std::lock_guard<std::mutex> lk(g_group_tile_mu);
            g_group_tile[key] = choice;
        }
        for (dfdm_ctx *c : members) g->tile[c] = choice;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

// A group's cases fall into shape classes: the same stage-kernel form, Nx, Nz and periodic Ny, so that every kernel
// family of a class is one instantiation, i.e. one launch.  Each branch (a class, or a run of its members) is
// captured on a graph branch of its own (forked from the group's stream and joined back), so the branches' launches
// overlap on the device as independent streams' would, while the cases of a branch share their launches.
int group_step_enqueue(dfdm_group *g) {
    const std::vector<std::vector<dfdm_ctx *>> branches = group_branches(g);
    if (branches.size() == 1) return members_step_enqueue(g->cs, g->stream, g->tile, g->walk_cap);
    cudaEvent_t fork = nullptr;
    int rc = DFDM_OK;
    auto check = [&](cudaError_t e, const char *what) {
        if (!rc && e != cudaSuccess) rc = fail(DFDM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    };
    check(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "fork event creation");
    if (fork) g->cap_events.push_back(fork);
    check(cudaEventRecord(fork, g->stream), "fork event record");
    for (auto &members : branches) {
        if (rc) break;
        cudaStream_t b = nullptr;
        cudaEvent_t j = nullptr;
        check(cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking), "branch stream creation");
        if (b) g->cap_streams.push_back(b);
        check(cudaEventCreateWithFlags(&j, cudaEventDisableTiming), "join event creation");
        if (j) g->cap_events.push_back(j);
        if (rc) break;
        check(cudaStreamWaitEvent(b, fork, 0), "branch wait on the fork");
        if (!rc) rc = members_step_enqueue(members, b, g->tile, g->walk_cap);
        check(cudaEventRecord(j, b), "join event record");
        check(cudaStreamWaitEvent(g->stream, j, 0), "wait on the join");
    }
    if (rc) g_err += " (" + std::to_string(branches.size()) + " branches)";
    return rc;
}

void release_capture_objects(dfdm_group *g) {
    for (cudaEvent_t e : g->cap_events) cudaEventDestroy(e);
    for (cudaStream_t b : g->cap_streams) cudaStreamDestroy(b);
    g->cap_events.clear();
    g->cap_streams.clear();
}

void group_destroy_graph(dfdm_group *g) {
    if (g->gexec) { cudaGraphExecDestroy(g->gexec); g->gexec = nullptr; }
    if (g->graph) { cudaGraphDestroy(g->graph); g->graph = nullptr; }
}

// dynamic shared memory of every grouped transform instantiation the group launches
int group_attributes(dfdm_group *g) {
    int rc = DFDM_OK;
    auto setattr = [&](const void *fn, size_t bytes) {
        if (rc || bytes <= 48 * 1024) return;
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) rc = fail(DFDM_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    };
    // the grouped y solve's shared memory depends on the members' Ny: its cap is the device's opt-in maximum (the
    // attribute holds for the whole process; a group of smaller grids must not lower it under another's launches)
    int optin = 0, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return fail(DFDM_ERR_CUDA, "device attribute query failed");
    setattr((const void *)kg_ysolve, (size_t)optin);
    for (dfdm_ctx *c : g->cs) {
        with_fft2l(c->d.Nx / 2, [&](auto n) {
            constexpr int M = decltype(n)::value;
            setattr((const void *)kg_fwd_x<M>, c->smem_x2);
            setattr((const void *)kg_inv_x<M>, c->smem_xi2);
        });
        with_fft2l(c->d.Nz, [&](auto n) {
            constexpr int L = decltype(n)::value;
            setattr((const void *)kg_col<0, L>, c->smem_z2);
            setattr((const void *)kg_col<1, L>, c->smem_z2);
        });
        if (c->yper)
            with_fft2l(c->d.Ny, [&](auto n) {
                constexpr int L = decltype(n)::value;
                setattr((const void *)kg_col<2, L>, c->smem_y2);
            });
    }
    return rc;
}

}  // namespace

extern "C" {

int dfdm_group_create(dfdm_ctx *const *ctxs, int n, void *stream, dfdm_group **out) {
    g_err.clear();
    if (!out) return fail(DFDM_ERR_INVALID, "null output");
    *out = nullptr;
    if (n < 1 || !ctxs) return fail(DFDM_ERR_INVALID, "a group needs at least one context");
    for (int q = 0; q < n; ++q) {
        if (int rc = check_ctx(ctxs[q])) return rc;
        if (int rc = group_eligible(ctxs[q])) return rc;
        for (int r = 0; r < q; ++r)
            if (ctxs[r] == ctxs[q]) return fail(DFDM_ERR_INVALID, "a context appears twice in the group");
    }
    dfdm_group *g = new dfdm_group;
    g->cs.assign(ctxs, ctxs + n);
    if (int rc = group_attributes(g)) { delete g; return rc; }
    if (cudaEventCreateWithFlags(&g->ev, cudaEventDisableTiming) != cudaSuccess) {
        delete g;
        return fail(DFDM_ERR_CUDA, "event creation failed");
    }
    if (stream) {
        g->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaEventDestroy(g->ev);
            delete g;
            return fail(DFDM_ERR_CUDA, "stream creation failed");
        }
        g->own_stream = true;
    }
    *out = g;
    return DFDM_OK;
}

int dfdm_group_step_async(dfdm_group *g, int nsteps) {
    g_err.clear();
    if (!g) return fail(DFDM_ERR_INVALID, "null group");
    if (nsteps < 0) return fail(DFDM_ERR_INVALID, "nsteps must be >= 0");
    if (nsteps == 0) return DFDM_OK;
    // each member's earlier work on its own stream comes before the group's steps (and the members' later work,
    // below, after them), without a host synchronisation
    for (dfdm_ctx *c : g->cs)
        if (c->stream != g->stream) {
            CK(cudaEventRecord(g->ev, c->stream));
            CK(cudaStreamWaitEvent(g->stream, g->ev, 0));
        }
    if (!g->tuned) {   // the grouped stage launches' tile shapes, before the first capture
        if (int rc = group_tune(g)) return rc;
        g->tuned = true;
    }
    for (int n = 0; n < nsteps; ++n) {
        if (!g->gexec) {   // one step of the whole group, captured once per group
            CK(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
            long long before = g_launches;
            int rc = group_step_enqueue(g);
            g->graph_launches = g_launches - before;
            g_launches = before;
            cudaGraph_t gr = nullptr;
            cudaError_t e = cudaStreamEndCapture(g->stream, &gr);
            release_capture_objects(g);
            if (rc) { if (gr) cudaGraphDestroy(gr); return rc; }
            if (e != cudaSuccess) return fail(DFDM_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            g->graph = gr;
            if (int rp = make_programmatic(g->graph)) return rp;
            CK(cudaGraphInstantiate(&g->gexec, g->graph, 0));
        }
        CK(cudaGraphLaunch(g->gexec, g->stream));
        g->launches += g->graph_launches;
        for (dfdm_ctx *c : g->cs) c->t += c->prm.dt;   // the group's kernels are counted on the group
    }
    CK(cudaEventRecord(g->ev, g->stream));
    for (dfdm_ctx *c : g->cs)
        if (c->stream != g->stream) CK(cudaStreamWaitEvent(c->stream, g->ev, 0));
    return DFDM_OK;
}

int dfdm_group_synchronize(dfdm_group *g) {
    if (!g) return fail(DFDM_ERR_INVALID, "null group");
    CK(cudaStreamSynchronize(g->stream));
    return DFDM_OK;
}

int dfdm_group_set_branch_cells(dfdm_group *g, long long cells) {
    if (!g || cells < 0) return fail(DFDM_ERR_INVALID, "null group or negative cell count");
    if (g->branch_cells != cells) {
        g->branch_cells = cells;
        group_destroy_graph(g);   // recaptured (and its tile shapes re-chosen) at the next step
        g->tuned = false;
    }
    return DFDM_OK;
}

int dfdm_group_set_stage_tiles(dfdm_group *g, int kc, int walk) {
    if (!g) return fail(DFDM_ERR_INVALID, "null group");
    g->forced = GroupTile{kc < 0 ? -1 : kc, walk != 0};
    g->tuned = false;
    group_destroy_graph(g);   // recaptured at the next step
    return DFDM_OK;
}

int dfdm_group_get_stream(dfdm_group *g, void **stream) {
    if (!g || !stream) return fail(DFDM_ERR_INVALID, "null argument");
    *stream = (void *)g->stream;
    return DFDM_OK;
}

int dfdm_group_launch_count(dfdm_group *g, long long *count) {
    if (!g || !count) return fail(DFDM_ERR_INVALID, "null argument");
    *count = g->launches;
    return DFDM_OK;
}

// no host wait: an executable graph and an event destroyed while in flight are released when the device is done
int dfdm_group_destroy(dfdm_group *g) {
    if (!g) return DFDM_OK;
    group_destroy_graph(g);
    if (g->ev) cudaEventDestroy(g->ev);
    if (g->own_stream) cudaStreamDestroy(g->stream);   // returns at once; released when its work is done
    delete g;
    return DFDM_OK;
}

}  // extern "C"
