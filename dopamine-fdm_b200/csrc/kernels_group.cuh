// kernels_group.cuh -- grouped launches of the FP32-mixed step: one launch runs one kernel family for every case of
// a serving group, on grids of uneven size.
//
// A grouped launch carries a job table in its parameter space (a __grid_constant__ struct, so the per-job
// arguments are read through the constant cache, as an ordinary launch reads its own): job j owns the linear
// blocks start[j] .. start[j+1]-1 of the launch.  Each block finds its job by binary search over `start`, turns its
// offset into block coordinates of that job's own grid, and runs the family's kernel body (the same __device__
// function the per-case kernel runs, given a JobBlock instead of the hardware block registers) with the job's
// arguments.  A job's arithmetic therefore depends on its own case only, never on the other jobs of the launch.  It is
// the per-case kernel's source; the two compilations may contract scalar multiply-adds differently, so a case agrees
// with its per-case steps to rounding.  The transform families are templated on their length, so a group launches
// them once per distinct length.
#pragma once

#include "kernels_diag.cuh"
#include "kernels_fft2l.cuh"
#include "kernels_step.cuh"

namespace dfdm {

constexpr int GROUP_MAX = 24;   // jobs per grouped launch (larger groups take several launches)

template <class Job> struct GroupTable {
    int njobs;
    int start[GROUP_MAX + 1];
    Job jobs[GROUP_MAX];
};

__device__ __forceinline__ int group_job(const int *start, int njobs, int b) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}
// block coordinates of linear tile b (of job j) in job j's own grid; at(g, j) is this block's
template <class Job> __device__ __forceinline__ JobBlock at(const GroupTable<Job> &g, int j, int b) {
    const dim3 gd = g.jobs[j].grid;
    const int local = b - g.start[j];
    JobBlock r;
    r.b.x = local % gd.x;
    const int t = local / gd.x;
    r.b.y = t % gd.y;
    r.b.z = t / gd.y;
    r.g = gd;
    return r;
}
template <class Job> __device__ __forceinline__ JobBlock at(const GroupTable<Job> &g, int j) { return at(g, j, (int)blockIdx.x); }

// ---- the stage kernel (DNS, no wall model): packed pairs (variant 1) or one cell per thread (variant 0) ----
struct StageJob {
    dim3 grid;
    StepArgs<float> a;
    const float *U, *V, *W;
    const double *tau_x, *tau_z;
    StageCoef sc;
    int kc;
    float *uo, *vo, *wo, *f1u, *f1v, *f1w, *us, *vs, *wsf;
    // null, passed as run-time values as the per-case launch passes them (not as constants the body would fold)
    const float *nu;
    float *rhs_only, *nut_out;
};
template <bool CORR>
__global__ void __launch_bounds__(256, 2) kg_stage2(const __grid_constant__ GroupTable<StageJob> g) {
    pdl_enter();
    const int j = group_job(g.start, g.njobs, blockIdx.x);
    const StageJob &J = g.jobs[j];
    k_tiled2_body<false, false, 8, false, CORR>(at(g, j), J.a, J.U, J.V, J.W, J.nu, J.tau_x, J.tau_z, J.sc, J.kc,
                                                J.uo, J.vo, J.wo, J.f1u, J.f1v, J.f1w, J.us, J.vs, J.wsf, J.rhs_only);
}
template <bool CORR>
__global__ void __launch_bounds__(256, 3) kg_stage1(const __grid_constant__ GroupTable<StageJob> g) {
    pdl_enter();
    const int j = group_job(g.start, g.njobs, blockIdx.x);
    const StageJob &J = g.jobs[j];
    k_tiled_body<float, false, false, 32, 8, 0, CORR>(at(g, j), J.a, J.U, J.V, J.W, J.nu, J.tau_x, J.tau_z, J.sc,
                                                      J.kc, J.uo, J.vo, J.wo, J.f1u, J.f1v, J.f1w, J.us, J.vs, J.wsf,
                                                      J.rhs_only, J.nut_out);
}

// The same stage kernels as persistent blocks: a grid of at most the resident capacity walks the table's tiles
// (tile b, b + gridDim.x, ...).  Between tiles a block waits for its last cp.async copies and synchronises, so the next
// tile's loads cannot overtake the previous tile's reads of shared memory.  The group's tuner times this form against
// one block per tile and keeps the faster.
template <bool CORR>
__global__ void __launch_bounds__(256, 2) kg_stage2_walk(const __grid_constant__ GroupTable<StageJob> g) {
    pdl_enter();
    const int total = g.start[g.njobs];
    for (int b = blockIdx.x; b < total; b += gridDim.x) {
        const int j = group_job(g.start, g.njobs, b);
        const StageJob &J = g.jobs[j];
        k_tiled2_body<false, false, 8, false, CORR>(at(g, j, b), J.a, J.U, J.V, J.W, J.nu, J.tau_x, J.tau_z, J.sc, J.kc,
                                                    J.uo, J.vo, J.wo, J.f1u, J.f1v, J.f1w, J.us, J.vs, J.wsf, J.rhs_only);
        cp_async_wait_all();
        __syncthreads();
    }
}
template <bool CORR>
__global__ void __launch_bounds__(256, 3) kg_stage1_walk(const __grid_constant__ GroupTable<StageJob> g) {
    pdl_enter();
    const int total = g.start[g.njobs];
    for (int b = blockIdx.x; b < total; b += gridDim.x) {
        const int j = group_job(g.start, g.njobs, b);
        const StageJob &J = g.jobs[j];
        k_tiled_body<float, false, false, 32, 8, 0, CORR>(at(g, j, b), J.a, J.U, J.V, J.W, J.nu, J.tau_x, J.tau_z, J.sc,
                                                          J.kc, J.uo, J.vo, J.wo, J.f1u, J.f1v, J.f1w, J.us, J.vs, J.wsf,
                                                          J.rhs_only, J.nut_out);
        cp_async_wait_all();
        __syncthreads();
    }
}

// ---- div u* + forward x transform, length Nx = 2M ----
struct FwdXJob {
    dim3 grid;
    PoissonArgs<float> a;
    int lx;
    const float *U, *V, *W;
    const float *src;   // null (run-time value, as in the per-case launch)
    float2 *spec;
    const float2 *tw, *twr;
};
template <int M>
__global__ void __launch_bounds__(256, 4) kg_fwd_x(const __grid_constant__ GroupTable<FwdXJob> g) {
    pdl_enter();
    const int j = group_job(g.start, g.njobs, blockIdx.x);
    const FwdXJob &J = g.jobs[j];
    k_fwd_x2_body<float, true, M>(at(g, j), J.a, J.lx, J.U, J.V, J.W, J.src, J.spec, J.tw, J.twr);
}

// ---- column transforms: z forward (MODE 0), z inverse (1), periodic-y solve (2), length L ----
struct ColJob {
    dim3 grid;
    Dims d;
    float2 *spec;
    const float2 *tw;
    const double *kxx, *kyy, *kzz;
};
template <int MODE, int L>
__global__ void __launch_bounds__(256) kg_col(const __grid_constant__ GroupTable<ColJob> g) {
    pdl_enter();
    typedef float T;
    constexpr int NL = 16;
    const int j = group_job(g.start, g.njobs, blockIdx.x);
    const ColJob &J = g.jobs[j];
    const JobBlock bc = at(g, j);
    const Dims &d = J.d;
    float2 *__restrict__ spec = J.spec;
    const float2 *__restrict__ tw = J.tw;
    const double *__restrict__ kxx = J.kxx, *__restrict__ kyy = J.kyy, *__restrict__ kzz = J.kzz;
#define DFDM_BLOCK_IDX bc.b
#include "k_col2_body.inc"
#undef DFDM_BLOCK_IDX
}

// ---- wall-bounded y solve: YS_COLS columns of the flattened (kz, kx) index per block (k_ysolve3) ----
struct YJob {
    dim3 grid;
    Dims d;
    float2 *spec;
    const double *rpiv, *lo, *up;
};
__global__ void __launch_bounds__(YS_COLS) kg_ysolve(const __grid_constant__ GroupTable<YJob> g) {
    pdl_enter();
    const int j = group_job(g.start, g.njobs, blockIdx.x);
    const YJob &J = g.jobs[j];
    k_ysolve3_body<float>(at(g, j), J.d, J.spec, J.rpiv, J.lo, J.up);
}

// ---- inverse x transform ----
struct InvXJob {
    dim3 grid;
    PoissonArgs<float> a;
    int lx;
    const float2 *spec;
    float *phi;
    const float2 *tw, *twr;
};
template <int M>
__global__ void __launch_bounds__(256) kg_inv_x(const __grid_constant__ GroupTable<InvXJob> g) {
    pdl_enter();
    const int j = group_job(g.start, g.njobs, blockIdx.x);
    const InvXJob &J = g.jobs[j];
    k_inv_x2_body<float, M>(at(g, j), J.a, J.lx, J.spec, J.phi, J.tw, J.twr);
}

// ---- velocity correction (+ P at stage 3), 64 x 4 threads of four x-faces ----
struct CorrJob {
    dim3 grid;
    PoissonArgs<float> a;
    const float *phi, *us, *vs, *ws;
    float *U, *V, *W, *P;
    const float *uo, *vo, *wo;
};
__global__ void __launch_bounds__(256) kg_correct4(const __grid_constant__ GroupTable<CorrJob> g) {
    pdl_enter();
    const int j = group_job(g.start, g.njobs, blockIdx.x);
    const CorrJob &J = g.jobs[j];
    k_correct4_body<float>(at(g, j), J.a, J.phi, J.us, J.vs, J.ws, J.U, J.V, J.W, J.P, J.uo, J.vo, J.wo);
}

// ---- constant flux: bulk-velocity partial sums, their final reduction (one block per case), the shift ----
struct BulkJob {
    dim3 grid;
    Dims d;
    const float *U;
    const double *dyc, *dzc, *ubd;
    double *part;
};
__global__ void __launch_bounds__(256) kg_bulk_partial(const __grid_constant__ GroupTable<BulkJob> g) {
    pdl_enter();
    const int j = group_job(g.start, g.njobs, blockIdx.x);
    const BulkJob &J = g.jobs[j];
    k_bulk_partial_body<float, true>(at(g, j), J.d, J.U, J.dyc, J.dzc, J.ubd, J.part);
}
struct FinalJob {
    dim3 grid;
    int nparts;
    const double *part;
    double Ub_target;
    double *out;
};
__global__ void __launch_bounds__(256) kg_bulk_final(const __grid_constant__ GroupTable<FinalJob> g) {
    pdl_enter();
    const int j = group_job(g.start, g.njobs, blockIdx.x);
    const FinalJob &J = g.jobs[j];
    k_bulk_final_body(at(g, j), J.nparts, J.part, J.Ub_target, J.out);
}
struct ShiftJob {
    dim3 grid;
    Dims d;
    float *U;
    const double *dU;
};
__global__ void __launch_bounds__(256) kg_shift(const __grid_constant__ GroupTable<ShiftJob> g) {
    pdl_enter();
    const int j = group_job(g.start, g.njobs, blockIdx.x);
    const ShiftJob &J = g.jobs[j];
    k_shift_body<float>(at(g, j), J.d, J.U, J.dU);
}

// kernel parameter space holds at most 32764 bytes
static_assert(sizeof(GroupTable<StageJob>) <= 32764, "stage job table too large");
static_assert(sizeof(GroupTable<FwdXJob>) <= 32764 && sizeof(GroupTable<InvXJob>) <= 32764, "x job table too large");
static_assert(sizeof(GroupTable<ColJob>) <= 32764 && sizeof(GroupTable<YJob>) <= 32764, "column job table too large");
static_assert(sizeof(GroupTable<CorrJob>) <= 32764 && sizeof(GroupTable<BulkJob>) <= 32764, "job table too large");

}  // namespace dfdm
