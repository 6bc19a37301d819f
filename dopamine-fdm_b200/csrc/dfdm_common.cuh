// dfdm_common.cuh -- device-side conventions shared by every kernel of the library.
//
// HBM layout.  Each field keeps only its independent cells, x fastest:  f[(k*Ny + j)*Nx + i].
//   U: face i (between centres i and i+1), centre j, centre k        -> reference U(i+2, j+2, k+2)
//   V: centre i, face j (between centres j and j+1), centre k        -> reference V(i+2, j+2, k+2)
//   W: centre i, centre j, face k                                    -> reference W(i+2, j+2, k+2)
//   P, nu_t, phi: centres                                            -> reference P(i+2, j+2, k+2)
// x and z are periodic: the reference's duplicated last cell and its ghosts are the wrap i -> i mod Nx.
// y is periodic (Ny cells, wrap) or bounded by no-slip walls (Ny cells): then the ghost centre j = -1 / Ny of U
// and W holds minus the first / last interior value (apply_Robin_bc_y with alpha = 0), V's wall faces j = -1 and
// j = Ny-1 are zero (row Ny-1 is stored and never written), and nu_t's ghosts are zero (sgs_fill_ghosts).
// The spectral array is complex, (Nx/2+1) x Ny x Nz, kx fastest.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dfdm {

// Programmatic dependent launch.  Every kernel of the library starts with pdl_enter(), which waits until the kernel
// before it has completed and its memory is visible, before this grid reads or writes anything.  The library turns
// the kernel-to-kernel edges of its captured graphs into programmatic edges, so the next grid is launched as the
// blocks of this one exit, without the launch gap of a full dependency; elsewhere (plain stream launches) the wait
// returns at once.  No kernel triggers its dependents early: blocks of later grids would then wait on SM slots that
// the running grid needs (measured: 23 % slower steps at 256 x 192 x 256).
__device__ __forceinline__ void pdl_enter() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

// Block coordinates of a kernel body.  A per-case kernel passes HwBlock, whose accessors read the hardware registers
// at each use (the body then compiles as if it named blockIdx / gridDim itself); a grouped launch (kernels_group.cuh)
// passes JobBlock, the block's coordinates in its own case's grid.
struct HwBlock {
    __device__ __forceinline__ uint3 idx() const { return blockIdx; }
    __device__ __forceinline__ dim3 dim() const { return gridDim; }
};
struct JobBlock {
    uint3 b;
    dim3 g;
    __device__ __forceinline__ uint3 idx() const { return b; }
    __device__ __forceinline__ dim3 dim() const { return g; }
};

template <typename T> struct cplx_t;
template <> struct cplx_t<double> { typedef double2 type; };
template <> struct cplx_t<float> { typedef float2 type; };

template <typename T> __host__ __device__ __forceinline__ typename cplx_t<T>::type mkc(T a, T b) {
    typename cplx_t<T>::type r; r.x = a; r.y = b; return r;
}

// Per-direction metric arrays, offset by one so index -1 is valid: m[j+1] holds the value of device index j.
//   dc[j] = y(j+2) - y(j+1)            width of centre j           ("y(j)-y(j-1)" in reference indices)
//   df[j] = yg(j+3) - yg(j+2)          centre spacing across face j ("yg(j+1)-yg(j)")
//   w0[j], w1[j] = weight_y_0(j+2), weight_y_1(j+2) of face j
// plus reciprocals for the FP32 path.  z uses the same layout.  Stored in double and in the storage type.
template <typename T> struct Metric1D {
    const T *dc, *df, *w0, *w1, *idc, *idf;   // all offset by +1 (point at element 1 of the allocation)
};

struct Dims {
    int Nx, Ny, Nz;      // independent cells
    int NyV;             // interior V rows: Ny-1 with walls, Ny when periodic
    int Nxc;             // Nx/2 + 1 spectral x modes
    int yper;            // 1 periodic y, 0 walls
    long long plane;     // Nx*Ny
    long long cells;     // Nx*Ny*Nz
};

__host__ __device__ __forceinline__ long long idx3(const Dims &d, int i, int j, int k) {
    return ((long long)k * d.Ny + j) * d.Nx + i;
}
__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// U or W at a centre-in-y index j that may be a ghost (j = -1 or Ny); i, k already wrapped.
template <typename T>
__device__ __forceinline__ T ld_yc(const T *__restrict__ f, const Dims &d, int i, int j, int k) {
    if (d.yper) { j = wrap(j, d.Ny); return __ldg(f + idx3(d, i, j, k)); }
    if (j < 0) return -__ldg(f + idx3(d, i, 0, k));
    if (j >= d.Ny) return -__ldg(f + idx3(d, i, d.Ny - 1, k));
    return __ldg(f + idx3(d, i, j, k));
}
// V at a face-in-y index j in [-1, Ny-1] (walls) or any wrapped index (periodic)
template <typename T>
__device__ __forceinline__ T ld_yf(const T *__restrict__ f, const Dims &d, int i, int j, int k) {
    if (d.yper) { j = wrap(j, d.Ny); return __ldg(f + idx3(d, i, j, k)); }
    if (j < 0) return T(0);
    return __ldg(f + idx3(d, i, j, k));
}
// nu_t at a centre-in-y index that may be a ghost: zero at the walls
template <typename T>
__device__ __forceinline__ T ld_nu(const T *__restrict__ f, const Dims &d, int i, int j, int k) {
    if (d.yper) { j = wrap(j, d.Ny); return __ldg(f + idx3(d, i, j, k)); }
    if (j < 0 || j >= d.Ny) return T(0);
    return __ldg(f + idx3(d, i, j, k));
}

// Divide / reciprocal helpers: the FP64 path divides exactly where the reference divides and forms 1/d where
// the reference forms 1/d, so its rounding follows the Fortran expressions; the FP32 path multiplies by the
// reciprocal precomputed in double.
template <typename T> struct Arith;
template <> struct Arith<double> {
    static __device__ __forceinline__ double div(double a, const double *d, const double *, int j) { return a / d[j]; }
    static __device__ __forceinline__ double inv(const double *d, const double *, int j) { return 1.0 / d[j]; }
};
template <> struct Arith<float> {
    static __device__ __forceinline__ float div(float a, const float *, const float *id, int j) { return a * id[j]; }
    static __device__ __forceinline__ float inv(const float *, const float *id, int j) { return id[j]; }
};

// Asynchronous global -> shared copies (cp.async, 4 or 8 bytes per element).
template <int B> __device__ __forceinline__ void cp_async(void *smem, const void *gmem) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(B));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

}  // namespace dfdm
