// fft_smem.cuh -- batched complex FFTs in shared memory (Stockham autosort, radix 2/3/4/5, runtime plan).
//
// Replaces the cuFFT plans of the reference's GPU Poisson backend (src/poisson_gpu.f90:94-117) and the FFTW
// plans of its CPU build (src/initialization.f90:385-412).  Convention: forward exp(-2 pi i jk/n), both
// directions unnormalised, as FFTW_FORWARD / FFTW_BACKWARD and CUFFT_FORWARD / CUFFT_INVERSE.
//
// Stockham pass with radix R over a line of length n (Ns = product of the radices already applied):
//   for every butterfly j in [0, n/R):  k = j mod Ns
//       v[r] = in[j + r n/R] * W_n^(r k n/(Ns R)),  v = DFT_R(v),  out[(j div Ns) Ns R + k + r Ns] = v[r]
// The output is in natural order after the last pass; src/dst ping-pong between two shared buffers.
#pragma once

#include "dfdm_common.cuh"

namespace dfdm {

// Division by a runtime constant with a multiply-high (Granlund & Montgomery, "Division by invariant integers
// using multiplication", 1994): for d >= 2, l = ceil(log2 d), m = ceil(2^(31+l)/d) < 2^32 and
// n / d = umulhi(n, m) >> (l-1) for every n < 2^22 (checked exhaustively for d <= 4096 when the plan is built).
struct FastDiv {
    unsigned d, m;
    int s;
};
inline FastDiv make_fastdiv(unsigned d) {
    FastDiv f;
    f.d = d; f.m = 0; f.s = 0;
    if (d <= 1) return f;
    int l = 0;
    while ((1u << l) < d) ++l;
    f.m = (unsigned)((((unsigned long long)1 << (31 + l)) + d - 1) / d);
    f.s = l - 1;
    return f;
}
__device__ __forceinline__ unsigned fdiv(unsigned n, const FastDiv &f) { return f.d <= 1 ? n : (__umulhi(n, f.m) >> f.s); }

struct FFTPlan {
    int n;           // transform length
    int nrad;        // number of passes
    int rad[16];     // radix of each pass
    FastDiv ns[16];  // division by Ns (product of the radices of the earlier passes)
    FastDiv nb[16];  // division by n / rad (butterflies per line)
};

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {   // a * conj(b)
    C r; r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; return r;
}
// multiply by -i (forward) or +i (inverse)
template <bool INV, typename C> __device__ __forceinline__ C mul_mi(C a) {
    C r;
    if (INV) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
    return r;
}

template <typename T, bool INV, typename C>
__device__ __forceinline__ void dft_small(C *v, int R) {
    if (R == 2) {
        C a = v[0], b = v[1];
        v[0] = cadd(a, b); v[1] = csub(a, b);
    } else if (R == 4) {
        C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]), t2 = cadd(v[1], v[3]), t3 = csub(v[1], v[3]);
        C it3 = mul_mi<INV>(t3);
        v[0] = cadd(t0, t2); v[2] = csub(t0, t2); v[1] = cadd(t1, it3); v[3] = csub(t1, it3);
    } else if (R == 3) {
        const T s = (T)0.86602540378443864676;   // sin(2 pi/3)
        C a = v[0], t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
        C m; m.x = a.x - (T)0.5 * t1.x; m.y = a.y - (T)0.5 * t1.y;
        C st2; st2.x = s * t2.x; st2.y = s * t2.y;
        C ist2 = mul_mi<INV>(st2);
        v[0] = cadd(a, t1); v[1] = cadd(m, ist2); v[2] = csub(m, ist2);
    } else if (R == 5) {
        const T c1 = (T)0.30901699437494742410, c2 = (T)-0.80901699437494742410;   // cos(2pi/5), cos(4pi/5)
        const T s1 = (T)0.95105651629515357212, s2 = (T)0.58778525229247312917;    // sin(2pi/5), sin(4pi/5)
        C a = v[0];
        C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]), t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        C m1, m2, n1, n2;
        m1.x = a.x + c1 * t1.x + c2 * t2.x; m1.y = a.y + c1 * t1.y + c2 * t2.y;
        m2.x = a.x + c2 * t1.x + c1 * t2.x; m2.y = a.y + c2 * t1.y + c1 * t2.y;
        n1.x = s1 * t3.x + s2 * t4.x; n1.y = s1 * t3.y + s2 * t4.y;
        n2.x = s2 * t3.x - s1 * t4.x; n2.y = s2 * t3.y - s1 * t4.y;
        C in1 = mul_mi<INV>(n1), in2 = mul_mi<INV>(n2);
        v[0] = cadd(a, cadd(t1, t2));
        v[1] = cadd(m1, in1); v[4] = csub(m1, in1);
        v[2] = cadd(m2, in2); v[3] = csub(m2, in2);
    }
}

// One Stockham pass of compile-time radix R over `nlines` lines (see the header comment for the index map).
template <typename T, bool INV, bool LINES_FAST, int NL, int R>
__device__ __forceinline__ void fft_pass(const typename cplx_t<T>::type *__restrict__ src,
                                         typename cplx_t<T>::type *__restrict__ dst, int nlines, int ldl, int lde,
                                         int n, int Ns, const FastDiv &fns, const FastDiv &fnb,
                                         const typename cplx_t<T>::type *__restrict__ tw) {
    typedef typename cplx_t<T>::type C;
    const int nb = n / R;
    const int total = nb * (LINES_FAST ? NL : nlines);
    const int twstep = n / (Ns * R);
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
        int line, j;
        if (LINES_FAST) { line = b % NL; j = b / NL; }
        else { line = (int)fdiv((unsigned)b, fnb); j = b - line * nb; }
        const int q = (int)fdiv((unsigned)j, fns);
        const int k = j - q * Ns;
        C v[R];
        const C *s = src + line * ldl;
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = s[(j + r * nb) * lde];
        if (k != 0) {
            const int tk = k * twstep;
#pragma unroll
            for (int r = 1; r < R; ++r) {
                C w = __ldg(tw + r * tk);
                v[r] = INV ? cmulc(v[r], w) : cmul(v[r], w);
            }
        }
        dft_small<T, INV>(v, R);
        C *d = dst + line * ldl;
        const int base = q * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) d[(base + r * Ns) * lde] = v[r];
    }
}

// Transforms `nlines` lines held in shared memory.  Element e of line l lives at buf[l*ldl + e*lde].
// LINES_FAST selects the thread mapping: consecutive threads take consecutive lines (column tiles, lde > 1, the
// line count NL is then a compile-time constant) or consecutive butterflies of one line (row tiles, lde == 1),
// which keeps shared-memory accesses unit-stride.  The radix of every pass is dispatched once per pass to a
// compile-time kernel body; no integer division is executed per butterfly.
// tw: global table W_n^k, k = 0..n-1 (storage precision).  Returns the buffer that holds the result.
template <typename T, bool INV, bool LINES_FAST, int NL = 1>
__device__ typename cplx_t<T>::type *fft_lines(typename cplx_t<T>::type *buf0, typename cplx_t<T>::type *buf1,
                                               int nlines, int ldl, int lde, const FFTPlan &p,
                                               const typename cplx_t<T>::type *__restrict__ tw) {
    typedef typename cplx_t<T>::type C;
    C *src = buf0, *dst = buf1;
    const int n = p.n;
    int Ns = 1;
    for (int ps = 0; ps < p.nrad; ++ps) {
        const int R = p.rad[ps];
        switch (R) {
        case 4: fft_pass<T, INV, LINES_FAST, NL, 4>(src, dst, nlines, ldl, lde, n, Ns, p.ns[ps], p.nb[ps], tw); break;
        case 2: fft_pass<T, INV, LINES_FAST, NL, 2>(src, dst, nlines, ldl, lde, n, Ns, p.ns[ps], p.nb[ps], tw); break;
        case 3: fft_pass<T, INV, LINES_FAST, NL, 3>(src, dst, nlines, ldl, lde, n, Ns, p.ns[ps], p.nb[ps], tw); break;
        default: fft_pass<T, INV, LINES_FAST, NL, 5>(src, dst, nlines, ldl, lde, n, Ns, p.ns[ps], p.nb[ps], tw); break;
        }
        __syncthreads();
        C *t = src; src = dst; dst = t;
        Ns *= R;
    }
    return src;
}

// Host helper: radix plan for n = 2^a 3^b 5^c (radix 4 first, then 2, 3, 5). Returns false otherwise.
inline bool make_fft_plan(int n, FFTPlan &p) {
    p.n = n; p.nrad = 0;
    if (n < 1) return false;
    int m = n;
    while (m % 4 == 0 && p.nrad < 16) { p.rad[p.nrad++] = 4; m /= 4; }
    while (m % 2 == 0 && p.nrad < 16) { p.rad[p.nrad++] = 2; m /= 2; }
    while (m % 3 == 0 && p.nrad < 16) { p.rad[p.nrad++] = 3; m /= 3; }
    while (m % 5 == 0 && p.nrad < 16) { p.rad[p.nrad++] = 5; m /= 5; }
    int Ns = 1;
    for (int ps = 0; ps < p.nrad; ++ps) {
        p.ns[ps] = make_fastdiv((unsigned)Ns);
        p.nb[ps] = make_fastdiv((unsigned)(n / p.rad[ps]));
        Ns *= p.rad[ps];
    }
    return m == 1;
}

}  // namespace dfdm
