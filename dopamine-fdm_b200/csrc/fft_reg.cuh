// fft_reg.cuh -- two-level FFTs with register codelets for the common transform lengths (8 ... 256, factors 2
// and 3); other lengths use the Stockham path of fft_smem.cuh.
//
// A length-N transform, N = N1 * N2, is split (Cooley-Tukey, n = n1*N2 + n2, k = k1 + N1*k2) as
//   step 1: for every n2, Y[k1][n2] = W_N^(n2*k1) * sum_n1 x[n1*N2 + n2] W_N1^(n1*k1)       (length-N1 DFT)
//   step 2: for every k1, X[k1 + N1*k2] = sum_n2 Y[k1][n2] W_N2^(n2*k2)                       (length-N2 DFT)
// Each DFT runs in registers with compile-time roots; between the steps the data crosses shared memory once.
// The callers feed step 1 straight from global memory and write step 2 straight to global memory where the
// access pattern allows it.  Conventions as the Stockham path: forward exp(-2 pi i jk/N), unnormalised.
#pragma once

#include "fft_smem.cuh"

namespace dfdm {

// cos(2 pi m / 48) for the roots of every codelet size used here (16 | 48 and 12 | 48), exact decimal values.
__host__ __device__ constexpr double cos48_first(int m) {   // 0 <= m <= 12
    return m == 0 ? 1.0
         : m == 1 ? 0.99144486137381041114    // cos(pi/24)
         : m == 2 ? 0.96592582628906828675    // cos(pi/12)
         : m == 3 ? 0.92387953251128675613    // cos(pi/8)
         : m == 4 ? 0.86602540378443864676    // cos(pi/6)
         : m == 5 ? 0.79335334029123516458    // cos(5pi/24)
         : m == 6 ? 0.70710678118654752440    // cos(pi/4)
         : m == 7 ? 0.60876142900872063942    // cos(7pi/24)
         : m == 8 ? 0.5
         : m == 9 ? 0.38268343236508977173    // cos(3pi/8)
         : m == 10 ? 0.25881904510252076235   // cos(5pi/12)
         : m == 11 ? 0.13052619222005159155   // cos(11pi/24)
         : 0.0;
}
__host__ __device__ constexpr double cos48_norm(int m) {   // 0 <= m < 48
    return m > 24 ? cos48_norm(48 - m) : (m > 12 ? -cos48_first(24 - m) : cos48_first(m));
}
__host__ __device__ constexpr double cos48(int m) { return cos48_norm(((m % 48) + 48) % 48); }
__host__ __device__ constexpr double sin48(int m) { return cos48(12 - m); }

// x * exp(-+2 pi i m / S) (forward sign unless INV) for a compile-time-known m; quarter turns cost no multiply.
template <typename T, bool INV, int S, typename C> __device__ __forceinline__ C rot(C x, int m) {
    m = ((m % S) + S) % S;
    if (m == 0) return x;
    if (4 * m == S) return mul_mi<INV>(x);
    if (2 * m == S) { C r; r.x = -x.x; r.y = -x.y; return r; }
    if (4 * m == 3 * S) return mul_mi<!INV>(x);
    const int q = m * (48 / S);
    C w;
    w.x = (T)cos48(q);
    w.y = INV ? (T)sin48(q) : (T)(-sin48(q));
    return cmul(x, w);
}

// In-register DFT of size S in {2, 3, 4, 5, 6, 8, 12, 16}; sizes above 5 are split S = A * B (A = 4, or 2 for 6)
// with the same Cooley-Tukey map as the two-level transform.
template <typename T, bool INV, int S> struct Codelet {
    typedef typename cplx_t<T>::type C;
    static __device__ __forceinline__ void run(C *v) {
        if constexpr (S <= 5) {
            dft_small<T, INV>(v, S);
        } else {
            constexpr int A = (S % 4 == 0) ? 4 : 2;
            constexpr int B = S / A;
            C t[S];
#pragma unroll
            for (int b = 0; b < B; ++b) {
                C x[A];
#pragma unroll
                for (int a = 0; a < A; ++a) x[a] = v[a * B + b];
                dft_small<T, INV>(x, A);
#pragma unroll
                for (int a = 0; a < A; ++a) t[a * B + b] = rot<T, INV, S>(x[a], a * b);
            }
#pragma unroll
            for (int a = 0; a < A; ++a) {
                C y[B];
#pragma unroll
                for (int b = 0; b < B; ++b) y[b] = t[a * B + b];
                Codelet<T, INV, B>::run(y);
#pragma unroll
                for (int b = 0; b < B; ++b) v[a + A * b] = y[b];
            }
        }
    }
};

// Factorisation N = N1 * N2 of the lengths handled by the two-level path (N2 = 8 or 16 where possible, which keeps
// the padded shared-memory accesses of step 2 free of bank conflicts).
template <int N> struct Split;
template <> struct Split<8> { static constexpr int N1 = 2, N2 = 4; };
template <> struct Split<16> { static constexpr int N1 = 4, N2 = 4; };
template <> struct Split<24> { static constexpr int N1 = 3, N2 = 8; };
template <> struct Split<32> { static constexpr int N1 = 4, N2 = 8; };
template <> struct Split<48> { static constexpr int N1 = 6, N2 = 8; };
template <> struct Split<64> { static constexpr int N1 = 8, N2 = 8; };
template <> struct Split<96> { static constexpr int N1 = 12, N2 = 8; };
template <> struct Split<128> { static constexpr int N1 = 16, N2 = 8; };
template <> struct Split<192> { static constexpr int N1 = 12, N2 = 16; };
template <> struct Split<256> { static constexpr int N1 = 16, N2 = 16; };

// Calls f(std::integral_constant<int, N>{}) when N has a two-level split; returns false otherwise.
template <typename F> inline bool with_fft2l(int n, F &&f) {
    switch (n) {
    case 8: f(std::integral_constant<int, 8>{}); return true;
    case 16: f(std::integral_constant<int, 16>{}); return true;
    case 24: f(std::integral_constant<int, 24>{}); return true;
    case 32: f(std::integral_constant<int, 32>{}); return true;
    case 48: f(std::integral_constant<int, 48>{}); return true;
    case 64: f(std::integral_constant<int, 64>{}); return true;
    case 96: f(std::integral_constant<int, 96>{}); return true;
    case 128: f(std::integral_constant<int, 128>{}); return true;
    case 192: f(std::integral_constant<int, 192>{}); return true;
    case 256: f(std::integral_constant<int, 256>{}); return true;
    }
    return false;
}

// Shared-memory row layouts of the row transforms (x lines), in complex elements:
//   LDA: stride of natural-order lines (padded to 8 mod 16 so two lines in one half-warp use disjoint banks)
//   LDT: stride of the step-1 output lines, element k1*N2 + n2 at k1*(N2+1) + n2
template <int N> struct RowLayout {
    static constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
    static constexpr int pad8(int x) { return x + ((8 - (x % 16) + 16) % 16); }
    static constexpr int LDA = pad8(N);
    static constexpr int LDT = pad8(N1 * (N2 + 1));
};

// x lines per block of the row transforms: as many as fit in 56 KB of shared memory (4 blocks of 256 threads per SM)
template <typename T, int N> struct RowLines {
    static constexpr int bytes = (RowLayout<N>::LDA + RowLayout<N>::LDT) * 2 * (int)sizeof(T);
    static constexpr int value = (57344 / bytes) < 1 ? 1 : ((57344 / bytes) > 64 ? 64 : (57344 / bytes));
};

// Step 1 of a row transform for one (line, n2) item: v holds x[n1*N2 + n2], n1 = 0..N1-1, on entry; the twiddled
// step-1 outputs go to t (layout LDT).
template <typename T, bool INV, int N>
__device__ __forceinline__ void row_step1(typename cplx_t<T>::type *v, typename cplx_t<T>::type *tl, int n2,
                                          const typename cplx_t<T>::type *__restrict__ tw) {
    typedef typename cplx_t<T>::type C;
    constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
    Codelet<T, INV, N1>::run(v);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
        C x = v[k1];
        if (k1 != 0 && n2 != 0) {
            C w = __ldg(tw + n2 * k1);
            x = INV ? cmulc(x, w) : cmul(x, w);
        }
        tl[k1 * (N2 + 1) + n2] = x;
    }
}

// Column transform step 1 / step 2 for tiles of NL columns, element e of column c at [e*NL + c].
template <typename T, bool INV, int N, int NL>
__device__ __forceinline__ void col_step1(typename cplx_t<T>::type *v, typename cplx_t<T>::type *t, int c, int n2,
                                          const typename cplx_t<T>::type *__restrict__ tw) {
    typedef typename cplx_t<T>::type C;
    constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
    Codelet<T, INV, N1>::run(v);
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
        C x = v[k1];
        if (k1 != 0 && n2 != 0) {
            C w = __ldg(tw + n2 * k1);
            x = INV ? cmulc(x, w) : cmul(x, w);
        }
        t[(k1 * N2 + n2) * NL + c] = x;
    }
}

}  // namespace dfdm
