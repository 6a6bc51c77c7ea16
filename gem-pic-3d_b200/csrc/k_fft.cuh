// Hand-written batched FFT of lengths 4..512 that are powers of two or three times a power of two (24..384), on lines
// held in shared memory.
//
// Algorithm: self-sorting Stockham, decimation in time. A length-N transform is a sequence of passes
// with radices R (the product of the radices of the earlier passes is L, m = N / (L R)); butterfly
// b = j L + k of a pass reads x[(q m + j) L + k], q < R, multiplies by exp(-2 pi i q k / (L R)), takes the
// length-R DFT and writes y[(j R + r) L + k], r < R. The passes here are one radix-2 or radix-4 pass
// (when log2 N is not a multiple of 3; it comes first, where the twiddles are all 1) followed by radix-8
// passes. A length 3 * 2^k takes a radix-3 pass first, then a radix-2 pass when k is odd, then radix-4 passes.
// Every thread owns E values of a line in registers during a pass (min(N, 8) for a power of two, 12 for three times
// one); a line is worked by N / E threads. The pass reads its inputs, synchronises the CTA, writes its outputs and
// synchronises again, so a line is transformed in place.
//
// The forward transform has the sign -1 and is unnormalised; the inverse is taken as
// conj(forward(conj(x))) by the callers, who also apply the 1/N factors (the reference's convention,
// src/fftmany.hpp:39-119: forward sign -1, inverse normalised).
#pragma once
#include "g3d_common.cuh"

namespace g3d {

constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }
constexpr bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
// the transform lengths of the library: powers of two in 4..512, three times a power of two in 24..384
constexpr bool fft_length_ok(int n) { return (is_pow2(n) && n >= 4 && n <= 512) || (n % 3 == 0 && is_pow2(n / 3) && n >= 24 && n <= 384); }

template <int N>
struct FftShape {
    static_assert(fft_length_ok(N), "FFT length must be a power of two in 4..512 or three times one in 24..384");
    static constexpr bool P3 = !is_pow2(N);                 // a radix-3 pass first
    static constexpr int B = P3 ? N / 3 : N;                // the power-of-two part
    static constexpr int LOG = ilog2(B);
    static constexpr int E = P3 ? 12 : (N < 8 ? N : 8);     // values per thread
    static constexpr int T = N / E;                         // threads per line
    static constexpr int REM = P3 ? ((LOG & 1) ? 2 : 1) : (N < 8 ? N : (1 << (LOG % 3)));   // radix of the next pass (1: none)
    static constexpr int NR8 = P3 ? 0 : (N < 8 ? 0 : LOG / 3);   // radix-8 passes (powers of two)
    static constexpr int NR4 = P3 ? LOG / 2 : 0;                 // radix-4 passes (three times a power of two)
};

// ---------------------------------------------------------------- small DFTs (forward, sign -1)
// Generic over the complex type T (double2: the FP64 form; float2: the FP32 transforms of the mixed form).
template <class T>
__device__ __forceinline__ void dft2(T* v) {
    const T a = v[0], b = v[1];
    v[0] = a + b; v[1] = a - b;
}
// length 3: with w = exp(-2 pi i / 3) = -1/2 - i sqrt(3)/2, y1,2 = a - (b + c)/2 -+ i (sqrt(3)/2) (b - c)
template <class T>
__device__ __forceinline__ void dft3(T* v) {
    typedef typename RealOf<T>::type Re;
    const Re h = Re(0.86602540378443864676);                 // sqrt(3) / 2
    const T s = v[1] + v[2], d = v[1] - v[2];
    const T m = mk<T>(v[0].x - Re(0.5) * s.x, v[0].y - Re(0.5) * s.y);
    const T r = mk<T>(h * d.y, -h * d.x);                    // -i (sqrt(3)/2) (b - c)
    v[0] = v[0] + s; v[1] = m + r; v[2] = m - r;
}
template <class T>
__device__ __forceinline__ void dft4(T* v) {
    const T s02 = v[0] + v[2], d02 = v[0] - v[2], s13 = v[1] + v[3], d13 = mul_mi(v[1] - v[3]);
    v[0] = s02 + s13; v[1] = d02 + d13; v[2] = s02 - s13; v[3] = d02 - d13;
}
template <class T>
__device__ __forceinline__ void dft8(T* v) {
    // even / odd split into two DFT4, combined with the eighth roots of unity
    typedef typename RealOf<T>::type Re;
    const Re r = Re(0.70710678118654752440);
    const T a0 = v[0] + v[4], a1 = v[0] - v[4], a2 = v[2] + v[6], a3 = mul_mi(v[2] - v[6]);
    const T a4 = v[1] + v[5], a5 = v[1] - v[5], a6 = v[3] + v[7], a7 = mul_mi(v[3] - v[7]);
    const T b0 = a0 + a2, b2 = a0 - a2, b1 = a1 + a3, b3 = a1 - a3;
    const T c0 = a4 + a6, c2 = a4 - a6, c1 = a5 + a7, c3 = a5 - a7;
    const T w1 = mk<T>(r * (c1.x + c1.y), r * (c1.y - c1.x));        // exp(-i pi/4) c1
    const T w2 = mul_mi(c2);                                          // -i c2
    const T w3 = mk<T>(r * (c3.y - c3.x), -r * (c3.x + c3.y));       // exp(-3i pi/4) c3
    v[0] = b0 + c0; v[4] = b0 - c0;
    v[1] = b1 + w1; v[5] = b1 - w1;
    v[2] = b2 + w2; v[6] = b2 - w2;
    v[3] = b3 + w3; v[7] = b3 - w3;
}
template <int R, class T>
__device__ __forceinline__ void dft(T* v) {
    if constexpr (R == 2) dft2(v);
    else if constexpr (R == 3) dft3(v);
    else if constexpr (R == 4) dft4(v);
    else dft8(v);
}

// One Stockham pass of radix R over a line. `A(p)` maps the position p of the line to its shared
// memory index; `t` is the thread's index among the T threads of the line; tw[s] = exp(-2 pi i s / N).
template <int N, int R, class Addr, class T>
__device__ __forceinline__ void fft_pass(T* sm, const Addr& A, int t, int L, const T* __restrict__ tw) {
    constexpr int E = FftShape<N>::E, TT = FftShape<N>::T, BPT = E / R;
    const int m = N / (L * R);
    T v[E];
#pragma unroll
    for (int u = 0; u < BPT; ++u) {
        const int b = t + u * TT, j = b / L, k = b - j * L;
#pragma unroll
        for (int q = 0; q < R; ++q) v[u * R + q] = sm[A((q * m + j) * L + k)];
        if (L > 1) {
#pragma unroll
            for (int q = 1; q < R; ++q) v[u * R + q] = v[u * R + q] * __ldg(&tw[q * k * m]);
        }
        dft<R>(&v[u * R]);
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < BPT; ++u) {
        const int b = t + u * TT, j = b / L, k = b - j * L;
#pragma unroll
        for (int r = 0; r < R; ++r) sm[A((j * R + r) * L + k)] = v[u * R + r];
    }
    __syncthreads();
}

// The whole forward transform of one line in shared memory (every thread of the CTA must call it
// the same number of times: the passes synchronise the CTA).
template <int N, class Addr, class T>
__device__ __forceinline__ void fft_line(T* sm, const Addr& A, int t, const T* __restrict__ tw) {
    using S = FftShape<N>;
    int L = 1;
    if constexpr (S::P3) { fft_pass<N, 3>(sm, A, t, L, tw); L *= 3; }
    if constexpr (S::REM > 1) { fft_pass<N, S::REM>(sm, A, t, L, tw); L *= S::REM; }
#pragma unroll
    for (int s = 0; s < S::NR4; ++s) { fft_pass<N, 4>(sm, A, t, L, tw); L *= 4; }
#pragma unroll
    for (int s = 0; s < S::NR8; ++s) { fft_pass<N, 8>(sm, A, t, L, tw); L *= 8; }
}

// NL lines of the same shape (one addressing A, bases sm[0..NL)) transformed together: per butterfly the twiddle
// is loaded once for all of them, the CTA synchronises once per pass for all of them, and the lines' loads and
// DFTs interleave. Each line gets the same operations as from fft_line.
template <int N, int R, int NL, class Addr, class T>
__device__ __forceinline__ void fft_pass_multi(T* const* sm, const Addr& A, int t, int L, const T* __restrict__ tw) {
    constexpr int E = FftShape<N>::E, TT = FftShape<N>::T, BPT = E / R;
    const int m = N / (L * R);
    T v[NL][E];
#pragma unroll
    for (int u = 0; u < BPT; ++u) {
        const int b = t + u * TT, j = b / L, k = b - j * L;
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const int a = A((q * m + j) * L + k);
#pragma unroll
            for (int l = 0; l < NL; ++l) v[l][u * R + q] = sm[l][a];
        }
        if (L > 1) {
#pragma unroll
            for (int q = 1; q < R; ++q) {
                const T w = __ldg(&tw[q * k * m]);
#pragma unroll
                for (int l = 0; l < NL; ++l) v[l][u * R + q] = v[l][u * R + q] * w;
            }
        }
#pragma unroll
        for (int l = 0; l < NL; ++l) dft<R>(&v[l][u * R]);
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < BPT; ++u) {
        const int b = t + u * TT, j = b / L, k = b - j * L;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int a = A((j * R + r) * L + k);
#pragma unroll
            for (int l = 0; l < NL; ++l) sm[l][a] = v[l][u * R + r];
        }
    }
    __syncthreads();
}
template <int N, int NL, class Addr, class T>
__device__ __forceinline__ void fft_lines(T* const* sm, const Addr& A, int t, const T* __restrict__ tw) {
    using S = FftShape<N>;
    int L = 1;
    if constexpr (S::P3) { fft_pass_multi<N, 3, NL>(sm, A, t, L, tw); L *= 3; }
    if constexpr (S::REM > 1) { fft_pass_multi<N, S::REM, NL>(sm, A, t, L, tw); L *= S::REM; }
#pragma unroll
    for (int s = 0; s < S::NR4; ++s) { fft_pass_multi<N, 4, NL>(sm, A, t, L, tw); L *= 4; }
#pragma unroll
    for (int s = 0; s < S::NR8; ++s) { fft_pass_multi<N, 8, NL>(sm, A, t, L, tw); L *= 8; }
}

// The same transform in a CTA that has more threads than it needs: only the threads with act (t < FftShape<N>::T
// per line set) load, compute and store; every thread of the CTA takes part in the barriers. For kernels with one
// thread per mode of a column around the transform.
template <int N, int R, int NL, class Addr, class T>
__device__ __forceinline__ void fft_pass_multi_some(T* const* sm, const Addr& A, int t, int L, const T* __restrict__ tw, bool act) {
    constexpr int E = FftShape<N>::E, TT = FftShape<N>::T, BPT = E / R;
    const int m = N / (L * R);
    T v[NL][E];
    if (act) {
#pragma unroll
        for (int u = 0; u < BPT; ++u) {
            const int b = t + u * TT, j = b / L, k = b - j * L;
#pragma unroll
            for (int q = 0; q < R; ++q) {
                const int a = A((q * m + j) * L + k);
#pragma unroll
                for (int l = 0; l < NL; ++l) v[l][u * R + q] = sm[l][a];
            }
            if (L > 1) {
#pragma unroll
                for (int q = 1; q < R; ++q) {
                    const T w = __ldg(&tw[q * k * m]);
#pragma unroll
                    for (int l = 0; l < NL; ++l) v[l][u * R + q] = v[l][u * R + q] * w;
                }
            }
#pragma unroll
            for (int l = 0; l < NL; ++l) dft<R>(&v[l][u * R]);
        }
    }
    __syncthreads();
    if (act) {
#pragma unroll
        for (int u = 0; u < BPT; ++u) {
            const int b = t + u * TT, j = b / L, k = b - j * L;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int a = A((j * R + r) * L + k);
#pragma unroll
                for (int l = 0; l < NL; ++l) sm[l][a] = v[l][u * R + r];
            }
        }
    }
    __syncthreads();
}
template <int N, int NL, class Addr, class T>
__device__ __forceinline__ void fft_lines_some(T* const* sm, const Addr& A, int t, const T* __restrict__ tw, bool act) {
    using S = FftShape<N>;
    int L = 1;
    if constexpr (S::P3) { fft_pass_multi_some<N, 3, NL>(sm, A, t, L, tw, act); L *= 3; }
    if constexpr (S::REM > 1) { fft_pass_multi_some<N, S::REM, NL>(sm, A, t, L, tw, act); L *= S::REM; }
#pragma unroll
    for (int s = 0; s < S::NR4; ++s) { fft_pass_multi_some<N, 4, NL>(sm, A, t, L, tw, act); L *= 4; }
#pragma unroll
    for (int s = 0; s < S::NR8; ++s) { fft_pass_multi_some<N, 8, NL>(sm, A, t, L, tw, act); L *= 8; }
}

// Shared-memory addressing of a row line: one padding slot per 8 values keeps the strided
// Stockham accesses free of bank conflicts.
struct RowAddr {
    int base;
    __device__ __forceinline__ int operator()(int p) const { return base + p + (p >> 3); }
};
template <int N>
constexpr int row_stride() { return N + N / 8 + 1; }
// Shared-memory layout of a tile of CW columns: column c stored contiguously at c * RS with the padding of a row,
// so that the transforms along y (RowAddr{c * RS}) read it without bank conflicts (a tile stored row-major puts a
// column's values CW elements apart: 2- to 8-way conflicts on every pass).
template <int N, int CW>
struct ColTile {
    static constexpr int RS = row_stride<N>();
    static constexpr int size = CW * RS;           // elements per array of the tile
    __device__ static __forceinline__ int at(int p, int c) { return c * RS + p + (p >> 3); }
};
}  // namespace g3d
