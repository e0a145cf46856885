// ld_fftx.cuh — Stockham FFT of a compile-time length and radix order.
//
// The same in-place Stockham stages as ld_fft.cuh (C interleaved sequences,
// s[idx * C + col], every thread's butterflies loaded before the CTA
// synchronises and written back after), but with the length, the radix of
// every stage, the stage's span NS and the thread count T all known at
// compile time:
//   * a butterfly's input addresses are b + r * (N / R) * C: one base and
//     immediate offsets, no per-element index arithmetic;
//   * its output addresses are one base and immediate offsets r * NS * C;
//   * (b / C) % NS divides by constants;
//   * the twiddles w^r (r < R) of butterfly k come from a per-stage table
//     of pairs (w^2q, w^(2q+1)) laid out [q][k] (q < RP / 2, RP = R rounded
//     up to even), read as R/2 16-byte loads that the threads of a warp
//     (consecutive k) make to consecutive addresses, instead of a serial
//     chain of R - 2 complex products.
// The stage tables are generated in FP64 on the host (fx_stage_table in
// ld_frame_fx.cu) and stored after one another for the stages after the
// first (the first stage's twiddles are all 1).
#pragma once

#include "ld_fft.cuh"

namespace ld {

template <int R>
struct FxPad {
    static constexpr int value = (R + 1) & ~1;
};

// One stage of radix R over span NS for C sequences of length N, T threads.
template <int N, int C, int T, bool INV, int R, int NS>
__device__ __forceinline__ void fx_stage(float2* s, const float2* __restrict__ stw) {
    constexpr int M = N / R;      // butterflies per sequence
    constexpr int NB = M * C;     // butterflies of the CTA
    constexpr int IT = (NB + T - 1) / T;
    constexpr int RP = FxPad<R>::value;
    const int tid = static_cast<int>(threadIdx.x);
    float2 v[IT][R];
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int b = tid + it * T;
        if ((it + 1) * T <= NB || b < NB) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[it][r] = s[b + r * NB];
        }
    }
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int b = tid + it * T;
        if ((it + 1) * T <= NB || b < NB) {
            if constexpr (NS > 1) {
                const int k = (b / C) % NS;
                const float4* t = reinterpret_cast<const float4*>(stw) + k;
#pragma unroll
                for (int q = 0; q < RP / 2; ++q) {
                    const float4 w = __ldg(t + q * NS);
                    if (2 * q >= 1 && 2 * q < R) {
                        const float2 w0 = make_float2(w.x, w.y);
                        v[it][2 * q] = INV ? cmulc(v[it][2 * q], w0) : cmul(v[it][2 * q], w0);
                    }
                    if (2 * q + 1 < R) {
                        const float2 w1 = make_float2(w.z, w.w);
                        v[it][2 * q + 1] = INV ? cmulc(v[it][2 * q + 1], w1) : cmul(v[it][2 * q + 1], w1);
                    }
                }
            }
            dft<R, INV>(v[it]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int b = tid + it * T;
        if ((it + 1) * T <= NB || b < NB) {
            const int j = b / C;
            const int col = b - j * C;
            const int k = j % NS;
            const int base = ((j - k) * R + k) * C + col;
#pragma unroll
            for (int r = 0; r < R; ++r) s[base + r * NS * C] = v[it][r];
        }
    }
    __syncthreads();
}

template <int N, int C, int T, bool INV, int NS, int R, int... Rest>
__device__ __forceinline__ void fx_stages(float2* s, const float2* stw) {
    fx_stage<N, C, T, INV, R, NS>(s, stw);
    if constexpr (sizeof...(Rest) > 0) fx_stages<N, C, T, INV, NS * R, Rest...>(s, NS > 1 ? stw + NS * FxPad<R>::value : stw);
}

// A transform of length N with the radix order Rs... (first stage first).
// run<C, INV, T>(s, stw): in place over C interleaved sequences in shared
// memory with T threads; the caller's fill ends with __syncthreads(), the
// transform ends with one.
template <int N, int... Rs>
struct FixedFft {
    static constexpr int n = N;
    static_assert((1 * ... * Rs) == N, "radix order does not multiply to the length");
    template <int C, bool INV, int T>
    static __device__ __forceinline__ void run(const FftPlan& plan, float2* s) {
        fx_stages<N, C, T, INV, 1, Rs...>(s, plan.stw);
    }
};

// The runtime-planned transform of ld_fft.cuh behind the same interface.
template <int E>
struct GenericFft {
    static constexpr int n = 0;
    template <int C, bool INV, int T>
    static __device__ __forceinline__ void run(const FftPlan& plan, float2* s) {
        fft_run<E, C, INV>(plan, s);
    }
};

}  // namespace ld
