// ld_fft.cuh — mixed-radix Stockham FFT building blocks for sm_100a.
//
// One CTA transforms C interleaved sequences of length n held in shared
// memory as s[index * C + column].  Every stage is in place: each thread takes
// its butterflies into registers (all loads issued before any math), the CTA
// synchronises, and the results are written back, so one n*C buffer suffices
// and the whole working set passes through the register file once per stage.
//
// Radices 2, 3, 4, 5, 8, and the composites 16 (4x4) and 25 (5x5), which do
// two radix layers per shared-memory pass: the 5-smooth grids the frame chain
// uses (3200 = 25*16*8, 2500 = 25*25*4, 1600 = 25*16*4, 2048 = 16*16*8) take
// three passes instead of five.
//
// Work split: the kernel is launched with T threads such that T * E >= n * C
// (E = elements per thread, a template parameter of the family), so a radix-R
// stage gives each thread at most ceil(E / R) butterflies.  Two families:
//   E = 25: n * C <= 12800, T <= 512, registers <= 128, every radix;
//   E = 16: n * C <= 16384, T <= 1024, registers <= 64, no radix 25 (the
//           host's planner leaves it out of plans for this family).
// Kernels fill the buffer from their producer (pupil generation, highlight
// extraction, zero padding, spectral multiply) and drain it into their
// consumer (|.|^2 windows, cropping, compositing), never through extra HBM
// passes.  Twiddles come from a table tw[k] = exp(-2 pi i k / n) generated in
// FP64 on the host and stored as float2.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ld {

constexpr int kMaxStages = 12;

// Elements-per-thread families (see the header comment).
constexpr int kE25 = 25;
constexpr int kE16 = 16;
constexpr int kE25MaxThreads = 512;
constexpr int kE16MaxThreads = 1024;

// Stages run grouped by radix in the fixed order 25, 5, 3, 16, 8, 4, 2 (odd
// radices first: their strided first-stage stores hit distinct shared-memory
// banks).  A plan stores how many stages of each radix it has, four bits per
// radix in that order, and is passed by value in registers.
constexpr int kPlanRadices[7] = {25, 5, 3, 16, 8, 4, 2};

struct FftPlan {
    int n;
    int nstages;
    unsigned long long codes;  // stage count of kPlanRadices[i] at bits 4i..4i+3
    const float2* tw;          // n entries, exp(-2 pi i k / n)
    // Compile-time plan (ld_fxplans.h) the launchers use for this length, 0
    // for none, and its per-stage twiddle tables (ld_fftx.cuh)
    int fixed;
    const float2* stw;
    // launch shape of the fixed plan's kernels (0: default; 1: one more CTA
    // per SM for the inverse row pass, under a tighter register cap)
    int shape;
};

__host__ __device__ inline int plan_count(const FftPlan& p, int i) {
    return static_cast<int>((p.codes >> (4 * i)) & 15ull);
}

// Values through opaque moves.  The thread index, block size and stage
// arguments are re-read in every stage, and twiddle constants are materialised
// where they are used, so the compiler cannot hoist the invariants of every
// radix body out of an enclosing loop (a persistent kernel's column loop) and
// keep them all live together.
__device__ __forceinline__ int opaque_tid() {
    int t;
    asm volatile("mov.u32 %0, %%tid.x;" : "=r"(t));
    return t;
}
__device__ __forceinline__ int opaque_ntid() {
    int t;
    asm volatile("mov.u32 %0, %%ntid.x;" : "=r"(t));
    return t;
}
__device__ __forceinline__ int opaque(int v) {
    int t;
    asm volatile("mov.b32 %0, %1;" : "=r"(t) : "r"(v));
    return t;
}
__device__ __forceinline__ unsigned long long opaque64(unsigned long long v) {
    unsigned long long t;
    asm volatile("mov.b64 %0, %1;" : "=l"(t) : "l"(v));
    return t;
}
__device__ __forceinline__ float kf(float c) {
    float t;
    asm volatile("mov.b32 %0, %1;" : "=f"(t) : "f"(c));
    return t;
}

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 rot90(float2 a) {
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// ---- small DFTs (forward: exp(-2 pi i jk/R); INV: conjugate kernel) -------
template <bool INV>
__device__ __forceinline__ void dft2(float2* v) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}

template <bool INV>
__device__ __forceinline__ void dft3(float2* v) {
    const float kS = kf(0.86602540378443864676f);  // sin(2 pi / 3)
    const float2 t1 = cadd(v[1], v[2]);
    const float2 t2 = csub(v[1], v[2]);
    const float2 y0 = cadd(v[0], t1);
    const float2 m = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
    const float2 s = rot90<INV>(cscale(t2, kS));
    v[0] = y0;
    v[1] = cadd(m, s);
    v[2] = csub(m, s);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2* v) {
    const float2 t0 = cadd(v[0], v[2]);
    const float2 t1 = csub(v[0], v[2]);
    const float2 t2 = cadd(v[1], v[3]);
    const float2 t3 = rot90<INV>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
}

template <bool INV>
__device__ __forceinline__ void dft5(float2* v) {
    const float c1 = kf(0.30901699437494742410f);   // cos(2 pi / 5)
    const float c2 = kf(-0.80901699437494742410f);  // cos(4 pi / 5)
    const float s1 = kf(0.95105651629515357212f);   // sin(2 pi / 5)
    const float s2 = kf(0.58778525229247312917f);   // sin(4 pi / 5)
    const float2 t1 = cadd(v[1], v[4]);
    const float2 t2 = cadd(v[2], v[3]);
    const float2 t3 = csub(v[1], v[4]);
    const float2 t4 = csub(v[2], v[3]);
    const float2 a0 = v[0];
    const float2 y0 = cadd(a0, cadd(t1, t2));
    const float2 m1 = make_float2(a0.x + c1 * t1.x + c2 * t2.x, a0.y + c1 * t1.y + c2 * t2.y);
    const float2 m2 = make_float2(a0.x + c2 * t1.x + c1 * t2.x, a0.y + c2 * t1.y + c1 * t2.y);
    const float2 n1 = rot90<INV>(make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
    const float2 n2 = rot90<INV>(make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
    v[0] = y0;
    v[1] = cadd(m1, n1);
    v[4] = csub(m1, n1);
    v[2] = cadd(m2, n2);
    v[3] = csub(m2, n2);
}

template <bool INV>
__device__ __forceinline__ void dft8(float2* v) {
    const float kR = kf(0.70710678118654752440f);
    float2 b[4], c[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        b[k] = cadd(v[k], v[k + 4]);
        c[k] = csub(v[k], v[k + 4]);
    }
    // c_k *= W8^k  (W8 = exp(-i pi/4) forward)
    c[1] = INV ? make_float2(kR * (c[1].x - c[1].y), kR * (c[1].x + c[1].y))
               : make_float2(kR * (c[1].x + c[1].y), kR * (c[1].y - c[1].x));
    c[2] = rot90<INV>(c[2]);
    c[3] = INV ? make_float2(-kR * (c[3].x + c[3].y), kR * (c[3].x - c[3].y))
               : make_float2(kR * (c[3].y - c[3].x), -kR * (c[3].x + c[3].y));
    dft4<INV>(b);
    dft4<INV>(c);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        v[2 * m] = b[m];
        v[2 * m + 1] = c[m];
    }
}

// cos / sin of 2 pi m / R for the composite radices (mathematical constants;
// the switch on the unrolled, compile-time m folds to one literal).
template <int R>
__device__ __forceinline__ float root_cos(int m) {
    if constexpr (R == 16) {
        switch (m & 15) {
            case 0: return 1.000000000f;
            case 1: case 15: return 0.923879533f;
            case 2: case 14: return 0.707106781f;
            case 3: case 13: return 0.382683432f;
            case 4: case 12: return 0.0f;
            case 5: case 11: return -0.382683432f;
            case 6: case 10: return -0.707106781f;
            case 7: case 9: return -0.923879533f;
            default: return -1.000000000f;
        }
    } else {
        switch (m % 25) {
            case 0: return 1.000000000f;
            case 1: case 24: return 0.968583161f;
            case 2: case 23: return 0.876306680f;
            case 3: case 22: return 0.728968627f;
            case 4: case 21: return 0.535826795f;
            case 5: case 20: return 0.309016994f;
            case 6: case 19: return 0.062790520f;
            case 7: case 18: return -0.187381315f;
            case 8: case 17: return -0.425779292f;
            case 9: case 16: return -0.637423990f;
            case 10: case 15: return -0.809016994f;
            case 11: case 14: return -0.929776486f;
            default: return -0.992114701f;
        }
    }
}
template <int R>
__device__ __forceinline__ float root_sin(int m) {
    if constexpr (R == 16) {
        switch (m & 15) {
            case 0: case 8: return 0.0f;
            case 1: case 7: return 0.382683432f;
            case 2: case 6: return 0.707106781f;
            case 3: case 5: return 0.923879533f;
            case 4: return 1.000000000f;
            case 9: case 15: return -0.382683432f;
            case 10: case 14: return -0.707106781f;
            case 11: case 13: return -0.923879533f;
            default: return -1.000000000f;
        }
    } else {
        switch (m % 25) {
            case 0: return 0.0f;
            case 1: return 0.248689887f;
            case 2: return 0.481753674f;
            case 3: return 0.684547106f;
            case 4: return 0.844327926f;
            case 5: return 0.951056516f;
            case 6: return 0.998026728f;
            case 7: return 0.982287251f;
            case 8: return 0.904827052f;
            case 9: return 0.770513243f;
            case 10: return 0.587785252f;
            case 11: return 0.368124553f;
            case 12: return 0.125333234f;
            case 13: return -0.125333234f;
            case 14: return -0.368124553f;
            case 15: return -0.587785252f;
            case 16: return -0.770513243f;
            case 17: return -0.904827052f;
            case 18: return -0.982287251f;
            case 19: return -0.998026728f;
            case 20: return -0.951056516f;
            case 21: return -0.844327926f;
            case 22: return -0.684547106f;
            case 23: return -0.481753674f;
            default: return -0.248689887f;
        }
    }
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2* v);

// Radix A*B in registers (Cooley-Tukey, r = B*r1 + r2, k = k1 + A*k2):
// DFT-A over r1 for every r2, twiddle by W_R^(r2 k1), DFT-B over r2 for
// every k1.  All indices are compile-time, so the data never leaves registers.
template <int A, int B, bool INV>
__device__ __forceinline__ void dft_composite(float2* v) {
    constexpr int R = A * B;
#pragma unroll
    for (int r2 = 0; r2 < B; ++r2) {
        float2 t[A];
#pragma unroll
        for (int r1 = 0; r1 < A; ++r1) t[r1] = v[B * r1 + r2];
        dft<A, INV>(t);
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) {
            const int e = (r2 * k1) % R;
            float2 x = t[k1];
            if (e != 0) {
                if (4 * e == R) {
                    x = rot90<INV>(x);
                } else if (2 * e == R) {
                    x = make_float2(-x.x, -x.y);
                } else {
                    const float2 w = make_float2(kf(root_cos<R>(e)), kf(-root_sin<R>(e)));
                    x = INV ? cmulc(x, w) : cmul(x, w);
                }
            }
            v[B * k1 + r2] = x;
        }
    }
    float2 o[R];
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
        float2 t[B];
#pragma unroll
        for (int r2 = 0; r2 < B; ++r2) t[r2] = v[B * k1 + r2];
        dft<B, INV>(t);
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) o[k1 + A * k2] = t[k2];
    }
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = o[r];
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2* v) {
    if constexpr (R == 2) dft2<INV>(v);
    else if constexpr (R == 3) dft3<INV>(v);
    else if constexpr (R == 4) dft4<INV>(v);
    else if constexpr (R == 5) dft5<INV>(v);
    else if constexpr (R == 8) dft8<INV>(v);
    else if constexpr (R == 16) dft_composite<4, 4, INV>(v);
    else dft_composite<5, 5, INV>(v);
}

// ---- one Stockham stage ------------------------------------------------------
// Reads x[j + r*n/R] (j < n/R), twiddles by tw[(j % ns) * r * n/(ns*R)],
// applies the radix-R DFT and writes y[(j/ns)*ns*R + j%ns + r*ns], in place.
template <int R, int E, int C, bool INV>
__device__ __forceinline__ void fft_stage(int n_in, int ns_in, const float2* __restrict__ tw, float2* s) {
    constexpr int MAXJ = (E + R - 1) / R;
    const int tid = opaque_tid();
    const int T = opaque_ntid();
    const int n = opaque(n_in);
    const int ns = opaque(ns_in);
    const int m = n / R;
    const int nb = m * C;
    const int stride = n / (ns * R);
    float2 v[MAXJ][R];
#pragma unroll
    for (int it = 0; it < MAXJ; ++it) {
        const int b = tid + it * T;
        if (b < nb) {
            const int col = b % C;
            const int j = b / C;
#pragma unroll
            for (int r = 0; r < R; ++r) v[it][r] = s[(j + r * m) * C + col];
        }
    }
#pragma unroll
    for (int it = 0; it < MAXJ; ++it) {
        const int b = tid + it * T;
        if (b < nb) {
            const int j = b / C;
            const int k = j % ns;
            if (k != 0) {
                // one table load per butterfly; w^r by repeated products
                // (relative error below r * 2^-23, far under the FP32 FFT noise)
                const float2 w1 = __ldg(&tw[k * stride]);
                float2 w = w1;
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    v[it][r] = INV ? cmulc(v[it][r], w) : cmul(v[it][r], w);
                    if (r + 1 < R) w = cmul(w, w1);
                }
            }
            dft<R, INV>(v[it]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < MAXJ; ++it) {
        const int b = tid + it * T;
        if (b < nb) {
            const int col = b % C;
            const int j = b / C;
            const int k = j % ns;
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) s[(base + r * ns) * C + col] = v[it][r];
        }
    }
    __syncthreads();
}

// All stages of one radix, in order.
template <int R, int E, int C, bool INV>
__device__ __forceinline__ void fft_stages(int count, int n, int& ns, const float2* tw, float2* s) {
#pragma unroll 1
    for (int i = 0; i < count; ++i) {
        fft_stage<R, E, C, INV>(n, ns, tw, s);
        ns *= R;
    }
}

// In-place transform of C interleaved sequences held in shared memory
// s[idx * C + col] (n * C float2).  The caller's fill must end with
// __syncthreads(); the transform ends with one.  Each radix body is inlined
// once, in its own loop: put behind one switch in a common stage loop, the
// bodies' register needs add up instead of overlapping.  Radix 25 is compiled
// only into the E >= 25 family (plans for E = 16 never contain it).
template <int E, int C, bool INV>
__device__ __forceinline__ void fft_run(const FftPlan plan, float2* s) {
    int ns = 1;
    const unsigned long long c = opaque64(plan.codes);
    const int n = plan.n;
    const float2* tw = plan.tw;
    if constexpr (E >= 25) fft_stages<25, E, C, INV>(static_cast<int>(c & 15ull), n, ns, tw, s);
    fft_stages<5, E, C, INV>(static_cast<int>((c >> 4) & 15ull), n, ns, tw, s);
    fft_stages<3, E, C, INV>(static_cast<int>((c >> 8) & 15ull), n, ns, tw, s);
    fft_stages<16, E, C, INV>(static_cast<int>((c >> 12) & 15ull), n, ns, tw, s);
    fft_stages<8, E, C, INV>(static_cast<int>((c >> 16) & 15ull), n, ns, tw, s);
    fft_stages<4, E, C, INV>(static_cast<int>((c >> 20) & 15ull), n, ns, tw, s);
    fft_stages<2, E, C, INV>(static_cast<int>((c >> 24) & 15ull), n, ns, tw, s);
}

// Fills all n*C entries: s[idx*C + col] = fn(idx, col).
template <int C, class Fn>
__device__ __forceinline__ void smem_fill(float2* s, int n, Fn fn) {
    for (int i = threadIdx.x; i < n * C; i += blockDim.x) s[i] = fn(i / C, i % C);
    __syncthreads();
}

// Threads for an n x C transform of family E, in whole warps.
__host__ __device__ constexpr int fft_threads(int n, int C, int E) {
    return ((n * C + E - 1) / E + 31) / 32 * 32;
}

// Family for an n x C transform: 25, 16, or 0 when it does not fit.
__host__ __device__ constexpr int fft_family(int n, int C) {
    return n * C <= kE25 * kE25MaxThreads ? kE25 : (n * C <= kE16 * kE16MaxThreads ? kE16 : 0);
}

}  // namespace ld
