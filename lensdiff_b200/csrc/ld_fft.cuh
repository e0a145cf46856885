// ld_fft.cuh — mixed-radix Stockham FFT building blocks for sm_100a.
//
// One CTA transforms C interleaved sequences of length n held in shared
// memory as s[index * C + column].  A stage of radix R lets every thread take
// ceil(n*C / (R*T)) butterflies into registers (all loads issued before any
// math), then writes them back in place after a barrier, so one n*C buffer
// suffices.  Kernels fuse their producers and consumers into the fill and
// drain of that buffer (pupil generation, highlight extraction, zero padding,
// spectral multiply, |.|^2, cropping, compositing), never into HBM passes.
// Twiddles come from a table tw[k] = exp(-2*pi*i*k/n) generated in FP64 on the
// host and stored as float2.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ld {

constexpr int kMaxStages = 16;

// A plan is passed by value and lives in registers: the stage radices are
// packed four bits each into `codes` (stage s uses (codes >> 4s) & 15), so no
// stage loop indexes an array in local memory.
struct FftPlan {
    int n;
    int nstages;
    unsigned long long codes;
    const float2* tw;  // n entries, exp(-2 pi i k / n)
};

__host__ __device__ inline int plan_radix(const FftPlan& p, int stage) {
    return static_cast<int>((p.codes >> (4 * stage)) & 15ull);
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
    const float kS = 0.86602540378443864676f;  // sin(2 pi / 3)
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
    const float c1 = 0.30901699437494742410f;   // cos(2 pi / 5)
    const float c2 = -0.80901699437494742410f;  // cos(4 pi / 5)
    const float s1 = 0.95105651629515357212f;   // sin(2 pi / 5)
    const float s2 = 0.58778525229247312917f;   // sin(4 pi / 5)
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
    const float kR = 0.70710678118654752440f;
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

template <int R, bool INV>
__device__ __forceinline__ void dft(float2* v) {
    if constexpr (R == 2) dft2<INV>(v);
    else if constexpr (R == 3) dft3<INV>(v);
    else if constexpr (R == 4) dft4<INV>(v);
    else if constexpr (R == 5) dft5<INV>(v);
    else dft8<INV>(v);
}

// ---- one Stockham stage ------------------------------------------------------
// Reads x[j + r*n/R] (j < n/R), twiddles by tw[(j % ns) * r * n/(ns*R)],
// applies the radix-R DFT and writes y[(j/ns)*ns*R + j%ns + r*ns].
// `load(idx, col)` and `store(idx, col, v)` address sequence element idx of
// interleaved column col.
template <int R, int T, int C, int NMAX, bool INV, class Load, class Store>
__device__ __forceinline__ void fft_stage(int n, int ns, const float2* __restrict__ tw, Load load,
                                          Store store) {
    constexpr int MAXJ = (NMAX / R * C + T - 1) / T;
    const int m = n / R;
    const int nb = m * C;
    const int stride = n / (ns * R);
    float2 v[MAXJ][R];
#pragma unroll
    for (int it = 0; it < MAXJ; ++it) {
        const int b = threadIdx.x + it * T;
        if (b < nb) {
            const int col = b % C;
            const int j = b / C;
#pragma unroll
            for (int r = 0; r < R; ++r) v[it][r] = load(j + r * m, col);
        }
    }
#pragma unroll
    for (int it = 0; it < MAXJ; ++it) {
        const int b = threadIdx.x + it * T;
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
        const int b = threadIdx.x + it * T;
        if (b < nb) {
            const int col = b % C;
            const int j = b / C;
            const int k = j % ns;
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) store(base + r * ns, col, v[it][r]);
        }
    }
    __syncthreads();
}

// Shared-memory accessors for s[idx * C + col].
template <int C>
struct SmemLoad {
    const float2* s;
    __device__ __forceinline__ float2 operator()(int idx, int col) const { return s[idx * C + col]; }
};
template <int C>
struct SmemStore {
    float2* s;
    __device__ __forceinline__ void operator()(int idx, int col, float2 v) const { s[idx * C + col] = v; }
};

// One radix per non-inlined function: inlined into the stage loop (or into a
// common switch), the loop-invariant address arithmetic of all five radix
// bodies is hoisted and stays live together, doubling the register need.
template <int R, int T, int C, int NMAX, bool INV>
__device__ __noinline__ void fft_stage_r(int n, int ns, const float2* tw, float2* s) {
    fft_stage<R, T, C, NMAX, INV>(n, ns, tw, SmemLoad<C>{s}, SmemStore<C>{s});
}

template <int T, int C, int NMAX, bool INV>
__device__ __forceinline__ void fft_stage_any(int radix, int n, int ns, const float2* tw, float2* s) {
    switch (radix) {
        case 8: fft_stage_r<8, T, C, NMAX, INV>(n, ns, tw, s); break;
        case 4: fft_stage_r<4, T, C, NMAX, INV>(n, ns, tw, s); break;
        case 5: fft_stage_r<5, T, C, NMAX, INV>(n, ns, tw, s); break;
        case 3: fft_stage_r<3, T, C, NMAX, INV>(n, ns, tw, s); break;
        default: fft_stage_r<2, T, C, NMAX, INV>(n, ns, tw, s); break;
    }
}

// In-place transform of C interleaved sequences held in shared memory
// s[idx * C + col] (n * C float2).  Callers fill `s` (fusing whatever produces
// the input: pupil generation, highlight extraction, zero padding, spectral
// multiply) and drain it (fusing |.|^2, windowing, cropping, compositing), so
// no intermediate goes back to HBM.  The fill must end with __syncthreads()
// (smem_fill does); the transform ends with one.
template <int T, int C, int NMAX, bool INV>
__device__ __forceinline__ void fft_run(const FftPlan plan, float2* s) {
    int ns = 1;
    unsigned long long codes = plan.codes;
    for (int st = 0; st < plan.nstages; ++st) {
        const int r = static_cast<int>(codes & 15ull);
        codes >>= 4;
        fft_stage_any<T, C, NMAX, INV>(r, plan.n, ns, plan.tw, s);
        ns *= r;
    }
}

// Fills all n*C entries: s[idx*C + col] = fn(idx, col).
template <int T, int C, class Fn>
__device__ __forceinline__ void smem_fill(float2* s, int n, Fn fn) {
    for (int i = threadIdx.x; i < n * C; i += T) s[i] = fn(i / C, i % C);
    __syncthreads();
}

}  // namespace ld
