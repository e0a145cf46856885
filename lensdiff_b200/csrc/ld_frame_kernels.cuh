// ld_frame_kernels.cuh — device kernels of the per-frame FFT convolution chain
// and of the kernel-spectrum build, shared by ld_frame.cu (runtime-planned
// transforms) and ld_frame_fx.cu (compile-time transforms of the fixed plans).
// Every FFT kernel takes its transform as the policy class FFT (ld_fftx.cuh):
// GenericFft<E> plays the plan the host built at run time, FixedFft<N, R...> a
// length and radix order fixed at compile time.
//
//
// Reference stages (LensDiffCpuReference.cpp):
//   buildSelectionMask / applyMask / applyMaskScalarDriver :1219-1279
//       -> fused into the fill of frame_rows_kernel
//   convolveScalar / paddedSpectrumFromKernel / convolveRgba :1153-1217
//       -> frame_rows_kernel (forward rows, real input)
//          frame_cols_kernel (forward column, spectral multiply, inverse columns)
//          frame_inverse_kernel (inverse rows, real output)
//   MapLensDiffSpectralBins (LensDiffSpectrum.cpp:462-497), composite
//   (:2200-2218) -> frame_inverse_kernel epilogue
//
// HBM layout (ld_internal.h): spectrum columns are stored column-major with
// their channels interleaved, so the column pass moves one column of every
// channel as one contiguous block with one bulk copy (cp.async.bulk, mbarrier
// completion) and writes its result back with one bulk store, and the row
// passes read and write C adjacent values per spectrum bin.
//
// The column passes run one column per CTA.  A transform loop inside a
// persistent column loop makes the compiler keep the register demands of all
// stage bodies live together (spilling); straight-line, each body needs its
// own registers only.  To keep HBM busy while an SM transforms, every CTA
// prefetches into L2 the column the CTA one generation later will load (the
// grid launches in blockIdx order, `ahead` CTAs resident at a time).
#pragma once

#include <algorithm>

#include <cuda_fp16.h>

#include "ld_async.cuh"
#include "ld_fftx.cuh"
#include "ld_internal.h"
#include "ld_pixel.cuh"

namespace ld {
namespace {


constexpr int kMaxSmem = 227 * 1024;

template <int E>
struct Fam {
    static constexpr int max_threads = E >= kE25 ? kE25MaxThreads : kE16MaxThreads;
};

// X[k] of a real length-2M sequence from Z = FFT_M(even + i*odd):
// X[k] = E + W^k O, E = (Z[k] + conj Z[M-k]) / 2, O = (Z[k] - conj Z[M-k]) / 2i.
__device__ __forceinline__ float2 r2c_post(float2 zk, float2 zmk, float2 wk) {
    const float2 zc = make_float2(zmk.x, -zmk.y);
    const float2 e = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
    const float2 d = csub(zk, zc);
    const float2 o = make_float2(0.5f * d.y, -0.5f * d.x);
    return cadd(e, cmul(wk, o));
}

// Z[k] = E + i O from X[k], X[M-k] (inverse of r2c_post).
__device__ __forceinline__ float2 c2r_pre(float2 xk, float2 xmk, float2 wk) {
    const float2 xc = make_float2(xmk.x, -xmk.y);
    const float2 e = make_float2(0.5f * (xk.x + xc.x), 0.5f * (xk.y + xc.y));
    const float2 d = csub(xk, xc);
    const float2 o = cmulc(make_float2(0.5f * d.x, 0.5f * d.y), wk);
    return make_float2(e.x - o.y, e.y + o.x);
}

// Column-pass outputs B are grouped four spectrum columns at a time,
// B[k / 4][row][k % 4][c]: a column writes 24- or 32-byte runs four apart
// (the four columns of a group run together and their partial sectors merge
// in L2), and a row of the inverse pass reads one aligned run of
// 4 * C * 8 bytes per group instead of C * 8 bytes per column.
constexpr int kBGroup = 4;
__device__ __forceinline__ int64_t b_index(int k, int row, int c, int Hp, int C) {
    return ((static_cast<int64_t>(k / kBGroup) * Hp + row) * kBGroup + (k % kBGroup)) * C + c;
}

// Writes a transformed column (rows [0, Hp) of s[row * C + c]) to B.
__device__ __forceinline__ void store_b_column(const float2* s, float2* B, int k, int Hp, int C) {
    for (int i = threadIdx.x; i < Hp * C; i += blockDim.x) {
        const int row = i / C;
        const int c = i - row * C;
        B[b_index(k, row, c, Hp, C)] = s[i];
    }
}

// ---- FP16 spectra with a per-column scale (the chosen form) ------------------------
// A spectrum column is stored as half2 values v * (kHalfTop / m), m = the
// largest |real| or |imag| of the column, with m / kHalfTop kept as the
// column's float scale: every value keeps FP16's 11-bit mantissa down to
// 4e-9 m, and nothing overflows.
constexpr float kHalfTop = 16384.0f;

// Largest m over the CTA's threads (all threads get it; a barrier for all).
__device__ float block_max(float m) {
    __shared__ float part[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) part[warp] = m;
    __syncthreads();
    m = lane < static_cast<int>((blockDim.x + 31) >> 5) ? part[lane] : 0.0f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __syncthreads();  // part[] may be reused
    return m;
}

// Largest |real| / |imag| of s[0, n) over the CTA (all threads get it).
__device__ float block_absmax(const float2* s, int n) {
    float m = 0.0f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmaxf(m, fmaxf(fabsf(s[i].x), fabsf(s[i].y)));
    return block_max(m);
}

__device__ __forceinline__ __half2 to_half2(float2 v, float s) { return __floats2half2_rn(v.x * s, v.y * s); }
__device__ __forceinline__ float2 from_half2(__half2 h, float scale) {
    const float2 f = __half22float2(h);
    return make_float2(f.x * scale, f.y * scale);
}

// Writes a transformed column to B in FP16 with its scale (see store_b_column).
__device__ __forceinline__ void store_b_column_h16(const float2* s, __half2* B, float* bscale, int k, int Hp, int C) {
    const float m = block_absmax(s, Hp * C);
    const float sc = m > 0.0f ? kHalfTop / m : 1.0f;
    if (threadIdx.x == 0) bscale[k] = m > 0.0f ? m / kHalfTop : 1.0f;
    for (int i = threadIdx.x; i < Hp * C; i += blockDim.x) {
        const int row = i / C;
        const int c = i - row * C;
        B[b_index(k, row, c, Hp, C)] = to_half2(s[i], sc);
    }
}

// Writes the M+1 bins of the C transformed sequences in smem (s[k*C + col])
// to a column-major array: bin k of sequence col goes to
// out[k * col_elems + base + col].  Consecutive threads write consecutive
// columns of one bin, so each bin is one contiguous C * 8-byte run.
__device__ __forceinline__ void store_bins(int M, int C, int64_t col_elems, int64_t base,
                                           const float2* __restrict__ tw_px, const float2* s, float2* out) {
    for (int i = threadIdx.x; i < (M + 1) * C; i += blockDim.x) {
        const int k = i / C;
        const int col = i - k * C;
        const float2 v = r2c_post(s[(k == M ? 0 : k) * C + col], s[(k == 0 ? 0 : M - k) * C + col], __ldg(&tw_px[k]));
        out[k * col_elems + base + col] = v;
    }
}

// 2^e as a float, e in [-126, 127] (exact; built from the exponent field).
__device__ __forceinline__ float exp2_int(int e) { return __int_as_float((127 + e) << 23); }

// Row-spectrum exponent of a tile whose largest component is m: every value
// times 2^-e lies below 2^14 in magnitude (FP16 keeps its 11-bit mantissa
// down to 2^-14 of that, and has room to 65504).
__device__ __forceinline__ int row_tile_exp(float m) {
    if (!(m > 0.0f)) return 0;
    int e;
    frexpf(m, &e);  // m < 2^e
    return min(110, max(-110, e - 14));
}

// FP16 row spectra (the chosen form, one driver per row): the bins of the C
// rows in smem are formed in place (bin M of row col goes to s[M * C + col],
// so smem holds (M + 1) * C values), the tile's largest component sets its
// exponent e (row_tile_exp), and bin k of row y0 + col is stored as half2
// values times 2^-e at out[k * Hp + y0 + col], with e in aexp[y0 + col].
__device__ __forceinline__ void store_bins_h16(int M, int C, int Hp, int y0, const float2* __restrict__ tw_px,
                                               float2* s, __half2* out, signed char* aexp) {
    // pairs (k, M - k): one thread forms both bins from Z[k], Z[M - k]
    // (k = 0: bins 0 and M from Z[0]; k = M / 2 of an even M pairs with itself)
    float m = 0.0f;
    for (int i = threadIdx.x; i < (M / 2 + 1) * C; i += blockDim.x) {
        const int k = i / C;
        const int col = i - k * C;
        const float2 zk = s[k * C + col];
        const float2 zm = s[(k == 0 ? 0 : M - k) * C + col];
        const float2 xk = r2c_post(zk, zm, __ldg(&tw_px[k]));
        const float2 xm = r2c_post(zm, zk, __ldg(&tw_px[M - k]));
        s[k * C + col] = xk;
        s[(M - k) * C + col] = xm;
        m = fmaxf(m, fmaxf(fmaxf(fabsf(xk.x), fabsf(xk.y)), fmaxf(fabsf(xm.x), fabsf(xm.y))));
    }
    const int e = row_tile_exp(block_max(m));  // its barrier publishes the bins
    const float sc = exp2_int(-e);
    if (static_cast<int>(threadIdx.x) < C) aexp[y0 + threadIdx.x] = static_cast<signed char>(e);
    for (int i = threadIdx.x; i < (M + 1) * C; i += blockDim.x) {
        const int k = i / C;
        const int col = i - k * C;
        out[static_cast<int64_t>(k) * Hp + y0 + col] = to_half2(s[i], sc);
    }
}

// ---- forward rows --------------------------------------------------------------------
// Shared memory of a forward row pass over C sequences of length M (one
// spare bin per sequence for the in-place bins of store_bins_h16).
constexpr size_t rows_smem(int M, int C) { return (static_cast<size_t>(M) + 1) * C * sizeof(float2); }

// Spectral (NDRV = 1): C = 4 frame rows per CTA, the scalar driver of each.
// Mono (NDRV = 3): C = 3, one frame row per CTA, its three colour drivers.
// Column col of the transform is row y0 + col / NDRV, driver col % NDRV; its
// spectrum goes to A[k][y0 + col / NDRV][col % NDRV].
// FROM_EFFECT (scatter, NDRV = 3): the drivers are the stored effect's RGB.
template <int E, int C, int NDRV, int MAXT = Fam<E>::max_threads, int MINB = 1, bool FROM_EFFECT = false,
          class FFT = GenericFft<E>>
__global__ void __launch_bounds__(MAXT, MINB) frame_rows_kernel(FrameArgs a) {
    extern __shared__ float2 smem[];
    constexpr int RPC = C / NDRV;  // frame rows per CTA
    const int y0 = blockIdx.x * RPC;
    const int64_t pitch = a.src_pitch;
    const bool aligned = ((reinterpret_cast<uintptr_t>(a.src) | static_cast<uintptr_t>(pitch)) & 15) == 0;
    const int W = a.W, H = a.H, M = a.g.M;
    const int tx0 = a.tile_x0, ty0 = a.tile_y0;  // grid origin in frame pixels (tiles)
    // the source rows of this CTA and of the CTA one resident generation
    // later (their part under the grid) go to L2 through the bulk-copy
    // engine while this CTA loads
    // (bit 1 of the row plan's launch shape turns the later generation's
    // prefetch off; the autotuner times both)
    if (!FROM_EFFECT && aligned && threadIdx.x == 0) {
        const int px0 = max(0, tx0), px1 = min(W, tx0 + 2 * M);
        const uint32_t span = px1 > px0 ? static_cast<uint32_t>(px1 - px0) * 16u : 0u;
        const int later = y0 + a.ahead * RPC;
        const bool ahead = a.ahead > 0 && (a.g.plan_m.shape & 2) == 0;
        for (int r = 0; r < RPC && span > 0; ++r) {
            const int fy = y0 + r + ty0, fl = later + r + ty0;
            if (fy >= 0 && fy < H) bulk_prefetch_l2(a.src + static_cast<int64_t>(fy) * pitch + px0 * 16, span);
            if (ahead && fl >= 0 && fl < H) bulk_prefetch_l2(a.src + static_cast<int64_t>(fl) * pitch + px0 * 16, span);
        }
    }
    const SelectionParams sel = a.sel;
    // one thread per (row, pixel pair): the selection mask is evaluated once
    // per pixel and feeds every driver plane.  kU pairs per thread are loaded
    // before any is used, so enough source reads are in flight to cover HBM
    // latency at one CTA per SM.
    constexpr int kU = 4;
    const int T = blockDim.x;
    for (int i0 = threadIdx.x; i0 < RPC * M; i0 += kU * T) {
        float4 px[kU][2];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int i = i0 + u * T;
            const int r = i / M;
            const int idx = i - r * M;
            const int y = y0 + r + ty0;   // frame row
            const int x0 = 2 * idx + tx0;  // frame column of the pair's first pixel
            const unsigned char* row = a.src + static_cast<int64_t>(y) * pitch;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const bool in = i < RPC * M && y >= 0 && y < H && x0 + h >= 0 && x0 + h < W;
                if constexpr (FROM_EFFECT)
                    px[u][h] = in ? a.effect[static_cast<int64_t>(y) * W + x0 + h] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                else
                    px[u][h] = in ? decode_px(a.transfer, load_px(row, x0 + h, aligned)) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int i = i0 + u * T;
            if (i >= RPC * M) break;
            const int r = i / M;
            const int idx = i - r * M;
            float2 v[NDRV];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const float4 p = px[u][h];
                float sig;
                // zero pixels (outside the frame or black) give a zero driver
                const float m = FROM_EFFECT ? 1.0f : selection_mask(sel, p.x, p.y, p.z, &sig) * sel.rscale;
                if (NDRV == 1) {
                    const float dv = sig * m;
                    if (h == 0) v[0].x = dv;
                    else v[0].y = dv;
                } else {
                    const float c3[3] = {p.x * m, p.y * m, p.z * m};
#pragma unroll
                    for (int d = 0; d < NDRV; ++d) {
                        if (h == 0) v[d].x = c3[d];
                        else v[d].y = c3[d];
                    }
                }
            }
#pragma unroll
            for (int d = 0; d < NDRV; ++d) smem[idx * C + r * NDRV + d] = v[d];
        }
    }
    __syncthreads();
    FFT::template run<C, false, MAXT>(a.g.plan_m, smem);
    if (NDRV == 1 && !FROM_EFFECT && a.h16)
        store_bins_h16(M, C, a.Hp, y0, a.g.tw_px, smem, reinterpret_cast<__half2*>(a.A), a.aexp);
    else
        store_bins(M, C, static_cast<int64_t>(a.Hp) * NDRV, static_cast<int64_t>(y0) * NDRV, a.g.tw_px, smem, a.A);
}

// ---- column pass, spectral: forward, multiply by NOUT kernel spectra, inverse ----------
// Column k = blockIdx.x.  Shared memory: F [Py] (the column's row spectra land
// in F[0, Hp), rows past Hp are the zero padding; transformed in place),
// Wk [Py][NOUT] (the column's NOUT kernel spectra land here, are multiplied by
// F in place and inverse-transformed together as NOUT interleaved sequences),
// two mbarriers.  The first Hp rows of Wk go to B with one bulk store.
// H16: the half2 row spectra land at the start of Wk and the rows' exponents
// right after them (a third mbarrier), and are widened into F; the half2
// kernel spectra land in the upper half of Wk and are widened in the multiply.
template <int E, int NOUT, int MAXT = Fam<E>::max_threads, int MINB = 1, bool H16 = false, class FFT = GenericFft<E>>
__global__ void __launch_bounds__(MAXT, MINB) frame_cols_kernel(FrameArgs a) {
    extern __shared__ __align__(128) unsigned char smraw[];
    const int Py = a.g.Py, Hp = a.Hp, cols = a.g.cols;
    const int k = blockIdx.x;
    float2* F = reinterpret_cast<float2*>(smraw);
    float2* Wk = F + Py;
    uint64_t* bars = reinterpret_cast<uint64_t*>(Wk + static_cast<size_t>(Py) * NOUT);
    const uint32_t a_bytes = static_cast<uint32_t>(Hp * (H16 ? sizeof(__half2) : sizeof(float2)));
    void* adst = H16 ? static_cast<void*>(Wk) : static_cast<void*>(F);
    const char* asrc = reinterpret_cast<const char*>(a.A) + static_cast<size_t>(k) * a_bytes;
    const size_t kn = static_cast<size_t>(Py) * NOUT;
    const uint32_t k_bytes = static_cast<uint32_t>(kn * (H16 ? sizeof(__half2) : sizeof(float2)));
    void* kdst = H16 ? static_cast<void*>(reinterpret_cast<__half2*>(Wk) + kn) : static_cast<void*>(Wk);
    const void* ksrc = H16 ? static_cast<const void*>(reinterpret_cast<const __half2*>(a.spectra) + k * kn)
                           : static_cast<const void*>(a.spectra + k * kn);
    const bool lead = threadIdx.x == 0;
    signed char* aex = reinterpret_cast<signed char*>(Wk) + static_cast<size_t>(Hp) * sizeof(__half2);
    if (lead) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        if (H16) mbar_init(&bars[2], 1);
        mbar_init_fence();
    }
    __syncthreads();  // barriers initialised before anyone waits on them
    if (lead) {
        bulk_load_checked(adst, asrc, a_bytes, &bars[0], smraw, a.err);
        if (H16) bulk_load_checked(aex, a.aexp, static_cast<uint32_t>((Hp + 15) & ~15), &bars[2], smraw, a.err);
        bulk_load_checked(kdst, ksrc, k_bytes, &bars[1], smraw, a.err);
        const int later = k + a.ahead;  // bit 1 of the column plan's shape: no look-ahead (autotuned)
        if (later < cols && (a.g.plan_py.shape & 2) == 0) {
            bulk_prefetch_l2(asrc + (later - k) * static_cast<size_t>(a_bytes), a_bytes);
            bulk_prefetch_l2(static_cast<const char*>(ksrc) + (later - k) * static_cast<size_t>(k_bytes), k_bytes);
        }
    }
    if constexpr (H16) {
        if (__syncthreads_or(!mbar_wait(&bars[0], 0, a.err) || !mbar_wait(&bars[2], 0, a.err))) return;
        const __half2* ah = reinterpret_cast<const __half2*>(Wk);
        for (int i = threadIdx.x; i < Py; i += blockDim.x)
            F[i] = i < Hp ? from_half2(ah[i], exp2_int(aex[i])) : make_float2(0.0f, 0.0f);
        __syncthreads();
    } else {
        for (int i = Hp + threadIdx.x; i < Py; i += blockDim.x) F[i] = make_float2(0.0f, 0.0f);
        if (__syncthreads_or(!mbar_wait(&bars[0], 0, a.err))) return;
    }
    FFT::template run<1, false, MAXT>(a.g.plan_py, F);
    if (__syncthreads_or(!mbar_wait(&bars[1], 0, a.err))) return;
    if constexpr (H16) {
        // every thread widens its (at most E) kernel values before any
        // product overwrites the half2 area they came from
        const float ks = a.kscale[k];
        const __half2* kh = reinterpret_cast<const __half2*>(Wk) + kn;
        float2 kv[E];
#pragma unroll
        for (int j = 0; j < E; ++j) {
            const int i = threadIdx.x + j * static_cast<int>(blockDim.x);
            kv[j] = i < static_cast<int>(kn) ? from_half2(kh[i], ks) : make_float2(0.0f, 0.0f);
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < E; ++j) {
            const int i = threadIdx.x + j * static_cast<int>(blockDim.x);
            if (i < static_cast<int>(kn)) Wk[i] = cmul(kv[j], F[i / NOUT]);
        }
    } else {
        for (int i = threadIdx.x; i < Py * NOUT; i += blockDim.x) Wk[i] = cmul(Wk[i], F[i / NOUT]);
    }
    __syncthreads();
    FFT::template run<NOUT, true, MAXT>(a.g.plan_py, Wk);
    if constexpr (H16)
        store_b_column_h16(Wk, reinterpret_cast<__half2*>(a.Bout), a.bscale, k, Hp, NOUT);
    else
        store_b_column(Wk, a.Bout, k, Hp, NOUT);
}

// ---- column pass, Mono: three colour drivers, one kernel spectrum -------------------
// Shared memory: X [Py][3] (the column's three row spectra land in X[0, Hp)),
// Kc [Py] (the kernel spectrum), two mbarriers.  Forward (3 sequences),
// multiply by Kc, inverse, bulk store of the first Hp rows.
template <int E>
__global__ void __launch_bounds__(Fam<E>::max_threads, 1) frame_cols_mono_kernel(FrameArgs a) {
    extern __shared__ __align__(128) unsigned char smraw[];
    const int Py = a.g.Py, Hp = a.Hp, cols = a.g.cols;
    const int k = blockIdx.x;
    float2* X = reinterpret_cast<float2*>(smraw);
    float2* Kc = X + static_cast<size_t>(Py) * 3;
    uint64_t* bars = reinterpret_cast<uint64_t*>(Kc + Py);
    const uint32_t a_bytes = static_cast<uint32_t>(static_cast<size_t>(Hp) * 3 * sizeof(float2));
    const uint32_t k_bytes = static_cast<uint32_t>(Py * sizeof(float2));
    const bool lead = threadIdx.x == 0;
    if (lead) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init_fence();
    }
    __syncthreads();  // barriers initialised before anyone waits on them
    if (lead) {
        bulk_load_checked(X, a.A + static_cast<size_t>(k) * Hp * 3, a_bytes, &bars[0], smraw, a.err);
        bulk_load_checked(Kc, a.spectra + static_cast<size_t>(k) * Py, k_bytes, &bars[1], smraw, a.err);
        const int later = k + a.ahead;
        if (later < cols) {
            bulk_prefetch_l2(a.A + static_cast<size_t>(later) * Hp * 3, a_bytes);
            bulk_prefetch_l2(a.spectra + static_cast<size_t>(later) * Py, k_bytes);
        }
    }
    for (int i = Hp * 3 + threadIdx.x; i < Py * 3; i += blockDim.x) X[i] = make_float2(0.0f, 0.0f);
    if (__syncthreads_or(!mbar_wait(&bars[0], 0, a.err))) return;
    fft_run<E, 3, false>(a.g.plan_py, X);
    if (__syncthreads_or(!mbar_wait(&bars[1], 0, a.err))) return;
    for (int i = threadIdx.x; i < Py * 3; i += blockDim.x) X[i] = cmul(X[i], Kc[i / 3]);
    __syncthreads();
    fft_run<E, 3, true>(a.g.plan_py, X);
    store_b_column(X, a.Bout, k, Hp, 3);
}

// ---- inverse rows + spectral map + composite ----------------------------------------
// The spectral map of pixel sx of the inverse-transformed row in smem.
template <int C>
__device__ __forceinline__ float3 mapped_effect(const FrameArgs& a, const float2* smem, int sx) {
    const int nn = sx >> 1;
    const bool odd = sx & 1;
    float e[C];
#pragma unroll
    for (int c = 0; c < C; ++c) {
        const float2 z = smem[nn * C + c];
        e[c] = odd ? z.y : z.x;
    }
    return map_effect<C>(a, e);
}

// softShoulder (LensDiffCpuReference.cpp:84-90): s (1 - exp(-max(0, v) / s)).
__device__ __forceinline__ float soft_shoulder(float v, float s) {
    const float x = fmaxf(0.0f, v);
    return s * (1.0f - expf(-x / s));
}

// Tent weight of field zone z along one axis (accumulateWeightedImage,
// LensDiffCpuReference.cpp:1458-1466; the reference's grid is n = 3).
__device__ __forceinline__ float zone_weight(int v, int extent, int z, int n) {
    const float denom = static_cast<float>(max(1, extent - 1));
    const float pv = (static_cast<float>(v) / denom) * static_cast<float>(n - 1);
    return fmaxf(0.0f, 1.0f - fabsf(pv - static_cast<float>(z)));
}

// One row per CTA; smem M * C float2 (C = n_out interleaved channels).  The
// row is output row out_y1 + blockIdx.x (kEffectComposite), source row
// blockIdx.x (kEffectStore, kEffectScatter) or source row row0 + blockIdx.x
// (kEffectAccumulate); see FrameArgs::effect_mode.
template <int E, int C, int MAXT = Fam<E>::max_threads, int MINB = 1, bool H16 = false, class FFT = GenericFft<E>>
__global__ void __launch_bounds__(MAXT, MINB) frame_inverse_kernel(FrameArgs a) {
    extern __shared__ float2 smem[];
    const int bid = static_cast<int>(blockIdx.x);
    const int yo = a.effect_mode == kEffectComposite ? a.out_y1 + bid
                                                     : a.src_y1 + (a.effect_mode == kEffectAccumulate ? a.row0 + bid : bid);
    const int sy = yo - a.src_y1;
    const int by = sy - a.tile_y0;  // the grid row of frame row sy
    const bool have = sy >= 0 && sy < a.H && by >= 0 && by < a.Hp;
    const int M = a.g.M;
    // composite: this row's source pixels, and those of the row one resident
    // generation later (unless bit 2 of the row plan's shape is set; the
    // autotuner times both), go to L2 while the row's spectrum loads and
    // transforms
    if (a.effect_mode == kEffectComposite && threadIdx.x == 0 &&
        ((reinterpret_cast<uintptr_t>(a.src) | static_cast<uintptr_t>(a.src_pitch)) & 15) == 0) {
        const uint32_t row_bytes = static_cast<uint32_t>(a.W) * 16u;
        if (have) bulk_prefetch_l2(a.src + static_cast<int64_t>(sy) * a.src_pitch, row_bytes);
        const int sl = sy + a.ahead;
        if (a.ahead > 0 && (a.g.plan_m.shape & 4) == 0 && sl >= 0 && sl < a.H &&
            bid + a.ahead < static_cast<int>(gridDim.x))
            bulk_prefetch_l2(a.src + static_cast<int64_t>(sl) * a.src_pitch, row_bytes);
    }
    if (have) {
        const float2* tw_px = a.g.tw_px;
        // Hermitian pairs: one load of X[p] and X[M-p] per channel gives both
        // Z[p] and Z[M-p] (p = 0 pairs with the Nyquist bin M and gives Z[0]
        // only; p = M/2 pairs with itself).  kU pairs per thread are loaded
        // before any is used: the reads are scattered, one run per bin group.
        const int Hp = a.Hp;
        const int half = M / 2;
        const int npair = (half + 1) * C;
        constexpr int kU = 4;
        const int T = blockDim.x;
        for (int i0 = threadIdx.x; i0 < npair; i0 += kU * T) {
            float2 xp[kU], xq[kU], wp[kU], wq[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int i = i0 + u * T;
                if (i < npair) {
                    const int pk = i / C;
                    const int c = i - pk * C;
                    if constexpr (H16) {
                        const __half2* Bh = reinterpret_cast<const __half2*>(a.Bout);
                        xp[u] = from_half2(__ldcs(&Bh[b_index(pk, by, c, Hp, C)]), __ldg(&a.bscale[pk]));
                        xq[u] = from_half2(__ldcs(&Bh[b_index(M - pk, by, c, Hp, C)]), __ldg(&a.bscale[M - pk]));
                    } else {
                        xp[u] = __ldcs(&a.Bout[b_index(pk, by, c, Hp, C)]);
                        xq[u] = __ldcs(&a.Bout[b_index(M - pk, by, c, Hp, C)]);
                    }
                    wp[u] = __ldg(&tw_px[pk]);
                    wq[u] = __ldg(&tw_px[M - pk]);
                }
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int i = i0 + u * T;
                if (i < npair) {
                    const int pk = i / C;
                    const int c = i - pk * C;
                    if (pk < M) smem[pk * C + c] = c2r_pre(xp[u], xq[u], wp[u]);
                    if (pk > 0 && M - pk != pk && M - pk < M) smem[(M - pk) * C + c] = c2r_pre(xq[u], xp[u], wq[u]);
                }
            }
        }
        __syncthreads();
        FFT::template run<C, true, MAXT>(a.g.plan_m, smem);
    }
    const bool aligned_s = ((reinterpret_cast<uintptr_t>(a.src) | static_cast<uintptr_t>(a.src_pitch)) & 15) == 0;
    const unsigned char* srow = a.src + static_cast<int64_t>(sy) * a.src_pitch;
    if (a.effect_mode == kEffectAccumulate) {
        if (!have) return;
        const float wy = a.zone_n > 0 ? zone_weight(sy, a.H, a.zone_y, a.zone_n) : 1.0f;
        if (wy <= 0.0f) return;
        const float gain = a.acc_gain, sh = a.acc_shoulder;
        float4* erow = a.effect + static_cast<int64_t>(sy) * a.W;
        for (int sx = a.acc_x0 + threadIdx.x; sx < a.acc_x1; sx += blockDim.x) {
            const float wgt = (a.zone_n > 0 ? zone_weight(sx, a.W, a.zone_x, a.zone_n) : 1.0f) * wy;
            if (wgt <= 0.0f) continue;
            float3 e = mapped_effect<C>(a, smem, sx - a.tile_x0);
            if (sh > 0.0f) e = make_float3(soft_shoulder(e.x, sh), soft_shoulder(e.y, sh), soft_shoulder(e.z, sh));
            float4 acc = erow[sx];
            acc.x += e.x * gain * wgt;
            acc.y += e.y * gain * wgt;
            acc.z += e.z * gain * wgt;
            erow[sx] = acc;
        }
        return;
    }
    if (a.effect_mode == kEffectScatter) {
        if (!have) return;
        const float amount = a.scatter;
        float4* erow = a.effect + static_cast<int64_t>(sy) * a.W;
        for (int sx = threadIdx.x; sx < a.W; sx += blockDim.x) {
            const float3 e = mapped_effect<C>(a, smem, sx);  // Mono map: max(0, value)
            float4 acc = erow[sx];
            if (a.scatter_replace) {
                acc = make_float4(e.x, e.y, e.z, 0.0f);
            } else {
                acc.x += e.x * amount;
                acc.y += e.y * amount;
                acc.z += e.z * amount;
            }
            erow[sx] = acc;
        }
        return;
    }
    if (a.effect_mode == kEffectStore) {
        double l_in = 0.0, l_eff = 0.0;
        float4* erow = a.effect + static_cast<int64_t>(sy) * a.W;
        for (int sx = threadIdx.x; sx < a.W; sx += blockDim.x) {
            const float3 e = mapped_effect<C>(a, smem, sx);
            erow[sx] = make_float4(e.x, e.y, e.z, 0.0f);
            if (!a.preserve) continue;
            const float4 p = decode_px(a.transfer, load_px(srow, sx, aligned_s));
            float sig;
            const float m = selection_mask(a.sel, p.x, p.y, p.z, &sig) * a.sel.rscale;
            l_in += static_cast<double>(luma(p.x * m, p.y * m, p.z * m));
            l_eff += static_cast<double>(luma(e.x, e.y, e.z));
        }
        if (a.preserve) block_add2(l_in, l_eff, a.sums);
        return;
    }
    const bool aligned_d = ((reinterpret_cast<uintptr_t>(a.dst) | static_cast<uintptr_t>(a.dst_pitch)) & 15) == 0;
    unsigned char* drow = a.dst + static_cast<int64_t>(yo - a.dst_y1) * a.dst_pitch;
    constexpr int kV = 4;  // source pixels loaded ahead of use, per thread
    const int T = blockDim.x;
    for (int x0 = a.out_x1 + threadIdx.x; x0 < a.out_x2; x0 += kV * T) {
        float4 px[kV];
#pragma unroll
        for (int u = 0; u < kV; ++u) {
            const int sx = x0 + u * T - a.src_x1;
            px[u] = (have && x0 + u * T < a.out_x2 && sx >= 0 && sx < a.W)
                        ? decode_px(a.transfer, load_px(srow, sx, aligned_s))
                                                                           : make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        }
#pragma unroll
        for (int u = 0; u < kV; ++u) {
            const int x = x0 + u * T;
            if (x >= a.out_x2) break;
            const int sx = x - a.src_x1;
            float4 out = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
            if (have && sx >= 0 && sx < a.W) out = composite_px(a, px[u], mapped_effect<C>(a, smem, sx));
            store_px(drow, x - a.dst_x1, aligned_d, encode_px(a.transfer, out));
        }
    }
}

// Luma sums of the redistributed source and of the stored effect over the
// whole source frame (field zones with Preserve energy); one source row per CTA.
__global__ void __launch_bounds__(256) effect_sums_kernel(FrameArgs a) {
    const int sy = blockIdx.x;
    const bool aligned_s = ((reinterpret_cast<uintptr_t>(a.src) | static_cast<uintptr_t>(a.src_pitch)) & 15) == 0;
    const unsigned char* srow = a.src + static_cast<int64_t>(sy) * a.src_pitch;
    const float4* erow = a.effect + static_cast<int64_t>(sy) * a.W;
    double l_in = 0.0, l_eff = 0.0;
    for (int sx = threadIdx.x; sx < a.W; sx += blockDim.x) {
        const float4 p = decode_px(a.transfer, load_px(srow, sx, aligned_s));
        float sig;
        const float m = selection_mask(a.sel, p.x, p.y, p.z, &sig) * a.sel.rscale;
        l_in += static_cast<double>(luma(p.x * m, p.y * m, p.z * m));
        const float4 e = erow[sx];
        l_eff += static_cast<double>(luma(e.x, e.y, e.z));
    }
    block_add2(l_in, l_eff, a.sums);
}

// One channel of the stored effect, bilinear at (fx, fy) clamped to the
// frame (sampleRgbaBilinear, LensDiffCpuReference.cpp:1477-1497).
__device__ __forceinline__ float effect_clamped(const float* e, int W, int H, float fx, float fy, int c) {
    const float x = fminf(fmaxf(fx, 0.0f), static_cast<float>(max(0, W - 1)));
    const float y = fminf(fmaxf(fy, 0.0f), static_cast<float>(max(0, H - 1)));
    const int x0 = static_cast<int>(floorf(x)), y0 = static_cast<int>(floorf(y));
    const int x1 = min(x0 + 1, W - 1), y1 = min(y0 + 1, H - 1);
    const float tx = __fsub_rn(x, static_cast<float>(x0)), ty = __fsub_rn(y, static_cast<float>(y0));
    const float p00 = __ldg(e + 4 * (static_cast<int64_t>(y0) * W + x0) + c);
    const float p10 = __ldg(e + 4 * (static_cast<int64_t>(y0) * W + x1) + c);
    const float p01 = __ldg(e + 4 * (static_cast<int64_t>(y1) * W + x0) + c);
    const float p11 = __ldg(e + 4 * (static_cast<int64_t>(y1) * W + x1) + c);
    const float u = p00 * (1.0f - tx) + p10 * tx;
    const float v = p01 * (1.0f - tx) + p11 * tx;
    return u * (1.0f - ty) + v * ty;
}

// The stored effect at working pixel (x, y), after the creative fringe when
// FRINGE: red sampled at +shift, blue at -shift along the direction from the
// frame centre, green unshifted (applyCreativeFringe :1499-1534).
template <bool FRINGE>
__device__ __forceinline__ float3 effect_px(const FrameArgs& a, int x, int y) {
    const float4 c = __ldg(a.effect + static_cast<int64_t>(y) * a.Ww + x);
    if (!FRINGE) return make_float3(c.x, c.y, c.z);
    const float cx = static_cast<float>(max(0, a.Ww - 1)) * 0.5f;
    const float cy = static_cast<float>(max(0, a.Hw - 1)) * 0.5f;
    const float dx = __fsub_rn(static_cast<float>(x), cx), dy = __fsub_rn(static_cast<float>(y), cy);
    const float len = sqrtf(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
    const float inv = len > 1e-6f ? __fdiv_rn(1.0f, len) : 0.0f;
    const float shx = __fmul_rn(__fmul_rn(dx, inv), a.fringe_px);
    const float shy = __fmul_rn(__fmul_rn(dy, inv), a.fringe_px);
    const float* e = reinterpret_cast<const float*>(a.effect);
    const float fxr = __fadd_rn(static_cast<float>(x), shx), fyr = __fadd_rn(static_cast<float>(y), shy);
    const float fxb = __fsub_rn(static_cast<float>(x), shx), fyb = __fsub_rn(static_cast<float>(y), shy);
    return make_float3(effect_clamped(e, a.Ww, a.Hw, fxr, fyr, 0), c.y, effect_clamped(e, a.Ww, a.Hw, fxb, fyb, 2));
}

__device__ __forceinline__ float3 lerp3(float3 a, float3 b, float t) {
    return make_float3(a.x + (b.x - a.x) * t, a.y + (b.y - a.y) * t, a.z + (b.z - a.z) * t);
}

// Selection mask of working pixel (x, y) (buildSelectionMask's value).
__device__ __forceinline__ float work_mask(const FrameArgs& a, int x, int y) {
    const float4 p = __ldg(a.work + static_cast<int64_t>(y) * a.Ww + x);
    float sig;
    return selection_mask(a.sel, p.x, p.y, p.z, &sig);
}

// What a working pixel contributes to an output pixel: the effect (after
// the fringe when FRINGE), the fringe preview |fringed - plain|
// (applyCreativeFringe's preview, LensDiffCpuReference.cpp:1527-1530), or the
// selection mask in .x.
template <int MODE, bool FRINGE>
__device__ __forceinline__ float3 tap_value(const FrameArgs& a, int x, int y) {
    if constexpr (MODE == kOutFringePreview) {
        const float3 f = effect_px<true>(a, x, y), e = effect_px<false>(a, x, y);
        return make_float3(fabsf(f.x - e.x), fabsf(f.y - e.y), fabsf(f.z - e.z));
    } else if constexpr (MODE == kOutSelection) {
        return make_float3(work_mask(a, x, y), 0.0f, 0.0f);
    } else {
        return effect_px<FRINGE>(a, x, y);
    }
}

// Output rows of the render window from the stored effect: scaled, with
// Preserve energy, by (luma sum of the redistributed source) / (luma sum of
// the effect) as LensDiffCpuReference.cpp:2172-2178 does (scaleImage with the
// float quotient of the two sums), then composited.  The scale is linear and
// commutes with the scatter, fringe and resample steps that follow it in the
// reference, so it is applied here, last.  RESAMPLE: the effect and the
// redistributed working source are sampled at the source pixel's position in
// the working frame (sampleRgbaBilinearImage :373-395: zero outside it), as
// resampleRgbaImage (:414-434) does for the whole image.
// MODE kOutComposite writes the composite (encoded to the source's
// transfer); the debug views (renderDebugView, :1789-1824) write, unencoded
// with alpha 1: kOutEffect the (scaled) effect, kOutFringePreview the fringe
// preview, kOutSelection the selection mask over its maximum
// (makeDebugFromScalar, :1370-1389; *a.mask_max from selection_max_kernel).
template <int MODE, bool FRINGE, bool RESAMPLE>
__global__ void __launch_bounds__(256) composite_kernel(FrameArgs a) {
    const int yo = a.out_y1 + blockIdx.x;
    const int sy = yo - a.src_y1;
    const bool have = sy >= 0 && sy < a.H;
    float scale = 1.0f;
    if (a.preserve) {
        const float in_e = static_cast<float>(a.sums[0]);
        const float eff_e = static_cast<float>(a.sums[1]);
        if (eff_e > 1e-6f) scale = in_e / eff_e;
    }
    float inv_max = 0.0f;
    if constexpr (MODE == kOutSelection) {
        const float mx = __uint_as_float(*a.mask_max);
        inv_max = mx > 0.0f ? 1.0f / mx : 0.0f;
    }
    const bool aligned_s = ((reinterpret_cast<uintptr_t>(a.src) | static_cast<uintptr_t>(a.src_pitch)) & 15) == 0;
    const bool aligned_d = ((reinterpret_cast<uintptr_t>(a.dst) | static_cast<uintptr_t>(a.dst_pitch)) & 15) == 0;
    const unsigned char* srow = a.src + static_cast<int64_t>(sy) * a.src_pitch;
    unsigned char* drow = a.dst + static_cast<int64_t>(yo - a.dst_y1) * a.dst_pitch;
    // resample coordinates (float, as the reference computes them)
    const float ksx = RESAMPLE ? __fdiv_rn(static_cast<float>(a.Ww), static_cast<float>(max(1, a.W))) : 1.0f;
    const float ksy = RESAMPLE ? __fdiv_rn(static_cast<float>(a.Hw), static_cast<float>(max(1, a.H))) : 1.0f;
    const float fy = __fsub_rn(__fmul_rn(__fadd_rn(static_cast<float>(sy), 0.5f), ksy), 0.5f);
    for (int x = a.out_x1 + threadIdx.x; x < a.out_x2; x += blockDim.x) {
        float4 out = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        const int sx = x - a.src_x1;
        if (have && sx >= 0 && sx < a.W) {
            const float4 p = decode_px(a.transfer, load_px(srow, sx, aligned_s));
            float3 rd = make_float3(0.0f, 0.0f, 0.0f), e = rd;
            if constexpr (!RESAMPLE) {
                if constexpr (MODE == kOutSelection) {
                    float sig;
                    e.x = selection_mask(a.sel, p.x, p.y, p.z, &sig);
                } else {
                    e = tap_value<MODE, FRINGE>(a, sx, sy);
                }
                if constexpr (MODE == kOutComposite) rd = redistributed(a, p);
            } else {
                const float fx = __fsub_rn(__fmul_rn(__fadd_rn(static_cast<float>(sx), 0.5f), ksx), 0.5f);
                if (!(fx < 0.0f || fy < 0.0f || fx > static_cast<float>(a.Ww - 1) ||
                      fy > static_cast<float>(a.Hw - 1))) {
                    const int x0 = static_cast<int>(floorf(fx)), y0 = static_cast<int>(floorf(fy));
                    const int x1 = min(x0 + 1, a.Ww - 1), y1 = min(y0 + 1, a.Hw - 1);
                    const float tx = __fsub_rn(fx, static_cast<float>(x0));
                    const float ty = __fsub_rn(fy, static_cast<float>(y0));
                    if constexpr (MODE == kOutComposite) {
                        const float4* wk = a.work;
                        const float3 r00 = redistributed(a, __ldg(wk + static_cast<int64_t>(y0) * a.Ww + x0));
                        const float3 r10 = redistributed(a, __ldg(wk + static_cast<int64_t>(y0) * a.Ww + x1));
                        const float3 r01 = redistributed(a, __ldg(wk + static_cast<int64_t>(y1) * a.Ww + x0));
                        const float3 r11 = redistributed(a, __ldg(wk + static_cast<int64_t>(y1) * a.Ww + x1));
                        rd = lerp3(lerp3(r00, r10, tx), lerp3(r01, r11, tx), ty);
                    }
                    const float3 e00 = tap_value<MODE, FRINGE>(a, x0, y0), e10 = tap_value<MODE, FRINGE>(a, x1, y0);
                    const float3 e01 = tap_value<MODE, FRINGE>(a, x0, y1), e11 = tap_value<MODE, FRINGE>(a, x1, y1);
                    e = lerp3(lerp3(e00, e10, tx), lerp3(e01, e11, tx), ty);
                }
            }
            if constexpr (MODE == kOutComposite) {
                out = composite_rd(a, p, rd, make_float3(e.x * scale, e.y * scale, e.z * scale));
            } else if constexpr (MODE == kOutSelection) {
                const float d = saturate(e.x * inv_max);
                out = make_float4(d, d, d, 1.0f);
            } else {
                out = make_float4(e.x * scale, e.y * scale, e.z * scale, 1.0f);
            }
        }
        store_px(drow, x - a.dst_x1, aligned_d, MODE == kOutComposite ? encode_px(a.transfer, out) : out);
    }
}

// Maximum of the selection mask over the whole source frame (resampled from
// the working frame when RESAMPLE, resampleScalarImage :397-412) into
// *a.mask_max as float bits; one source row per CTA.
template <bool RESAMPLE>
__global__ void __launch_bounds__(256) selection_max_kernel(FrameArgs a) {
    const int sy = blockIdx.x;
    const bool aligned_s = ((reinterpret_cast<uintptr_t>(a.src) | static_cast<uintptr_t>(a.src_pitch)) & 15) == 0;
    const unsigned char* srow = a.src + static_cast<int64_t>(sy) * a.src_pitch;
    const float ksx = RESAMPLE ? __fdiv_rn(static_cast<float>(a.Ww), static_cast<float>(max(1, a.W))) : 1.0f;
    const float ksy = RESAMPLE ? __fdiv_rn(static_cast<float>(a.Hw), static_cast<float>(max(1, a.H))) : 1.0f;
    const float fy = __fsub_rn(__fmul_rn(__fadd_rn(static_cast<float>(sy), 0.5f), ksy), 0.5f);
    float m = 0.0f;
    for (int sx = threadIdx.x; sx < a.W; sx += blockDim.x) {
        float v = 0.0f;
        if constexpr (!RESAMPLE) {
            const float4 p = decode_px(a.transfer, load_px(srow, sx, aligned_s));
            float sig;
            v = selection_mask(a.sel, p.x, p.y, p.z, &sig);
        } else {
            const float fx = __fsub_rn(__fmul_rn(__fadd_rn(static_cast<float>(sx), 0.5f), ksx), 0.5f);
            if (!(fx < 0.0f || fy < 0.0f || fx > static_cast<float>(a.Ww - 1) || fy > static_cast<float>(a.Hw - 1))) {
                const int x0 = static_cast<int>(floorf(fx)), y0 = static_cast<int>(floorf(fy));
                const int x1 = min(x0 + 1, a.Ww - 1), y1 = min(y0 + 1, a.Hw - 1);
                const float tx = __fsub_rn(fx, static_cast<float>(x0));
                const float ty = __fsub_rn(fy, static_cast<float>(y0));
                const float v00 = work_mask(a, x0, y0), v10 = work_mask(a, x1, y0);
                const float v01 = work_mask(a, x0, y1), v11 = work_mask(a, x1, y1);
                const float vx0 = v00 + (v10 - v00) * tx, vx1 = v01 + (v11 - v01) * tx;
                v = vx0 + (vx1 - vx0) * ty;
            }
        }
        m = fmaxf(m, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0f) atomicMax(a.mask_max, __float_as_uint(m));
}

// Working source of the resolution-aware path: pixel (x, y) of the a.Ww x
// a.Hw working frame samples the source at ((x + .5) * W / Ww - .5, ...)
// bilinearly, zero outside [0, W-1] x [0, H-1] (resampleRgbaImage
// :414-434 with sampleRgbaBilinearImage :373-395).
__global__ void __launch_bounds__(256) resample_source_kernel(FrameArgs a) {
    const int y = blockIdx.y;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= a.Ww) return;
    const float ksx = __fdiv_rn(static_cast<float>(a.W), static_cast<float>(max(1, a.Ww)));
    const float ksy = __fdiv_rn(static_cast<float>(a.H), static_cast<float>(max(1, a.Hw)));
    const float fx = __fsub_rn(__fmul_rn(__fadd_rn(static_cast<float>(x), 0.5f), ksx), 0.5f);
    const float fy = __fsub_rn(__fmul_rn(__fadd_rn(static_cast<float>(y), 0.5f), ksy), 0.5f);
    float4 out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (!(fx < 0.0f || fy < 0.0f || fx > static_cast<float>(a.W - 1) || fy > static_cast<float>(a.H - 1))) {
        const bool aligned = ((reinterpret_cast<uintptr_t>(a.src) | static_cast<uintptr_t>(a.src_pitch)) & 15) == 0;
        const int x0 = static_cast<int>(floorf(fx)), y0 = static_cast<int>(floorf(fy));
        const int x1 = min(x0 + 1, a.W - 1), y1 = min(y0 + 1, a.H - 1);
        const float tx = __fsub_rn(fx, static_cast<float>(x0)), ty = __fsub_rn(fy, static_cast<float>(y0));
        const unsigned char* r0 = a.src + static_cast<int64_t>(y0) * a.src_pitch;
        const unsigned char* r1 = a.src + static_cast<int64_t>(y1) * a.src_pitch;
        const int tf = a.transfer;
        const float4 p00 = decode_px(tf, load_px(r0, x0, aligned)), p10 = decode_px(tf, load_px(r0, x1, aligned));
        const float4 p01 = decode_px(tf, load_px(r1, x0, aligned)), p11 = decode_px(tf, load_px(r1, x1, aligned));
        const float4 u = make_float4(p00.x + (p10.x - p00.x) * tx, p00.y + (p10.y - p00.y) * tx,
                                     p00.z + (p10.z - p00.z) * tx, p00.w + (p10.w - p00.w) * tx);
        const float4 v = make_float4(p01.x + (p11.x - p01.x) * tx, p01.y + (p11.y - p01.y) * tx,
                                     p01.z + (p11.z - p01.z) * tx, p01.w + (p11.w - p01.w) * tx);
        out = make_float4(u.x + (v.x - u.x) * ty, u.y + (v.y - u.y) * ty, u.z + (v.z - u.z) * ty,
                          u.w + (v.w - u.w) * ty);
    }
    a.work[static_cast<int64_t>(y) * a.Ww + x] = out;
}

// ---- kernel spectra ----------------------------------------------------------------------
// Canvas column j sits at grid column (j - R) mod Px; canvas row i at grid row
// (i - R) mod Py (the kernel centre at the origin, paddedSpectrumFromKernel
// LensDiffCpuReference.cpp:1153-1165).
__device__ __forceinline__ int canvas_index(int g, int P, int R) {
    if (g <= R) return g + R;
    if (g >= P - R) return g - P + R;
    return -1;
}

// One canvas row i = blockIdx.x of all C kernels per CTA (rows >= K are zero):
// KR[k][i][c], k < M + 1.
template <int E, int C, int MAXT = Fam<E>::max_threads, int MINB = 1, class FFT = GenericFft<E>>
__global__ void __launch_bounds__(MAXT, MINB) kspec_rows_kernel(KernelSpectraArgs a) {
    extern __shared__ float2 smem[];
    const int i = blockIdx.x;
    const int Px = a.g.Px, R = a.R, K = a.K;
    const size_t kk = static_cast<size_t>(K) * K;
    const float* crow = a.canvas + static_cast<size_t>(i < K ? i : 0) * K;
    smem_fill<C>(smem, a.g.M, [=](int idx, int c) -> float2 {
        if (i >= K) return make_float2(0.0f, 0.0f);
        const float* p = crow + c * kk;
        const int j0 = canvas_index(2 * idx, Px, R);
        const int j1 = canvas_index(2 * idx + 1, Px, R);
        return make_float2(j0 >= 0 ? p[j0] : 0.0f, j1 >= 0 ? p[j1] : 0.0f);
    });
    FFT::template run<C, false, MAXT>(a.g.plan_m, smem);
    store_bins(a.g.M, C, static_cast<int64_t>(a.Kp) * C, static_cast<int64_t>(i) * C, a.g.tw_px, smem, a.rows);
}

// Column k = blockIdx.x: the KR column (Kp x C, contiguous) arrives by bulk
// copy; the wrap map places canvas row ci at grid row v and folds in the
// inverse scale; the transformed column KS[k] (Py x C, contiguous) leaves by
// one bulk store.
template <int E, int C, int MAXT = Fam<E>::max_threads, int MINB = 1, bool H16 = false, class FFT = GenericFft<E>>
__global__ void __launch_bounds__(MAXT, MINB) kspec_cols_kernel(KernelSpectraArgs a) {
    extern __shared__ __align__(128) unsigned char smraw[];
    const int Py = a.g.Py, cols = a.g.cols, Kp = a.Kp, R = a.R;
    const int k = blockIdx.x;
    float2* W = reinterpret_cast<float2*>(smraw);
    float2* Rb = W + static_cast<size_t>(Py) * C;
    uint64_t* bar = reinterpret_cast<uint64_t*>(Rb + static_cast<size_t>(Kp) * C);
    const uint32_t r_bytes = static_cast<uint32_t>(static_cast<size_t>(Kp) * C * sizeof(float2));
    const bool lead = threadIdx.x == 0;
    if (lead) {
        mbar_init(bar, 1);
        mbar_init_fence();
    }
    __syncthreads();  // barrier initialised before anyone waits on it
    if (lead) {
        bulk_load_checked(Rb, a.rows + static_cast<size_t>(k) * Kp * C, r_bytes, bar, smraw, a.err);
        const int later = k + a.ahead;
        if (later < cols) bulk_prefetch_l2(a.rows + static_cast<size_t>(later) * Kp * C, r_bytes);
    }
    if (__syncthreads_or(!mbar_wait(bar, 0, a.err))) return;
    const float sc = a.scale;
    for (int i = threadIdx.x; i < Py * C; i += blockDim.x) {
        const int v = i / C;
        const int c = i - v * C;
        const int ci = canvas_index(v, Py, R);
        W[i] = ci >= 0 ? cscale(Rb[ci * C + c], sc) : make_float2(0.0f, 0.0f);
    }
    __syncthreads();
    FFT::template run<C, false, MAXT>(a.g.plan_py, W);
    if constexpr (H16) {
        const float m = block_absmax(W, Py * C);
        const float sc = m > 0.0f ? kHalfTop / m : 1.0f;
        if (lead) a.kscale[k] = m > 0.0f ? m / kHalfTop : 1.0f;
        __half2* out = reinterpret_cast<__half2*>(a.spectra) + static_cast<size_t>(k) * Py * C;
        for (int i = threadIdx.x; i < Py * C; i += blockDim.x) out[i] = to_half2(W[i], sc);
        return;
    }
    fence_proxy_async_smem();
    __syncthreads();
    const uint32_t s_bytes = static_cast<uint32_t>(static_cast<size_t>(Py) * C * sizeof(float2));
    float2* sdst = a.spectra + static_cast<size_t>(k) * Py * C;
    if (lead && bulk_args_ok(sdst, W, s_bytes, smraw, a.err)) {
        bulk_copy_s2g(sdst, W, s_bytes);
        bulk_commit();
        bulk_wait_read();
    }
}

// Dynamic shared-memory opt-in, leaving 1 KB for a kernel's static arrays.
template <class F>
void set_smem(F f) {
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem - 1024);
}

// CTAs of `f` resident at once on the current device (the L2 prefetch distance).
template <class F>
int resident_ctas(F f, int threads, size_t smem) {
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, f, threads, smem) != cudaSuccess || per < 1) per = 1;
    return sms * per;
}

}  // namespace
}  // namespace ld
