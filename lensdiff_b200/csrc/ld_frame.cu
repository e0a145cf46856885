// ld_frame.cu — per-frame FFT convolution chain and kernel-spectrum build.
//
// Reference stages (LensDiffCpuReference.cpp):
//   buildSelectionMask / applyMask / applyMaskScalarDriver :1219-1279
//       -> fused into the first stage of frame_rows_kernel
//   convolveScalar / paddedSpectrumFromKernel / convolveRgba :1153-1217
//       -> frame_rows_kernel (forward rows, real input)
//          frame_cols_kernel (forward columns, spectral multiply, inverse columns)
//          frame_inverse_kernel (inverse rows, real output)
//   MapLensDiffSpectralBins (LensDiffSpectrum.cpp:462-497), composite
//   (:2200-2218) -> frame_inverse_kernel epilogue
//
// Layout in HBM: row spectra A[ch][y][u] and column outputs B[o][y][u] are
// row-major with a padded width Pw (a multiple of the 4-column tile) holding the
// Px/2+1 non-redundant bins of a real row; kernel spectra are stored per column
// tile, KS[k][tile][v][4], so the column pass streams them contiguously.
#include <algorithm>

#include "ld_internal.h"

namespace ld {
namespace {

constexpr int C4 = kColTile;

__device__ __forceinline__ float saturate(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

// buildSelectionMask per pixel (LensDiffCpuReference.cpp:1225-1245).
__device__ __forceinline__ float selection_mask(const SelectionParams& s, float r, float g, float b, float* signal) {
    const float maxrgb = fmaxf(fmaxf(r, g), b);
    const float sig = s.luma ? 0.2126f * r + 0.7152f * g + 0.0722f * b : maxrgb;
    *signal = sig;
    float gate = 0.0f;
    if (sig > 0.0f) {
        const float stops = log2f(fmaxf(sig, 1e-6f) / 0.18f);
        const float t = saturate((stops - s.edge0) / fmaxf(s.edge1 - s.edge0, 1e-4f));
        gate = t * t * (3.0f - 2.0f * t);
    }
    const float boost = 1.0f + s.point_emphasis * fmaxf(0.0f, maxrgb / fmaxf(s.thr_linear, 1e-4f) - 1.0f);
    return saturate(gate * boost);
}

__device__ __forceinline__ float4 load_px(const unsigned char* row, int x, bool aligned) {
    if (aligned) return __ldg(reinterpret_cast<const float4*>(row) + x);
    const float* p = reinterpret_cast<const float*>(row) + 4 * x;
    return make_float4(__ldg(p), __ldg(p + 1), __ldg(p + 2), __ldg(p + 3));
}

// Driver value of one pixel for channel `ch`: the scalar driver
// (signal * mask * scale) for spectral modes, the redistributed colour
// src_c * (mask * scale) for Mono.
__device__ __forceinline__ float driver_value(const FrameArgs& a, float4 p, int ch) {
    float sig;
    const float m = selection_mask(a.sel, p.x, p.y, p.z, &sig);
    if (a.n_drv == 1) return sig * m * a.sel.rscale;
    const float mm = m * a.sel.rscale;
    return (ch == 0 ? p.x : (ch == 1 ? p.y : p.z)) * mm;
}

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

// ---- forward rows ------------------------------------------------------------------
// grid H, smem M * NCH float2.  Element n of the half-length complex sequence is
// (driver[2n], driver[2n+1]); pixels past W are the zero padding.
template <int T, int NMAX, int NCH>
__global__ void __launch_bounds__(T) frame_rows_kernel(FrameArgs a) {
    extern __shared__ float2 smem[];
    const int y = blockIdx.x;
    const unsigned char* row = a.src + static_cast<int64_t>(y) * a.src_pitch;
    const bool aligned = ((reinterpret_cast<uintptr_t>(a.src) | static_cast<uintptr_t>(a.src_pitch)) & 15) == 0;
    const int W = a.W;
    smem_fill<T, NCH>(smem, a.g.M, [&](int idx, int col) -> float2 {
        const int x0 = 2 * idx;
        float v0 = 0.0f, v1 = 0.0f;
        if (x0 < W) v0 = driver_value(a, load_px(row, x0, aligned), col);
        if (x0 + 1 < W) v1 = driver_value(a, load_px(row, x0 + 1, aligned), col);
        return make_float2(v0, v1);
    });
    fft_run<T, NCH, NMAX, false>(a.g.plan_m, smem);
    const int M = a.g.M, Pw = a.g.Pw;
    for (int k = threadIdx.x; k < Pw; k += T) {
#pragma unroll
        for (int ch = 0; ch < NCH; ++ch) {
            float2 v = make_float2(0.0f, 0.0f);
            if (k <= M) {
                const float2 zk = smem[(k == M ? 0 : k) * NCH + ch];
                const float2 zmk = smem[(k == 0 ? 0 : M - k) * NCH + ch];
                v = r2c_post(zk, zmk, __ldg(&a.g.tw_px[k]));
            }
            a.A[(static_cast<size_t>(ch) * a.H + y) * Pw + k] = v;
        }
    }
}

// ---- column pass: forward, multiply by kernel spectra, inverse -----------------------
// Persistent grid; CTA `blockIdx.x` walks column tiles and keeps the forward
// column spectrum of its tile in its own scratch slot (L2 resident).
template <int T, int NMAX>
__global__ void __launch_bounds__(T) frame_cols_kernel(FrameArgs a) {
    extern __shared__ float2 smem[];
    const int Py = a.g.Py, Pw = a.g.Pw, H = a.H;
    float2* scratch = a.scratch + static_cast<size_t>(blockIdx.x) * Py * C4;
    const int n = Py * C4;
    for (int tile = blockIdx.x; tile < a.g.tiles; tile += gridDim.x) {
        const int u0 = tile * C4;
        for (int o = 0; o < a.n_out; ++o) {
            const int d = a.n_drv == 1 ? 0 : o;
            const int k = a.n_ker == 1 ? 0 : o;
            const float2* ks = a.spectra + (static_cast<size_t>(k) * a.g.tiles + tile) * Py * C4;
            if (o == 0 || a.n_drv > 1) {
                const float2* Ad = a.A + static_cast<size_t>(d) * H * Pw + u0;
                smem_fill<T, C4>(smem, Py, [&](int v, int col) -> float2 {
                    return v < H ? __ldcs(&Ad[static_cast<size_t>(v) * Pw + col]) : make_float2(0.0f, 0.0f);
                });
                fft_run<T, C4, NMAX, false>(a.g.plan_py, smem);
                // keep the forward spectrum for the other outputs, multiply in place
                const bool keep = a.n_drv == 1 && a.n_out > 1;
                for (int i = threadIdx.x; i < n; i += T) {
                    const float2 dv = smem[i];
                    if (keep) scratch[i] = dv;
                    smem[i] = cmul(dv, __ldcs(&ks[i]));
                }
                __syncthreads();
            } else {
                smem_fill<T, C4>(smem, Py, [&](int v, int col) -> float2 {
                    const int i = v * C4 + col;
                    return cmul(scratch[i], __ldcs(&ks[i]));
                });
            }
            fft_run<T, C4, NMAX, true>(a.g.plan_py, smem);
            float2* Bo = a.Bout + static_cast<size_t>(o) * H * Pw + u0;
            for (int i = threadIdx.x; i < H * C4; i += T) {
                const int v = i / C4, col = i % C4;
                __stcs(&Bo[static_cast<size_t>(v) * Pw + col], smem[i]);
            }
            __syncthreads();
        }
    }
}

// ---- inverse rows + spectral map + composite ----------------------------------------
// grid = output rows, smem M * C float2 (C = n_out interleaved channels).
template <int T, int NMAX, int C>
__global__ void __launch_bounds__(T) frame_inverse_kernel(FrameArgs a) {
    extern __shared__ float2 smem[];
    const int yo = a.out_y1 + blockIdx.x;
    const int sy = yo - a.src_y1;
    const bool have = sy >= 0 && sy < a.H;
    const int M = a.g.M, Pw = a.g.Pw;
    if (have) {
        const float2* Brow = a.Bout + static_cast<size_t>(sy) * Pw;
        const size_t plane = static_cast<size_t>(a.H) * Pw;
        smem_fill<T, C>(smem, M, [&](int k, int col) -> float2 {
            const float2* p = Brow + col * plane;
            return c2r_pre(__ldcs(&p[k]), __ldcs(&p[M - k]), __ldg(&a.g.tw_px[k]));
        });
        fft_run<T, C, NMAX, true>(a.g.plan_m, smem);
    }
    const bool aligned_s = ((reinterpret_cast<uintptr_t>(a.src) | static_cast<uintptr_t>(a.src_pitch)) & 15) == 0;
    const bool aligned_d = ((reinterpret_cast<uintptr_t>(a.dst) | static_cast<uintptr_t>(a.dst_pitch)) & 15) == 0;
    const unsigned char* srow = a.src + static_cast<int64_t>(sy) * a.src_pitch;
    unsigned char* drow = a.dst + static_cast<int64_t>(yo - a.dst_y1) * a.dst_pitch;
    for (int x = a.out_x1 + threadIdx.x; x < a.out_x2; x += T) {
        float4 out = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        const int sx = x - a.src_x1;
        if (have && sx >= 0 && sx < a.W) {
            const int n = sx >> 1;
            const bool odd = sx & 1;
            float e[C];
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const float2 z = smem[n * C + c];
                e[c] = odd ? z.y : z.x;
            }
            float r, g, b;
            if (a.mono) {
                r = fmaxf(0.0f, e[0]);
                g = fmaxf(0.0f, e[1]);
                b = fmaxf(0.0f, e[2]);
            } else {
                r = fmaxf(0.0f, e[0]);
                g = fmaxf(0.0f, e[1]);
                b = fmaxf(0.0f, e[2]);
                if (a.saturation != 1.0f) {
                    const float gray = 0.2126f * r + 0.7152f * g + 0.0722f * b;
                    r = gray + (r - gray) * a.saturation;
                    g = gray + (g - gray) * a.saturation;
                    b = gray + (b - gray) * a.saturation;
                }
                if (C == 4 && a.luma_lock) {
                    const float cur = 0.2126f * r + 0.7152f * g + 0.0722f * b;
                    if (cur > 1e-6f) {
                        const float sc = e[C - 1] / cur;
                        r *= sc;
                        g *= sc;
                        b *= sc;
                    }
                }
            }
            const float4 p = load_px(srow, sx, aligned_s);
            float sig;
            const float m = selection_mask(a.sel, p.x, p.y, p.z, &sig) * a.sel.rscale;
            const float rr = p.x * m, rg = p.y * m, rb = p.z * m;
            out.x = fmaxf(fmaxf(0.0f, p.x - a.core_comp * rr + a.effect_gain * r), fmaxf(0.0f, p.x - rr * a.max_sub));
            out.y = fmaxf(fmaxf(0.0f, p.y - a.core_comp * rg + a.effect_gain * g), fmaxf(0.0f, p.y - rg * a.max_sub));
            out.z = fmaxf(fmaxf(0.0f, p.z - a.core_comp * rb + a.effect_gain * b), fmaxf(0.0f, p.z - rb * a.max_sub));
            out.w = p.w;
        }
        const int dx = x - a.dst_x1;
        if (aligned_d) {
            reinterpret_cast<float4*>(drow)[dx] = out;
        } else {
            float* q = reinterpret_cast<float*>(drow) + 4 * dx;
            q[0] = out.x;
            q[1] = out.y;
            q[2] = out.z;
            q[3] = out.w;
        }
    }
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

template <int T, int NMAX>
__global__ void __launch_bounds__(T) kspec_rows_kernel(KernelSpectraArgs a) {
    extern __shared__ float2 smem[];
    const int i = blockIdx.x;
    const int k = blockIdx.y;
    const float* crow = a.canvas + (static_cast<size_t>(k) * a.K + i) * a.K;
    const int Px = a.g.Px, R = a.R;
    smem_fill<T, 1>(smem, a.g.M, [&](int idx, int) -> float2 {
        const int j0 = canvas_index(2 * idx, Px, R);
        const int j1 = canvas_index(2 * idx + 1, Px, R);
        return make_float2(j0 >= 0 ? crow[j0] : 0.0f, j1 >= 0 ? crow[j1] : 0.0f);
    });
    fft_run<T, 1, NMAX, false>(a.g.plan_m, smem);
    const int M = a.g.M, Pw = a.g.Pw;
    float2* out = a.rows + (static_cast<size_t>(k) * a.K + i) * Pw;
    for (int u = threadIdx.x; u < Pw; u += T) {
        float2 v = make_float2(0.0f, 0.0f);
        if (u <= M) v = r2c_post(smem[u == M ? 0 : u], smem[u == 0 ? 0 : M - u], __ldg(&a.g.tw_px[u]));
        out[u] = v;
    }
}

template <int T, int NMAX>
__global__ void __launch_bounds__(T) kspec_cols_kernel(KernelSpectraArgs a) {
    extern __shared__ float2 smem[];
    const int tile = blockIdx.x;
    const int k = blockIdx.y;
    const int Py = a.g.Py, Pw = a.g.Pw, R = a.R;
    const int u0 = tile * C4;
    const float2* rows = a.rows + static_cast<size_t>(k) * a.K * Pw + u0;
    smem_fill<T, C4>(smem, Py, [&](int v, int col) -> float2 {
        const int i = canvas_index(v, Py, R);
        return i >= 0 ? rows[static_cast<size_t>(i) * Pw + col] : make_float2(0.0f, 0.0f);
    });
    fft_run<T, C4, NMAX, false>(a.g.plan_py, smem);
    float2* out = a.spectra + (static_cast<size_t>(k) * a.g.tiles + tile) * Py * C4;
    const float sc = a.scale;
    for (int i = threadIdx.x; i < Py * C4; i += T) out[i] = cscale(smem[i], sc);
}

// ---- launch tables ------------------------------------------------------------------
template <class F>
void set_smem(F f, size_t bytes) {
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
}

}  // namespace

// Row transforms: length M = Px/2 (<= 6912).  Column transforms: Py (<= 6912);
// 6912 x 4 interleaved float2 is the largest tile that fits 227 KB of shared memory.
void launch_frame_rows(const FrameArgs& a, cudaStream_t s) {
    const int M = a.g.M;
    const dim3 grid(a.H);
    if (a.n_drv == 1) {
        const size_t sm = static_cast<size_t>(M) * sizeof(float2);
        if (M <= 1024) frame_rows_kernel<64, 1024, 1><<<grid, 64, sm, s>>>(a);
        else if (M <= 2048) frame_rows_kernel<128, 2048, 1><<<grid, 128, sm, s>>>(a);
        else if (M <= 4096) frame_rows_kernel<256, 4096, 1><<<grid, 256, sm, s>>>(a);
        else frame_rows_kernel<512, 8192, 1><<<grid, 512, sm, s>>>(a);
    } else {
        const size_t sm = static_cast<size_t>(M) * 3 * sizeof(float2);
        if (M <= 1024) frame_rows_kernel<192, 1024, 3><<<grid, 192, sm, s>>>(a);
        else if (M <= 2048) frame_rows_kernel<384, 2048, 3><<<grid, 384, sm, s>>>(a);
        else if (M <= 4096) frame_rows_kernel<768, 4096, 3><<<grid, 768, sm, s>>>(a);
        else frame_rows_kernel<1024, 6912, 3><<<grid, 1024, sm, s>>>(a);
    }
}

int column_pass_blocks_per_sm(int Py) {
    // dynamic shared memory per CTA is Py * 4 * 8 bytes; at most 227 KB per SM
    const size_t sm = static_cast<size_t>(Py) * C4 * sizeof(float2);
    int threads = Py <= 1024 ? 256 : (Py <= 2048 ? 512 : 1024);
    int by_smem = static_cast<int>((228u * 1024u) / (sm + 1024));
    int by_threads = 2048 / threads;
    return std::max(1, std::min(by_smem, by_threads));
}

void launch_frame_cols(const FrameArgs& a, cudaStream_t s) {
    const int Py = a.g.Py;
    const size_t sm = static_cast<size_t>(Py) * C4 * sizeof(float2);
    const dim3 grid(a.col_grid);
    if (Py <= 1024) frame_cols_kernel<256, 1024><<<grid, 256, sm, s>>>(a);
    else if (Py <= 2048) frame_cols_kernel<512, 2048><<<grid, 512, sm, s>>>(a);
    else if (Py <= 4096) frame_cols_kernel<1024, 4096><<<grid, 1024, sm, s>>>(a);
    else frame_cols_kernel<1024, 6912><<<grid, 1024, sm, s>>>(a);
}

void launch_frame_inverse(const FrameArgs& a, cudaStream_t s) {
    const int M = a.g.M;
    const int rows = a.out_y2 - a.out_y1;
    if (rows <= 0) return;
    const dim3 grid(rows);
    if (a.n_out == 4) {
        const size_t sm = static_cast<size_t>(M) * 4 * sizeof(float2);
        if (M <= 1024) frame_inverse_kernel<256, 1024, 4><<<grid, 256, sm, s>>>(a);
        else if (M <= 2048) frame_inverse_kernel<512, 2048, 4><<<grid, 512, sm, s>>>(a);
        else if (M <= 4096) frame_inverse_kernel<1024, 4096, 4><<<grid, 1024, sm, s>>>(a);
        else frame_inverse_kernel<1024, 6912, 4><<<grid, 1024, sm, s>>>(a);
    } else {
        const size_t sm = static_cast<size_t>(M) * 3 * sizeof(float2);
        if (M <= 1024) frame_inverse_kernel<192, 1024, 3><<<grid, 192, sm, s>>>(a);
        else if (M <= 2048) frame_inverse_kernel<384, 2048, 3><<<grid, 384, sm, s>>>(a);
        else if (M <= 4096) frame_inverse_kernel<768, 4096, 3><<<grid, 768, sm, s>>>(a);
        else frame_inverse_kernel<1024, 6912, 3><<<grid, 1024, sm, s>>>(a);
    }
}

void launch_kspec_rows(const KernelSpectraArgs& a, cudaStream_t s) {
    const int M = a.g.M;
    const dim3 grid(a.K, a.n_ker);
    const size_t sm = static_cast<size_t>(M) * sizeof(float2);
    if (M <= 1024) kspec_rows_kernel<64, 1024><<<grid, 64, sm, s>>>(a);
    else if (M <= 2048) kspec_rows_kernel<128, 2048><<<grid, 128, sm, s>>>(a);
    else if (M <= 4096) kspec_rows_kernel<256, 4096><<<grid, 256, sm, s>>>(a);
    else kspec_rows_kernel<512, 8192><<<grid, 512, sm, s>>>(a);
}

void launch_kspec_cols(const KernelSpectraArgs& a, cudaStream_t s) {
    const int Py = a.g.Py;
    const dim3 grid(a.g.tiles, a.n_ker);
    const size_t sm = static_cast<size_t>(Py) * C4 * sizeof(float2);
    if (Py <= 1024) kspec_cols_kernel<256, 1024><<<grid, 256, sm, s>>>(a);
    else if (Py <= 2048) kspec_cols_kernel<512, 2048><<<grid, 512, sm, s>>>(a);
    else if (Py <= 4096) kspec_cols_kernel<1024, 4096><<<grid, 1024, sm, s>>>(a);
    else kspec_cols_kernel<1024, 6912><<<grid, 1024, sm, s>>>(a);
}

void configure_psf_kernels();

void configure_kernels() {
    configure_psf_kernels();
    set_smem(frame_rows_kernel<512, 8192, 1>, 8192 * 8);
    set_smem(frame_rows_kernel<256, 4096, 1>, 4096 * 8);
    set_smem(frame_rows_kernel<1024, 6912, 3>, 6912 * 3 * 8);
    set_smem(frame_rows_kernel<768, 4096, 3>, 4096 * 3 * 8);
    set_smem(frame_rows_kernel<384, 2048, 3>, 2048 * 3 * 8);
    set_smem(frame_cols_kernel<256, 1024>, 1024 * C4 * 8);
    set_smem(frame_cols_kernel<512, 2048>, 2048 * C4 * 8);
    set_smem(frame_cols_kernel<1024, 4096>, 4096 * C4 * 8);
    set_smem(frame_cols_kernel<1024, 6912>, 6912 * C4 * 8);
    set_smem(frame_inverse_kernel<1024, 4096, 4>, 4096 * 4 * 8);
    set_smem(frame_inverse_kernel<1024, 6912, 4>, 6912 * 4 * 8);
    set_smem(frame_inverse_kernel<512, 2048, 4>, 2048 * 4 * 8);
    set_smem(frame_inverse_kernel<768, 4096, 3>, 4096 * 3 * 8);
    set_smem(frame_inverse_kernel<1024, 6912, 3>, 6912 * 3 * 8);
    set_smem(frame_inverse_kernel<384, 2048, 3>, 2048 * 3 * 8);
    set_smem(kspec_rows_kernel<512, 8192>, 8192 * 8);
    set_smem(kspec_rows_kernel<256, 4096>, 4096 * 8);
    set_smem(kspec_cols_kernel<256, 1024>, 1024 * C4 * 8);
    set_smem(kspec_cols_kernel<512, 2048>, 2048 * C4 * 8);
    set_smem(kspec_cols_kernel<1024, 4096>, 4096 * C4 * 8);
    set_smem(kspec_cols_kernel<1024, 6912>, 6912 * C4 * 8);
}

}  // namespace ld
