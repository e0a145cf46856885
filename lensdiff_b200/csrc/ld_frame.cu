// ld_frame.cu — per-frame FFT convolution chain and kernel-spectrum build.
//
// Reference stages (LensDiffCpuReference.cpp):
//   buildSelectionMask / applyMask / applyMaskScalarDriver :1219-1279
//       -> fused into the fill of frame_rows_kernel
//   convolveScalar / paddedSpectrumFromKernel / convolveRgba :1153-1217
//       -> frame_rows_kernel (forward rows, real input, two rows per CTA)
//          frame_cols_kernel (forward columns, spectral multiply, inverse columns)
//          frame_inverse_kernel (inverse rows, real output)
//   MapLensDiffSpectralBins (LensDiffSpectrum.cpp:462-497), composite
//   (:2200-2218) -> frame_inverse_kernel epilogue
//
// HBM layout (ld_internal.h): every array the column passes touch is stored
// tile-major, so one column tile is one contiguous block.  The column passes
// are persistent (one CTA per SM) and double-buffer their inputs: while a tile
// is transformed, the bulk-copy engine (cp.async.bulk, mbarrier completion)
// already streams the next tile's row spectra and kernel spectra into shared
// memory.
#include <algorithm>

#include "ld_async.cuh"
#include "ld_internal.h"

namespace ld {
namespace {

constexpr int kMaxSmem = 227 * 1024;

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

// Driver value of one pixel for plane `ch`: the scalar driver
// (signal * mask * scale) for spectral modes, the redistributed colour
// src_c * (mask * scale) for Mono.
__device__ __forceinline__ float driver_value(const SelectionParams& sel, int n_drv, float4 p, int ch) {
    float sig;
    const float m = selection_mask(sel, p.x, p.y, p.z, &sig);
    if (n_drv == 1) return sig * m * sel.rscale;
    const float mm = m * sel.rscale;
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

// Writes the Px/2+1 bins of two transformed rows (interleaved in smem as
// s[n*2 + r]) to a tile-major array out[t][row0 + r][kk] with k = t*ct + kk;
// bins past M are zero.  The two rows of one tile are 2*ct adjacent float2.
__device__ __forceinline__ void store_row_pair(int M, int ct, int Pw, const float2* __restrict__ tw_px,
                                               const float2* s, float2* out, int rows_total, int row0, int T) {
    for (int i = threadIdx.x; i < Pw * 2; i += T) {
        const int t = i / (2 * ct);
        const int rem = i - t * 2 * ct;
        const int r = rem / ct;
        const int kk = rem - r * ct;
        const int k = t * ct + kk;
        float2 v = make_float2(0.0f, 0.0f);
        if (k <= M) v = r2c_post(s[(k == M ? 0 : k) * 2 + r], s[(k == 0 ? 0 : M - k) * 2 + r], __ldg(&tw_px[k]));
        out[(static_cast<size_t>(t) * rows_total + row0 + r) * ct + kk] = v;
    }
}

// ---- forward rows: two rows per CTA -------------------------------------------------
// (The kernels copy what their fill/drain lambdas need into registers and
// capture by value: a lambda holding a reference to the kernel's parameter
// block would force a copy of the block into local memory.)
template <int T, int NMAX>
__global__ void __launch_bounds__(T, 1) frame_rows_kernel(FrameArgs a) {
    extern __shared__ float2 smem[];
    const int y0 = blockIdx.x * 2;
    const int64_t pitch = a.src_pitch;
    const bool aligned = ((reinterpret_cast<uintptr_t>(a.src) | static_cast<uintptr_t>(pitch)) & 15) == 0;
    const unsigned char* row0 = a.src + static_cast<int64_t>(y0) * pitch;
    const int W = a.W, H = a.H, n_drv = a.n_drv;
    const SelectionParams sel = a.sel;
    const FftPlan plan = a.g.plan_m;
    const int M = a.g.M, ct = a.g.ct, Pw = a.g.Pw, Hp = a.Hp;
    const float2* tw_px = a.g.tw_px;
    float2* A = a.A;
    const size_t plane = static_cast<size_t>(a.g.tiles) * Hp * ct;
    for (int d = 0; d < n_drv; ++d) {
        smem_fill<T, 2>(smem, M, [=](int idx, int r) -> float2 {
            if (y0 + r >= H) return make_float2(0.0f, 0.0f);
            const unsigned char* row = row0 + r * pitch;
            const int x0 = 2 * idx;
            float v0 = 0.0f, v1 = 0.0f;
            if (x0 < W) v0 = driver_value(sel, n_drv, load_px(row, x0, aligned), d);
            if (x0 + 1 < W) v1 = driver_value(sel, n_drv, load_px(row, x0 + 1, aligned), d);
            return make_float2(v0, v1);
        });
        fft_run<T, 2, NMAX, false>(plan, smem);
        store_row_pair(M, ct, Pw, tw_px, smem, A + d * plane, Hp, y0, T);
        __syncthreads();
    }
}

// ---- column pass: forward, multiply by kernel spectra, inverse -----------------------
// One CTA per SM walks column tiles.  Shared memory: W (work, Py x CT),
// D (forward spectrum kept for every output, spectral only), Abuf (next row-
// spectrum tile, Hp x CT), Kbuf (next kernel-spectrum tile, Py x CT), two
// mbarriers.  Thread 0 issues the bulk copies; everyone waits on the barriers.
template <int T, int CT, int NMAX>
__global__ void __launch_bounds__(T, 1) frame_cols_kernel(FrameArgs a) {
    extern __shared__ __align__(128) unsigned char smraw[];
    const int Py = a.g.Py, H = a.H, Hp = a.Hp, tiles = a.g.tiles;
    const int n = Py * CT;
    const int n_drv = a.n_drv, n_out = a.n_out;
    const bool spectral = n_drv == 1;
    const FftPlan plan = a.g.plan_py;
    const float2* Asrc = a.A;
    const float2* Ksrc = a.spectra;
    float2* Bdst = a.Bout;
    int* err = a.err;
    float2* W = reinterpret_cast<float2*>(smraw);
    float2* D = W + n;
    float2* Abuf = spectral ? D + n : W + n;
    float2* Kbuf = Abuf + Hp * CT;
    uint64_t* bars = reinterpret_cast<uint64_t*>(Kbuf + n);
    const uint32_t a_bytes = static_cast<uint32_t>(Hp * CT * sizeof(float2));
    const uint32_t k_bytes = static_cast<uint32_t>(n * sizeof(float2));
    int tile = blockIdx.x;
    if (tile >= tiles) return;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init_fence();
    }
    __syncthreads();
    auto a_src = [=](int t, int d) { return Asrc + (static_cast<size_t>(d) * tiles + t) * Hp * CT; };
    auto k_src = [=](int t, int k) { return Ksrc + (static_cast<size_t>(k) * tiles + t) * Py * CT; };
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(&bars[0], a_bytes);
        bulk_copy_g2s(Abuf, a_src(tile, 0), a_bytes, &bars[0]);
        mbar_arrive_expect_tx(&bars[1], k_bytes);
        bulk_copy_g2s(Kbuf, k_src(tile, 0), k_bytes, &bars[1]);
    }
    uint32_t pa = 0, pk = 0;
    for (; tile < tiles; tile += gridDim.x) {
        const int next = tile + gridDim.x;
        for (int o = 0; o < a.n_out; ++o) {
            if (o == 0 || !spectral) {
                const int d = spectral ? 0 : o;
                const bool ok = mbar_wait(&bars[0], pa, a.err);
                pa ^= 1u;
                if (__syncthreads_or(!ok)) return;
                float2* F = spectral ? D : W;
                const int filled = Hp * CT;
                for (int i = threadIdx.x; i < n; i += T) F[i] = i < filled ? Abuf[i] : make_float2(0.0f, 0.0f);
                __syncthreads();
                if (threadIdx.x == 0) {  // Abuf is free: stream the next plane / tile
                    int nt = tile, nd = d + 1;
                    if (nd >= a.n_drv) {
                        nt = next;
                        nd = 0;
                    }
                    if (nt < tiles) {
                        fence_proxy_async_smem();
                        mbar_arrive_expect_tx(&bars[0], a_bytes);
                        bulk_copy_g2s(Abuf, a_src(nt, nd), a_bytes, &bars[0]);
                    }
                }
                fft_run<T, CT, NMAX, false>(a.g.plan_py, F);
            }
            if (o == 0 || spectral) {
                const bool ok = mbar_wait(&bars[1], pk, a.err);
                pk ^= 1u;
                if (__syncthreads_or(!ok)) return;
            }
            if (spectral) {
                for (int i = threadIdx.x; i < n; i += T) W[i] = cmul(D[i], Kbuf[i]);
            } else {
                for (int i = threadIdx.x; i < n; i += T) W[i] = cmul(W[i], Kbuf[i]);
            }
            __syncthreads();
            if (threadIdx.x == 0) {  // Kbuf is free: stream the next kernel spectrum
                int nt = -1, nk = 0;
                if (spectral) {
                    if (o + 1 < a.n_out) {
                        nt = tile;
                        nk = o + 1;
                    } else {
                        nt = next;
                    }
                } else if (o + 1 == a.n_out) {
                    nt = next;
                }
                if (nt >= 0 && nt < tiles) {
                    fence_proxy_async_smem();
                    mbar_arrive_expect_tx(&bars[1], k_bytes);
                    bulk_copy_g2s(Kbuf, k_src(nt, nk), k_bytes, &bars[1]);
                }
            }
            fft_run<T, CT, NMAX, true>(a.g.plan_py, W);
            float2* Bo = a.Bout + (static_cast<size_t>(o) * tiles + tile) * H * CT;
            for (int i = threadIdx.x; i < H * CT; i += T) __stcs(&Bo[i], W[i]);
            __syncthreads();
        }
    }
}

// ---- inverse rows + spectral map + composite ----------------------------------------
// grid = output rows, smem M * C float2 (C = n_out interleaved channels).
template <int T, int NMAX, int C>
__global__ void __launch_bounds__(T, 1) frame_inverse_kernel(FrameArgs a) {
    extern __shared__ float2 smem[];
    const int yo = a.out_y1 + blockIdx.x;
    const int sy = yo - a.src_y1;
    const bool have = sy >= 0 && sy < a.H;
    const int M = a.g.M, ct = a.g.ct, tiles = a.g.tiles, H = a.H;
    if (have) {
        const float2* Bsrc = a.Bout;
        const float2* tw_px = a.g.tw_px;
        smem_fill<T, C>(smem, M, [=](int k, int col) -> float2 {
            const float2* p = Bsrc + (static_cast<size_t>(col) * tiles) * H * ct;
            const int km = M - k;
            const float2 xk = __ldcs(&p[(static_cast<size_t>(k / ct) * H + sy) * ct + k % ct]);
            const float2 xm = __ldcs(&p[(static_cast<size_t>(km / ct) * H + sy) * ct + km % ct]);
            return c2r_pre(xk, xm, __ldg(&tw_px[k]));
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
            const int nn = sx >> 1;
            const bool odd = sx & 1;
            float e[C];
#pragma unroll
            for (int c = 0; c < C; ++c) {
                const float2 z = smem[nn * C + c];
                e[c] = odd ? z.y : z.x;
            }
            float r = fmaxf(0.0f, e[0]);
            float g = fmaxf(0.0f, e[1]);
            float b = fmaxf(0.0f, e[2]);
            if (!a.mono) {
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

// grid (Kp/2, n_ker): two canvas rows per CTA -> KR tile-major.
template <int T, int NMAX>
__global__ void __launch_bounds__(T, 1) kspec_rows_kernel(KernelSpectraArgs a) {
    extern __shared__ float2 smem[];
    const int i0 = blockIdx.x * 2;
    const int k = blockIdx.y;
    const int Px = a.g.Px, R = a.R, K = a.K;
    const float* canvas = a.canvas + static_cast<size_t>(k) * K * K;
    smem_fill<T, 2>(smem, a.g.M, [=](int idx, int r) -> float2 {
        const int i = i0 + r;
        if (i >= K) return make_float2(0.0f, 0.0f);
        const float* crow = canvas + static_cast<size_t>(i) * K;
        const int j0 = canvas_index(2 * idx, Px, R);
        const int j1 = canvas_index(2 * idx + 1, Px, R);
        return make_float2(j0 >= 0 ? crow[j0] : 0.0f, j1 >= 0 ? crow[j1] : 0.0f);
    });
    fft_run<T, 2, NMAX, false>(a.g.plan_m, smem);
    store_row_pair(a.g.M, a.g.ct, a.g.Pw, a.g.tw_px, smem,
                   a.rows + static_cast<size_t>(k) * a.g.tiles * a.Kp * a.g.ct, a.Kp, i0, T);
}

// Persistent: CTA walks (kernel, tile) items; the next item's KR tile streams
// into shared memory while the current one is transformed.
template <int T, int CT, int NMAX>
__global__ void __launch_bounds__(T, 1) kspec_cols_kernel(KernelSpectraArgs a) {
    extern __shared__ __align__(128) unsigned char smraw[];
    const int Py = a.g.Py, tiles = a.g.tiles, Kp = a.Kp, R = a.R;
    const int n = Py * CT;
    float2* W = reinterpret_cast<float2*>(smraw);
    float2* Rbuf = W + n;
    uint64_t* bar = reinterpret_cast<uint64_t*>(Rbuf + Kp * CT);
    const uint32_t r_bytes = static_cast<uint32_t>(Kp * CT * sizeof(float2));
    const int items = a.n_ker * tiles;
    int item = blockIdx.x;
    if (item >= items) return;
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_init_fence();
    }
    __syncthreads();
    const float2* rows = a.rows;
    auto r_src = [=](int it) { return rows + static_cast<size_t>(it) * Kp * CT; };  // [k][t] == item order
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(bar, r_bytes);
        bulk_copy_g2s(Rbuf, r_src(item), r_bytes, bar);
    }
    uint32_t ph = 0;
    for (; item < items; item += gridDim.x) {
        const bool ok = mbar_wait(bar, ph, a.err);
        ph ^= 1u;
        if (__syncthreads_or(!ok)) return;
        for (int i = threadIdx.x; i < n; i += T) {
            const int v = i / CT, col = i - (i / CT) * CT;
            const int ci = canvas_index(v, Py, R);
            W[i] = ci >= 0 ? Rbuf[ci * CT + col] : make_float2(0.0f, 0.0f);
        }
        __syncthreads();
        const int nxt = item + gridDim.x;
        if (threadIdx.x == 0 && nxt < items) {
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(bar, r_bytes);
            bulk_copy_g2s(Rbuf, r_src(nxt), r_bytes, bar);
        }
        fft_run<T, CT, NMAX, false>(a.g.plan_py, W);
        float2* out = a.spectra + static_cast<size_t>(item) * Py * CT;  // [k][t][v][CT]
        const float sc = a.scale;
        for (int i = threadIdx.x; i < n; i += T) out[i] = cscale(W[i], sc);
        __syncthreads();
    }
}

template <class F>
void set_smem(F f) {
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmem);
}

}  // namespace

size_t frame_cols_smem(const FrameArgs& a) {
    const size_t n = static_cast<size_t>(a.g.Py) * a.g.ct;
    const size_t bufs = (a.n_drv == 1 ? 3 : 2) * n + static_cast<size_t>(a.Hp) * a.g.ct;
    return bufs * sizeof(float2) + 2 * sizeof(uint64_t);
}

size_t kspec_cols_smem(const GridGeom& g, int Kp) {
    return (static_cast<size_t>(g.Py) + Kp) * g.ct * sizeof(float2) + sizeof(uint64_t);
}

int frame_cols_threads(int Py) { return Py <= 1024 ? 256 : (Py <= 2048 ? 512 : 1024); }

// Row transforms: two rows per CTA, length M = Px/2 <= 6912.
void launch_frame_rows(const FrameArgs& a, cudaStream_t s) {
    const int M = a.g.M;
    const dim3 grid(a.Hp / 2);
    const size_t sm = static_cast<size_t>(M) * 2 * sizeof(float2);
    if (M <= 1024) frame_rows_kernel<256, 1024><<<grid, 256, sm, s>>>(a);
    else if (M <= 2048) frame_rows_kernel<512, 2048><<<grid, 512, sm, s>>>(a);
    else if (M <= 4096) frame_rows_kernel<1024, 4096><<<grid, 1024, sm, s>>>(a);
    else frame_rows_kernel<1024, 6912><<<grid, 1024, sm, s>>>(a);
}

template <int CT>
static void cols_launch_ct(const FrameArgs& a, cudaStream_t s) {
    const int Py = a.g.Py;
    const size_t sm = frame_cols_smem(a);
    const dim3 grid(a.col_grid);
    if (Py <= 1024) frame_cols_kernel<256, CT, 1024><<<grid, 256, sm, s>>>(a);
    else if (Py <= 2048) frame_cols_kernel<512, CT, 2048><<<grid, 512, sm, s>>>(a);
    else if (Py <= 4096) frame_cols_kernel<1024, CT, 4096><<<grid, 1024, sm, s>>>(a);
    else frame_cols_kernel<1024, CT, 6912><<<grid, 1024, sm, s>>>(a);
}

void launch_frame_cols(const FrameArgs& a, cudaStream_t s) {
    if (a.g.ct == 2) cols_launch_ct<2>(a, s);
    else cols_launch_ct<1>(a, s);
}

void launch_frame_inverse(const FrameArgs& a, cudaStream_t s) {
    const int M = a.g.M;
    const int rows = a.out_y2 - a.out_y1;
    if (rows <= 0) return;
    const dim3 grid(rows);
    if (a.n_out == 4) {
        const size_t sm = static_cast<size_t>(M) * 4 * sizeof(float2);
        if (M <= 1024) frame_inverse_kernel<512, 1024, 4><<<grid, 512, sm, s>>>(a);
        else if (M <= 2048) frame_inverse_kernel<1024, 2048, 4><<<grid, 1024, sm, s>>>(a);
        else if (M <= 4096) frame_inverse_kernel<1024, 4096, 4><<<grid, 1024, sm, s>>>(a);
        else frame_inverse_kernel<1024, 6912, 4><<<grid, 1024, sm, s>>>(a);
    } else {
        const size_t sm = static_cast<size_t>(M) * 3 * sizeof(float2);
        if (M <= 1024) frame_inverse_kernel<384, 1024, 3><<<grid, 384, sm, s>>>(a);
        else if (M <= 2048) frame_inverse_kernel<768, 2048, 3><<<grid, 768, sm, s>>>(a);
        else if (M <= 4096) frame_inverse_kernel<1024, 4096, 3><<<grid, 1024, sm, s>>>(a);
        else frame_inverse_kernel<1024, 6912, 3><<<grid, 1024, sm, s>>>(a);
    }
}

void launch_kspec_rows(const KernelSpectraArgs& a, cudaStream_t s) {
    const int M = a.g.M;
    const dim3 grid(a.Kp / 2, a.n_ker);
    const size_t sm = static_cast<size_t>(M) * 2 * sizeof(float2);
    if (M <= 1024) kspec_rows_kernel<256, 1024><<<grid, 256, sm, s>>>(a);
    else if (M <= 2048) kspec_rows_kernel<512, 2048><<<grid, 512, sm, s>>>(a);
    else if (M <= 4096) kspec_rows_kernel<1024, 4096><<<grid, 1024, sm, s>>>(a);
    else kspec_rows_kernel<1024, 6912><<<grid, 1024, sm, s>>>(a);
}

template <int CT>
static void kcols_launch_ct(const KernelSpectraArgs& a, cudaStream_t s) {
    const int Py = a.g.Py;
    const size_t sm = kspec_cols_smem(a.g, a.Kp);
    const dim3 grid(a.grid);
    if (Py <= 1024) kspec_cols_kernel<256, CT, 1024><<<grid, 256, sm, s>>>(a);
    else if (Py <= 2048) kspec_cols_kernel<512, CT, 2048><<<grid, 512, sm, s>>>(a);
    else if (Py <= 4096) kspec_cols_kernel<1024, CT, 4096><<<grid, 1024, sm, s>>>(a);
    else kspec_cols_kernel<1024, CT, 6912><<<grid, 1024, sm, s>>>(a);
}

void launch_kspec_cols(const KernelSpectraArgs& a, cudaStream_t s) {
    if (a.g.ct == 2) kcols_launch_ct<2>(a, s);
    else kcols_launch_ct<1>(a, s);
}

void configure_psf_kernels();

template <int CT>
static void configure_ct() {
    set_smem(frame_cols_kernel<256, CT, 1024>);
    set_smem(frame_cols_kernel<512, CT, 2048>);
    set_smem(frame_cols_kernel<1024, CT, 4096>);
    set_smem(frame_cols_kernel<1024, CT, 6912>);
    set_smem(kspec_cols_kernel<256, CT, 1024>);
    set_smem(kspec_cols_kernel<512, CT, 2048>);
    set_smem(kspec_cols_kernel<1024, CT, 4096>);
    set_smem(kspec_cols_kernel<1024, CT, 6912>);
}

void configure_kernels() {
    configure_psf_kernels();
    set_smem(frame_rows_kernel<256, 1024>);
    set_smem(frame_rows_kernel<512, 2048>);
    set_smem(frame_rows_kernel<1024, 4096>);
    set_smem(frame_rows_kernel<1024, 6912>);
    configure_ct<2>();
    configure_ct<1>();
    set_smem(frame_inverse_kernel<512, 1024, 4>);
    set_smem(frame_inverse_kernel<1024, 2048, 4>);
    set_smem(frame_inverse_kernel<1024, 4096, 4>);
    set_smem(frame_inverse_kernel<1024, 6912, 4>);
    set_smem(frame_inverse_kernel<384, 1024, 3>);
    set_smem(frame_inverse_kernel<768, 2048, 3>);
    set_smem(frame_inverse_kernel<1024, 4096, 3>);
    set_smem(frame_inverse_kernel<1024, 6912, 3>);
    set_smem(kspec_rows_kernel<256, 1024>);
    set_smem(kspec_rows_kernel<512, 2048>);
    set_smem(kspec_rows_kernel<1024, 4096>);
    set_smem(kspec_rows_kernel<1024, 6912>);
}

}  // namespace ld
