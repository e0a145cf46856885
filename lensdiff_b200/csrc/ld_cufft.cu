// ld_cufft.cu — the comparator form (fft_form LD_FFT_CUFFT): the same PSF
// bank and frame chain with every transform done by cuFFT, the library the
// reference CUDA backend calls (LensDiffCuda.cu buildShiftedRawPsfOnCuda
// :3269-3378, makeImageSpectrum :2928-2953, convolveSpectrumToPlane
// :3038-3074).  Everything around the transforms stays as in the own chain:
// the pupil pre-pass, the lambda-rescale and shaping kernels, the spectral map
// and the composite, so the two forms differ only in how the FFTs are done.
//
// Layouts are cuFFT's natural row-major ones: raw PSF grids [b][S][S]
// complex; frame planes [c][Py][Px] real; half spectra [c][Py][Px/2+1].
#include <cufft.h>

#include <tuple>

#include "ld_internal.h"
#include "ld_pixel.cuh"

namespace ld {
namespace {

constexpr int kThreads = 256;

int blocks_for(size_t n) { return static_cast<int>(std::min<size_t>((n + kThreads - 1) / kThreads, 148 * 64)); }

// Pupil field embedded at offset (S - N_p) / 2 of wavelengths b0..b0+nb
// (the fill of psf_rows_kernel, every row).
__global__ void cf_psf_field_kernel(PsfBankArgs a, int b0, int nb, float2* grid) {
    const size_t SS = static_cast<size_t>(a.S) * a.S;
    const size_t total = SS * nb;
    const int np = a.pupil.size;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int bi = static_cast<int>(i / SS);
        const size_t r = i - bi * SS;
        const int Y = static_cast<int>(r / a.S), X = static_cast<int>(r - static_cast<size_t>(Y) * a.S);
        const int y = Y - a.off, x = X - a.off;
        float2 v = make_float2(0.0f, 0.0f);
        if (y >= 0 && y < np && x >= 0 && x < np) {
            const float4 q = a.pupil_pre[static_cast<size_t>(y) * np + x];
            if (q.x > 0.0f) {
                const WavelengthInfo* w = a.wl + b0 + bi;
                const float ph = (w->phase.enabled && q.w != 0.0f) ? q.y + w->phase.c[4] * q.z : 0.0f;
                if (ph == 0.0f) {
                    v = make_float2(q.x, 0.0f);
                } else {
                    float sn, cs;
                    sincosf(ph * 2.0f * kPiF, &sn, &cs);
                    v = make_float2(q.x * cs, q.x * sn);
                }
            }
        }
        grid[i] = v;
    }
}

// |F|^2 of the fftshifted window of every wavelength of the chunk (the drain
// of psf_cols_kernel), plus the FP64 energy when asked.  grid (wins, nb).
__global__ void __launch_bounds__(kThreads) cf_psf_window_kernel(PsfBankArgs a, int b0, const float2* grid) {
    const int bi = blockIdx.y;
    const int b = b0 + bi;
    const WavelengthInfo* w = a.wl + b;
    const int wn = w->win_n, w0 = w->win_x0, S = a.S;
    const float2* g = grid + static_cast<size_t>(bi) * S * S;
    float* outw = a.win + static_cast<size_t>(b) * a.win_stride * a.win_stride;
    double esum = 0.0;
    const size_t total = static_cast<size_t>(wn) * wn;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int wy = static_cast<int>(i / wn), wx = static_cast<int>(i - static_cast<size_t>(wy) * wn);
        int u = w0 + wx + a.half;
        if (u >= S) u -= S;
        int v = w0 + wy + a.half;
        if (v >= S) v -= S;
        const float2 f = g[static_cast<size_t>(v) * S + u];
        const float I = f.x * f.x + f.y * f.y;
        outw[static_cast<size_t>(wy) * a.win_stride + wx] = I;
        esum += I;
    }
    if (a.want_energy) {
        __shared__ double part[kThreads / 32];
        for (int o = 16; o > 0; o >>= 1) esum += __shfl_xor_sync(0xffffffffu, esum, o);
        if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = esum;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int k = 0; k < kThreads / 32; ++k) t += part[k];
            atomicAdd(&a.scalars[b].energy, t);
        }
    }
}

__device__ __forceinline__ int wrap_index(int g, int P, int R) {
    if (g <= R) return g + R;
    if (g >= P - R) return g - P + R;
    return -1;
}

// RGB kernels wrapped with their centre at the origin of a Py x Px real
// plane each (paddedSpectrumFromKernel, LensDiffCpuReference.cpp:1153-1165),
// the inverse scale 1 / (Px Py) folded in.
__global__ void cf_kernel_place_kernel(KernelSpectraArgs a, float scale, float* planes) {
    const int Px = a.g.Px, Py = a.g.Py;
    const size_t P = static_cast<size_t>(Px) * Py;
    const size_t total = P * a.n_ker;
    const size_t kk = static_cast<size_t>(a.K) * a.K;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int k = static_cast<int>(i / P);
        const size_t r = i - k * P;
        const int y = static_cast<int>(r / Px), x = static_cast<int>(r - static_cast<size_t>(y) * Px);
        const int ci = wrap_index(y, Py, a.R), cj = wrap_index(x, Px, a.R);
        planes[i] = (ci >= 0 && cj >= 0) ? a.canvas[k * kk + static_cast<size_t>(ci) * a.K + cj] * scale : 0.0f;
    }
}

// Highlight extraction into n_drv zero-padded Py x Px driver planes.
__global__ void cf_extract_kernel(FrameArgs a, float* planes) {
    const int Px = a.g.Px, Py = a.g.Py;
    const size_t P = static_cast<size_t>(Px) * Py;
    const bool aligned = ((reinterpret_cast<uintptr_t>(a.src) | static_cast<uintptr_t>(a.src_pitch)) & 15) == 0;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < P;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int y = static_cast<int>(i / Px), x = static_cast<int>(i - static_cast<size_t>(y) * Px);
        float v[3] = {0.0f, 0.0f, 0.0f};
        if (y < a.H && x < a.W) {
            const float4 p = decode_px(a.transfer, load_px(a.src + static_cast<int64_t>(y) * a.src_pitch, x, aligned));
            float sig;
            const float m = selection_mask(a.sel, p.x, p.y, p.z, &sig) * a.sel.rscale;
            if (a.n_drv == 1) {
                v[0] = sig * m;
            } else {
                v[0] = p.x * m;
                v[1] = p.y * m;
                v[2] = p.z * m;
            }
        }
        for (int d = 0; d < a.n_drv; ++d) planes[d * P + i] = v[d];
    }
}

// Spectral multiply: spectral, out o = driver x kernel o; Mono, out d =
// driver d x the single kernel.  n = Py * (Px/2 + 1) bins per plane.
__global__ void cf_multiply_kernel(const float2* sd, const float2* ks, float2* prod, int n_out, int spectral,
                                   size_t n) {
    const size_t total = n * n_out;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int o = static_cast<int>(i / n);
        const size_t j = i - o * n;
        const float2 d = spectral ? sd[j] : sd[i];
        const float2 k = spectral ? ks[i] : ks[j];
        prod[i] = cmul(d, k);
    }
}

// Effect of output pixels from the C inverse planes: composited directly
// (kEffectComposite, render window rows) or stored with its luma sums
// (kEffectStore, every source pixel; composite_kernel finishes).
template <int C>
__global__ void __launch_bounds__(kThreads) cf_effect_kernel(FrameArgs a, const float* planes) {
    const size_t P = static_cast<size_t>(a.g.Px) * a.g.Py;
    const bool aligned_s = ((reinterpret_cast<uintptr_t>(a.src) | static_cast<uintptr_t>(a.src_pitch)) & 15) == 0;
    if (a.effect_mode == kEffectStore) {
        const int sy = blockIdx.x;
        const unsigned char* srow = a.src + static_cast<int64_t>(sy) * a.src_pitch;
        double l_in = 0.0, l_eff = 0.0;
        for (int sx = threadIdx.x; sx < a.W; sx += blockDim.x) {
            float e[C];
#pragma unroll
            for (int c = 0; c < C; ++c) e[c] = planes[c * P + static_cast<size_t>(sy) * a.g.Px + sx];
            const float3 m3 = map_effect<C>(a, e);
            a.effect[static_cast<int64_t>(sy) * a.W + sx] = make_float4(m3.x, m3.y, m3.z, 0.0f);
            const float4 p = decode_px(a.transfer, load_px(srow, sx, aligned_s));
            float sig;
            const float m = selection_mask(a.sel, p.x, p.y, p.z, &sig) * a.sel.rscale;
            l_in += static_cast<double>(luma(p.x * m, p.y * m, p.z * m));
            l_eff += static_cast<double>(luma(m3.x, m3.y, m3.z));
        }
        block_add2(l_in, l_eff, a.sums);
        return;
    }
    const int yo = a.out_y1 + blockIdx.x;
    const int sy = yo - a.src_y1;
    const bool have = sy >= 0 && sy < a.H;
    const bool aligned_d = ((reinterpret_cast<uintptr_t>(a.dst) | static_cast<uintptr_t>(a.dst_pitch)) & 15) == 0;
    const unsigned char* srow = a.src + static_cast<int64_t>(sy) * a.src_pitch;
    unsigned char* drow = a.dst + static_cast<int64_t>(yo - a.dst_y1) * a.dst_pitch;
    for (int x = a.out_x1 + threadIdx.x; x < a.out_x2; x += blockDim.x) {
        float4 out = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        const int sx = x - a.src_x1;
        if (have && sx >= 0 && sx < a.W) {
            float e[C];
#pragma unroll
            for (int c = 0; c < C; ++c) e[c] = planes[c * P + static_cast<size_t>(sy) * a.g.Px + sx];
            out = composite_px(a, decode_px(a.transfer, load_px(srow, sx, aligned_s)), map_effect<C>(a, e));
        }
        store_px(drow, x - a.dst_x1, aligned_d, encode_px(a.transfer, out));
    }
}

void check_cufft(cufftResult r, const char* what) {
    if (r != CUFFT_SUCCESS) throw CufftError{static_cast<int>(r), what};
}

}  // namespace

CufftPlanCache::~CufftPlanCache() { release(); }

void CufftPlanCache::release() {
    for (auto& kv : plans) cufftDestroy(kv.second);
    plans.clear();
}

int CufftPlanCache::get(int type, int ny, int nx, int batch) {
    const auto key = std::make_tuple(type, ny, nx, batch);
    auto it = plans.find(key);
    if (it != plans.end()) return it->second;
    cufftHandle h = 0;
    int n[2] = {ny, nx};
    check_cufft(cufftPlanMany(&h, 2, n, nullptr, 1, 0, nullptr, 1, 0, static_cast<cufftType>(type), batch),
                "cufft-plan");
    plans[key] = h;
    return h;
}

size_t cf_psf_chunk(int S, int B) {
    const size_t per = static_cast<size_t>(S) * S * sizeof(float2);
    const size_t cap = std::max<size_t>(1, (size_t(1) << 30) / per);
    return std::min<size_t>(cap, static_cast<size_t>(B));
}

void cf_psf_transform(const PsfBankArgs& a, float2* grid, CufftPlanCache& plans, cudaStream_t s) {
    const int chunk = static_cast<int>(cf_psf_chunk(a.S, a.B));
    for (int b0 = 0; b0 < a.B; b0 += chunk) {
        const int nb = std::min(chunk, a.B - b0);
        const size_t total = static_cast<size_t>(a.S) * a.S * nb;
        cf_psf_field_kernel<<<blocks_for(total), kThreads, 0, s>>>(a, b0, nb, grid);
        const cufftHandle h = plans.get(CUFFT_C2C, a.S, a.S, nb);
        check_cufft(cufftSetStream(h, s), "cufft-stream");
        check_cufft(cufftExecC2C(h, reinterpret_cast<cufftComplex*>(grid), reinterpret_cast<cufftComplex*>(grid),
                                 CUFFT_FORWARD),
                    "cufft-psf");
        const int wins = std::max(1, std::min(1024, (a.win_stride * a.win_stride + kThreads - 1) / kThreads));
        cf_psf_window_kernel<<<dim3(wins, nb), kThreads, 0, s>>>(a, b0, grid);
    }
}

void cf_kernel_spectra(const KernelSpectraArgs& a, float* planes, CufftPlanCache& plans, cudaStream_t s) {
    const size_t P = static_cast<size_t>(a.g.Px) * a.g.Py;
    const float scale = static_cast<float>(1.0 / (static_cast<double>(a.g.Px) * a.g.Py));
    cf_kernel_place_kernel<<<blocks_for(P * a.n_ker), kThreads, 0, s>>>(a, scale, planes);
    const cufftHandle h = plans.get(CUFFT_R2C, a.g.Py, a.g.Px, a.n_ker);
    check_cufft(cufftSetStream(h, s), "cufft-stream");
    check_cufft(cufftExecR2C(h, planes, reinterpret_cast<cufftComplex*>(a.spectra)), "cufft-kernel-spectra");
}

void cf_frame_forward(const FrameArgs& a, float* planes, float2* sd, CufftPlanCache& plans, cudaStream_t s) {
    const size_t P = static_cast<size_t>(a.g.Px) * a.g.Py;
    cf_extract_kernel<<<blocks_for(P), kThreads, 0, s>>>(a, planes);
    const cufftHandle h = plans.get(CUFFT_R2C, a.g.Py, a.g.Px, a.n_drv);
    check_cufft(cufftSetStream(h, s), "cufft-stream");
    check_cufft(cufftExecR2C(h, planes, reinterpret_cast<cufftComplex*>(sd)), "cufft-frame-forward");
}

void cf_frame_multiply(const FrameArgs& a, const float2* sd, float2* prod, cudaStream_t s) {
    const size_t n = static_cast<size_t>(a.g.Py) * (a.g.Px / 2 + 1);
    cf_multiply_kernel<<<blocks_for(n * a.n_out), kThreads, 0, s>>>(sd, a.spectra, prod, a.n_out, a.n_drv == 1, n);
}

void cf_frame_inverse(const FrameArgs& a, float2* prod, float* planes, CufftPlanCache& plans, cudaStream_t s) {
    const cufftHandle h = plans.get(CUFFT_C2R, a.g.Py, a.g.Px, a.n_out);
    check_cufft(cufftSetStream(h, s), "cufft-stream");
    check_cufft(cufftExecC2R(h, reinterpret_cast<cufftComplex*>(prod), planes), "cufft-frame-inverse");
    const int rows = a.effect_mode == kEffectStore ? a.H : a.out_y2 - a.out_y1;
    if (rows <= 0) return;
    if (a.n_out == 4) cf_effect_kernel<4><<<rows, kThreads, 0, s>>>(a, planes);
    else cf_effect_kernel<3><<<rows, kThreads, 0, s>>>(a, planes);
}

}  // namespace ld
