// ld_pixel.cuh — per-pixel device functions shared by the frame chains:
// highlight extraction, the spectral map of the effect, the composite, and a
// two-value block reduction.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ld_internal.h"

namespace ld {

__device__ __forceinline__ float saturate(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

// buildSelectionMask per pixel (LensDiffCpuReference.cpp:1225-1245).  A
// non-positive signal gives a zero gate; so does one whose clamped value
// max(sig, 1e-6) is at or below s.sig_zero (its stops lie below edge0, t = 0)
// whatever the boost: such pixels (most of a frame) return at once.
__device__ __forceinline__ float selection_mask(const SelectionParams& s, float r, float g, float b, float* signal) {
    const float maxrgb = fmaxf(fmaxf(r, g), b);
    const float sig = s.luma ? 0.2126f * r + 0.7152f * g + 0.0722f * b : maxrgb;
    *signal = sig;
    if (sig <= 0.0f || fmaxf(sig, 1e-6f) <= s.sig_zero) return 0.0f;
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

// DaVinci Intermediate, Blackmagic's published log encoding: the decode the
// reference applies as it loads the source (ColorManagement.cpp:168-169 via
// loadSourceRgba, LensDiffCpuReference.cpp:174-192) and the encode of its
// final pixels (LensDiffTransfer.cpp:8-20, LensDiffCpuReference.cpp:2248-2250).
__device__ __forceinline__ float davinci_decode(float x) {
    return x <= 0.02740668f ? x / 10.44426855f : exp2f(x / 0.07329248f - 7.0f) - 0.0075f;
}
__device__ __forceinline__ float davinci_encode(float x) {
    return x <= 0.00262409f ? x * 10.44426855f : (log2f(fmaxf(x, 0.0f) + 0.0075f) + 7.0f) * 0.07329248f;
}
// Source pixel in linear light (alpha untouched).
__device__ __forceinline__ float4 decode_px(int transfer, float4 p) {
    if (transfer == kTransferDavinci) {
        p.x = davinci_decode(p.x);
        p.y = davinci_decode(p.y);
        p.z = davinci_decode(p.z);
    }
    return p;
}
// Output pixel in the source's encoding (alpha untouched).
__device__ __forceinline__ float4 encode_px(int transfer, float4 p) {
    if (transfer == kTransferDavinci) {
        p.x = davinci_encode(p.x);
        p.y = davinci_encode(p.y);
        p.z = davinci_encode(p.z);
    }
    return p;
}

// MapLensDiffSpectralBins (LensDiffSpectrum.cpp:462-497) on one pixel whose
// C channel values are e[0..C): clamp, saturation, luma lock.
template <int C>
__device__ __forceinline__ float3 map_effect(const FrameArgs& a, const float* e) {
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
    return make_float3(r, g, b);
}

// Final composite of one pixel (LensDiffCpuReference.cpp:2200-2218): the
// effect is already multiplied by its energy scale.
// `rd`: the redistributed source at the pixel (src * mask * (1 - corePreserve)).
__device__ __forceinline__ float4 composite_rd(const FrameArgs& a, float4 p, float3 rd, float3 eff) {
    const float rr = rd.x, rg = rd.y, rb = rd.z;
    float4 out;
    out.x = fmaxf(fmaxf(0.0f, p.x - a.core_comp * rr + a.effect_gain * eff.x), fmaxf(0.0f, p.x - rr * a.max_sub));
    out.y = fmaxf(fmaxf(0.0f, p.y - a.core_comp * rg + a.effect_gain * eff.y), fmaxf(0.0f, p.y - rg * a.max_sub));
    out.z = fmaxf(fmaxf(0.0f, p.z - a.core_comp * rb + a.effect_gain * eff.z), fmaxf(0.0f, p.z - rb * a.max_sub));
    out.w = p.w;
    return out;
}

__device__ __forceinline__ float3 redistributed(const FrameArgs& a, float4 p) {
    float sig;
    const float m = selection_mask(a.sel, p.x, p.y, p.z, &sig) * a.sel.rscale;
    return make_float3(p.x * m, p.y * m, p.z * m);
}

__device__ __forceinline__ float4 composite_px(const FrameArgs& a, float4 p, float3 eff) {
    return composite_rd(a, p, redistributed(a, p), eff);
}

__device__ __forceinline__ void store_px(unsigned char* drow, int dx, bool aligned, float4 out) {
    if (aligned) {
        reinterpret_cast<float4*>(drow)[dx] = out;
    } else {
        float* q = reinterpret_cast<float*>(drow) + 4 * dx;
        q[0] = out.x;
        q[1] = out.y;
        q[2] = out.z;
        q[3] = out.w;
    }
}

__device__ __forceinline__ float luma(float r, float g, float b) { return 0.2126f * r + 0.7152f * g + 0.0722f * b; }

// Block sum of two doubles added to out[0], out[1] (one atomic each per CTA).
__device__ __forceinline__ void block_add2(double v0, double v1, double* out) {
    __shared__ double part[2][32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v0 += __shfl_xor_sync(0xffffffffu, v0, o);
        v1 += __shfl_xor_sync(0xffffffffu, v1, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    if (lane == 0) {
        part[0][warp] = v0;
        part[1][warp] = v1;
    }
    __syncthreads();
    if (warp == 0) {
        v0 = lane < nw ? part[0][lane] : 0.0;
        v1 = lane < nw ? part[1][lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v0 += __shfl_xor_sync(0xffffffffu, v0, o);
            v1 += __shfl_xor_sync(0xffffffffu, v1, o);
        }
        if (lane == 0) {
            atomicAdd(&out[0], v0);
            atomicAdd(&out[1], v1);
        }
    }
}

}  // namespace ld
