// ld_psf.cu — PSF-bank kernels: pupil -> |FFT|^2 window -> lambda-rescale ->
// kernel shaping -> adaptive crop/taper -> weighted combination.
//
// Reference stages (LensDiffCpuReference.cpp):
//   buildPupilAmplitude / BuildLensDiffPupilPhaseWaves :758-829
//                           -> pupil_pre_kernel (once per bank)
//   buildShiftedRawPsf      :831-859   -> psf_rows_kernel + psf_cols_kernel
//   makeResampledKernel     :1060-1086 -> resample_kernel
//   azimuthalMeanKernel / reshapeAnisotropy / estimateAdaptiveSupportRadius
//                           :1088-1135, :984-1031 -> shape_stats_kernel, support_kernel
//   cropKernelToRadius + applySupportBoundaryTaper :1038-1058, :957-982
//                           -> crop_sum_kernel, combine_kernel
//   estimateFirstMinimumRadius :865-955 -> profile_kernel + first_zero_scan_kernel
//
// All wavelengths of a bank run in the same launches (blockIdx.y / .z is the
// wavelength).  No stage returns to the host.  The canvas of a wavelength is
// overwritten stage by stage: resampled value -> shaped value (shape_stats) ->
// shaped * taper inside the crop box, 0 outside (crop_sum); the final,
// normalised kernel is that value / (s3 * s4).
#include <climits>

#include "ld_internal.h"

namespace ld {
namespace {

constexpr int kTile = 32;       // canvas tile side for the per-pixel kernels
constexpr int kRingSpan = 64;   // ring indices one 32x32 tile can touch
// The ring-statistics passes (resample, shape_stats) take 32 x 128 tiles:
// sixteen rows per thread amortise each CTA's ring setup, flush and sums.
constexpr int kTallH = 128;
constexpr int kRingSpanTall = 160;  // >= sqrt(31^2 + 127^2) + 3

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of one double; result valid in thread 0.
__device__ double block_sum(double v) {
    __shared__ double part[32];
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int lane = tid & 31, warp = tid >> 5;
    v = warp_sum(v);
    const int nwarps = (blockDim.x * blockDim.y + 31) >> 5;
    __syncthreads();
    if (lane == 0) part[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (warp == 0) {
        r = lane < nwarps ? part[lane] : 0.0;
        r = warp_sum(r);
    }
    return r;
}

// Adds each lane's v to ring[slot] (and, with PEAK, maxes it into
// peak[slot] as float bits) where the lanes' slots form runs of equal values
// in consecutive lanes (slot < 0: nothing to add), v >= 0.  A warp is 32
// pixels of a canvas row, along which the ring index is monotonic on each
// side of the centre, so equal slots are contiguous.  One inclusive
// segmented scan over the warp (five shuffles) gives each run's sum (and
// maximum) in its last lane, which adds it with one shared-memory atomic:
// a fixed cost per warp whatever the number of runs.
template <bool PEAK>
__device__ __forceinline__ void warp_runs_accumulate(int slot, float v, float* ring, unsigned int* peak) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int prev = __shfl_up_sync(full, slot, 1);
    const unsigned heads = __ballot_sync(full, lane == 0 || prev != slot);
    const int head = 31 - __clz(heads & (full >> (31 - lane)));  // first lane of this lane's run
    float sum = v, m = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const float t = __shfl_up_sync(full, sum, o);
        const float u = PEAK ? __shfl_up_sync(full, m, o) : 0.0f;
        if (lane - o >= head) {
            sum += t;
            if (PEAK) m = fmaxf(m, u);
        }
    }
    const bool tail = lane == 31 || ((heads >> (lane + 1)) & 1u) != 0u;
    if (tail && slot >= 0) {
        if (sum != 0.0f) atomicAdd(&ring[slot], sum);
        if (PEAK && m != 0.0f) atomicMax(&peak[slot], __float_as_uint(m));
    }
}

// ---- pupil, once per bank --------------------------------------------------------
__global__ void __launch_bounds__(256) pupil_pre_kernel(PsfBankArgs a) {
    const int n = a.pupil.size;
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= n * n) return;
    const int x = i % n, y = i / n;
    const float amp = pupil_amplitude(a.pupil, x, y);
    float phi0 = 0.0f, z4 = 0.0f, valid = 0.0f;
    if (amp > 0.0f) pupil_phase_split(a.pupil, a.base_phase, x, y, &phi0, &z4, &valid);
    a.pupil_pre[i] = make_float4(amp, phi0, z4, valid);
}

// ---- raw PSF: row pass ---------------------------------------------------------
// grid (row_n, B).  Pupil row y = row_lo + blockIdx.x, embedded at (S-N_p)/2 of
// a length-S row; the field A exp(i 2 pi phi) is generated in the fill, the
// window columns are written by the drain.
template <int E>
__global__ void __launch_bounds__(E >= kE25 ? kE25MaxThreads : kE16MaxThreads, 1) psf_rows_kernel(PsfBankArgs a) {
    extern __shared__ float2 smem[];
    const int yr = blockIdx.x;
    const int y = a.row_lo + yr;
    const int b = blockIdx.y;
    const WavelengthInfo* w = a.wl + b;
    const int np = a.pupil.size;
    const int off = a.off;
    const int enabled = w->phase.enabled;
    const float c4 = w->phase.c[4];
    const float4* pre = a.pupil_pre + static_cast<size_t>(y) * np;
    smem_fill<1>(smem, a.S, [=](int idx, int) -> float2 {
        const int x = idx - off;
        if (x < 0 || x >= np) return make_float2(0.0f, 0.0f);
        const float4 q = pre[x];
        if (q.x <= 0.0f) return make_float2(0.0f, 0.0f);
        const float ph = (enabled && q.w != 0.0f) ? q.y + c4 * q.z : 0.0f;
        if (ph == 0.0f) return make_float2(q.x, 0.0f);
        float sn, cs;
        sincosf(ph * 2.0f * kPiF, &sn, &cs);
        return make_float2(q.x * cs, q.x * sn);
    });
    fft_run<E, 1, false>(a.plan_s, smem);
    const int wn = w->win_n;
    const int wx0 = w->win_x0;
    const int S = a.S;
    float2* out = a.rows + (static_cast<size_t>(b) * a.row_n + yr) * a.win_stride;
    for (int wx = threadIdx.x; wx < wn; wx += blockDim.x) {
        int u = wx0 + wx + a.half;  // shifted column X -> unshifted (X + S/2) mod S
        if (u >= S) u -= S;
        out[wx] = smem[u];
    }
}

// ---- raw PSF: column pass + |.|^2 + fftshift window -----------------------------
// grid (ceil(win/C), B).  Columns X0..X0+C of the window; only the pupil rows
// that can be non-zero are read, |F|^2 of the window rows is written.
template <int E, int C>
__global__ void __launch_bounds__(E >= kE25 ? kE25MaxThreads : kE16MaxThreads, 1) psf_cols_kernel(PsfBankArgs a) {
    extern __shared__ float2 smem[];
    const int b = blockIdx.y;
    const WavelengthInfo* w = a.wl + b;
    const int wn = w->win_n;
    const int X0 = blockIdx.x * C;
    if (X0 >= wn) return;
    const int lo = a.off + a.row_lo;
    const int rn = a.row_n;
    const int stride = a.win_stride;
    const float2* in = a.rows + static_cast<size_t>(b) * rn * stride;
    float* outw = a.win + static_cast<size_t>(b) * stride * stride;
    smem_fill<C>(smem, a.S, [=](int idx, int col) -> float2 {
        const int g = idx - lo;
        const int X = X0 + col;
        if (g < 0 || g >= rn || X >= wn) return make_float2(0.0f, 0.0f);
        return in[static_cast<size_t>(g) * stride + X];
    });
    fft_run<E, C, false>(a.plan_s, smem);
    const int S = a.S;
    const int wy0 = w->win_x0;
    double esum = 0.0;
    for (int i = threadIdx.x; i < wn * C; i += blockDim.x) {
        const int wy = i / C, col = i % C;
        const int X = X0 + col;
        if (X >= wn) continue;
        int v = wy0 + wy + a.half;  // shifted row Y -> unshifted (Y + S/2) mod S
        if (v >= S) v -= S;
        const float2 f = smem[v * C + col];
        const float I = f.x * f.x + f.y * f.y;
        outw[static_cast<size_t>(wy) * stride + X] = I;
        esum += I;
    }
    if (a.want_energy) {
        const double tot = block_sum(esum);
        if (threadIdx.x == 0) atomicAdd(&a.scalars[b].energy, tot);
    }
}

// ---- lambda-rescale -----------------------------------------------------------------
struct Window {
    const float* p;
    int stride, x0, n, S;
};

// sampleSquareBilinear (LensDiffCpuReference.cpp:316-336) reading the |F|^2
// window; the window covers every pixel the kernel touches.
__device__ __forceinline__ float sample_bilinear(const Window& w, float x, float y) {
    const float lim = static_cast<float>(w.S - 1);
    if (x < 0.0f || y < 0.0f || x > lim || y > lim) return 0.0f;
    const int x0 = static_cast<int>(floorf(x));
    const int y0 = static_cast<int>(floorf(y));
    const int x1 = min(x0 + 1, w.S - 1);
    const int y1 = min(y0 + 1, w.S - 1);
    const float tx = x - static_cast<float>(x0);
    const float ty = y - static_cast<float>(y0);
    const int hi = w.n - 1;
    const int ax0 = min(max(x0 - w.x0, 0), hi), ax1 = min(max(x1 - w.x0, 0), hi);
    const int ay0 = min(max(y0 - w.x0, 0), hi), ay1 = min(max(y1 - w.x0, 0), hi);
    const float v00 = w.p[static_cast<size_t>(ay0) * w.stride + ax0];
    const float v10 = w.p[static_cast<size_t>(ay0) * w.stride + ax1];
    const float v01 = w.p[static_cast<size_t>(ay1) * w.stride + ax0];
    const float v11 = w.p[static_cast<size_t>(ay1) * w.stride + ax1];
    const float vx0 = v00 + (v10 - v00) * tx;
    const float vx1 = v01 + (v11 - v01) * tx;
    return vx0 + (vx1 - vx0) * ty;
}

// sampleSquareFiltered (LensDiffCpuReference.cpp:338-353)
__device__ __forceinline__ float sample_filtered(const Window& w, float x, float y, float footprint, int taps,
                                                 float step) {
    if (taps == 0) return sample_bilinear(w, x, y);
    float sum = 0.0f;
    for (int ty = 0; ty < taps; ++ty) {
        const float oy = (static_cast<float>(ty) + 0.5f) * step - footprint * 0.5f;
        for (int tx = 0; tx < taps; ++tx) {
            const float ox = (static_cast<float>(tx) + 0.5f) * step - footprint * 0.5f;
            sum += sample_bilinear(w, x + ox, y + oy);
        }
    }
    return sum / static_cast<float>(taps * taps);
}

// First ring index a 32 x TH tile can touch, for a centre at (c, c) and ring
// indices clamped to `cap`: every pixel of the tile has a ring index in
// [base, base + span) with span <= the tile's diagonal + 3 (kRingSpan for
// 32 x 32 tiles, kRingSpanTall for the 32 x 128 tiles of the ring-statistics
// passes).
template <int TH = kTile>
__device__ __forceinline__ int tile_ring_base(int tx0, int ty0, int c, int cap) {
    const int dx = tx0 > c ? tx0 - c : (tx0 + kTile - 1 < c ? c - (tx0 + kTile - 1) : 0);
    const int dy = ty0 > c ? ty0 - c : (ty0 + TH - 1 < c ? c - (ty0 + TH - 1) : 0);
    const float r = sqrtf(static_cast<float>(dx * dx + dy * dy));
    return min(cap, max(0, static_cast<int>(r) - 1));
}

// The column half of a bilinear sample of the |F|^2 window at x
// (sampleSquareBilinear's x terms): the same for every row a thread samples.
struct ColTap {
    bool in;       // x inside [0, S - 1]
    int ax0, ax1;  // window columns of x0 and x1
    float tx;
};
__device__ __forceinline__ ColTap col_tap(const Window& w, float x) {
    ColTap c;
    c.in = !(x < 0.0f || x > static_cast<float>(w.S - 1));
    const int x0 = static_cast<int>(floorf(x));
    const int x1 = min(x0 + 1, w.S - 1);
    c.tx = x - static_cast<float>(x0);
    const int hi = w.n - 1;
    c.ax0 = min(max(x0 - w.x0, 0), hi);
    c.ax1 = min(max(x1 - w.x0, 0), hi);
    return c;
}
// sample_bilinear with the column half precomputed (identical arithmetic).
__device__ __forceinline__ float sample_row(const Window& w, const ColTap& c, float y) {
    if (!c.in || y < 0.0f || y > static_cast<float>(w.S - 1)) return 0.0f;
    const int y0 = static_cast<int>(floorf(y));
    const int y1 = min(y0 + 1, w.S - 1);
    const float ty = y - static_cast<float>(y0);
    const int hi = w.n - 1;
    const float* r0 = w.p + min(max(y0 - w.x0, 0), hi) * w.stride;
    const float* r1 = w.p + min(max(y1 - w.x0, 0), hi) * w.stride;
    const float v00 = __ldg(r0 + c.ax0), v10 = __ldg(r0 + c.ax1);
    const float v01 = __ldg(r1 + c.ax0), v11 = __ldg(r1 + c.ax1);
    const float vx0 = v00 + (v10 - v00) * c.tx;
    const float vx1 = v01 + (v11 - v01) * c.tx;
    return vx0 + (vx1 - vx0) * ty;
}

// grid (ceil(K/32), ceil(K/128), B), block (32, 8).
// FUSED (anisotropy gain 1): reshapeAnisotropy (LensDiffCpuReference.cpp:1122-1134)
// then gives mean + (base - mean) * 1, the base kernel itself up to one
// rounding, so the canvas keeps the resampled values unnormalised and this
// pass takes the shaped kernel's statistics that shape_stats_kernel takes
// otherwise (s3 = s1, the ceil(r) ring energies and peaks, the peak) in
// place of the round(r) ring sums, which only the Split look's ring means
// need (ring_sums_kernel, run when a Split render first uses the bank).
// The bilinear path (no box filter: the canvas samples the |F|^2 window at
// most one window pixel apart, scaleFactor >= 1) stages the window pixels a
// 32 x 128 tile reads in shared memory first: at most 33 x 129 of them, with
// one more on each side so that the span holds whatever the rounding of the
// sample positions.
constexpr int kStageW = kTile + 4, kStageH = kTallH + 4;

// Rows / columns of the window that canvas coordinates c0 .. c1 sample
// (sample_bilinear's x0 .. x1 of the first and last sample, clamped to the
// window as it clamps them): [lo, hi] in window indices.
__device__ __forceinline__ void stage_span(const Window& w, float rc, float kc, float inv, int c0, int c1, int* lo,
                                           int* hi) {
    const float p0 = rc + (static_cast<float>(c0) - kc) * inv;
    const float p1 = rc + (static_cast<float>(c1) - kc) * inv;
    const int whi = w.n - 1;
    const int a0 = static_cast<int>(floorf(fmaxf(p0, 0.0f)));
    const int a1 = min(static_cast<int>(floorf(fminf(fmaxf(p1, 0.0f), static_cast<float>(w.S - 1)))) + 1, w.S - 1);
    *lo = min(max(a0 - 1 - w.x0, 0), whi);
    *hi = min(max(a1 + 1 - w.x0, 0), whi);
}

// Shared memory of one λ-rescale tile.
template <bool FUSED>
struct ResampleSmem {
    float ring[kRingSpanTall];  // FUSED: the ceil(r) ring energies, else the round(r) sums
    unsigned int ring_p[FUSED ? kRingSpanTall : 1];
    float stage[kStageH][kStageW];
};

// Ring slot of canvas pixel (x, y) relative to the tile's first ring `rbase`
// (-1: no pixel): ceil(r) (FUSED) or round(r) of its distance to the centre.
template <bool FUSED>
__device__ __forceinline__ int ring_slot(bool in, float dx, float dy, int R, int rbase) {
    if (!in) return -1;
    const float rr = sqrtf(dx * dx + dy * dy);
    return min(R, static_cast<int>(FUSED ? ceilf(rr) : roundf(rr))) - rbase;
}

// The window pixels (rows cy0.., columns cx0..) a staged tile samples.
struct StageBox {
    int cx0, cy0, sw, sh;
};

// The staged box of wavelength `w`'s window for the tile at (tx0, ty0);
// ok = false when the samples are box-filtered or the span is too wide.
__device__ __forceinline__ bool stage_box(const Window& w, float rc, float kc, float inv, int taps, int tx0, int ty0,
                                          int K, StageBox* b) {
    if (taps != 0) return false;
    int cx1 = -1, cy1 = -1;
    stage_span(w, rc, kc, inv, tx0, min(tx0 + kTile, K) - 1, &b->cx0, &cx1);
    stage_span(w, rc, kc, inv, ty0, min(ty0 + kTallH, K) - 1, &b->cy0, &cy1);
    b->sw = cx1 - b->cx0 + 1;
    b->sh = cy1 - b->cy0 + 1;
    return b->sw <= kStageW && b->sh <= kStageH;
}

__device__ __forceinline__ void stage_load(const Window& w, const StageBox& b, float (*stage)[kStageW], int tid) {
    for (int i = tid; i < b.sw * b.sh; i += 256) {
        const int r = i / b.sw, c = i - r * b.sw;
        stage[r][c] = __ldg(w.p + static_cast<size_t>(b.cy0 + r) * w.stride + b.cx0 + c);
    }
}

// sample_row's arithmetic on staged pixels: the bilinear sample at window
// row coordinate yy of the column tap ct (sx0, sx1: its columns in the box).
__device__ __forceinline__ float staged_sample(const Window& w, const ColTap& ct, int sx0, int sx1, int cy0,
                                              const float (*stage)[kStageW], bool in, float yy) {
    const float lim = static_cast<float>(w.S - 1);
    if (!(in && ct.in && !(yy < 0.0f || yy > lim))) return 0.0f;
    const int hi = w.n - 1;
    const int y0 = static_cast<int>(floorf(yy));
    const int y1 = min(y0 + 1, w.S - 1);
    const float ty = yy - static_cast<float>(y0);
    const int sy0 = min(max(y0 - w.x0, 0), hi) - cy0;
    const int sy1 = min(max(y1 - w.x0, 0), hi) - cy0;
    const float v00 = stage[sy0][sx0], v10 = stage[sy0][sx1];
    const float v01 = stage[sy1][sx0], v11 = stage[sy1][sx1];
    const float vx0 = v00 + (v10 - v00) * ct.tx;
    const float vx1 = v01 + (v11 - v01) * ct.tx;
    return vx0 + (vx1 - vx0) * ty;
}

// The end of one wavelength's tile: the CTA's ring sums and peaks, the peak
// and the canvas sum go to the wavelength's global statistics.
template <bool FUSED>
__device__ __forceinline__ void resample_flush(const PsfBankArgs& a, int b, int rbase, ResampleSmem<FUSED>& sm,
                                               float lsum, unsigned int lpeak, int tid) {
    __syncthreads();
    const int R = a.R;
    const size_t ro = static_cast<size_t>(b) * (R + 1);
    for (int i = tid; i < kRingSpanTall; i += 256) {
        if (rbase + i > R) continue;
        if (sm.ring[i] != 0.0f)
            atomicAdd(&(FUSED ? a.ring_ceil : a.ring_round)[ro + rbase + i], static_cast<double>(sm.ring[i]));
        if constexpr (FUSED) {
            if (sm.ring_p[i] != 0u) atomicMax(&a.ring_peak[ro + rbase + i], sm.ring_p[i]);
        }
    }
    if constexpr (FUSED) {
        for (int o = 16; o > 0; o >>= 1) lpeak = max(lpeak, __shfl_xor_sync(0xffffffffu, lpeak, o));
        if ((tid & 31) == 0 && lpeak != 0u) atomicMax(&a.scalars[b].peak, lpeak);
    }
    const double tot = block_sum(static_cast<double>(lsum));
    if (tid == 0) {
        atomicAdd(&a.scalars[b].s1, tot);
        if constexpr (FUSED) atomicAdd(&a.scalars[b].s3, tot);
    }
}

// One wavelength's 32 x 128 canvas tile (grid (ceil(K/32), ceil(K/128), .),
// block (32, 8); 16 rows per thread).
// FUSED (anisotropy gain 1): reshapeAnisotropy (LensDiffCpuReference.cpp:1122-1134)
// then gives mean + (base - mean) * 1, the base kernel itself up to one
// rounding, so the canvas keeps the resampled values unnormalised and this
// pass takes the shaped kernel's statistics that shape_stats_kernel takes
// otherwise (s3 = s1, the ceil(r) ring energies and peaks, the peak) in
// place of the round(r) ring sums, which only the Split look's ring means
// need (ring_sums_kernel, run when a Split render first uses the bank).
// The bilinear path (no box filter: the canvas samples the |F|^2 window at
// most one window pixel apart, scaleFactor >= 1) stages the window pixels the
// tile reads in shared memory first (stage_box); box-filtered samples, and
// any span too wide to stage, read the window directly.
template <bool FUSED>
__device__ void resample_tile(const PsfBankArgs& a, int b, int rbase, ResampleSmem<FUSED>& sm, int tid) {
    for (int i = tid; i < kRingSpanTall; i += 256) {
        sm.ring[i] = 0.0f;
        if constexpr (FUSED) sm.ring_p[i] = 0u;
    }
    const WavelengthInfo* wi = a.wl + b;
    const int K = a.K, R = a.R;
    const int tx0 = blockIdx.x * kTile, ty0 = blockIdx.y * kTallH;
    const Window w{a.win + static_cast<size_t>(b) * a.win_stride * a.win_stride, a.win_stride, wi->win_x0,
                   wi->win_n, a.S};
    const float kc = static_cast<float>(K - 1) * 0.5f;
    const float inv = wi->inv_scale;
    const int taps = wi->taps;
    const float step = wi->step;
    const float rc = a.raw_center;
    float* canvas = a.canvas + static_cast<size_t>(b) * K * K;
    float lsum = 0.0f;  // this thread's pixels; one double add per thread at the flush
    unsigned int lpeak = 0u;
    const int x = tx0 + threadIdx.x;
    const bool in = x < K;
    const float dx = static_cast<float>(x) - kc;
    StageBox bx;
    if (stage_box(w, rc, kc, inv, taps, tx0, ty0, K, &bx)) {  // uniform per CTA
        stage_load(w, bx, sm.stage, tid);
        __syncthreads();
        const ColTap ct = col_tap(w, rc + dx * inv);
        const int sx0 = ct.ax0 - bx.cx0, sx1 = ct.ax1 - bx.cx0;
#pragma unroll 4
        for (int i = 0; i < kTallH / 8; ++i) {
            const int y = ty0 + threadIdx.y + 8 * i;
            if (y >= K) break;  // uniform: a warp is one canvas row
            const float dy = static_cast<float>(y) - kc;
            const float v = staged_sample(w, ct, sx0, sx1, bx.cy0, sm.stage, in, rc + dy * inv);
            if (in) canvas[static_cast<size_t>(y) * K + x] = v;
            lsum += v;
            if constexpr (FUSED) lpeak = max(lpeak, __float_as_uint(v));
            warp_runs_accumulate<FUSED>(ring_slot<FUSED>(in, dx, dy, R, rbase), v, sm.ring, sm.ring_p);
        }
    } else {
        __syncthreads();
        const ColTap ct = col_tap(w, rc + dx * inv);
#pragma unroll 4
        for (int i = 0; i < kTallH / 8; ++i) {
            const int y = ty0 + threadIdx.y + 8 * i;
            if (y >= K) break;  // uniform: a warp is one canvas row (the last tile row is mostly past K)
            const float dy = static_cast<float>(y) - kc;
            float v = 0.0f;
            if (in) {
                v = taps == 0 ? sample_row(w, ct, rc + dy * inv)
                              : sample_filtered(w, rc + dx * inv, rc + dy * inv, inv, taps, step);
                canvas[static_cast<size_t>(y) * K + x] = v;
                lsum += v;
                if constexpr (FUSED) lpeak = max(lpeak, __float_as_uint(v));
            }
            warp_runs_accumulate<FUSED>(ring_slot<FUSED>(in, dx, dy, R, rbase), v, sm.ring, sm.ring_p);
        }
    }
    resample_flush<FUSED>(a, b, rbase, sm, lsum, lpeak, tid);
}

// grid (ceil(K/32), ceil(K/128), B), block (32, 8): wavelength blockIdx.z.
template <bool FUSED>
__global__ void __launch_bounds__(256) resample_kernel(PsfBankArgs a) {
    __shared__ ResampleSmem<FUSED> sm;
    const int tid = threadIdx.x + threadIdx.y * 32;
    const int rbase = tile_ring_base<kTallH>(blockIdx.x * kTile, blockIdx.y * kTallH, a.R, a.R);
    resample_tile<FUSED>(a, blockIdx.z, rbase, sm, tid);
}

// warp_runs_accumulate for the same pixels of two wavelengths: one ring
// geometry (slot, run heads) for both, each wavelength's run sums and peaks
// formed by the same scan steps in the same order as the single form.
template <bool PEAK>
__device__ __forceinline__ void warp_runs_accumulate2(int slot, float v0, float v1, float* ring0,
                                                      unsigned int* peak0, float* ring1, unsigned int* peak1) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int prev = __shfl_up_sync(full, slot, 1);
    const unsigned heads = __ballot_sync(full, lane == 0 || prev != slot);
    const int head = 31 - __clz(heads & (full >> (31 - lane)));
    float s0 = v0, s1 = v1, m0 = v0, m1 = v1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const float t0 = __shfl_up_sync(full, s0, o);
        const float t1 = __shfl_up_sync(full, s1, o);
        const float u0 = PEAK ? __shfl_up_sync(full, m0, o) : 0.0f;
        const float u1 = PEAK ? __shfl_up_sync(full, m1, o) : 0.0f;
        if (lane - o >= head) {
            s0 += t0;
            s1 += t1;
            if (PEAK) {
                m0 = fmaxf(m0, u0);
                m1 = fmaxf(m1, u1);
            }
        }
    }
    const bool tail = lane == 31 || ((heads >> (lane + 1)) & 1u) != 0u;
    if (tail && slot >= 0) {
        if (s0 != 0.0f) atomicAdd(&ring0[slot], s0);
        if (s1 != 0.0f) atomicAdd(&ring1[slot], s1);
        if (PEAK && m0 != 0.0f) atomicMax(&peak0[slot], __float_as_uint(m0));
        if (PEAK && m1 != 0.0f) atomicMax(&peak1[slot], __float_as_uint(m1));
    }
}

// grid (ceil(K/32), ceil(K/128), B / 2), block (32, 8): wavelengths 2z and
// 2z + 1 of the same tile.  When both are staged, one pass over the tile
// samples both from their staged windows and takes each pixel's ring slot and
// run boundaries once for the two; otherwise the two tiles run in turn.  The
// canvases and every statistic equal those of resample_kernel.
template <bool FUSED>
__global__ void __launch_bounds__(256) resample_pair_kernel(PsfBankArgs a) {
    __shared__ ResampleSmem<FUSED> sm[2];
    const int tid = threadIdx.x + threadIdx.y * 32;
    const int K = a.K, R = a.R;
    const int tx0 = blockIdx.x * kTile, ty0 = blockIdx.y * kTallH;
    const int rbase = tile_ring_base<kTallH>(tx0, ty0, R, R);
    const int b0 = 2 * blockIdx.z, b1 = b0 + 1;
    const WavelengthInfo* wi0 = a.wl + b0;
    const WavelengthInfo* wi1 = a.wl + b1;
    const size_t wsz = static_cast<size_t>(a.win_stride) * a.win_stride;
    const Window w0{a.win + b0 * wsz, a.win_stride, wi0->win_x0, wi0->win_n, a.S};
    const Window w1{a.win + b1 * wsz, a.win_stride, wi1->win_x0, wi1->win_n, a.S};
    const float kc = static_cast<float>(K - 1) * 0.5f;
    const float rc = a.raw_center;
    const float inv0 = wi0->inv_scale, inv1 = wi1->inv_scale;
    StageBox bx0, bx1;
    const bool joint = stage_box(w0, rc, kc, inv0, wi0->taps, tx0, ty0, K, &bx0) &&
                       stage_box(w1, rc, kc, inv1, wi1->taps, tx0, ty0, K, &bx1);  // uniform per CTA
    if (!joint) {
        resample_tile<FUSED>(a, b0, rbase, sm[0], tid);
        resample_tile<FUSED>(a, b1, rbase, sm[1], tid);
        return;
    }
    for (int i = tid; i < kRingSpanTall; i += 256) {
        sm[0].ring[i] = 0.0f;
        sm[1].ring[i] = 0.0f;
        if constexpr (FUSED) {
            sm[0].ring_p[i] = 0u;
            sm[1].ring_p[i] = 0u;
        }
    }
    stage_load(w0, bx0, sm[0].stage, tid);
    stage_load(w1, bx1, sm[1].stage, tid);
    __syncthreads();
    const int x = tx0 + threadIdx.x;
    const bool in = x < K;
    const float dx = static_cast<float>(x) - kc;
    const ColTap ct0 = col_tap(w0, rc + dx * inv0), ct1 = col_tap(w1, rc + dx * inv1);
    const int s00 = ct0.ax0 - bx0.cx0, s01 = ct0.ax1 - bx0.cx0;
    const int s10 = ct1.ax0 - bx1.cx0, s11 = ct1.ax1 - bx1.cx0;
    float* canvas0 = a.canvas + static_cast<size_t>(b0) * K * K;
    float* canvas1 = a.canvas + static_cast<size_t>(b1) * K * K;
    float lsum0 = 0.0f, lsum1 = 0.0f;
    unsigned int lpeak0 = 0u, lpeak1 = 0u;
#pragma unroll 2
    for (int i = 0; i < kTallH / 8; ++i) {
        const int y = ty0 + threadIdx.y + 8 * i;
        if (y >= K) break;  // uniform: a warp is one canvas row
        const float dy = static_cast<float>(y) - kc;
        const float v0 = staged_sample(w0, ct0, s00, s01, bx0.cy0, sm[0].stage, in, rc + dy * inv0);
        const float v1 = staged_sample(w1, ct1, s10, s11, bx1.cy0, sm[1].stage, in, rc + dy * inv1);
        if (in) {
            canvas0[static_cast<size_t>(y) * K + x] = v0;
            canvas1[static_cast<size_t>(y) * K + x] = v1;
        }
        lsum0 += v0;
        lsum1 += v1;
        if constexpr (FUSED) {
            lpeak0 = max(lpeak0, __float_as_uint(v0));
            lpeak1 = max(lpeak1, __float_as_uint(v1));
        }
        warp_runs_accumulate2<FUSED>(ring_slot<FUSED>(in, dx, dy, R, rbase), v0, v1, sm[0].ring, sm[0].ring_p,
                                     sm[1].ring, sm[1].ring_p);
    }
    resample_flush<FUSED>(a, b0, rbase, sm[0], lsum0, lpeak0, tid);
    resample_flush<FUSED>(a, b1, rbase, sm[1], lsum1, lpeak1, tid);
}

// Sum over rings of the unnormalised azimuthal mean, i.e. the normaliser of
// azimuthalMeanKernel: sum_r count[r] * (ring[r] / s1) / count[r].
__device__ double mean_kernel_sum(const double* ring, const int* count, int R, double s1) {
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int nth = blockDim.x * blockDim.y;
    double acc = 0.0;
    for (int r = tid; r <= R; r += nth) {
        const int c = max(1, count[r]);
        acc += static_cast<double>(count[r]) * ((ring[r] / s1) / c);
    }
    __shared__ double s2_shared;
    const double t = block_sum(acc);
    if (tid == 0) s2_shared = t;
    __syncthreads();
    return s2_shared;
}

// grid (B), block 256: s2 (the normaliser of azimuthalMeanKernel) and the
// normalised azimuthal mean of every round(r) ring, once per wavelength, for
// shape_stats_kernel to read.
__global__ void __launch_bounds__(256) ring_mean_kernel(PsfBankArgs a) {
    const int b = blockIdx.x;
    const int R = a.R;
    const double s1 = a.scalars[b].s1;
    const double* rr = a.ring_round + static_cast<size_t>(b) * (R + 1);
    const double s2 = mean_kernel_sum(rr, a.count_round, R, s1);
    if (threadIdx.x == 0) a.scalars[b].s2 = s2;
    float* out = a.ring_mean + static_cast<size_t>(b) * (R + 1);
    for (int r = threadIdx.x; r <= R; r += blockDim.x)
        out[r] = static_cast<float>(((rr[r] / s1) / max(1, a.count_round[r])) / s2);
}

// grid (ceil(K/32), ceil(K/128), B), block (32, 8): the round(r) ring sums
// of a canvas that resample_kernel<true> filled (the unnormalised resampled
// kernel), for the ring means of the Split look.
__global__ void __launch_bounds__(256) ring_sums_kernel(PsfBankArgs a) {
    __shared__ float ring[kRingSpanTall];
    const int b = blockIdx.z;
    const int K = a.K, R = a.R;
    const int tx0 = blockIdx.x * kTile, ty0 = blockIdx.y * kTallH;
    const int tid = threadIdx.x + threadIdx.y * 32;
    const int rbase = tile_ring_base<kTallH>(tx0, ty0, R, R);
    for (int i = tid; i < kRingSpanTall; i += 256) ring[i] = 0.0f;
    __syncthreads();
    const float kc = static_cast<float>(K - 1) * 0.5f;
    const float* canvas = a.canvas + static_cast<size_t>(b) * K * K;
    const int x = tx0 + threadIdx.x;
    const float dx = static_cast<float>(x) - kc;
    for (int i = 0; i < kTallH / 8; ++i) {
        const int y = ty0 + threadIdx.y + 8 * i;
        if (y >= K) break;  // uniform: a warp is one canvas row
        float v = 0.0f;
        int slot = -1;
        if (x < K) {
            const float dy = static_cast<float>(y) - kc;
            v = __ldg(canvas + static_cast<size_t>(y) * K + x);
            slot = min(R, static_cast<int>(roundf(sqrtf(dx * dx + dy * dy)))) - rbase;
        }
        warp_runs_accumulate<false>(slot, v, ring, nullptr);
    }
    __syncthreads();
    const size_t ro = static_cast<size_t>(b) * (R + 1);
    for (int i = tid; i < kRingSpanTall; i += 256)
        if (ring[i] != 0.0f && rbase + i <= R) atomicAdd(&a.ring_round[ro + rbase + i], static_cast<double>(ring[i]));
}

// grid (ceil(K/32), ceil(K/128), B): shaped kernel (reshapeAnisotropy of the
// base kernel against its azimuthal mean, LensDiffCpuReference.cpp:1088-1135)
// written in place, its sum, and its ring energy / peak by ceil(r)
// (estimateAdaptiveSupportRadius, :984-1007).
__global__ void __launch_bounds__(256) shape_stats_kernel(PsfBankArgs a) {
    __shared__ float ring_e[kRingSpanTall];
    __shared__ unsigned int ring_p[kRingSpanTall];
    __shared__ float mean_r[kRingSpanTall];
    const int b = blockIdx.z;
    const int tid = threadIdx.x + threadIdx.y * 32;
    const double s1 = a.scalars[b].s1;
    const int K = a.K, R = a.R;
    const int tx0 = blockIdx.x * kTile, ty0 = blockIdx.y * kTallH;
    const int rbase = tile_ring_base<kTallH>(tx0, ty0, R, R);
    // ring means (round(r) rings) the tile can touch
    const float* rm = a.ring_mean + static_cast<size_t>(b) * (R + 1);
    for (int i = tid; i < kRingSpanTall; i += 256) {
        ring_e[i] = 0.0f;
        ring_p[i] = 0u;
        const int r = rbase + i;
        mean_r[i] = r <= R ? rm[r] : 0.0f;
    }
    __syncthreads();
    const float inv_s1 = static_cast<float>(1.0 / s1);
    const float gain = a.gain;
    const float kc = static_cast<float>(K - 1) * 0.5f;
    float* canvas = a.canvas + static_cast<size_t>(b) * K * K;
    float lsum = 0.0f;  // this thread's pixels; one double add per thread below
    unsigned int lpeak = 0u;
    const int x = tx0 + threadIdx.x;
    // the thread's four canvas reads are issued before any is used (each
    // element is read, then written, by this thread only)
    float raw[kTallH / 8];
#pragma unroll
    for (int i = 0; i < kTallH / 8; ++i) {
        const int y = ty0 + threadIdx.y + 8 * i;
        raw[i] = (x < K && y < K) ? __ldg(canvas + static_cast<size_t>(y) * K + x) : 0.0f;
    }
#pragma unroll
    for (int i = 0; i < kTallH / 8; ++i) {
        const int y = ty0 + threadIdx.y + 8 * i;
        const bool in = x < K && y < K;
        float v = 0.0f;
        int slot = -1;
        if (in) {
            const float dx = static_cast<float>(x) - kc;
            const float dy = static_cast<float>(y) - kc;
            const float rad = sqrtf(dx * dx + dy * dy);
            const size_t idx = static_cast<size_t>(y) * K + x;
            const float base = raw[i] * inv_s1;
            const float mean = mean_r[min(R, static_cast<int>(roundf(rad))) - rbase];
            v = fmaxf(0.0f, mean + (base - mean) * gain);
            canvas[idx] = v;
            lsum += v;
            lpeak = max(lpeak, __float_as_uint(v));
            slot = min(R, static_cast<int>(ceilf(rad))) - rbase;
        }
        warp_runs_accumulate<true>(slot, v, ring_e, ring_p);
    }
    __syncthreads();
    const size_t ro = static_cast<size_t>(b) * (R + 1);
    for (int i = tid; i < kRingSpanTall; i += 256) {
        if (rbase + i <= R) {
            if (ring_e[i] != 0.0f) atomicAdd(&a.ring_ceil[ro + rbase + i], static_cast<double>(ring_e[i]));
            if (ring_p[i] != 0u) atomicMax(&a.ring_peak[ro + rbase + i], ring_p[i]);
        }
    }
    for (int o = 16; o > 0; o >>= 1) lpeak = max(lpeak, __shfl_xor_sync(0xffffffffu, lpeak, o));
    if ((tid & 31) == 0 && lpeak != 0u) atomicMax(&a.scalars[b].peak, lpeak);
    const double tot = block_sum(static_cast<double>(lsum));
    if (tid == 0) atomicAdd(&a.scalars[b].s3, tot);
}

// grid (B), block 256: adaptive support radius and taper constants
// (estimateAdaptiveSupportRadius :1009-1030, paddedAdaptiveSupportRadius
// :1033-1036, cropKernelToRadius :1039, applySupportBoundaryTaper :962-965).
// Suffix maxima of the ring peaks and prefix sums of the ring energies are
// block scans over per-thread chunks of rings.
__global__ void __launch_bounds__(256) support_kernel(PsfBankArgs a) {
    __shared__ float chunk_max[256];
    __shared__ double chunk_sum[256];
    __shared__ int first_hit;
    const int b = blockIdx.x;
    const int tid = threadIdx.x;
    PsfScalars& sc = a.scalars[b];
    const int R = a.R;
    const int rm = min(R, a.K / 2);
    const int nr = rm + 1;
    const int per = (nr + 255) / 256;
    const int r0 = tid * per, r1 = min(nr, r0 + per);
    const double* e = a.ring_ceil + static_cast<size_t>(b) * (R + 1);
    const unsigned int* pk = a.ring_peak + static_cast<size_t>(b) * (R + 1);
    const double total = sc.s3;
    const float peak = __uint_as_float(sc.peak);
    float lmax = 0.0f;
    double lsum = 0.0;
    for (int r = r0; r < r1; ++r) {
        lmax = fmaxf(lmax, __uint_as_float(pk[r]));
        lsum += e[r];
    }
    chunk_max[tid] = lmax;
    chunk_sum[tid] = lsum;
    if (tid == 0) first_hit = 1 << 30;
    __syncthreads();
    if (tid == 0) {  // exclusive prefix sums / suffix maxima over the 256 chunks
        double run = 0.0;
        for (int t = 0; t < 256; ++t) {
            const double s = chunk_sum[t];
            chunk_sum[t] = run;
            run += s;
        }
        float m = 0.0f;
        for (int t = 255; t >= 0; --t) {
            const float v = chunk_max[t];
            chunk_max[t] = m;  // maximum over the chunks after t
            m = fmaxf(m, v);
        }
    }
    __syncthreads();
    // the normalised kernel has total 1 and peak = peak / total
    const bool degenerate = !(total > 0.0) || (static_cast<double>(peak) / total <= 1e-6);
    if (!degenerate && r0 < r1) {
        // suffix maxima inside this chunk, then the first ring that passes
        float suffix[64];
        const int len = r1 - r0;  // <= 64 for R <= 16383
        float m = chunk_max[tid];
        for (int k = len - 1; k >= 0; --k) {
            suffix[k] = m;  // maximum over rings > r0 + k
            m = fmaxf(m, __uint_as_float(pk[r0 + k]));
        }
        double cum = chunk_sum[tid];
        const double thr_cap = static_cast<double>(0.9999f);
        const float thr_peak = peak * 2e-4f;
        for (int k = 0; k < len; ++k) {
            cum += e[r0 + k];
            if (cum / total >= thr_cap && suffix[k] <= thr_peak) {
                atomicMin(&first_hit, r0 + k);
                break;
            }
        }
    }
    __syncthreads();
    if (tid != 0) return;
    int est = max(4, rm);
    if (!degenerate && first_hit < (1 << 30)) est = max(4, first_hit + 1);
    const int pad = max(6, min(24, static_cast<int>(ceilf(static_cast<float>(max(1, est)) * 0.05f))));
    int rho = min(max(est + pad, 4), max(4, R));
    rho = min(max(rho, 1), a.K / 2);
    sc.radius = rho;
    const float extent = fmaxf(1.0f, static_cast<float>(rho));
    const float fade = fmaxf(6.0f, fminf(24.0f, extent * 0.04f));
    sc.extent = extent;
    sc.fade = fade;
    sc.start = fmaxf(0.0f, extent - fade);
}

// grid (ceil(K/8), B), block 256: s4 = sum over the crop box of taper *
// normalised shaped kernel, the normaliser of cropKernelToRadius and
// applySupportBoundaryTaper (LensDiffCpuReference.cpp:1038-1058, :957-982).
// The canvas keeps the shaped kernel; the crop and the taper are applied
// where the kernel is read (combine_kernel, split_sums_kernel, export_kernel).
// The taper is 1 up to radius `start` and 0 from `extent` on, and every pixel
// with r < extent lies in the crop box, so s4 = (the ceil(r) ring energies of
// rings 0 .. S0 = floor(start)) / s3 + the annulus S0 < r < extent pixel by
// pixel.  A pixel's ring is ceil(sqrtf(dx^2 + dy^2)) <= S0 exactly when
// dx^2 + dy^2 <= S0^2 (integers; exact below 2^24), so each crop row reads
// only its |dx| > isqrt(S0^2 - dy^2) part.  One warp per crop row, eight
// reads in flight per thread.
constexpr int kCropRows = 8;

__device__ __forceinline__ int isqrt_floor(int v) {  // floor(sqrt(v)), v >= 0
    int r = static_cast<int>(sqrtf(static_cast<float>(v)));
    while (r > 0 && r * r > v) --r;
    while ((r + 1) * (r + 1) <= v) ++r;
    return r;
}

__global__ void __launch_bounds__(256) crop_sum_kernel(PsfBankArgs a) {
    const int b = blockIdx.y;
    const PsfScalars& sc = a.scalars[b];
    const int rho = sc.radius;
    const int K = a.K, R = a.R;
    const int y0 = R - rho + static_cast<int>(blockIdx.x) * kCropRows;
    if (y0 > R + rho) return;  // uniform
    const float inv_s3 = static_cast<float>(1.0 / sc.s3);
    const float extent = sc.extent, fade = sc.fade, start = sc.start;
    const int s0 = static_cast<int>(floorf(start));
    const int lane = threadIdx.x & 31;
    const int y = y0 + static_cast<int>(threadIdx.x >> 5);  // one warp per crop row
    float lsum = 0.0f;
    if (y <= R + rho) {
        const float* row = a.canvas + static_cast<size_t>(b) * K * K + static_cast<size_t>(y) * K + R;  // dx = 0
        const int dyi = y - R;
        const int in2 = s0 * s0 - dyi * dyi;
        // |dx| <= xin lies inside ring s0; a row that misses that disc reads
        // all of [-rho, rho] (left part [-rho, 0], right part [1, rho])
        const int xin = in2 >= 0 ? isqrt_floor(in2) : -1;
        const int nl = xin >= 0 ? rho - xin : rho + 1;  // left part: dx = -rho .. -rho + nl - 1
        const int r0 = xin >= 0 ? xin + 1 : 1;          // right part: dx = r0 .. rho
        const int n = nl + (rho - r0 + 1);
        const float dy2 = static_cast<float>(dyi) * static_cast<float>(dyi);
        constexpr int kU = 8;
        for (int t0 = lane; t0 < n; t0 += kU * 32) {
            float v[kU];
            int dxs[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int t = t0 + u * 32;
                dxs[u] = t < nl ? t - rho : r0 + (t - nl);
                v[u] = t < n ? __ldg(row + dxs[u]) : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                if (t0 + u * 32 >= n) break;
                const float dx = static_cast<float>(dxs[u]);
                lsum += (v[u] * inv_s3) * taper_weight(sqrtf(dx * dx + dy2), extent, fade, start);
            }
        }
    }
    double tot = block_sum(static_cast<double>(lsum));
    if (blockIdx.x == 0) {  // the rings inside the taper's flat part
        const double* e = a.ring_ceil + static_cast<size_t>(b) * (R + 1);
        double ring = 0.0;
        for (int r = threadIdx.x; r <= s0; r += blockDim.x) ring += e[r];
        ring = block_sum(ring);
        if (threadIdx.x == 0) tot += ring / sc.s3;
    }
    if (threadIdx.x == 0) atomicAdd(&a.scalars[b].s4, tot);
}

// grid (ceil(K/32), ceil(K/32), B): the Split look's normalisers after the
// crop (the canvas holds the shaped kernel; taper applied here):
// s_core = sum of mean * taper, s_struct = sum of max(0, shaped * taper / s3
// - mean * taper) over the crop box.
__global__ void __launch_bounds__(256) split_sums_kernel(PsfBankArgs a) {
    const int b = blockIdx.z;
    const PsfScalars& sc = a.scalars[b];
    const float inv_s3 = static_cast<float>(1.0 / sc.s3);
    const int rho = sc.radius;
    const int K = a.K, R = a.R;
    const float* canvas = a.canvas + static_cast<size_t>(b) * K * K;
    const float* rm = a.ring_mean + static_cast<size_t>(b) * (R + 1);
    const int x = blockIdx.x * kTile + threadIdx.x;
    double lcore = 0.0, lstruct = 0.0;
#pragma unroll
    for (int i = 0; i < kTile / 8; ++i) {
        const int y = blockIdx.y * kTile + threadIdx.y + 8 * i;
        if (x < K && y < K) {
            const int ix = x - R, iy = y - R;
            if (abs(ix) <= rho && abs(iy) <= rho) {
                const float dx = static_cast<float>(ix), dy = static_cast<float>(iy);
                const float rad = sqrtf(dx * dx + dy * dy);
                const float wgt = taper_weight(rad, sc.extent, sc.fade, sc.start);
                const float mt = rm[min(R, static_cast<int>(roundf(rad)))] * wgt;
                lcore += static_cast<double>(mt);
                lstruct += static_cast<double>(fmaxf(0.0f, (canvas[static_cast<size_t>(y) * K + x] * wgt) * inv_s3 - mt));
            }
        }
    }
    const double tc = block_sum(lcore);
    if (threadIdx.x == 0 && threadIdx.y == 0) atomicAdd(&a.scalars[b].s_core, tc);
    __syncthreads();
    const double ts = block_sum(lstruct);
    if (threadIdx.x == 0 && threadIdx.y == 0) atomicAdd(&a.scalars[b].s_struct, ts);
}

// grid (ceil(K/32), ceil(K/32)), block (32, 8): out[k] = sum_b coef[k][b] *
// final_b with final_b = crop_b(canvas_b * taper_b) / (s3_b * s4_b): the crop
// box and boundary taper of each wavelength (cropKernelToRadius,
// applySupportBoundaryTaper, LensDiffCpuReference.cpp:1038-1058, :957-982)
// are applied here as the shaped kernels are read.  Eight wavelengths'
// reads are issued before any is used.  SPLIT: the core and structure
// kernels of the Split look instead.
struct CombineBin {
    float w[4];                // coef[k][b] / (s3 s4)
    float ext, fade, start;    // taper
    int rho;                   // crop radius
};

// NK: kernel sets of the Physical look (1 Mono, 3 spectral; 4 covers any n_ker <= 4).
template <bool SPLIT, int NK>
__global__ void __launch_bounds__(256) combine_kernel(CombineArgs a) {
    __shared__ float inv[kMaxBins], inv_s3[kMaxBins], inv_core[kMaxBins], inv_struct[kMaxBins];
    __shared__ float ext[kMaxBins], fade[kMaxBins], start[kMaxBins];
    __shared__ int rho[kMaxBins];
    __shared__ CombineBin bin[kMaxBins];
    const int tid = threadIdx.x + threadIdx.y * 32;
    const int B = a.bank.B;
    for (int b = tid; b < B; b += 256) {
        const PsfScalars& sc = a.bank.scalars[b];
        const float ib = static_cast<float>(1.0 / (sc.s3 * sc.s4));
        for (int k = 0; k < 4; ++k) bin[b].w[k] = a.coef[k][b] * ib;
        bin[b].ext = sc.extent;
        bin[b].fade = sc.fade;
        bin[b].start = sc.start;
        bin[b].rho = sc.radius;
        inv[b] = ib;
        inv_s3[b] = static_cast<float>(1.0 / sc.s3);
        inv_core[b] = sc.s_core > 0.0 ? static_cast<float>(1.0 / sc.s_core) : 0.0f;
        inv_struct[b] = sc.s_struct > 0.0 ? static_cast<float>(1.0 / sc.s_struct) : 0.0f;
        ext[b] = sc.extent;
        fade[b] = sc.fade;
        start[b] = sc.start;
        rho[b] = sc.radius;
    }
    __syncthreads();
    const int x = blockIdx.x * kTile + threadIdx.x;
    const int K = a.bank.K, R = a.bank.R;
    const size_t plane = static_cast<size_t>(K) * K;
    if constexpr (!SPLIT) {
        // four pixels per thread (rows 8 apart) share each wavelength's bin
        // constants; per pixel the wavelengths are summed in order, as below
        constexpr int kP = kTile / 8;
        float acc[kP][NK], rad[kP];
        int aix[kP];
        size_t idx[kP];
#pragma unroll
        for (int p = 0; p < kP; ++p) {
            const int y = blockIdx.y * kTile + threadIdx.y + 8 * p;
            const bool in = x < K && y < K;
            const int ix = x - R, iy = y - R;
            aix[p] = in ? max(abs(ix), abs(iy)) : INT_MAX;  // inside the crop box of b iff aix <= rho[b]
            const float dx = static_cast<float>(ix), dy = static_cast<float>(iy);
            rad[p] = sqrtf(dx * dx + dy * dy);
            idx[p] = in ? static_cast<size_t>(y) * K + x : 0;
#pragma unroll
            for (int k = 0; k < NK; ++k) acc[p][k] = 0.0f;
        }
        // kL wavelengths' reads are issued before any of them is used, so
        // kL * kP reads per thread are in flight over the canvases
        constexpr int kL = 4;
        for (int b0 = 0; b0 < B; b0 += kL) {
            float v[kL][kP];
#pragma unroll
            for (int l = 0; l < kL; ++l) {
                const int b = b0 + l;
                const int rho_b = b < B ? bin[b].rho : -1;
                const float* cv = a.bank.canvas + static_cast<size_t>(b < B ? b : 0) * plane;
#pragma unroll
                for (int p = 0; p < kP; ++p) v[l][p] = aix[p] <= rho_b ? __ldg(cv + idx[p]) : 0.0f;
            }
#pragma unroll
            for (int l = 0; l < kL; ++l) {  // per pixel the wavelengths are summed in order
                const int b = b0 + l;
                if (b >= B) break;
                const CombineBin& cb = bin[b];
                const float ext_b = cb.ext, fade_b = cb.fade, start_b = cb.start;
                float w[NK];
#pragma unroll
                for (int k = 0; k < NK; ++k) w[k] = cb.w[k];
#pragma unroll
                for (int p = 0; p < kP; ++p) {
                    if (v[l][p] != 0.0f) {  // else outside the crop box, or a zero kernel value
                        const float f = v[l][p] * taper_weight(rad[p], ext_b, fade_b, start_b);
#pragma unroll
                        for (int k = 0; k < NK; ++k) acc[p][k] += w[k] * f;
                    }
                }
            }
        }
#pragma unroll
        for (int p = 0; p < kP; ++p) {
            if (aix[p] == INT_MAX) continue;
#pragma unroll
            for (int k = 0; k < NK; ++k)
                if (k < a.n_ker) a.out[k * plane + idx[p]] = acc[p][k];
        }
        return;
    }
#pragma unroll 1
    for (int i = 0; i < kTile / 8; ++i) {  // Split look
        const int y = blockIdx.y * kTile + threadIdx.y + 8 * i;
        if (x >= K || y >= K) continue;
        const size_t idx = static_cast<size_t>(y) * K + x;
        const int ix = x - R, iy = y - R;
        const int aix = max(abs(ix), abs(iy));  // inside the crop box of b iff aix <= rho[b]
        const float dx = static_cast<float>(ix), dy = static_cast<float>(iy);
        const float rad = sqrtf(dx * dx + dy * dy);
        {
        // Split: core = mean * taper / s_core, structure = max(0, shaped *
        // taper / s3 - mean * taper) / s_struct
        const int ring = min(R, static_cast<int>(roundf(rad)));
        float core[4] = {0.0f, 0.0f, 0.0f, 0.0f}, strc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (int b = 0; b < B; ++b) {
            if (aix > rho[b]) continue;
            const float wgt = taper_weight(rad, ext[b], fade[b], start[b]);
            const float mt = a.bank.ring_mean[static_cast<size_t>(b) * (R + 1) + ring] * wgt;
            const float c = mt * inv_core[b];
            const float st = fmaxf(0.0f, (a.bank.canvas[b * plane + idx] * wgt) * inv_s3[b] - mt) * inv_struct[b];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                core[k] += a.coef[k][b] * c;
                strc[k] += a.coef[k][b] * st;
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k >= a.n_ker) break;
            a.out[k * plane + idx] = core[k];
            a.out[(a.n_ker + k) * plane + idx] = strc[k];
        }
        }
    }
}

// grid (ceil(K/32), ceil(K/32), B): final kernels packed at offsets[b].
__global__ void __launch_bounds__(256) export_kernel(PsfBankArgs a, const int64_t* offsets, float* out) {
    const int b = blockIdx.z;
    const PsfScalars& sc = a.scalars[b];
    const int rho = sc.radius;
    const int side = 2 * rho + 1;
    const float inv = static_cast<float>(1.0 / (sc.s3 * sc.s4));
    const float* canvas = a.canvas + static_cast<size_t>(b) * a.K * a.K;
    const int x = blockIdx.x * kTile + threadIdx.x;
    for (int i = 0; i < kTile / 8; ++i) {
        const int y = blockIdx.y * kTile + threadIdx.y + 8 * i;
        if (x >= a.K || y >= a.K) continue;
        const int ix = x - a.R + rho, iy = y - a.R + rho;
        if (ix < 0 || iy < 0 || ix >= side || iy >= side) continue;
        const float dx = static_cast<float>(x - a.R), dy = static_cast<float>(y - a.R);
        const float wgt = taper_weight(sqrtf(dx * dx + dy * dy), sc.extent, sc.fade, sc.start);
        out[offsets[b] + static_cast<int64_t>(iy) * side + ix] = (canvas[static_cast<size_t>(y) * a.K + x] * wgt) * inv;
    }
}

// ---- first-minimum calibration ------------------------------------------------------
// grid (ceil(S/32), ceil(S/32)), block (32, 8): sums and counts of the shifted
// intensity by round(r) around shiftedSpectrumCenterCoordinate.
// The window psf[y * stride + x], x, y < n, is the square of the shifted PSF
// starting at (x0, x0); total == null: the caller supplies the full PSF's sum.
__global__ void __launch_bounds__(256) profile_kernel(const float* psf, int stride, int n, int x0, int S,
                                                      double* sums, int* counts, double* total) {
    __shared__ double rs[kRingSpan];
    __shared__ int rc[kRingSpan];
    const int tid = threadIdx.x + threadIdx.y * 32;
    const float c = (S & 1) == 0 ? static_cast<float>(S) * 0.5f : static_cast<float>(S - 1) * 0.5f;
    const int ci = static_cast<int>(c);
    const int rmax = S / 2;
    const int tx0 = blockIdx.x * kTile, ty0 = blockIdx.y * kTile;
    const int rbase = tile_ring_base(x0 + tx0, x0 + ty0, ci, rmax);
    for (int i = tid; i < kRingSpan; i += 256) {
        rs[i] = 0.0;
        rc[i] = 0;
    }
    __syncthreads();
    double lsum = 0.0;
    const int x = tx0 + threadIdx.x;
    for (int i = 0; i < kTile / 8; ++i) {
        const int y = ty0 + threadIdx.y + 8 * i;
        if (x < n && y < n) {
            const float dx = static_cast<float>(x0 + x) - c;
            const float dy = static_cast<float>(x0 + y) - c;
            const int r = min(rmax, static_cast<int>(roundf(sqrtf(dx * dx + dy * dy))));
            const float v = psf[static_cast<size_t>(y) * stride + x];
            lsum += v;
            atomicAdd(&rs[r - rbase], static_cast<double>(v));
            atomicAdd(&rc[r - rbase], 1);
        }
    }
    __syncthreads();
    for (int i = tid; i < kRingSpan; i += 256) {
        if (rc[i] != 0 && rbase + i <= rmax) {
            atomicAdd(&sums[rbase + i], rs[i]);
            atomicAdd(&counts[rbase + i], rc[i]);
        }
    }
    if (total) {
        const double tot = block_sum(lsum);
        if (tid == 0) atomicAdd(total, tot);
    }
}

__device__ float refine_parabolic(double l, double c, double r) {
    const double den = l - 2.0 * c + r;
    if (fabs(den) < 1e-6) return 0.0f;
    return static_cast<float>(fmin(fmax(0.5 * (l - r) / den, -0.5), 0.5));
}

// One thread: radialMeanProfile normalised by the total, [1,2,1]/4 smoothing,
// first local minimum after >= 2 descents with parabolic refinement, fallback
// argmin over [1, max(4, S/8)] (LensDiffCpuReference.cpp:897-955).
// n: rings profiled (S / 2 + 1 for the whole PSF); truncated: the rings past
// n exist but were not profiled, so a scan that finds no minimum inside them
// reports r0 = -1 instead of taking the fallback over all rings.
__global__ void first_zero_scan_kernel(const double* sums, const int* counts, const double* total, int S, int n,
                                       int truncated, double* prof, float* r0) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double t = *total > 0.0 ? *total : 1.0;
    for (int r = 0; r < n; ++r) prof[r] = (sums[r] / t) / max(1, counts[r]);
    if (n < 4) {
        *r0 = 1.0f;
        return;
    }
    double* sm = prof + n;
    for (int i = 0; i < n; ++i) {
        const double left = prof[i == 0 ? 0 : i - 1];
        const double right = prof[i + 1 < n ? i + 1 : i];
        sm[i] = (left + 2.0 * prof[i] + right) * 0.25;
    }
    int best = 1;
    double bestv = sm[1];
    int desc = sm[1] < sm[0] ? 1 : 0;
    for (int i = 2; i + 1 < n; ++i) {
        if (sm[i] <= sm[i - 1]) {
            desc += 1;
            if (sm[i] < bestv) {
                bestv = sm[i];
                best = i;
            }
            continue;
        }
        if (desc >= 2 && best > 0 && best + 1 < n) {
            *r0 = fmaxf(1.0f, static_cast<float>(best) + refine_parabolic(sm[best - 1], sm[best], sm[best + 1]));
            return;
        }
        best = i;
        bestv = sm[i];
        desc = 0;
    }
    if (truncated) {
        *r0 = -1.0f;
        return;
    }
    const int limit = max(2, min(n - 1, max(4, S / 8)));
    best = 1;
    bestv = sm[1];
    for (int i = 2; i <= limit; ++i) {
        if (sm[i] < bestv) {
            bestv = sm[i];
            best = i;
        }
    }
    if (best > 0 && best + 1 < n)
        *r0 = fmaxf(1.0f, static_cast<float>(best) + refine_parabolic(sm[best - 1], sm[best], sm[best + 1]));
    else
        *r0 = static_cast<float>(best);
}

// scale * sum of the squared pupil amplitude: by Parseval, the sum of the
// unnormalised S x S PSF when scale = S^2.
__global__ void __launch_bounds__(256) pupil_energy_kernel(PsfBankArgs a, double scale, double* out) {
    const int n = a.pupil.size * a.pupil.size;
    double acc = 0.0;
    for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
        const float amp = a.pupil_pre[i].x;
        acc += static_cast<double>(amp) * amp;
    }
    const double t = block_sum(acc);
    if (threadIdx.x == 0) atomicAdd(out, t * scale);
}

__global__ void normalize_psf_kernel(float* psf, int64_t n, const PsfScalars* sc) {
    const double e = sc->energy;
    const float inv = e > 0.0 ? static_cast<float>(1.0 / e) : 1.0f;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x)
        psf[i] *= inv;
}

// ---- launch helpers ---------------------------------------------------------------
// Row pass: one length-S transform per CTA.  Column pass: C adjacent window
// columns per CTA, C = 4 / 2 / 1 for S <= 2048 / 4096 / larger (S * C <= 8192
// keeps the E = 25 family up to S = 4096).
template <int E>
void rows_launch(const PsfBankArgs& a, cudaStream_t s) {
    dim3 grid(a.row_n, a.B);
    psf_rows_kernel<E><<<grid, fft_threads(a.S, 1, E), a.S * sizeof(float2), s>>>(a);
}

template <int E, int C>
void cols_launch(const PsfBankArgs& a, cudaStream_t s) {
    dim3 grid((a.win_stride + C - 1) / C, a.B);
    psf_cols_kernel<E, C><<<grid, fft_threads(a.S, C, E), static_cast<size_t>(a.S) * C * sizeof(float2), s>>>(a);
}

dim3 tall_grid(const PsfBankArgs& a) {
    return dim3((a.K + kTile - 1) / kTile, (a.K + kTallH - 1) / kTallH, a.B);
}

dim3 canvas_grid(const PsfBankArgs& a, int z) {
    return dim3((a.K + kTile - 1) / kTile, (a.K + kTile - 1) / kTile, z);
}

template <class Kern>
void opt_in(Kern k, size_t bytes) {
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
}

}  // namespace

void launch_pupil_pre(const PsfBankArgs& a, cudaStream_t s) {
    const int n = a.pupil.size * a.pupil.size;
    pupil_pre_kernel<<<(n + 255) / 256, 256, 0, s>>>(a);
}

void launch_psf_rows(const PsfBankArgs& a, cudaStream_t s) {
    if (fft_family(a.S, 1) == kE25) rows_launch<kE25>(a, s);
    else rows_launch<kE16>(a, s);
}

void launch_psf_cols(const PsfBankArgs& a, cudaStream_t s) {
    if (a.S <= 2048) cols_launch<kE25, 4>(a, s);
    else if (a.S <= 4096) cols_launch<kE25, 2>(a, s);
    else if (fft_family(a.S, 1) == kE25) cols_launch<kE25, 1>(a, s);
    else cols_launch<kE16, 1>(a, s);
}

bool fused_shaping(const PsfBankArgs& a) { return a.gain == 1.0f; }

// The bank's wavelengths from b0 on, as a bank of their own (the per-wavelength
// arrays the canvas passes index by wavelength, advanced to b0).
PsfBankArgs bank_from(const PsfBankArgs& a, int b0) {
    PsfBankArgs t = a;
    const size_t rr = static_cast<size_t>(a.R) + 1;
    t.wl = a.wl + b0;
    t.win = a.win + static_cast<size_t>(b0) * a.win_stride * a.win_stride;
    t.canvas = a.canvas + static_cast<size_t>(b0) * a.K * a.K;
    t.ring_round = a.ring_round + b0 * rr;
    t.ring_ceil = a.ring_ceil + b0 * rr;
    t.ring_peak = a.ring_peak + b0 * rr;
    t.ring_mean = a.ring_mean ? a.ring_mean + b0 * rr : nullptr;
    t.scalars = a.scalars + b0;
    t.B = a.B - b0;
    return t;
}

// Wavelengths in pairs (resample_pair_kernel) when none is box-filtered, the
// last one of an odd count on its own; else one per CTA.
void launch_resample(const PsfBankArgs& a, bool pairs, cudaStream_t s) {
    const bool fused = fused_shaping(a);
    if (!pairs) {
        if (fused) resample_kernel<true><<<tall_grid(a), dim3(32, 8), 0, s>>>(a);
        else resample_kernel<false><<<tall_grid(a), dim3(32, 8), 0, s>>>(a);
        return;
    }
    if (a.B >= 2) {
        dim3 g = tall_grid(a);
        g.z = a.B / 2;
        if (fused) resample_pair_kernel<true><<<g, dim3(32, 8), 0, s>>>(a);
        else resample_pair_kernel<false><<<g, dim3(32, 8), 0, s>>>(a);
    }
    if (a.B & 1) {
        const PsfBankArgs t = bank_from(a, a.B - 1);
        if (fused) resample_kernel<true><<<tall_grid(t), dim3(32, 8), 0, s>>>(t);
        else resample_kernel<false><<<tall_grid(t), dim3(32, 8), 0, s>>>(t);
    }
}

void launch_shape_stats(const PsfBankArgs& a, cudaStream_t s) {
    ring_mean_kernel<<<a.B, 256, 0, s>>>(a);
    shape_stats_kernel<<<tall_grid(a), dim3(32, 8), 0, s>>>(a);
}

void launch_ring_means(const PsfBankArgs& a, cudaStream_t s) {
    ring_sums_kernel<<<tall_grid(a), dim3(32, 8), 0, s>>>(a);
    ring_mean_kernel<<<a.B, 256, 0, s>>>(a);
}

void launch_support(const PsfBankArgs& a, cudaStream_t s) { support_kernel<<<a.B, 256, 0, s>>>(a); }

void launch_crop_sum(const PsfBankArgs& a, cudaStream_t s) {
    crop_sum_kernel<<<dim3((a.K + kCropRows - 1) / kCropRows, a.B), 256, 0, s>>>(a);
}

void launch_split_sums(const PsfBankArgs& a, cudaStream_t s) {
    split_sums_kernel<<<canvas_grid(a, a.B), dim3(32, 8), 0, s>>>(a);
}

void launch_combine(const CombineArgs& a, cudaStream_t s) {
    const dim3 grid = canvas_grid(a.bank, 1), block(32, 8);
    if (a.split) combine_kernel<true, 4><<<grid, block, 0, s>>>(a);
    else if (a.n_ker == 1) combine_kernel<false, 1><<<grid, block, 0, s>>>(a);
    else if (a.n_ker == 3) combine_kernel<false, 3><<<grid, block, 0, s>>>(a);
    else combine_kernel<false, 4><<<grid, block, 0, s>>>(a);
}

void launch_export(const PsfBankArgs& a, const int64_t* offsets_dev, float* out, cudaStream_t s) {
    export_kernel<<<canvas_grid(a, a.B), dim3(32, 8), 0, s>>>(a, offsets_dev, out);
}

void launch_first_zero(const float* psf, int S, double* ring_sums, int* ring_counts, double* total, float* r0_out,
                       cudaStream_t s) {
    launch_first_zero_window(psf, S, S, 0, S, S / 2 + 1, ring_sums, ring_counts, total, true, r0_out, s);
}

void launch_first_zero_window(const float* psf, int stride, int n, int x0, int S, int rings, double* ring_sums,
                              int* ring_counts, double* total, bool own_total, float* r0_out, cudaStream_t s) {
    dim3 grid((n + kTile - 1) / kTile, (n + kTile - 1) / kTile);
    profile_kernel<<<grid, dim3(32, 8), 0, s>>>(psf, stride, n, x0, S, ring_sums, ring_counts,
                                                own_total ? total : nullptr);
    // profile scratch follows the ring sums: 2 * (S/2 + 1) doubles
    first_zero_scan_kernel<<<1, 32, 0, s>>>(ring_sums, ring_counts, total, S, rings, rings < S / 2 + 1 ? 1 : 0,
                                            ring_sums + (S / 2 + 1), r0_out);
}

void launch_pupil_energy(const PsfBankArgs& a, double scale, double* out, cudaStream_t s) {
    pupil_energy_kernel<<<64, 256, 0, s>>>(a, scale, out);
}

void launch_normalize_psf(float* psf, int n, const PsfScalars* sc, cudaStream_t s) {
    normalize_psf_kernel<<<592, 256, 0, s>>>(psf, static_cast<int64_t>(n), sc);
}

void configure_psf_kernels() {
    opt_in(psf_rows_kernel<kE25>, 12800 * 8);
    opt_in(psf_rows_kernel<kE16>, 16384 * 8);
    opt_in(psf_cols_kernel<kE25, 4>, 2048 * 4 * 8);
    opt_in(psf_cols_kernel<kE25, 2>, 4096 * 2 * 8);
    opt_in(psf_cols_kernel<kE25, 1>, 12800 * 8);
    opt_in(psf_cols_kernel<kE16, 1>, 16384 * 8);
}

}  // namespace ld
