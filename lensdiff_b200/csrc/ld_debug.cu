// ld_debug.cu — the lens's static debug views (BuildLensDiffStaticDebugRgba,
// LensDiffCpuReference.cpp:1909-1970): the pupil, the PSF and its OTF, the
// pupil phase, the field-edge PSF and phase, and the chromatic split, each
// drawn into the centred square of the output frame.
//
// Square images (the pupil amplitude, the phase in waves, a bank kernel
// after its crop, taper and normalisation, the OTF magnitude) are built on
// the device with their maxima (float bits, atomicMax; every value is >= 0,
// the phase's by its absolute value); the view kernels then sample them
// bilinearly (sampleSquareBilinear, :316-336) at each output pixel's place in
// the square (visualizeSquareCentered :1416-1450, visualizeSignedPhaseCentered
// :1536-1595).  Image sizes that depend on a kernel's support radius are
// read on the device from the bank's scalars, so nothing returns to the host.
#include <cuda_runtime.h>
#include <stdint.h>

#include "ld_internal.h"
#include "ld_pixel.cuh"

namespace ld {
namespace {

__device__ __forceinline__ void max_bits(unsigned int* m, float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0 && v > 0.0f) atomicMax(m, __float_as_uint(v));
}

// Side of kernel b after its crop (2 radius + 1), or `fixed` when sc is null.
__device__ __forceinline__ int square_side(const PsfScalars* sc, int fixed) {
    return sc ? 2 * sc->radius + 1 : fixed;
}

// Kernel b of the bank as the bank's kernels are exported: the crop box of
// radius rho around the centre, tapered, divided by s3 * s4; row-major with
// side 2 rho + 1 at `out`.  grid (ceil(K / 256), K), block 256.
__global__ void __launch_bounds__(256) kernel_image_kernel(PsfBankArgs a, int b, float* out, unsigned int* maxv) {
    const PsfScalars& sc = a.scalars[b];
    const int rho = sc.radius, side = 2 * rho + 1;
    const int iy = blockIdx.y;
    const int ix = blockIdx.x * 256 + threadIdx.x;
    float v = 0.0f;
    if (iy < side && ix < side) {
        const int y = a.R - rho + iy, x = a.R - rho + ix;
        const float dx = static_cast<float>(x - a.R), dy = static_cast<float>(y - a.R);
        const float wgt = taper_weight(sqrtf(dx * dx + dy * dy), sc.extent, sc.fade, sc.start);
        const float inv = static_cast<float>(1.0 / (sc.s3 * sc.s4));
        v = (a.canvas[static_cast<size_t>(b) * a.K * a.K + static_cast<size_t>(y) * a.K + x] * wgt) * inv;
        out[static_cast<size_t>(iy) * side + ix] = v;
    }
    max_bits(maxv, v);
}

// Pupil amplitude and phase in waves (buildPupilAmplitude :758-822,
// BuildLensDiffPupilPhaseWaves LensDiffPhase.cpp:215-243 with the lens's own
// coefficients); maxima of the amplitude and of |phase|.
__global__ void __launch_bounds__(256) pupil_image_kernel(PupilParams pp, PhaseCoeffs c, float* amp, float* phase,
                                                          unsigned int* amp_max, unsigned int* phase_max) {
    const int n = pp.size;
    const int i = blockIdx.x * 256 + threadIdx.x;
    float av = 0.0f, pv = 0.0f;
    if (i < n * n) {
        const int x = i % n, y = i / n;
        av = pupil_amplitude(pp, x, y);
        pv = pupil_phase(pp, c, x, y);
        amp[i] = av;
        phase[i] = pv;
    }
    max_bits(amp_max, av);
    max_bits(phase_max, fabsf(pv));
}

// OTF magnitude of a square kernel of side n (computeOtfMagnitude
// :1403-1414): |2-D DFT| of the kernel wrapped with its centre at the origin
// (the wrap only multiplies the DFT by a phase), fftshifted by n / 2
// (fftShiftSquare :303-314).  Direct transforms in FP64 with the angles
// reduced exactly (j u mod n): rows then columns.  Pass 1: grid (n, n) over
// (u, row), one output per thread block row; pass 2 the columns with the
// magnitude, shift and maximum.
__global__ void __launch_bounds__(256) otf_rows_kernel(const float* img, const PsfScalars* sc, int fixed,
                                                       double2* t) {
    const int n = square_side(sc, fixed);
    const int row = blockIdx.y;
    const int u = blockIdx.x * 256 + threadIdx.x;
    if (row >= n || u >= n) return;
    double re = 0.0, im = 0.0;
    const float* r = img + static_cast<size_t>(row) * n;
    for (int j = 0; j < n; ++j) {
        const int k = static_cast<int>((static_cast<int64_t>(j) * u) % n);
        double s, cs;
        sincospi(-2.0 * static_cast<double>(k) / static_cast<double>(n), &s, &cs);
        const double v = static_cast<double>(r[j]);
        re += v * cs;
        im += v * s;
    }
    t[static_cast<size_t>(row) * n + u] = make_double2(re, im);
}

__global__ void __launch_bounds__(256) otf_cols_kernel(const double2* t, const PsfScalars* sc, int fixed, float* out,
                                                       unsigned int* maxv) {
    const int n = square_side(sc, fixed);
    const int v = blockIdx.y;
    const int u = blockIdx.x * 256 + threadIdx.x;
    float mag = 0.0f;
    if (v < n && u < n) {
        double re = 0.0, im = 0.0;
        for (int i = 0; i < n; ++i) {
            const int k = static_cast<int>((static_cast<int64_t>(i) * v) % n);
            double s, cs;
            sincospi(-2.0 * static_cast<double>(k) / static_cast<double>(n), &s, &cs);
            const double2 a = t[static_cast<size_t>(i) * n + u];
            re += a.x * cs - a.y * s;
            im += a.x * s + a.y * cs;
        }
        mag = static_cast<float>(sqrt(re * re + im * im));
        // shifted[y][x] = src[(y + n/2) % n][(x + n/2) % n]: src (v, u) lands at
        // ((v - n/2) mod n, (u - n/2) mod n)
        const int h = n / 2;
        const int ys = (v - h + n) % n, xs = (u - h + n) % n;
        out[static_cast<size_t>(ys) * n + xs] = mag;
    }
    max_bits(maxv, mag);
}

// sampleSquareBilinear (LensDiffCpuReference.cpp:316-336) on a row-major
// square of side n.
__device__ __forceinline__ float sample_square(const float* img, int n, float x, float y) {
    if (x < 0.0f || y < 0.0f || x > static_cast<float>(n - 1) || y > static_cast<float>(n - 1)) return 0.0f;
    const int x0 = static_cast<int>(floorf(x)), y0 = static_cast<int>(floorf(y));
    const int x1 = min(x0 + 1, n - 1), y1 = min(y0 + 1, n - 1);
    const float tx = x - static_cast<float>(x0), ty = y - static_cast<float>(y0);
    const float v00 = img[static_cast<size_t>(y0) * n + x0], v10 = img[static_cast<size_t>(y0) * n + x1];
    const float v01 = img[static_cast<size_t>(y1) * n + x0], v11 = img[static_cast<size_t>(y1) * n + x1];
    const float vx0 = v00 + (v10 - v00) * tx;
    const float vx1 = v01 + (v11 - v01) * tx;
    return vx0 + (vx1 - vx0) * ty;
}

// Place of output pixel (sx, sy) of a W x H frame in the centred square, as
// coordinates of a square image of side n; false outside the square.
__device__ __forceinline__ bool square_coords(int sx, int sy, int W, int H, int n, float* px, float* py) {
    const int sq = min(W, H);
    const int xo = (W - sq) / 2, yo = (H - sq) / 2;
    if (sx < xo || sx >= xo + sq || sy < yo || sy >= yo + sq) return false;
    const float nx = static_cast<float>(sx - xo) / static_cast<float>(max(1, sq - 1));
    const float ny = static_cast<float>(sy - yo) / static_cast<float>(max(1, sq - 1));
    *px = nx * static_cast<float>(n - 1);
    *py = ny * static_cast<float>(n - 1);
    return true;
}

// visualizeSquareCentered (:1416-1450) written into the render window of
// the destination: `channels` bit c writes channel c (the chromatic split
// draws one kernel per channel); `first` also writes the other channels (0)
// and alpha 1, and pixels outside the source frame as (0, 0, 0, 1).  One
// output row per CTA.
__global__ void __launch_bounds__(256) square_view_kernel(FrameArgs a, const float* img, const PsfScalars* sc,
                                                          int fixed, const unsigned int* maxv, int log_view,
                                                          int channels, int first) {
    const int n = square_side(sc, fixed);
    const int yo = a.out_y1 + blockIdx.x;
    const int sy = yo - a.src_y1;
    const float mx = __uint_as_float(*maxv);
    const float log_max = log1pf(fmaxf(0.0f, mx) * 1024.0f);
    float* drow = reinterpret_cast<float*>(a.dst + static_cast<int64_t>(yo - a.dst_y1) * a.dst_pitch);
    for (int x = a.out_x1 + threadIdx.x; x < a.out_x2; x += blockDim.x) {
        const int sx = x - a.src_x1;
        float* q = drow + 4 * (x - a.dst_x1);
        const bool inside = sy >= 0 && sy < a.H && sx >= 0 && sx < a.W;
        float d = 0.0f, px, py;
        if (inside && square_coords(sx, sy, a.W, a.H, n, &px, &py)) {
            const float v = sample_square(img, n, px, py);
            if (log_view) d = log_max > 0.0f ? log1pf(fmaxf(0.0f, v) * 1024.0f) / log_max : 0.0f;
            else d = mx > 0.0f ? v / mx : 0.0f;
        }
        if (first) {
            q[0] = (channels & 1) ? d : 0.0f;
            q[1] = (channels & 2) ? d : 0.0f;
            q[2] = (channels & 4) ? d : 0.0f;
            q[3] = 1.0f;
        } else if (inside) {
            if (channels & 1) q[0] = d;
            if (channels & 2) q[1] = d;
            if (channels & 4) q[2] = d;
        }
    }
}

// visualizeSignedPhaseCentered (:1536-1595): black outside the pupil
// (amplitude <= 1e-4), grey where the phase is 0, warm for positive and cool
// for negative phase, scaled by the phase's largest magnitude.
__global__ void __launch_bounds__(256) phase_view_kernel(FrameArgs a, const float* amp, const float* phase, int n,
                                                         const unsigned int* phase_max) {
    const int yo = a.out_y1 + blockIdx.x;
    const int sy = yo - a.src_y1;
    const float mabs = __uint_as_float(*phase_max);
    float* drow = reinterpret_cast<float*>(a.dst + static_cast<int64_t>(yo - a.dst_y1) * a.dst_pitch);
    for (int x = a.out_x1 + threadIdx.x; x < a.out_x2; x += blockDim.x) {
        const int sx = x - a.src_x1;
        float4 out = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        float px, py;
        if (sy >= 0 && sy < a.H && sx >= 0 && sx < a.W && square_coords(sx, sy, a.W, a.H, n, &px, &py) &&
            sample_square(amp, n, px, py) > 1e-4f) {
            const float pv = sample_square(phase, n, px, py);
            const float nv = mabs > 0.0f ? fminf(fmaxf(pv / mabs, -1.0f), 1.0f) : 0.0f;
            const float m = fabsf(nv);
            const float g = 0.18f;
            if (m <= 1e-6f) out = make_float4(g, g, g, 1.0f);
            else if (nv > 0.0f) out = make_float4(g + 0.82f * m, g + 0.28f * m, fmaxf(0.0f, g - 0.12f * m), 1.0f);
            else out = make_float4(fmaxf(0.0f, g - 0.10f * m), g + 0.34f * m, g + 0.80f * m, 1.0f);
        }
        float* q = drow + 4 * (x - a.dst_x1);
        q[0] = out.x;
        q[1] = out.y;
        q[2] = out.z;
        q[3] = out.w;
    }
}

}  // namespace

void launch_kernel_image(const PsfBankArgs& a, int b, float* out, unsigned int* maxv, cudaStream_t s) {
    kernel_image_kernel<<<dim3((a.K + 255) / 256, a.K), 256, 0, s>>>(a, b, out, maxv);
}

void launch_pupil_image(const PupilParams& pp, const PhaseCoeffs& c, float* amp, float* phase,
                        unsigned int* amp_max, unsigned int* phase_max, cudaStream_t s) {
    const int n = pp.size * pp.size;
    pupil_image_kernel<<<(n + 255) / 256, 256, 0, s>>>(pp, c, amp, phase, amp_max, phase_max);
}

void launch_otf_image(const float* img, const PsfScalars* sc, int max_side, double2* tmp, float* out,
                      unsigned int* maxv, cudaStream_t s) {
    const dim3 grid((max_side + 255) / 256, max_side);
    otf_rows_kernel<<<grid, 256, 0, s>>>(img, sc, 0, tmp);
    otf_cols_kernel<<<grid, 256, 0, s>>>(tmp, sc, 0, out, maxv);
}

void launch_square_view(const FrameArgs& a, const float* img, const PsfScalars* sc, int fixed,
                        const unsigned int* maxv, bool log_view, int channels, bool first, cudaStream_t s) {
    const int rows = a.out_y2 - a.out_y1;
    if (rows <= 0) return;
    square_view_kernel<<<rows, 256, 0, s>>>(a, img, sc, fixed, maxv, log_view ? 1 : 0, channels, first ? 1 : 0);
}

void launch_phase_view(const FrameArgs& a, const float* amp, const float* phase, int n,
                       const unsigned int* phase_max, cudaStream_t s) {
    const int rows = a.out_y2 - a.out_y1;
    if (rows <= 0) return;
    phase_view_kernel<<<rows, 256, 0, s>>>(a, amp, phase, n, phase_max);
}

}  // namespace ld
