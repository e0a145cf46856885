// ld_frame.cu — per-frame FFT convolution chain and kernel-spectrum build.
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
#include "ld_frame_kernels.cuh"

namespace ld {
namespace {


// ---- launch helpers -------------------------------------------------------------------
// Launch with a.ahead = the CTAs of f resident at once (the L2 prefetch distance).
template <class Kern>
void launch_ahead(Kern f, FrameArgs a, int grid, int T, size_t sm, cudaStream_t s) {
    a.ahead = resident_ctas(f, T, sm);
    f<<<grid, T, sm, s>>>(a);
}

template <int E>
void rows_e(const FrameArgs& a, cudaStream_t s) {
    const int M = a.g.M;
    if (a.n_drv == 1) {
        // two rows per CTA and three CTAs per SM (register cap 80) when the
        // transform fits 224 threads; else four rows per CTA
        if (fft_threads(M, 2, E) <= 224) {
            const size_t sm = rows_smem(M, 2);
            launch_ahead(frame_rows_kernel<E, 2, 1, 224, 3>, a, a.Hp / 2, fft_threads(M, 2, E), sm, s);
        } else {
            const size_t sm = rows_smem(M, 4);
            launch_ahead(frame_rows_kernel<E, 4, 1>, a, a.Hp / 4, fft_threads(M, 4, E), sm, s);
        }
    } else {
        const size_t sm = rows_smem(M, 3);
        if (a.drv_effect)
            frame_rows_kernel<E, 3, 3, Fam<E>::max_threads, 1, true><<<a.Hp, fft_threads(M, 3, E), sm, s>>>(a);
        else
            launch_ahead(frame_rows_kernel<E, 3, 3>, a, a.Hp, fft_threads(M, 3, E), sm, s);
    }
}

template <int E, class Kern>
void cols_launch(Kern f, FrameArgs a, int C, size_t sm, cudaStream_t s) {
    const int T = fft_threads(a.g.Py, C, E);
    a.ahead = resident_ctas(f, T, sm);
    f<<<a.g.cols, T, sm, s>>>(a);
}

// Spectral column pass: two CTAs per SM (register cap 85) when the transform
// fits 384 threads and two working sets fit shared memory.
template <int E, int NOUT, bool H16>
void cols_spectral_h(const FrameArgs& a, cudaStream_t s) {
    const size_t sm = frame_cols_smem(a.g.Py, NOUT);
    if (fft_threads(a.g.Py, NOUT, E) <= 384 && 2 * sm + 2048 <= static_cast<size_t>(kMaxSmem))
        cols_launch<E>(frame_cols_kernel<E, NOUT, 384, 2, H16>, a, NOUT, sm, s);
    else
        cols_launch<E>(frame_cols_kernel<E, NOUT, Fam<E>::max_threads, 1, H16>, a, NOUT, sm, s);
}

template <int E, int NOUT>
void cols_spectral(const FrameArgs& a, cudaStream_t s) {
    if (a.h16) cols_spectral_h<E, NOUT, true>(a, s);
    else cols_spectral_h<E, NOUT, false>(a, s);
}

template <int E>
void cols_e(const FrameArgs& a, cudaStream_t s) {
    if (a.n_drv == 3) {
        cols_launch<E>(frame_cols_mono_kernel<E>, a, 3, frame_cols_smem(a.g.Py, 0), s);
    } else if (a.n_out == 4) {
        cols_spectral<E, 4>(a, s);
    } else {
        cols_spectral<E, 3>(a, s);
    }
}

template <int E, int C, bool H16>
void inverse_c(const FrameArgs& a, int rows, cudaStream_t s) {
    const int M = a.g.M;
    const int T = fft_threads(M, C, E);
    const size_t sm = static_cast<size_t>(M) * C * sizeof(float2);
    // two CTAs per SM when the transform fits 320 threads (register cap 102)
    if (T <= 320) launch_ahead(frame_inverse_kernel<E, C, 320, 2, H16>, a, rows, T, sm, s);
    else launch_ahead(frame_inverse_kernel<E, C, Fam<E>::max_threads, 1, H16>, a, rows, T, sm, s);
}

template <int E>
void inverse_e(const FrameArgs& a, int rows, cudaStream_t s) {  // rows: grid size
    if (a.n_out == 4) {
        if (a.h16) inverse_c<E, 4, true>(a, rows, s);
        else inverse_c<E, 4, false>(a, rows, s);
    } else {
        if (a.h16) inverse_c<E, 3, true>(a, rows, s);
        else inverse_c<E, 3, false>(a, rows, s);
    }
}

template <int E, int C>
void kspec_rows_c(const KernelSpectraArgs& a, cudaStream_t s) {
    kspec_rows_kernel<E, C><<<a.Kp, fft_threads(a.g.M, C, E), static_cast<size_t>(a.g.M) * C * sizeof(float2), s>>>(
        a);
}

template <int E, int C, bool H16>
void kspec_cols_h(KernelSpectraArgs a, cudaStream_t s) {
    const int T = fft_threads(a.g.Py, C, E);
    const size_t sm = kspec_cols_smem(a.g.Py, a.Kp, C);
    if (C > 1 && T <= 384 && 2 * sm + 2048 <= static_cast<size_t>(kMaxSmem)) {  // C == 1: Mono, one kernel
        // two CTAs per SM (register cap 80)
        auto f = kspec_cols_kernel<E, C, 384, 2, H16>;
        a.ahead = resident_ctas(f, T, sm);
        f<<<a.g.cols, T, sm, s>>>(a);
    } else {
        auto f = kspec_cols_kernel<E, C, Fam<E>::max_threads, 1, H16>;
        a.ahead = resident_ctas(f, T, sm);
        f<<<a.g.cols, T, sm, s>>>(a);
    }
}

template <int E, int C>
void kspec_cols_c(const KernelSpectraArgs& a, cudaStream_t s) {
    if (a.h16) kspec_cols_h<E, C, true>(a, s);
    else kspec_cols_h<E, C, false>(a, s);
}

template <int E>
void kspec_rows_e(const KernelSpectraArgs& a, cudaStream_t s) {
    if (a.n_ker == 4) kspec_rows_c<E, 4>(a, s);
    else if (a.n_ker == 3) kspec_rows_c<E, 3>(a, s);
    else kspec_rows_c<E, 1>(a, s);
}

template <int E>
void kspec_cols_e(const KernelSpectraArgs& a, cudaStream_t s) {
    if (a.n_ker == 4) kspec_cols_c<E, 4>(a, s);
    else if (a.n_ker == 3) kspec_cols_c<E, 3>(a, s);
    else kspec_cols_c<E, 1>(a, s);
}

template <int E>
void configure_e() {
    set_smem(frame_rows_kernel<E, 4, 1>);
    set_smem(frame_rows_kernel<E, 3, 3>);
    set_smem(frame_rows_kernel<E, 3, 3, Fam<E>::max_threads, 1, true>);
    set_smem(frame_cols_kernel<E, 3>);
    set_smem(frame_cols_kernel<E, 4>);
    set_smem(frame_cols_mono_kernel<E>);
    set_smem(frame_inverse_kernel<E, 3>);
    set_smem(frame_inverse_kernel<E, 4>);
    set_smem(frame_inverse_kernel<E, 3, 320, 2>);
    set_smem(frame_cols_kernel<E, 3, 384, 2>);
    set_smem(frame_cols_kernel<E, 4, 384, 2>);
    set_smem(frame_cols_kernel<E, 3, 384, 2, true>);
    set_smem(frame_cols_kernel<E, 4, 384, 2, true>);
    set_smem(frame_cols_kernel<E, 3, Fam<E>::max_threads, 1, true>);
    set_smem(frame_cols_kernel<E, 4, Fam<E>::max_threads, 1, true>);
    set_smem(frame_inverse_kernel<E, 3, 320, 2, true>);
    set_smem(frame_inverse_kernel<E, 4, 320, 2, true>);
    set_smem(frame_inverse_kernel<E, 3, Fam<E>::max_threads, 1, true>);
    set_smem(frame_inverse_kernel<E, 4, Fam<E>::max_threads, 1, true>);
    set_smem(kspec_cols_kernel<E, 3, 384, 2, true>);
    set_smem(kspec_cols_kernel<E, 4, 384, 2, true>);
    set_smem(kspec_cols_kernel<E, 1, Fam<E>::max_threads, 1, true>);
    set_smem(kspec_cols_kernel<E, 3, Fam<E>::max_threads, 1, true>);
    set_smem(kspec_cols_kernel<E, 4, Fam<E>::max_threads, 1, true>);
    set_smem(frame_rows_kernel<E, 2, 1, 224, 3>);
    set_smem(kspec_cols_kernel<E, 3, 384, 2>);
    set_smem(kspec_cols_kernel<E, 4, 384, 2>);
    set_smem(frame_inverse_kernel<E, 4, 320, 2>);
    set_smem(kspec_rows_kernel<E, 1>);
    set_smem(kspec_rows_kernel<E, 3>);
    set_smem(kspec_rows_kernel<E, 4>);
    set_smem(kspec_cols_kernel<E, 1>);
    set_smem(kspec_cols_kernel<E, 3>);
    set_smem(kspec_cols_kernel<E, 4>);
}

}  // namespace

size_t frame_cols_smem(int Py, int n_out) {
    const size_t n = static_cast<size_t>(Py);
    const size_t bufs = n_out == 0 ? 4 * n : (1 + static_cast<size_t>(n_out)) * n;
    return bufs * sizeof(float2) + 4 * sizeof(uint64_t);
}

size_t kspec_cols_smem(int Py, int Kp, int n_ker) {
    return (static_cast<size_t>(Py) + Kp) * n_ker * sizeof(float2) + sizeof(uint64_t);
}

void launch_frame_rows(const FrameArgs& a, cudaStream_t s) {
    if (fx_launch_frame_rows(a, s)) return;
    if (a.g.fam_m == kE25) rows_e<kE25>(a, s);
    else rows_e<kE16>(a, s);
}

void launch_frame_cols(const FrameArgs& a, cudaStream_t s) {
    if (fx_launch_frame_cols(a, s)) return;
    if (a.g.fam_py == kE25) cols_e<kE25>(a, s);
    else cols_e<kE16>(a, s);
}

void launch_frame_inverse(const FrameArgs& a, cudaStream_t s) {
    const int rows = a.effect_mode == kEffectComposite ? a.out_y2 - a.out_y1 : a.H;
    if (rows <= 0) return;
    if (fx_launch_frame_inverse(a, rows, s)) return;
    if (a.g.fam_m == kE25) inverse_e<kE25>(a, rows, s);
    else inverse_e<kE16>(a, rows, s);
}

void launch_frame_inverse_rows(const FrameArgs& a, int rows, cudaStream_t s) {
    if (rows <= 0) return;
    if (fx_launch_frame_inverse(a, rows, s)) return;
    if (a.g.fam_m == kE25) inverse_e<kE25>(a, rows, s);
    else inverse_e<kE16>(a, rows, s);
}

void launch_effect_sums(const FrameArgs& a, cudaStream_t s) { effect_sums_kernel<<<a.H, 256, 0, s>>>(a); }

template <int MODE>
void composite_launch(const FrameArgs& a, bool fringe, bool rs, int rows, cudaStream_t s) {
    if (rs) {
        if (fringe) composite_kernel<MODE, true, true><<<rows, 256, 0, s>>>(a);
        else composite_kernel<MODE, false, true><<<rows, 256, 0, s>>>(a);
    } else {
        if (fringe) composite_kernel<MODE, true, false><<<rows, 256, 0, s>>>(a);
        else composite_kernel<MODE, false, false><<<rows, 256, 0, s>>>(a);
    }
}

void launch_composite(const FrameArgs& a, cudaStream_t s) {
    const int rows = a.out_y2 - a.out_y1;
    if (rows <= 0) return;
    const bool fringe = a.fringe_px > 0.0f, rs = a.work != nullptr;
    switch (a.debug) {
        case kOutEffect:
            composite_launch<kOutEffect>(a, fringe, rs, rows, s);
            break;
        case kOutFringePreview:
            if (rs) composite_kernel<kOutFringePreview, true, true><<<rows, 256, 0, s>>>(a);
            else composite_kernel<kOutFringePreview, true, false><<<rows, 256, 0, s>>>(a);
            break;
        case kOutSelection:
            if (rs) {
                selection_max_kernel<true><<<a.H, 256, 0, s>>>(a);
                composite_kernel<kOutSelection, false, true><<<rows, 256, 0, s>>>(a);
            } else {
                selection_max_kernel<false><<<a.H, 256, 0, s>>>(a);
                composite_kernel<kOutSelection, false, false><<<rows, 256, 0, s>>>(a);
            }
            break;
        default:
            composite_launch<kOutComposite>(a, fringe, rs, rows, s);
    }
}

void launch_resample_source(const FrameArgs& a, cudaStream_t s) {
    if (a.Ww <= 0 || a.Hw <= 0) return;
    resample_source_kernel<<<dim3((a.Ww + 255) / 256, a.Hw), 256, 0, s>>>(a);
}

void launch_kspec_rows(const KernelSpectraArgs& a, cudaStream_t s) {
    if (fx_launch_kspec_rows(a, s)) return;
    if (a.g.fam_m == kE25) kspec_rows_e<kE25>(a, s);
    else kspec_rows_e<kE16>(a, s);
}

void launch_kspec_cols(const KernelSpectraArgs& a, cudaStream_t s) {
    if (fx_launch_kspec_cols(a, s)) return;
    if (a.g.fam_py == kE25) kspec_cols_e<kE25>(a, s);
    else kspec_cols_e<kE16>(a, s);
}

void configure_psf_kernels();

void configure_kernels() {
    configure_psf_kernels();
    configure_dft_kernels();
    configure_e<kE25>();
    configure_e<kE16>();
    fx_configure();
}

}  // namespace ld
