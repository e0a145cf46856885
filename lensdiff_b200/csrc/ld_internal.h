// ld_internal.h — argument blocks and launchers shared by the host
// orchestration (ld_host.cu) and the kernels (ld_psf.cu, ld_frame.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <tuple>
#include <vector>

#include "ld_fft.cuh"
#include "ld_optics.cuh"

namespace ld {

constexpr int kMaxBins = 64;  // LD_MAX_WAVELENGTHS

// ---- PSF bank -----------------------------------------------------------------
// Per-wavelength constants, computed on the host with the reference's float
// expressions (LensDiffCpuReference.cpp:1720-1731, :1069-1071, :343-345).
struct WavelengthInfo {
    PhaseCoeffs phase;
    float inv_scale;   // 1 / max(scaleFactor, 0.05f)
    int taps;          // box-filter taps (0: plain bilinear)
    float step;        // footprint / taps
    int win_x0;        // window origin in shifted PSF coordinates
    int win_n;         // window side (<= S)
};

struct PsfScalars {      // per wavelength, FP64 sums of the shaping chain
    double s1;           // sum of resampled values
    double s2;           // sum of the azimuthal-mean kernel (unnormalised)
    double s3;           // sum of the shaped kernel (unnormalised)
    double s4;           // sum of the cropped, tapered, normalised kernel
    double energy;       // sum of |F|^2 over the computed window (raw PSF export)
    double s_core;       // Split look: sum of mean * taper over the crop box
    double s_struct;     // Split look: sum of max(0, shaped / s3 - mean) * taper over the crop box
    unsigned int peak;   // max shaped value (float bits)
    int radius;          // adaptive support radius
    float extent, fade, start;  // taper constants
};

struct PsfBankArgs {
    PupilParams pupil;
    PhaseCoeffs base_phase;      // every coefficient but defocus (λ independent)
    float4* pupil_pre;           // [N_p][N_p]: amplitude, phi0, z4, phase valid
    int row_lo, row_n;           // pupil rows that can be non-zero
    const WavelengthInfo* wl;    // [B]
    int B;
    int S;                       // raw PSF size
    int half;                    // S / 2 (integer)
    int off;                     // (S - N_p) / 2
    int win_stride;              // max window side over wavelengths
    float raw_center;            // shiftedSpectrumCenterCoordinate(S)
    int R;                       // R_max
    int K;                       // 2 R_max + 1
    float gain;                  // 1 + 4 max(0, anisotropy)
    FftPlan plan_s;              // length S
    float2* rows;                // [B][N_p][win_stride] row-pass output
    float* win;                  // [B][win_stride][win_stride] |F|^2 windows
    float* canvas;               // [B][K][K] resampled kernels
    double* ring_round;          // [B][R+1] sums by round(r)
    double* ring_ceil;           // [B][R+1] sums by ceil(r)
    unsigned int* ring_peak;     // [B][R+1] max by ceil(r) (float bits)
    float* ring_mean;            // [B][R+1] normalised azimuthal mean by round(r)
    const int* count_round;      // [R+1] pixel counts by round(r)
    PsfScalars* scalars;         // [B]
    int want_energy;
};

void launch_pupil_pre(const PsfBankArgs& a, cudaStream_t s);
void launch_psf_rows(const PsfBankArgs& a, cudaStream_t s);
void launch_psf_cols(const PsfBankArgs& a, cudaStream_t s);
// pairs: every wavelength samples without a box filter (taps 0), so a tile's
// two wavelengths can share one staged pass (resample_pair_kernel)
void launch_resample(const PsfBankArgs& a, bool pairs, cudaStream_t s);
void launch_shape_stats(const PsfBankArgs& a, cudaStream_t s);
// Anisotropy gain 1: shaping is the identity; launch_resample then takes the
// shaped kernel's statistics and launch_shape_stats is not needed.  The ring
// means (Split look) then come from launch_ring_means when first needed.
bool fused_shaping(const PsfBankArgs& a);
void launch_ring_means(const PsfBankArgs& a, cudaStream_t s);
void launch_support(const PsfBankArgs& a, cudaStream_t s);
void launch_crop_sum(const PsfBankArgs& a, cudaStream_t s);
void launch_split_sums(const PsfBankArgs& a, cudaStream_t s);  // s_core, s_struct (Split look)

// Combination of the per-wavelength final kernels into n_ker output kernels:
// out[k][i] = sum_b coef[k][b] * final_b[i].
// Split look: 2 * n_ker planes, the core kernels (azimuthal mean, cropped,
// tapered, normalised; populatePsfBankCacheFromBaseKernels,
// LensDiffCpuReference.cpp:1631-1645) then the structure kernels (positive
// residual of the shaped kernel over the mean, same crop).
struct CombineArgs {
    PsfBankArgs bank;
    int n_ker;
    int split;
    float coef[4][kMaxBins];
    float* out;                  // [n_ker][K][K], Split: [2][n_ker][K][K]
};
void launch_combine(const CombineArgs& a, cudaStream_t s);

// Packs each wavelength's final (cropped) kernel back to back at offsets[b].
void launch_export(const PsfBankArgs& a, const int64_t* offsets_dev, float* out, cudaStream_t s);

// Radial profile of a full S x S intensity and the first-minimum scan
// (LensDiffCpuReference.cpp:865-955).
void launch_first_zero(const float* psf, int S, double* ring_sums, int* ring_counts, double* total,
                       float* r0_out, cudaStream_t s);
// The same scan over a window of the shifted PSF: psf[y * stride + x] for
// x, y < n is the PSF at (x0 + x, x0 + y); the first `rings` rings are
// complete in it.  own_total = false: *total already holds the whole PSF's
// sum.  r0 = -1 when the window holds no minimum.
void launch_first_zero_window(const float* psf, int stride, int n, int x0, int S, int rings, double* ring_sums,
                              int* ring_counts, double* total, bool own_total, float* r0_out, cudaStream_t s);
// scale * sum of the squared pupil amplitude added to *out.
void launch_pupil_energy(const PsfBankArgs& a, double scale, double* out, cudaStream_t s);

// Shifted full raw PSF export: window covers all of S x S; writes psf / energy.
void launch_normalize_psf(float* psf, int n, const PsfScalars* sc, cudaStream_t s);

// ---- kernel spectra and frame chain ------------------------------------------------
// Spectrum columns k = 0..M (the M + 1 bins of the real row transforms) are
// stored column-major with their channels interleaved, so one column of every
// channel is one contiguous block that a single bulk copy moves, and a row
// pass reads or writes C adjacent values per bin:
//   A  [cols][Hp][n_drv]   forward row spectra (Hp = H rounded up to 4)
//   B  [cols][Hp][n_out]   column-pass outputs (rows >= H unused)
//   KR [cols][Kp][n_ker]   kernel row spectra (Kp = K rounded up to even)
//   KS [cols][Py][n_ker]   kernel spectra, scaled by 1 / (M * Py)
struct GridGeom {
    int Px, Py;        // FFT grid
    int M;             // Px / 2
    int cols;          // M + 1 spectrum columns
    int fam_m, fam_py; // FFT families (elements per thread) of the row / column transforms
    FftPlan plan_m;    // length M (real rows via half-length complex)
    FftPlan plan_py;   // length Py (columns)
    const float2* tw_px;  // exp(-2 pi i k / Px), k < Px
};

struct KernelSpectraArgs {
    GridGeom g;
    int n_ker;
    int R, K, Kp;
    const float* canvas;  // [n_ker][K][K]
    float2* rows;         // KR
    float2* spectra;      // KS
    float scale;          // 1 / (M * Py)
    int h16;              // chosen form: KS in FP16 (half2) with one float scale per column
    float* kscale;        // [cols] (h16)
    int ahead;            // column-pass CTAs resident at once (set by the launcher)
    int* err;             // device error word
};
void launch_kspec_rows(const KernelSpectraArgs& a, cudaStream_t s);
void launch_kspec_cols(const KernelSpectraArgs& a, cudaStream_t s);
// Fixed-plan launches (ld_frame_fx.cu): false when no compiled fixed plan
// covers the launch, which then takes the runtime-planned kernel.
struct FrameArgs;
bool fx_launch_frame_rows(const FrameArgs& a, cudaStream_t s);
bool fx_launch_frame_cols(const FrameArgs& a, cudaStream_t s);
bool fx_launch_frame_inverse(const FrameArgs& a, int rows, cudaStream_t s);
bool fx_launch_kspec_rows(const KernelSpectraArgs& a, cudaStream_t s);
bool fx_launch_kspec_cols(const KernelSpectraArgs& a, cudaStream_t s);
void fx_configure();
// ld_selftest.cu: one bounded-wait self-test (LD_SELFTEST_*) on `err`.
int launch_wait_selftest(int mode, long long budget, float4* scratch, int* err, cudaStream_t s);
// FP64 stage twiddle tables of fixed plan `id` (ld_fxplans.h).
std::vector<float2> fx_stage_table(int id);
size_t kspec_cols_smem(int Py, int Kp, int n_ker);

struct SelectionParams {
    int luma;              // extraction mode
    float thr_stops;       // threshold in stops
    float edge0, edge1;    // smoothstep edges in stops
    float thr_linear;      // 0.18 * 2^threshold
    float point_emphasis;
    float rscale;          // 1 - corePreserve
    // signals at or below this give a zero mask: their stops lie below edge0
    // by more than log2f's rounding (0.18 * 2^edge0 * 0.999)
    float sig_zero;
};

// FrameArgs::transfer values (the public LD_TRANSFER_* enum)
constexpr int kTransferLinear = 0;
constexpr int kTransferDavinci = 1;

enum { kEffectComposite = 0, kEffectStore = 1, kEffectAccumulate = 2, kEffectScatter = 3 };
// FrameArgs::debug: what composite_kernel writes (the composite, or a debug view)
enum { kOutComposite = 0, kOutEffect = 1, kOutFringePreview = 2, kOutSelection = 3 };

struct FrameArgs {
    GridGeom g;
    SelectionParams sel;
    int W, H, Hp;
    const unsigned char* src;  // device, row-major float RGBA
    int64_t src_pitch;
    unsigned char* dst;
    int64_t dst_pitch;
    int src_x1, src_y1;        // src bounds origin
    int dst_x1, dst_y1;        // dst bounds origin
    int out_x1, out_y1, out_x2, out_y2;  // render window intersect dst bounds
    int n_drv;                 // 1 (spectral scalar driver) or 3 (Mono RGB)
    int n_out;                 // 3 or 4 (4th: luma-lock target)
    int n_ker;                 // kernels (1 for Mono)
    float2* A;
    float2* Bout;
    const float2* spectra;     // KS; half2 when h16
    int h16;                   // chosen form: KS and B in FP16 with per-column scales, A per row tile
    const float* kscale;       // [cols] (h16)
    float* bscale;             // [cols] (h16)
    // h16 row spectra (n_drv = 1): A holds half2 values, column-major
    // [bin][Hp]; row r's values are its spectrum times 2^-aexp[r] (one
    // exponent per row tile of the forward row pass, stored for each row)
    signed char* aexp;         // [Hp] (h16)
    int ahead;                // CTAs of the launch resident at once: the L2 prefetch distance (set by each launcher)
    int* err;                  // device error word
    // What the inverse pass does with the mapped effect of a row:
    //   kEffectComposite: composite the render window directly (Augment);
    //   kEffectStore: write every source pixel's effect to `effect` and add the
    //     luma sums of the redistributed source and of the effect to sums[0],
    //     sums[1] (Preserve energy, LensDiffCpuReference.cpp:2172-2178);
    //   kEffectAccumulate: add the tent-weighted effect of field zone
    //     (zone_x, zone_y) of a zone_n x zone_n grid to `effect`, source rows
    //     row0 + blockIdx.x (accumulateWeightedImage, :1452-1475).
    //   kEffectScatter: the scatter convolution's inverse pass (Mono chain over
    //     the stored effect, one Gaussian kernel): add scatter * max(0, value)
    //     to every source pixel of `effect` (CpuReference.cpp:2180-2186).
    // composite_kernel then finishes the stored effect, scaling it by
    // sums[0] / sums[1] when `preserve`.  Store skips the sums without it.
    int effect_mode;
    int preserve;
    int zone_x, zone_y, zone_n, row0;  // zone_n = 0: no field zones (weight 1)
    // Overlap-add tiles (field zones): the FFT grid's origin in working-frame
    // pixels (0, 0 for the whole frame; may be negative, pixels outside the
    // frame read as zero).  Grid row / column g is frame row / column
    // g + tile_y0 / g + tile_x0; A and B hold grid rows [0, Hp).  The inverse
    // pass's accumulate mode writes the frame columns [acc_x0, acc_x1).
    int tile_x0, tile_y0;
    int acc_x0, acc_x1;
    // kEffectAccumulate adds weight * gain * shoulder(effect): Split look
    // (core / structure gains and soft shoulders, LensDiffCpuReference.cpp:
    // 2123-2146, :1340-1352); 1 and 0 otherwise
    float acc_gain, acc_shoulder;
    float4* effect;            // [H][W]
    double* sums;              // [2]
    // epilogue
    int mono;
    float saturation;
    int luma_lock;
    float effect_gain, core_comp, max_sub;
    // scatter chain: the forward rows take their three drivers from `effect`
    // (drv_effect = 1) and the inverse adds scatter * max(0, value)
    int drv_effect;
    float scatter;
    // composite of a stored effect (composite_kernel): the creative fringe
    // shift in working pixels (0: off, applyCreativeFringe :1499-1534), and
    // the resolution-aware working frame (work == null: the effect has the
    // source's size).  With `work`, `effect` is [Hw][Ww] and both it and
    // the redistributed working source are resampled to the source frame
    // (resampleRgbaImage :414-434) before the composite.
    float fringe_px;
    float4* work;
    int Ww, Hw;
    // source / output encoding (LD_TRANSFER_*): source pixels are decoded to
    // linear as they are read, output pixels encoded as they are written
    int transfer;
    // composite_kernel output (kOut*); kOutSelection reads the mask maximum
    // (float bits, zeroed by the host) from mask_max
    int debug;
    unsigned int* mask_max;
    // kEffectScatter: store max(0, value) in place of the effect (the scatter
    // debug view) instead of adding scatter * max(0, value)
    int scatter_replace;
};
void launch_frame_rows(const FrameArgs& a, cudaStream_t s);
void launch_frame_cols(const FrameArgs& a, cudaStream_t s);
void launch_frame_inverse(const FrameArgs& a, cudaStream_t s);
void launch_composite(const FrameArgs& a, cudaStream_t s);
// Inverse pass over `rows` CTAs (kEffectAccumulate: source rows row0 + i).
void launch_frame_inverse_rows(const FrameArgs& a, int rows, cudaStream_t s);
void launch_effect_sums(const FrameArgs& a, cudaStream_t s);
// Resolution-aware working source: the source frame (a.src, a.W x a.H)
// resampled to a.Ww x a.Hw into a.work (resampleRgbaImage,
// CpuReference.cpp:414-434).
void launch_resample_source(const FrameArgs& a, cudaStream_t s);
// Column-pass shared memory: spectral (n_out 3 or 4) or Mono (n_out = 0).
size_t frame_cols_smem(int Py, int n_out);

// shared-memory opt-in for every kernel instantiation (once per device)
void configure_kernels();

// ---- chosen form: the pupil-to-PSF transform as DFT-as-GEMM on the tensor
// cores (ld_dftgemm.cu).  Operands are BF16 hi/lo images in the tensor core's
// shared-memory layout, one slab of `rows` x 128 bytes per K-chunk of 32
// complex values.
enum { kDftRows = 0, kDftCols = 1 };
struct DftLambda {
    int n0;     // first window column computed (relative to the union origin; multiple of 4)
    int shift;  // window column 0 is computed column `shift`
    int nt;     // 128-column tiles computed
    int pad;
};
struct DftPlan {
    int col_lo, col_n;         // pupil columns that can be non-zero
    int mt_rows;               // row pass: 128-row tiles of pupil rows
    int kc_rows, kc_cols;      // K-chunks of the row pass (pupil columns) and the column pass (pupil rows)
    int nt_max;                // max tiles over wavelengths
    int x0;                    // union window origin (shifted PSF coordinates)
    int basis_rows;            // rows of the basis images: 2 x padded union width
    unsigned char *pf_hi, *pf_lo;  // pupil fields [B][kc_rows][mt_rows * 128 rows]
    size_t pf_lambda, pf_slab;
    unsigned char *dx_hi, *dx_lo;  // row-pass basis [kc_rows][basis_rows]
    unsigned char *dy_hi, *dy_lo;  // column-pass basis [kc_cols][basis_rows]
    size_t dx_slab, dy_slab;
    unsigned char *yt_hi, *yt_lo;  // row-pass output [B][mt_rows * 4][nt_max * 128 rows]
    size_t yt_lambda, yt_slab;
};
struct DftBasisArgs {
    unsigned char *hi, *lo;
    size_t slab;
    int rows, kc, k_valid, koff, x0, half, S;
};
// One pass of one wavelength of one lens for dft_gemm_kernel: its operands
// (A: 128-row tiles along M; B: the basis, 2 rows per complex output), the
// K-chunks and tile counts, and where the output goes.
struct DftProblem {
    const unsigned char *a_hi, *a_lo;
    const unsigned char *b_hi, *b_lo;
    unsigned char *y_hi, *y_lo;  // kDftRows: the column pass's A images of this problem
    float* win;                  // kDftCols: the window (row-major, win_stride)
    double* energy;              // kDftCols: sum of the window added here (null: none)
    uint32_t a_slab, b_slab, y_slab;  // bytes per K-chunk
    int kc, mt, nt;              // K-chunks; 128-row M tiles; 128-complex N tiles
    int n0, shift;               // first basis column (multiple of 4); window column 0 = computed `shift`
    int win_n, win_stride;
};
struct DftBatchArgs {
    const DftProblem* probs;     // [problems]
    const int* tile_start;       // [problems + 1]: first tile of each problem (mt * nt tiles each)
    int problems, tiles;
    int mode;                    // kDftRows or kDftCols
    int* counter;                // work-queue counter, zero before the launch
    int* err;
};
size_t dft_gemm_smem();
void launch_dft_basis(const DftBasisArgs& a, cudaStream_t s);
void launch_pupil_field(const PsfBankArgs& a, const DftPlan& d, cudaStream_t s);
void launch_dft_gemm(const DftBatchArgs& g, cudaStream_t s);
void configure_dft_kernels();

// ---- static debug views (ld_debug.cu) ----------------------------------------------
// Kernel b of the bank after its crop, taper and normalisation (side
// 2 radius + 1, row-major at out); its maximum (float bits) into *maxv.
void launch_kernel_image(const PsfBankArgs& a, int b, float* out, unsigned int* maxv, cudaStream_t s);
// Pupil amplitude and phase in waves (N_p^2 each) and their maxima.
void launch_pupil_image(const PupilParams& pp, const PhaseCoeffs& c, float* amp, float* phase,
                        unsigned int* amp_max, unsigned int* phase_max, cudaStream_t s);
// OTF magnitude (fftshifted) of a kernel image whose side is 2 sc->radius + 1
// (<= max_side); tmp holds max_side^2 complex doubles.
void launch_otf_image(const float* img, const PsfScalars* sc, int max_side, double2* tmp, float* out,
                      unsigned int* maxv, cudaStream_t s);
// A square image (side 2 sc->radius + 1, or `fixed` when sc is null) drawn
// into the centred square of the output frame: see ld_debug.cu.
void launch_square_view(const FrameArgs& a, const float* img, const PsfScalars* sc, int fixed,
                        const unsigned int* maxv, bool log_view, int channels, bool first, cudaStream_t s);
void launch_phase_view(const FrameArgs& a, const float* amp, const float* phase, int n,
                       const unsigned int* phase_max, cudaStream_t s);

// ---- comparator form: the same chain with cuFFT transforms (ld_cufft.cu) -----------
struct CufftError {
    int code;
    const char* what;
};

// cuFFT plans by (type, ny, nx, batch), destroyed with the cache.
struct CufftPlanCache {
    std::map<std::tuple<int, int, int, int>, int> plans;
    int get(int type, int ny, int nx, int batch);
    void release();
    ~CufftPlanCache();
};

size_t cf_psf_chunk(int S, int B);  // wavelengths per batched S x S transform
void cf_psf_transform(const PsfBankArgs& a, float2* grid, CufftPlanCache& plans, cudaStream_t s);
void cf_kernel_spectra(const KernelSpectraArgs& a, float* planes, CufftPlanCache& plans, cudaStream_t s);
void cf_frame_forward(const FrameArgs& a, float* planes, float2* sd, CufftPlanCache& plans, cudaStream_t s);
void cf_frame_multiply(const FrameArgs& a, const float2* sd, float2* prod, cudaStream_t s);
void cf_frame_inverse(const FrameArgs& a, float2* prod, float* planes, CufftPlanCache& plans, cudaStream_t s);

}  // namespace ld
