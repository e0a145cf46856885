/*
 * lensdiff_b200.h — C ABI of the B200 (sm_100a) LensDiff diffraction path.
 *
 * The library replaces one call of the LensDiff OpenFX plugin:
 *
 *     bool RunLensDiffCuda(const LensDiffRenderRequest& request,
 *                          const LensDiffParams& params,
 *                          LensDiffPsfBankCache& cache,
 *                          std::string* error);
 *
 * declared at source/src/cuda/LensDiffCuda.h:7-10 and called from
 * source/src/LensDiff.cpp:3833.  The structs below are plain-old-data mirrors
 * of the reference's request and parameter types (source/src/core/
 * LensDiffTypes.h:94-208); enum values keep the reference's declaration order
 * (LensDiffTypes.h:14-91) so a field can be copied with a cast.  No torch or
 * CUDA type appears in a signature: device pointers and the stream travel as
 * `void*`.
 *
 * Every entry point returns an ld_status_code.  On failure `status->stage`
 * holds a short stage string in the reference's style
 * ("missing-source-or-destination-cuda-buffer", ...).  The library never falls
 * back to a CPU path.
 */
#ifndef LENSDIFF_B200_H
#define LENSDIFF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LD_ABI_VERSION 1
#define LD_MAX_WAVELENGTHS 64   /* reference caps at 9 (LensDiffTypes.h:12) */
#define LD_NOLL_COUNT 23        /* Noll index j = 0..22; j = 0 unused      */
#define LD_STAGE_LEN 128

/* ---- status codes ------------------------------------------------------ */
typedef enum {
    LD_OK = 0,
    LD_ERR_ARG = 1,         /* malformed request or parameter             */
    LD_ERR_OOM = 2,         /* device allocation failed                   */
    LD_ERR_BUDGET = 3,      /* request does not fit the HBM budget        */
    LD_ERR_TIMEOUT = 4,     /* a bounded device wait ran out              */
    LD_ERR_CUDA = 5,        /* a CUDA runtime / launch error              */
    LD_ERR_UNSUPPORTED = 6  /* valid reference setting not on this path   */
} ld_status_code;

/* ---- enums (values mirror LensDiffTypes.h:14-91) ------------------------ */
enum { LD_EXTRACT_MAXRGB = 0, LD_EXTRACT_LUMA = 1 };
enum {
    LD_APERTURE_CIRCLE = 0, LD_APERTURE_POLYGON = 1, LD_APERTURE_STAR = 2,
    LD_APERTURE_SPIRAL = 3, LD_APERTURE_CUSTOM = 4, LD_APERTURE_HEXAGON = 5,
    LD_APERTURE_SQUAREGRID = 6, LD_APERTURE_SNOWFLAKE = 7
};
enum { LD_APOD_FLAT = 0, LD_APOD_COSINE = 1, LD_APOD_GAUSSIAN = 2 };
enum { LD_SPECTRAL_MONO = 0, LD_SPECTRAL_TRISTIMULUS = 1, LD_SPECTRAL_5 = 2, LD_SPECTRAL_9 = 3 };
enum { LD_STYLE_NATURAL = 0, LD_STYLE_CYANMAGENTA = 1, LD_STYLE_WARMCOOL = 2 };
enum { LD_LOOK_PHYSICAL = 0, LD_LOOK_SPLIT = 1 };
enum { LD_ENERGY_PRESERVE = 0, LD_ENERGY_AUGMENT = 1 };
/* LensDiffDebugView (LensDiffTypes.h:66-81), same order */
enum {
    LD_DEBUG_FINAL = 0, LD_DEBUG_SELECTION, LD_DEBUG_PUPIL, LD_DEBUG_PSF, LD_DEBUG_OTF, LD_DEBUG_CORE,
    LD_DEBUG_STRUCTURE, LD_DEBUG_EFFECT, LD_DEBUG_PHASE, LD_DEBUG_PHASE_EDGE, LD_DEBUG_FIELD_PSF,
    LD_DEBUG_CHROMATIC_SPLIT, LD_DEBUG_CREATIVE_FRINGE, LD_DEBUG_SCATTER
};
enum { LD_TRANSFER_LINEAR = 0, LD_TRANSFER_DAVINCI_INTERMEDIATE = 1 };
enum { LD_PHASE_OFF = 0, LD_PHASE_ENABLED = 1 };

/* ---- extensions (not in the reference) ---------------------------------- */
enum {
    LD_RGB_FROM_CALLER = 0,  /* natural/style matrices supplied by the caller
                                (the plugin computes them with its own
                                BuildLensDiffSpectrumConfig, LensDiffSpectrum.cpp:380) */
    LD_RGB_GAUSSIAN = 1      /* Gaussian RGB responses: rgb_gauss_center/sigma */
};
enum {
    LD_FFT_OWN_FP32 = 0,     /* hand-written FP32 Stockham chain ("plain")   */
    LD_FFT_OWN_CHOSEN = 1,   /* hand-written chain, FP16 tile-scaled spectra */
    LD_FFT_CUFFT = 2         /* same chain with cuFFT transforms (comparator) */
};

/* ---- request (mirrors LensDiffRenderRequest, LensDiffTypes.h:94-126) ---- */
typedef struct {
    int32_t x1, y1, x2, y2;
} ld_rect;

typedef struct {
    void* data;              /* DEVICE pointer to float RGBA rows           */
    int64_t row_bytes;
    ld_rect bounds;
    int32_t origin_x, origin_y;
    int32_t components;      /* must be 4                                   */
    int32_t bytes_per_component; /* must be 4                               */
} ld_image_view;

typedef struct {
    ld_rect render_window;
    ld_rect frame_bounds;
    ld_image_view src;
    ld_image_view dst;
    int32_t frame_short_side_px;
    int32_t host_enabled_cuda_render;
    void* cuda_stream;       /* cudaStream_t of the host                    */
} ld_render_request;

/* ---- parameters (mirrors LensDiffParams, LensDiffTypes.h:128-208) ------- */
typedef struct {
    int32_t extraction_mode;
    int32_t aperture_mode;
    int32_t apodization_mode;
    int32_t spectral_mode;
    int32_t spectrum_style;
    int32_t look_mode;
    int32_t energy_mode;
    int32_t debug_view;
    int32_t input_transfer;
    int32_t resolution_aware;

    double threshold;
    double softness_stops;
    double point_emphasis;
    double core_preserve;

    int32_t blade_count;
    int32_t vane_count;
    double roundness;
    double rotation_deg;
    double central_obstruction;
    double vane_thickness;
    double diffraction_scale_px;   /* percent of the optics short side      */
    int32_t pupil_resolution;
    int32_t frame_short_side_px;
    double max_kernel_radius_px;   /* percent of the optics short side      */

    int32_t phase_mode;
    int32_t chromatic_affects_luma;
    double phase_defocus;          /* Noll 4  */
    double phase_astigmatism0;     /* Noll 6  */
    double phase_astigmatism45;    /* Noll 5  */
    double phase_coma_x;           /* Noll 8  */
    double phase_coma_y;           /* Noll 7  */
    double phase_spherical;        /* Noll 11 */
    double phase_trefoil_x;        /* Noll 10 */
    double phase_trefoil_y;        /* Noll 9  */
    double phase_secondary_astigmatism0;  /* Noll 12 */
    double phase_secondary_astigmatism45; /* Noll 13 */
    double phase_quadrafoil0;      /* Noll 14 */
    double phase_quadrafoil45;     /* Noll 15 */
    double phase_secondary_coma_x; /* Noll 16 */
    double phase_secondary_coma_y; /* Noll 17 */
    double pupil_decenter_x;
    double pupil_decenter_y;

    double phase_field_strength;
    double phase_field_edge_bias;
    double phase_field_defocus;
    double phase_field_astig_radial;
    double phase_field_astig_tangential;
    double phase_field_coma_radial;
    double phase_field_coma_tangential;
    double phase_field_spherical;
    double phase_field_trefoil_radial;
    double phase_field_trefoil_tangential;
    double phase_field_secondary_astig_radial;
    double phase_field_secondary_astig_tangential;
    double phase_field_quadrafoil_radial;
    double phase_field_quadrafoil_tangential;
    double phase_field_secondary_coma_radial;
    double phase_field_secondary_coma_tangential;

    double spectrum_force;
    double spectrum_saturation;
    double chromatic_focus;
    double chromatic_spread;
    double creative_fringe;
    double scatter_amount;
    double scatter_radius;

    double effect_gain;
    double core_compensation;
    double anisotropy_emphasis;
    double core_gain;
    double structure_gain;
    double core_shoulder;
    double structure_shoulder;

    /* ---- extensions; all-zero keeps the reference's behaviour ---------- */
    int32_t wavelength_count;      /* 0: the spectral_mode's wavelengths    */
    float wavelengths_nm[LD_MAX_WAVELENGTHS];
    int32_t rgb_mode;              /* LD_RGB_FROM_CALLER / LD_RGB_GAUSSIAN   */
    int32_t field_grid;            /* 0: reference 3x3 when field phase on   */
    float natural_matrix[3 * LD_MAX_WAVELENGTHS]; /* row-major 3 x count     */
    float style_matrix[3 * LD_MAX_WAVELENGTHS];
    float rgb_gauss_center_nm[3];  /* R, G, B                                */
    float rgb_gauss_sigma_nm;
    double noll[LD_NOLL_COUNT];    /* added to the named terms; j=2,3,18..22 */
    int32_t fft_form;              /* LD_FFT_OWN_FP32 / _CHOSEN / _CUFFT      */
    int32_t reserved[7];
} ld_params;

typedef struct {
    int32_t code;                  /* ld_status_code                          */
    char stage[LD_STAGE_LEN];      /* reference-style stage string            */
    int32_t bank_rebuilt;          /* 1 if this call rebuilt the PSF bank     */
    int32_t spectra_rebuilt;       /* 1 if the kernel spectra were rebuilt    */
    int32_t pupil_size;            /* N_p                                     */
    int32_t raw_psf_size;          /* S                                       */
    int32_t max_kernel_radius;     /* R_max                                   */
    int32_t support_radius;        /* max adaptive support radius (export)    */
    int32_t grid_requested_w, grid_requested_h;  /* W+K-1, H+K-1              */
    int32_t grid_used_w, grid_used_h;            /* smooth FFT grid used      */
    int32_t wavelength_count;
    int32_t kernel_launches;       /* kernels this call launched              */
} ld_status;

typedef struct ld_ctx ld_ctx;

/* ---- context ------------------------------------------------------------ */
/* Creates a context on `device`.  hbm_budget_bytes = 0 means no budget. */
int ld_create(ld_ctx** out, int device, size_t hbm_budget_bytes);
void ld_destroy(ld_ctx* ctx);
int ld_abi_version(void);
/* Device bytes the context holds (work buffers + caches). */
size_t ld_device_bytes(const ld_ctx* ctx);
/* Drops the cached PSF banks, kernel spectra, DFT bases and pupil pre-pass. */
void ld_clear_caches(ld_ctx* ctx);
/* Reads and clears the context's device error word (synchronising the
 * device): LD_OK if no kernel reported a problem since the last check,
 * LD_ERR_TIMEOUT if a bounded device wait (bulk-copy barrier) gave up. */
int ld_check_device_errors(ld_ctx* ctx, int32_t* error_word);

/* ---- stage timing (CUDA events on the launching stream) ---------------- */
/* Stage ids reported by ld_profile_collect. */
enum {
    LD_STAGE_PSF_ROWS = 0, LD_STAGE_PSF_COLS, LD_STAGE_RESAMPLE, LD_STAGE_SHAPE_STATS,
    LD_STAGE_SUPPORT, LD_STAGE_CROP_SUM, LD_STAGE_COMBINE, LD_STAGE_KSPEC_ROWS,
    LD_STAGE_KSPEC_COLS, LD_STAGE_FRAME_ROWS, LD_STAGE_FRAME_COLS, LD_STAGE_FRAME_INVERSE,
    LD_STAGE_PUPIL, LD_STAGE_COMPOSITE, LD_STAGE_SCATTER, LD_STAGE_WORKING_SOURCE,
    LD_STAGE_DFT_GEMM, LD_STAGE_COUNT
};
/* Per-frame chains are captured into CUDA graphs on first use and replayed
 * when a later frame issues identical launches (same buffers, geometry and
 * parameters); enable = 0 launches every kernel directly.  On by default;
 * graphs are never used while stage profiling is on or when the caller's
 * stream is being captured.  No counterpart in the reference. */
int ld_set_graphs(ld_ctx* ctx, int enable);

/* Autotuner of the frame chain's transforms.  The row length M and column
 * length Py of a frame grid can each run on one of several compiled radix
 * orders (ld_fxplans.h).  With autotuning on (the default), the first frame
 * rendered at a grid, when it composites directly (no field zones, Preserve
 * energy or scatter) and the caller's stream is not being captured, times
 * every order of both lengths on that frame's own buffers with CUDA events
 * (the timed kernels rewrite the same results) and keeps the fastest for
 * later frames of the context: that first frame synchronises its stream a
 * few times.  mode 1: tune (the default); 0: the first compiled order of each
 * length; 2 + k (k <= 7): the k-th compiled order of each length (its last
 * when it has fewer), for tests and offline tuning; -1: the
 * runtime-planned transforms only, no compiled orders.  No counterpart in
 * the reference. */
int ld_set_autotune(ld_ctx* ctx, int mode);
/* The radix order chosen for transform length n: writes up to 4 radices
 * (first stage first) and returns how many, 0 when n has no compiled order
 * or has not been tuned yet.  *shape_out (may be null): the launch shape
 * bits: for a row length 1: the inverse row pass at one more CTA per SM;
 * 2: the forward row pass, 4: the inverse row pass without the L2 prefetch
 * of the rows one resident generation later; for a column length 2: the
 * column pass without its look-ahead prefetch.  *ms_out (may be null): the
 * winner's time per tuned launch group. */
int ld_autotune_choice(ld_ctx* ctx, int32_t n, int32_t* radices_out, int32_t* shape_out, double* ms_out);

/* The Custom aperture mode's image (LD_APERTURE_CUSTOM).  The reference
 * loads it from LensDiffParams::customAperturePath with WIC or ImageIO
 * (LensDiffApertureImage.cpp:301-365), decoding each pixel to an amplitude,
 * then normalises and inverts it as customApertureNormalize /
 * customApertureInvert ask (:367-399) and samples it into the pupil
 * (LensDiffCpuReference.cpp:707-756).  Here the host decodes the file and
 * passes the amplitudes (height rows of width floats, host memory); the
 * library normalises and inverts them the same way, keeps them on the
 * context's device and samples them as the reference does.  Renders in the
 * Custom mode without an image return LD_ERR_ARG
 * "custom-aperture-image-not-set"; values = null clears the image.  A new
 * image invalidates the cached banks of Custom lenses. */
int ld_set_custom_aperture(ld_ctx* ctx, const float* values, int32_t width, int32_t height, int32_t normalize,
                           int32_t invert);

/* ---- kernel spectra between contexts (no counterpart in the reference) ---
 * The kernel spectra of a lens for a width x height source frame (the FFT of
 * the RGB kernels on the frame's grid, what a cold frame builds before its
 * convolution) as one opaque device block, so that one GPU can build them and
 * others take them over NVLink instead of rebuilding: ld_export_kernel_spectra
 * builds them if the context does not hold them yet and copies them to
 * device_dst on `stream` (device_dst null: only *bytes_out is written);
 * ld_import_kernel_spectra installs a block exported for the same parameters
 * and frame size into the context's spectra cache, so the next ld_render of
 * that lens and size starts from them.  Not with field zones or the cuFFT
 * form (LD_ERR_UNSUPPORTED). */
int ld_export_kernel_spectra(ld_ctx* ctx, const ld_params* params, int32_t width, int32_t height, void* device_dst,
                             size_t capacity, size_t* bytes_out, void* stream, ld_status* status);
int ld_import_kernel_spectra(ld_ctx* ctx, const ld_params* params, int32_t width, int32_t height,
                             const void* device_src, size_t bytes, void* stream, ld_status* status);

/* ---- failure detection without a fault (no counterpart in the reference) --
 * ld_selftest_wait runs one CTA that exercises the device-side failure paths
 * every bulk-copy wait of the library relies on, and returns what the
 * context's device error word recorded (cleared afterwards):
 *   LD_SELFTEST_WAIT_TIMEOUT   waits on a barrier nothing will complete; the
 *                              wait gives up after budget_cycles SM cycles
 *                              (1e3 .. 2e9) and records 1: LD_ERR_TIMEOUT;
 *   LD_SELFTEST_BAD_COPY_ARGS  asks for a bulk copy of 20 bytes, which the
 *                              argument check refuses without issuing it,
 *                              recording 2: LD_ERR_TIMEOUT;
 *   LD_SELFTEST_VALID_COPY     one valid copy: nothing recorded, LD_OK.
 * Synchronises `stream`.  The error word must be clear when it is called. */
enum { LD_SELFTEST_WAIT_TIMEOUT = 0, LD_SELFTEST_BAD_COPY_ARGS = 1, LD_SELFTEST_VALID_COPY = 2 };
int ld_selftest_wait(ld_ctx* ctx, int32_t mode, int64_t budget_cycles, void* stream, int32_t* error_word);
/* Host-side fault injection: the allocation after `after` more successful
 * ones fails as a refused cudaMalloc would (LD_ERR_OOM, stage
 * "device-allocation-failed (injected)"); -1 turns it off.  The failing call
 * returns the error and the context stays usable. */
int ld_inject_alloc_failure(ld_ctx* ctx, int32_t after);

/* When enabled, every kernel launch of ld_render / ld_build_psf_bank is
 * bracketed by a pair of CUDA events on its stream. */
int ld_set_profiling(ld_ctx* ctx, int enable);
/* Synchronises the recorded events and writes, per stage id, the summed
 * device milliseconds and the launch count since the last collect; resets. */
int ld_profile_collect(ld_ctx* ctx, double* ms_per_stage, int32_t* launches_per_stage, int32_t count);
/* Tensor-core MMA flops issued by the DFT-as-GEMM launches (LD_STAGE_DFT_GEMM)
 * since the last call, the BF16x3 split's three products counted; resets. */
int ld_profile_tensor_flops(ld_ctx* ctx, double* flops);

/* ---- the drop-in render (replaces RunLensDiffCuda, LensDiffCuda.h:7-10) -- */
/* Enqueues the whole frame on request->cuda_stream; no host synchronisation
 * except the one-time first-zero calibration per (pupil size, PSF size). */
int ld_render(ld_ctx* ctx, const ld_render_request* request,
              const ld_params* params, ld_status* status);

/* ---- PSF bank (EnsureLensDiffPsfBank, LensDiffCpuReference.h:62-63) ----- */
/* Builds (or finds cached) the bank for `params` on `stream`. */
int ld_build_psf_bank(ld_ctx* ctx, const ld_params* params, void* stream,
                      ld_status* status);

/* Builds the banks of `count` unrelated lenses on `stream` (pupil size, PSF
 * size, wavelength count and phase terms may all differ), each as
 * EnsureLensDiffPsfBank builds one (LensDiffCpuReference.cpp:2068-2071).
 * With the tensor-core form the windows of every (lens, wavelength) pair
 * come from one persistent GEMM launch per transform pass, in chunks of at
 * most 32 GiB of scratch (a quarter of the HBM budget when that is less).
 * The banks stay in the context until the next call or ld_clear_caches;
 * ld_export_psf_bank and ld_render find them by their parameters.  Banks
 * already held for the same lens at the same position are kept;
 * status->bank_rebuilt counts the banks built and the size fields describe
 * params[0]. */
int ld_build_psf_banks(ld_ctx* ctx, const ld_params* params, int32_t count,
                       void* stream, ld_status* status);

/* Copies the bank's `full` kernels to HOST memory: for wavelength i,
 * sizes[i] = 2*radius_i+1 and a sizes[i]^2 row-major kernel is written at
 * kernels_out + offsets[i].  `capacity` is the float count of kernels_out.
 * Synchronises `stream`. */
int ld_export_psf_bank(ld_ctx* ctx, const ld_params* params, void* stream,
                       float* wavelengths_out, int32_t* sizes, int64_t* offsets,
                       float* kernels_out, int64_t capacity, ld_status* status);

/* Writes the normalised, fft-shifted raw PSF (S x S floats, DEVICE pointer)
 * of wavelength `wavelength_index`, as BuildLensDiffShiftedRawPsf does
 * (LensDiffCpuReference.cpp:831-859, chromatic focus applied as at :1720-1728). */
int ld_raw_psf(ld_ctx* ctx, const ld_params* params, int wavelength_index,
               float* psf_out_device, void* stream, ld_status* status);

/* ---- device memory estimate ------------------------------------------------------
 * Upper estimate of the device bytes one context grows to for rendering a
 * width x height frame with these parameters (PSF bank, kernel spectra, frame
 * work buffers; field zones counted); used for HBM admission.  No counterpart
 * in the reference (it allocates per call). */
size_t ld_estimate_device_bytes(const ld_params* params, int32_t width, int32_t height);

/* ---- frame serving with continuous batching ----------------------------------------
 * No counterpart in the reference (it renders one frame per host call,
 * LensDiff.cpp:3833).  A server keeps `slots` contexts, each with its own
 * stream, device PSF-bank cache and worker thread, on one GPU.  Submitted
 * frames (host RGBA float32, width x height, rows packed) wait in FIFO order
 * and start the moment a slot is free and the HBM budget (0: none) allows;
 * frames with the same lens parameters go to the slot that has them cached.
 * Host buffers must stay valid until ld_server_wait returns for the ticket. */
typedef struct ld_server ld_server;

typedef struct ld_server_stats {
    uint64_t completed, pending, cache_hits, max_concurrent;
    double p50_ms, p99_ms, mean_ms;   /* submit -> result on the host */
    double frames_per_s;              /* completed / (first submit -> last completion) */
    size_t device_bytes, reserved_bytes;
} ld_server_stats;

int ld_server_create(ld_server** out, int device, int slots, size_t hbm_budget_bytes);
void ld_server_destroy(ld_server* server);
int ld_server_submit(ld_server* server, const float* src_host, float* dst_host, int32_t width, int32_t height,
                     const ld_params* params, uint64_t* ticket);
/* Waits up to timeout_s for the frame; LD_ERR_TIMEOUT if it is not done (the
 * ticket stays valid), else the frame's status code (the ticket is released). */
int ld_server_wait(ld_server* server, uint64_t ticket, double timeout_s, ld_status* status, double* latency_ms);
int ld_server_get_stats(ld_server* server, ld_server_stats* out);
void ld_server_reset_stats(ld_server* server);


/* Same output as ld_raw_psf, for callers that cannot allocate device memory
 * (an OpenFX host that owns and budgets all GPU memory, a real-time thread
 * that must not take cudaMalloc's implicit synchronisation, a fixed memory
 * reservation).  No context and no allocation: the scratch is a 12 MiB
 * file-scope device array that every GPU loading the library holds until
 * exit.  Limit: pupil <= 512 and PSF grid <= 1024 (maximum kernel radius
 * <= 256 px); larger requests return LD_ERR_ARG.  A PSF grid whose size has
 * a prime factor above 5 (e.g. 4R with R = 131) returns LD_ERR_UNSUPPORTED
 * "fft-length-not-5-smooth"; the aperture checks and their codes are those of
 * ld_raw_psf.  All calls on a device share the array, so calls that overlap
 * on the GPU race.  The array's address is looked up in the calling thread's
 * current CUDA context on every call outside a stream capture; the first call
 * in a context must precede any stream capture in it.
 * This entry point has no counterpart in the reference. */
int ld_raw_psf_noalloc(const ld_params* params, int wavelength_index, float* psf_out_device, void* stream,
                       ld_status* status);

/* Resolved sizes of the path for `params` (N_p, S, R_max, wavelength count). */
int ld_resolve_sizes(const ld_params* params, int32_t* pupil_size,
                     int32_t* raw_psf_size, int32_t* max_kernel_radius,
                     int32_t* wavelength_count);

/* Fills a 3 x count natural matrix of Gaussian RGB responses (row-normalised
 * to unit sum), the weighting used for wavelength sets the reference cannot
 * express (more than 9 bins). */
int ld_gaussian_rgb_matrix(const float* wavelengths_nm, int32_t count,
                           const float* center_nm, float sigma_nm,
                           float* matrix_out);

#ifdef __cplusplus
}
#endif
#endif /* LENSDIFF_B200_H */
