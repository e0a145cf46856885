// ld_host.cu — host orchestration and the C ABI (include/lensdiff_b200.h).
//
// ld_render replaces RunLensDiffCuda (reference source/src/cuda/LensDiffCuda.h:7-10,
// implemented at LensDiffCuda.cu:4642-7587).  The sequence per frame is
//   [bank miss]    pupil/|FFT|^2 window -> lambda-rescale -> shaping -> crop
//   [spectra miss] weighted combination -> kernel spectra on the FFT grid
//   frame          forward rows (+extraction) -> columns (+multiply) ->
//                  inverse rows (+spectral map +composite)
// all enqueued on the caller's stream.  The only host synchronisation is the
// one-time first-zero calibration per (pupil size, PSF size), the analogue of
// the reference's process-wide GetLensDiffReferenceRawPsfCached
// (LensDiffCpuReference.cpp:2018-2038).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/lensdiff_b200.h"
#include "ld_fxplans.h"
#include "ld_internal.h"

using namespace ld;

namespace {

// ---------------------------------------------------------------------------
// device memory
// ---------------------------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

// A custom aperture image (ld_set_custom_aperture): the prepared amplitude
// values on the device and a digest of them for the bank key.
struct CustomAperture {
    DevBuf img;
    int w = 0, h = 0;
    uint64_t digest = 0;
};

// The context whose entry point is running on this thread: pupil set-up and
// the bank key read its custom aperture image through it.
thread_local const CustomAperture* t_custom = nullptr;
struct CustomScope {
    const CustomAperture* prev;
    explicit CustomScope(const CustomAperture* c) : prev(t_custom) { t_custom = c; }
    ~CustomScope() { t_custom = prev; }
};

struct BankEntry {
    bool valid = false;
    std::string key;
    int B = 0, np = 0, S = 0, R = 0, K = 0;
    int win_stride = 0;
    std::vector<float> wavelengths;
    bool cufft = false;  // built with the comparator form (its spectra follow)
    bool h16 = false;    // chosen form: kernel spectra in FP16 with per-column scales
    bool split_sums = false;  // s_core / s_struct computed (first Split render of the bank)
    bool ring_means = false;  // ring means computed (built unfused, or on first Split use)
    DevBuf canvas, ring_round, ring_ceil, ring_peak, ring_mean, scalars, wl;
    PsfBankArgs args{};
};

struct SpectraEntry {
    bool valid = false;
    uint64_t last_use = 0;
    std::string key;
    DevBuf spectra;
    GridGeom g{};
    int n_ker = 0;
    // recorded on the render stream after the last frame chain that read
    // these spectra: a rebuild on the bank stream waits for it
    cudaEvent_t free_ev = nullptr;
    bool free_pending = false;
};

}  // namespace

struct ld_ctx {
    int device = 0;
    size_t budget = 0;
    size_t held = 0;
    bool configured = false;
    std::mutex mu;
    std::map<int, DevBuf> twiddles;
    std::map<int, DevBuf> stage_twiddles;  // by fixed plan id
    std::map<int, int> fixed_choice;       // transform length -> fixed plan id | shape << 8 (autotuner)
    std::map<int, double> fixed_ms;        // transform length -> the winner's timed ms
    int autotune = 1;  // 1: tune, 0: first compiled order, -1: runtime-planned transforms only
    int fail_alloc_after = -1;  // fault injection: allocations until one fails (-1: off)
    CustomAperture custom;      // the Custom aperture mode's image
    std::map<std::pair<int, int>, float> r0_cache;
    std::map<int, DevBuf> ring_counts;  // by R
    BankEntry bank;
    SpectraEntry spectra;
    std::vector<SpectraEntry> zone_spectra;  // field zones, zy * n + zx
    // field zones' pupils, wavelength tables and windows of one batched transform
    std::vector<DevBuf> zone_pupil, zone_wl, zone_win;
    // banks of unrelated lenses built together (ld_build_psf_banks), kept
    // until the next such build; the pupils, wavelength tables and windows of
    // one chunk of their batched transform
    std::vector<BankEntry> set_banks;
    std::vector<DevBuf> set_pupil, set_wl, set_win;
    // kernel spectra of recent (lens, frame size) pairs, least recently used
    // replaced first: a context serving one lens at several frame sizes keeps
    // them all without rebuilding the bank
    std::vector<SpectraEntry> spectra_lru;
    uint64_t spectra_clock = 0;
    // per-frame chains captured as CUDA graphs, by the bytes of their arguments
    struct GraphEntry {
        std::string key;
        cudaGraphExec_t exec = nullptr;
        int launches = 0;
        uint64_t last_use = 0;
    };
    std::vector<GraphEntry> graphs;
    uint64_t graph_clock = 0;
    bool graphs_enabled = true;
    // work buffers, grown on demand
    DevBuf rows, win, combine_out, kspec_rows, frameA, frameB, calib, calib_psf, pupil_pre, effect;
    // resolution-aware working source; scatter kernel canvas and spectrum
    DevBuf work, scatter_canvas, scatter_ks;
    // chosen form's DFT-as-GEMM operand images and per-wavelength tiles
    DevBuf dft;
    // the DFT basis images of the last single-lens bank: they depend only on
    // the transform geometry (PSF size, pupil extent, union window), which a
    // lens keeps from frame to frame when only its phase changes
    DevBuf basis;
    std::vector<int> basis_key;
    std::string pupil_key;  // what pupil_pre holds (setup_pupil)
    DevBuf debug;  // static debug views: maxima, square images, OTF scratch
    // side stream for the source's row transforms while a bank is built
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    // bank stream: cold frames build their bank and kernel spectra here while
    // the render stream still runs earlier frames' chains (bank_done joins
    // them); other users of the bank's buffers join it first and leave a
    // fence that the next build waits for
    cudaStream_t bank_s = nullptr;
    cudaEvent_t bank_done = nullptr, bank_fence = nullptr;
    bool fence_pending = false;
    DevBuf scatter_rows;  // the scatter spectrum's row transforms (not shared with the bank stream)
    // pinned staging ring for the small per-bank uploads (upload_async)
    void* stage_host = nullptr;
    std::vector<cudaEvent_t> stage_ev;
    std::vector<bool> stage_pending;
    int stage_next = 0;
    // pinned buffers for uploads larger than a staging slot (the problem
    // tables of a lens set's batched transform), reused round-robin
    struct BigStage {
        void* host = nullptr;
        size_t bytes = 0;
        cudaEvent_t ev = nullptr;
        bool pending = false;
    };
    std::vector<BigStage> big_stage;
    int big_next = 0;
    std::string scatter_key;
    // comparator form (cuFFT): plans and its own work buffers
    CufftPlanCache cufft;
    DevBuf cf_grid, cf_planes, cf_sd, cf_prod;
    DevBuf err_word;    // device int: nonzero after a bounded wait gave up
    int* err = nullptr;
    DevBuf selftest;    // ld_selftest_wait's source and destination
    int launches = 0;
    // stage timing
    bool profiling = false;
    std::vector<cudaEvent_t> event_pool;
    size_t events_used = 0;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
    double tensor_flops = 0.0;  // MMA flops issued by DFT-GEMM launches (ld_profile_tensor_flops)
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

struct Fail {
    int code;
    std::string stage;
};

void set_status(ld_status* st, int code, const std::string& stage) {
    if (!st) return;
    st->code = code;
    std::strncpy(st->stage, stage.c_str(), LD_STAGE_LEN - 1);
    st->stage[LD_STAGE_LEN - 1] = '\0';
}

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Fail{LD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

void check_launch(const char* what) { check_cuda(cudaGetLastError(), what); }

void free_buf(ld_ctx* c, DevBuf& b) {
    if (b.p) {
        cudaFree(b.p);
        c->held -= b.bytes;
    }
    b.p = nullptr;
    b.bytes = 0;
}

void* ensure(ld_ctx* c, DevBuf& b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return b.p;
    const size_t old = b.bytes;
    if (c->budget && c->held - old + bytes > c->budget)
        throw Fail{LD_ERR_BUDGET, "hbm-budget-exceeded"};
    // host-side fault injection (ld_inject_alloc_failure): this allocation
    // fails as a refused cudaMalloc would, before anything is freed
    if (c->fail_alloc_after >= 0 && c->fail_alloc_after-- == 0)
        throw Fail{LD_ERR_OOM, "device-allocation-failed (injected)"};
    free_buf(c, b);
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        throw Fail{LD_ERR_OOM, "device-allocation-failed"};
    }
    b.p = p;
    b.bytes = bytes;
    c->held += bytes;
    return p;
}

// ---------------------------------------------------------------------------
// stage timing
// ---------------------------------------------------------------------------
constexpr size_t kStageSlot = 16384;
constexpr int kStageSlots = 64;  // 16 cold frames of uploads in flight
constexpr int kBigStages = 8;

// One CTA copies `words` 4-byte words from mapped pinned host memory (`src`
// 16-byte aligned): 16 bytes per thread where `dst` allows, so a staging
// slot's reads are all in flight at once and the copy costs about one PCIe
// round trip.
constexpr int kHostWordsThreads = 1024;
__global__ void __launch_bounds__(kHostWordsThreads) host_words_kernel(uint32_t* dst, const uint32_t* src, int words) {
    int i0 = 0;
    if ((reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
        const int q = words / 4;
        for (int k = threadIdx.x; k < q; k += kHostWordsThreads)
            reinterpret_cast<uint4*>(dst)[k] = reinterpret_cast<const uint4*>(src)[k];
        i0 = 4 * q;
    }
    for (int k = i0 + threadIdx.x; k < words; k += kHostWordsThreads) dst[k] = src[k];
}

// Host -> device copy of a small host array that leaves the host free: the
// bytes go through a slot of a mapped pinned staging ring and a one-CTA
// kernel on the stream reads them, so a frame that rebuilds its bank neither
// waits for the frames before it (as a copy from pageable memory does) nor
// queues behind a caller's large frame copies on the copy engine.  A slot is
// refilled only after the kernel that last read it has finished.  Arrays
// above one slot take a plain copy.
void upload_async(ld_ctx* c, void* dst, const void* src, size_t bytes, cudaStream_t s, const char* what) {
    if ((bytes & 3) != 0 || (reinterpret_cast<uintptr_t>(dst) & 3) != 0) {
        check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), what);
        return;
    }
    if (bytes > kStageSlot) {  // a pinned copy: no wait for the stream, as a pageable one would
        if (c->big_stage.empty()) c->big_stage.resize(kBigStages);
        ld_ctx::BigStage& b = c->big_stage[static_cast<size_t>(c->big_next)];
        c->big_next = (c->big_next + 1) % kBigStages;
        if (b.pending) check_cuda(cudaEventSynchronize(b.ev), what);
        b.pending = false;
        if (!b.ev) check_cuda(cudaEventCreateWithFlags(&b.ev, cudaEventDisableTiming), what);
        if (b.bytes < bytes) {
            if (b.host) cudaFreeHost(b.host);
            b.host = nullptr;
            b.bytes = 0;
            check_cuda(cudaHostAlloc(&b.host, bytes, cudaHostAllocDefault), what);
            b.bytes = bytes;
        }
        std::memcpy(b.host, src, bytes);
        check_cuda(cudaMemcpyAsync(dst, b.host, bytes, cudaMemcpyHostToDevice, s), what);
        check_cuda(cudaEventRecord(b.ev, s), what);
        b.pending = true;
        return;
    }
    if (!c->stage_host) {
        check_cuda(cudaHostAlloc(&c->stage_host, kStageSlot * kStageSlots, cudaHostAllocMapped), what);
        c->stage_ev.assign(kStageSlots, nullptr);
        for (auto& e : c->stage_ev) check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), what);
        c->stage_pending.assign(kStageSlots, false);
    }
    const int i = c->stage_next;
    c->stage_next = (i + 1) % kStageSlots;
    if (c->stage_pending[static_cast<size_t>(i)])
        check_cuda(cudaEventSynchronize(c->stage_ev[static_cast<size_t>(i)]), what);
    char* h = static_cast<char*>(c->stage_host) + static_cast<size_t>(i) * kStageSlot;
    std::memcpy(h, src, bytes);
    void* hd = nullptr;
    check_cuda(cudaHostGetDevicePointer(&hd, h, 0), what);
    host_words_kernel<<<1, kHostWordsThreads, 0, s>>>(static_cast<uint32_t*>(dst), static_cast<const uint32_t*>(hd),
                                                       static_cast<int>(bytes / 4));
    check_launch(what);
    ++c->launches;
    check_cuda(cudaEventRecord(c->stage_ev[static_cast<size_t>(i)], s), what);
    c->stage_pending[static_cast<size_t>(i)] = true;
}

// The context's bank stream and its events, created on first use.
cudaStream_t bank_stream(ld_ctx* c) {
    if (!c->bank_s) {
        check_cuda(cudaStreamCreateWithFlags(&c->bank_s, cudaStreamNonBlocking), "bank-stream");
        check_cuda(cudaEventCreateWithFlags(&c->bank_done, cudaEventDisableTiming), "bank-stream");
        check_cuda(cudaEventCreateWithFlags(&c->bank_fence, cudaEventDisableTiming), "bank-stream");
    }
    return c->bank_s;
}

// Stream s is about to use the bank's buffers outside the bank stream: wait
// for the bank stream's work so far.
void join_bank(ld_ctx* c, cudaStream_t s) {
    if (!c->bank_s || s == c->bank_s) return;
    check_cuda(cudaEventRecord(c->bank_done, c->bank_s), "bank-join");
    check_cuda(cudaStreamWaitEvent(s, c->bank_done, 0), "bank-join");
}

// Stream s has enqueued uses of the bank's buffers: the next build on the
// bank stream waits for them.
void fence_bank(ld_ctx* c, cudaStream_t s) {
    if (!c->bank_s || s == c->bank_s) return;
    check_cuda(cudaEventRecord(c->bank_fence, s), "bank-fence");
    c->fence_pending = true;
}

// An entry about to be rebuilt on stream s: wait until no frame chain reads it.
void wait_free(SpectraEntry& e, cudaStream_t s) {
    if (e.free_pending) check_cuda(cudaStreamWaitEvent(s, e.free_ev, 0), "spectra-reuse");
}

// Record, on the render stream, that a chain has finished with entry e.
void mark_used(SpectraEntry& e, cudaStream_t s) {
    if (!e.free_ev) check_cuda(cudaEventCreateWithFlags(&e.free_ev, cudaEventDisableTiming), "spectra-event");
    check_cuda(cudaEventRecord(e.free_ev, s), "spectra-event");
    e.free_pending = true;
}

// The context's side stream and its fork / join events, created on first use.
cudaStream_t side_stream(ld_ctx* c) {
    if (!c->side) {
        check_cuda(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking), "side-stream");
        check_cuda(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming), "side-stream");
        check_cuda(cudaEventCreateWithFlags(&c->join_ev, cudaEventDisableTiming), "side-stream");
    }
    return c->side;
}

cudaEvent_t next_event(ld_ctx* c) {
    if (c->events_used == c->event_pool.size()) {
        cudaEvent_t e;
        check_cuda(cudaEventCreate(&e), "event-create");
        c->event_pool.push_back(e);
    }
    return c->event_pool[c->events_used++];
}

// Runs `launch` bracketed by events when profiling is on.
template <class F>
void staged(ld_ctx* c, int stage, cudaStream_t s, F launch) {
    if (!c->profiling) {
        launch();
        ++c->launches;
        return;
    }
    cudaEvent_t a = next_event(c), b = next_event(c);
    cudaEventRecord(a, s);
    launch();
    cudaEventRecord(b, s);
    c->marks.push_back({stage, {a, b}});
    ++c->launches;
}

// ---------------------------------------------------------------------------
// FFT plans and twiddles
// ---------------------------------------------------------------------------
// Radices for a 5-smooth n: pairs of fives as 25 (when allowed: E = 25
// family only), fours of twos as 16, the rest as 8 / 4 / 2 (16*2 becomes 8*4),
// threes as 3.  The transform runs them in the order of kPlanRadices.
bool factor_radices(int n, bool allow25, std::vector<int>* out) {
    if (n < 2) return false;
    int m = n, a = 0, b = 0, c5 = 0;
    while (m % 2 == 0) { m /= 2; ++a; }
    while (m % 3 == 0) { m /= 3; ++b; }
    while (m % 5 == 0) { m /= 5; ++c5; }
    if (m != 1) return false;
    out->clear();
    if (allow25) {
        for (int i = 0; i < c5 / 2; ++i) out->push_back(25);
        if (c5 % 2) out->push_back(5);
    } else {
        for (int i = 0; i < c5; ++i) out->push_back(5);
    }
    for (int i = 0; i < b; ++i) out->push_back(3);
    int q16 = a / 4;
    const int rem = a % 4;
    if (rem == 1 && q16 > 0) {
        --q16;
        out->push_back(8);
        out->push_back(4);
    }
    for (int i = 0; i < q16; ++i) out->push_back(16);
    if (rem == 3) out->push_back(8);
    else if (rem == 2) out->push_back(4);
    else if (rem == 1 && a == 1) out->push_back(2);
    if (out->size() > static_cast<size_t>(kMaxStages)) return false;
    for (int i = 0; i < 7; ++i)
        if (std::count(out->begin(), out->end(), kPlanRadices[i]) > 15) return false;
    return true;
}

bool factor_plan(int n, bool allow25, FftPlan* plan) {
    std::vector<int> r;
    if (!factor_radices(n, allow25, &r)) return false;
    plan->n = n;
    plan->nstages = static_cast<int>(r.size());
    plan->codes = 0ull;
    for (int i = 0; i < 7; ++i) {
        const unsigned long long cnt =
            static_cast<unsigned long long>(std::count(r.begin(), r.end(), kPlanRadices[i]));
        plan->codes |= cnt << (4 * i);
    }
    return true;
}

bool smooth(int n) {
    if (n <= 0) return false;
    for (int p : {2, 3, 5})
        while (n % p == 0) n /= p;
    return n == 1;
}

const float2* twiddles(ld_ctx* c, int n) {
    auto it = c->twiddles.find(n);
    if (it != c->twiddles.end()) return static_cast<const float2*>(it->second.p);
    std::vector<float2> h(static_cast<size_t>(n));
    for (int k = 0; k < n; ++k) {
        const double a = -2.0 * M_PI * static_cast<double>(k) / static_cast<double>(n);
        h[static_cast<size_t>(k)] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
    }
    DevBuf b;
    ensure(c, b, h.size() * sizeof(float2));
    check_cuda(cudaMemcpy(b.p, h.data(), h.size() * sizeof(float2), cudaMemcpyHostToDevice), "twiddle-upload");
    c->twiddles[n] = b;
    return static_cast<const float2*>(b.p);
}

// Per-stage twiddle tables of a fixed plan (ld_fxplans.h), uploaded once.
const float2* stage_twiddles(ld_ctx* c, int id) {
    auto it = c->stage_twiddles.find(id);
    if (it != c->stage_twiddles.end()) return static_cast<const float2*>(it->second.p);
    const std::vector<float2> h = fx_stage_table(id);
    DevBuf b;
    ensure(c, b, std::max<size_t>(16, h.size() * sizeof(float2)));
    if (!h.empty())
        check_cuda(cudaMemcpy(b.p, h.data(), h.size() * sizeof(float2), cudaMemcpyHostToDevice), "stage-twiddle-upload");
    c->stage_twiddles[id] = b;
    return static_cast<const float2*>(b.p);
}

// The fixed plan a length runs on: the autotuner's choice when it has made
// one, else the first compiled radix order of that length (0: none).
// Mode 2 + k pins the k-th compiled order of every length (its last when it
// has fewer).
int fixed_plan_for(ld_ctx* c, int n, bool allow25) {
    if (!allow25 || c->autotune < 0) return 0;  // the fixed launchers serve grids of the 25-element family
    int ids[8];
    const int count = fx_candidates(n, ids, 8);
    if (c->autotune >= 2) return count > 0 ? ids[std::min(c->autotune - 2, count - 1)] : 0;
    auto it = c->fixed_choice.find(n);
    if (it != c->fixed_choice.end()) return it->second;
    return count > 0 ? ids[0] : 0;
}

FftPlan make_plan(ld_ctx* c, int n, bool allow25) {
    FftPlan p{};
    if (!factor_plan(n, allow25, &p)) throw Fail{LD_ERR_UNSUPPORTED, "fft-length-not-5-smooth"};
    p.tw = twiddles(c, n);
    const int choice = fixed_plan_for(c, n, allow25);
    p.fixed = choice & 255;
    p.shape = choice >> 8;
    p.stw = p.fixed ? stage_twiddles(c, p.fixed) : nullptr;
    return p;
}

// ---------------------------------------------------------------------------
// parameter resolution (reference float/double expressions)
// ---------------------------------------------------------------------------
constexpr float kPiRef = 3.14159265358979323846f;  // kPi, LensDiffCpuReference.cpp:25

int frame_short_side(const ld_params& p) { return std::max(1, p.frame_short_side_px); }  // LensDiffTypes.h:294-296
int optics_short_side(const ld_params& p) {  // LensDiffTypes.h:302-305
    return p.resolution_aware ? 2160 : std::max(1, p.frame_short_side_px);
}
double percent_to_px(double pct, int side) {  // LensDiffTypes.h:312-314
    return std::max(0.0, pct) * 0.01 * static_cast<double>(std::max(1, side));
}
int max_kernel_radius(const ld_params& p) {  // LensDiffTypes.h:316-320 + CpuReference.cpp:1710
    const int r = std::max(0, static_cast<int>(std::ceil(percent_to_px(p.max_kernel_radius_px, optics_short_side(p)))));
    return std::max(4, r);
}
int pupil_size(const ld_params& p) { return std::min(std::max(p.pupil_resolution, 64), 1024); }
int raw_psf_size(int np, int rmax) {  // chooseRawPsfSize, CpuReference.cpp:112-115
    return std::min(std::max(std::max(np * 2, std::max(512, rmax * 4)), 128), 16384);
}

bool is_mono(const ld_params& p) { return p.spectral_mode == LD_SPECTRAL_MONO; }

// Chosen form: kernel spectra and column outputs in FP16 with per-column
// scales (spectral modes; Mono keeps FP32 spectra).
bool chosen_h16(const ld_params& p) { return p.fft_form == LD_FFT_OWN_CHOSEN && !is_mono(p); }

std::vector<float> wavelengths_of(const ld_params& p) {  // CpuReference.cpp:1602-1614
    if (!is_mono(p) && p.wavelength_count > 0) {
        return std::vector<float>(p.wavelengths_nm, p.wavelengths_nm + p.wavelength_count);
    }
    switch (p.spectral_mode) {
        case LD_SPECTRAL_9: return {420.f, 450.f, 480.f, 510.f, 540.f, 570.f, 600.f, 630.f, 660.f};
        case LD_SPECTRAL_5: return {440.f, 490.f, 540.f, 590.f, 640.f};
        case LD_SPECTRAL_TRISTIMULUS: return {460.f, 550.f, 610.f};
        default: return {550.f};
    }
}

constexpr int kMaxFieldGrid = 16;

bool has_field_phase(const ld_params& p) {  // LensDiffPhase.cpp:40-57
    if (p.phase_mode != LD_PHASE_ENABLED || std::abs(p.phase_field_strength) <= 1e-6) return false;
    const double v[] = {p.phase_field_defocus, p.phase_field_astig_radial, p.phase_field_astig_tangential,
                        p.phase_field_coma_radial, p.phase_field_coma_tangential, p.phase_field_spherical,
                        p.phase_field_trefoil_radial, p.phase_field_trefoil_tangential,
                        p.phase_field_secondary_astig_radial, p.phase_field_secondary_astig_tangential,
                        p.phase_field_quadrafoil_radial, p.phase_field_quadrafoil_tangential,
                        p.phase_field_secondary_coma_radial, p.phase_field_secondary_coma_tangential};
    for (double x : v)
        if (std::abs(x) > 1e-6) return true;
    return false;
}

// ResolveLensDiffFieldZoneParams (LensDiffPhase.cpp:98-168), FP64 as the
// reference: the zone's own Zernike coefficients at normalised field position
// (nx, ny); the field terms are cleared so the zone bank has no zones.
void add_orientation_pair(double radial, double tangential, double angle, int harmonic, double* x, double* y) {
    const double base = static_cast<double>(harmonic) * angle;
    const double cs = std::cos(base), sn = std::sin(base);
    *x += radial * cs - tangential * sn;
    *y += radial * sn + tangential * cs;
}

ld_params zone_params(const ld_params& p, float nx, float ny) {
    ld_params q = p;
    q.phase_field_strength = 0.0;
    const double radial = std::min(1.0, std::sqrt(static_cast<double>(nx) * nx + static_cast<double>(ny) * ny) /
                                            std::sqrt(2.0));
    const double bias = std::min(std::max(p.phase_field_edge_bias, 0.0), 1.0);
    const double scale = p.phase_field_strength * std::pow(radial, 1.0 + bias * 2.0);
    if (std::abs(scale) <= 1e-9) return q;
    const double angle = std::atan2(static_cast<double>(ny), static_cast<double>(nx));
    q.phase_defocus += p.phase_field_defocus * scale;
    q.phase_spherical += p.phase_field_spherical * scale;
    add_orientation_pair(p.phase_field_astig_radial * scale, p.phase_field_astig_tangential * scale, angle, 2,
                         &q.phase_astigmatism0, &q.phase_astigmatism45);
    add_orientation_pair(p.phase_field_coma_radial * scale, p.phase_field_coma_tangential * scale, angle, 1,
                         &q.phase_coma_x, &q.phase_coma_y);
    add_orientation_pair(p.phase_field_trefoil_radial * scale, p.phase_field_trefoil_tangential * scale, angle, 3,
                         &q.phase_trefoil_x, &q.phase_trefoil_y);
    add_orientation_pair(p.phase_field_secondary_astig_radial * scale,
                         p.phase_field_secondary_astig_tangential * scale, angle, 2,
                         &q.phase_secondary_astigmatism0, &q.phase_secondary_astigmatism45);
    add_orientation_pair(p.phase_field_quadrafoil_radial * scale, p.phase_field_quadrafoil_tangential * scale,
                         angle, 4, &q.phase_quadrafoil0, &q.phase_quadrafoil45);
    add_orientation_pair(p.phase_field_secondary_coma_radial * scale,
                         p.phase_field_secondary_coma_tangential * scale, angle, 1, &q.phase_secondary_coma_x,
                         &q.phase_secondary_coma_y);
    return q;
}

// Noll-indexed coefficients for one wavelength: the named terms
// (LensDiffPhase.cpp:199-212) with the chromatic defocus offset
// (CpuReference.cpp:1721-1726) plus the extension vector.
PhaseCoeffs phase_for_wavelength(const ld_params& p, float wavelength) {
    PhaseCoeffs pc{};
    const float off = (wavelength - 550.0f) / 110.0f;
    const double defocus = p.phase_defocus + p.chromatic_focus * static_cast<double>(off);
    const bool enabled = p.phase_mode == LD_PHASE_ENABLED || std::abs(defocus) > 1e-6;
    double c[LD_NOLL_COUNT] = {0};
    c[4] = defocus;
    c[5] = p.phase_astigmatism45;
    c[6] = p.phase_astigmatism0;
    c[7] = p.phase_coma_y;
    c[8] = p.phase_coma_x;
    c[9] = p.phase_trefoil_y;
    c[10] = p.phase_trefoil_x;
    c[11] = p.phase_spherical;
    c[12] = p.phase_secondary_astigmatism0;
    c[13] = p.phase_secondary_astigmatism45;
    c[14] = p.phase_quadrafoil0;
    c[15] = p.phase_quadrafoil45;
    c[16] = p.phase_secondary_coma_x;
    c[17] = p.phase_secondary_coma_y;
    bool nonflat = std::abs(p.pupil_decenter_x) > 1e-6 || std::abs(p.pupil_decenter_y) > 1e-6;
    for (int j = 1; j < LD_NOLL_COUNT; ++j) {
        c[j] += p.noll[j];
        if (std::abs(c[j]) > 1e-6) nonflat = true;
    }
    pc.enabled = (enabled && nonflat) ? 1 : 0;
    for (int j = 0; j < LD_NOLL_COUNT; ++j) pc.c[j] = static_cast<float>(c[j]);
    return pc;
}

PupilParams pupil_params(const ld_params& p, bool circle_reference) {
    PupilParams pp{};
    pp.size = pupil_size(p);
    if (circle_reference) {  // GetLensDiffReferenceRawPsfCached, CpuReference.cpp:2028-2033
        pp.mode = 0;
        pp.sides = 6;
        pp.apod = 0;
        pp.roundness = 1.0f;
        pp.phase_cs = 1.0f;
        return pp;
    }
    pp.mode = p.aperture_mode;
    pp.sides = p.aperture_mode == LD_APERTURE_HEXAGON ? 6 : std::max(3, p.blade_count);
    if (pp.mode == LD_APERTURE_HEXAGON) pp.mode = LD_APERTURE_POLYGON;
    pp.apod = p.apodization_mode;
    pp.roundness = static_cast<float>(std::min(std::max(p.roundness, 0.0), 1.0));
    pp.rotation = static_cast<float>(p.rotation_deg * static_cast<double>(kPiRef) / 180.0);
    pp.obstruction = static_cast<float>(std::max(0.0, std::min(0.95, p.central_obstruction))) * 0.86f;
    const float thick = static_cast<float>(std::max(0.0, p.vane_thickness));
    pp.vane_half = thick * 0.86f;
    pp.vanes = (p.vane_count <= 0 || thick <= 0.0f) ? 0 : std::max(1, p.vane_count);
    for (int i = 0; i < pp.vanes; ++i) {  // blockedByVanes, CpuReference.cpp:477-479
        const float ang = pp.rotation + static_cast<float>(i) * kPiRef / static_cast<float>(pp.vanes);
        pp.vane_cs[i] = std::cos(ang);
        pp.vane_sn[i] = std::sin(ang);
    }
    pp.decx = static_cast<float>(p.pupil_decenter_x);
    pp.decy = static_cast<float>(p.pupil_decenter_y);
    pp.phase_cs = std::cos(-pp.rotation);  // LensDiffPhase.cpp:225-226
    pp.phase_sn = std::sin(-pp.rotation);
    if (p.aperture_mode == LD_APERTURE_CUSTOM) {  // buildCustomPupilAmplitude, CpuReference.cpp:715-721
        const CustomAperture* ca = t_custom;
        if (ca == nullptr || ca->img.p == nullptr) throw Fail{LD_ERR_ARG, "custom-aperture-image-not-set"};
        pp.custom = static_cast<const float*>(ca->img.p);
        pp.cw = ca->w;
        pp.ch = ca->h;
        const float aspect = static_cast<float>(ca->w) / static_cast<float>(std::max(1, ca->h));
        pp.fit_hw = aspect >= 1.0f ? 1.0f : aspect;
        pp.fit_hh = aspect >= 1.0f ? 1.0f / aspect : 1.0f;
        pp.vanes = 0;
        pp.obstruction = 0.0f;
    }
    // per-mode constants with the reference's float expressions
    const float outer = 0.86f;
    const float rnd = pp.roundness;
    auto clampf = [](float v, float lo, float hi) { return std::min(std::max(v, lo), hi); };
    pp.star_inner = outer * clampf(0.18f + rnd * 0.62f, 0.1f, 0.95f);  // CpuReference.cpp:776, :520
    pp.spiral_twist = 4.0f + (1.0f - clampf(rnd, 0.0f, 1.0f)) * 8.0f;  // :663-664
    pp.spiral_opening = 0.18f + clampf(rnd, 0.0f, 1.0f) * 0.26f;
    pp.grid_half = outer * 0.82f;  // :586-594
    pp.grid_pitch = (2.0f * pp.grid_half) / static_cast<float>(pp.sides);
    pp.grid_bar = pp.grid_pitch * (0.06f + (1.0f - clampf(rnd, 0.0f, 1.0f)) * 0.12f);
    pp.snow_levels = std::min(std::max(std::max(2, std::max(3, p.blade_count) / 2), 2), 5);  // :619-623
    pp.snow_main = outer * 0.92f;
    pp.snow_thick = outer * (0.045f + (1.0f - clampf(rnd, 0.0f, 1.0f)) * 0.05f);
    const float branch_angle = kPiRef / 5.5f;
    for (int arm = 0; arm < 6; ++arm) {
        const float angle = pp.rotation - kPiRef * 0.5f + static_cast<float>(arm) * (kPiRef / 3.0f);
        pp.snow_arm_cs[arm] = std::cos(angle);
        pp.snow_arm_sn[arm] = std::sin(angle);
        for (int side = 0; side < 2; ++side) {
            const float theta = angle + static_cast<float>(side == 0 ? -1 : 1) * branch_angle;
            pp.snow_br_cs[arm][side] = std::cos(theta);
            pp.snow_br_sn[arm][side] = std::sin(theta);
        }
    }
    for (int level = 0; level < pp.snow_levels; ++level) {
        pp.snow_t[level] = 0.34f + static_cast<float>(level) * (0.44f / static_cast<float>(std::max(1, pp.snow_levels - 1)));
        pp.snow_len[level] = outer * (0.16f + 0.03f * static_cast<float>(level));
    }
    return pp;
}

std::string append_bytes(std::string s, const void* p, size_t n) {
    s.append(static_cast<const char*>(p), n);
    return s;
}

// Identity of a PSF bank: every parameter the bank depends on
// (MakeLensDiffPsfBankKey, CpuReference.cpp:1836-1875, plus the extensions).
std::string bank_key(const ld_params& p, const std::vector<float>& wl) {
    std::string k;
    const int ints[] = {p.aperture_mode, p.apodization_mode, p.blade_count, p.vane_count, pupil_size(p),
                        optics_short_side(p), p.phase_mode};
    const double dbl[] = {p.roundness, p.rotation_deg, p.central_obstruction, p.vane_thickness,
                          p.max_kernel_radius_px, p.diffraction_scale_px, p.anisotropy_emphasis,
                          p.phase_defocus, p.phase_astigmatism0, p.phase_astigmatism45, p.phase_coma_x,
                          p.phase_coma_y, p.phase_spherical, p.phase_trefoil_x, p.phase_trefoil_y,
                          p.phase_secondary_astigmatism0, p.phase_secondary_astigmatism45,
                          p.phase_quadrafoil0, p.phase_quadrafoil45, p.phase_secondary_coma_x,
                          p.phase_secondary_coma_y, p.pupil_decenter_x, p.pupil_decenter_y,
                          p.chromatic_focus, p.chromatic_spread};
    k = append_bytes(k, ints, sizeof(ints));
    k = append_bytes(k, dbl, sizeof(dbl));
    k = append_bytes(k, p.noll, sizeof(p.noll));
    k = append_bytes(k, wl.data(), wl.size() * sizeof(float));
    k = append_bytes(k, &p.fft_form, sizeof(p.fft_form));
    if (p.aperture_mode == LD_APERTURE_CUSTOM && t_custom != nullptr) {  // the image, as the reference keys its path
        const uint64_t img[3] = {t_custom->digest, static_cast<uint64_t>(t_custom->w), static_cast<uint64_t>(t_custom->h)};
        k = append_bytes(k, img, sizeof(img));
    }
    return k;
}

static_assert(LD_TRANSFER_LINEAR == kTransferLinear && LD_TRANSFER_DAVINCI_INTERMEDIATE == kTransferDavinci,
              "FrameArgs::transfer takes the public LD_TRANSFER_* values");

// The steps after the effect (CpuReference.cpp:2089-2094, :2180-2198): the
// resolution-aware working frame, scatter and creative fringe.
// Field zone z (of n per side) over `extent` working pixels: the pixels its
// tent weight can reach, [lo, hi) (accumulateWeightedImage's weight
// max(0, 1 - |x (n - 1) / (extent - 1) - z|), LensDiffCpuReference.cpp:
// 1458-1466, is zero outside ((z - 1) step, (z + 1) step); one pixel of margin
// each side, the inverse pass evaluates the weight itself).
void zone_span(int extent, int n, int z, int* lo, int* hi) {
    const double step = static_cast<double>(std::max(1, extent - 1)) / static_cast<double>(n - 1);
    *lo = std::max(0, static_cast<int>(std::floor((z - 1) * step)) - 1);
    *hi = std::min(extent, static_cast<int>(std::ceil((z + 1) * step)) + 2);
}

// The largest zone window of an n x n zone grid: the output size every
// zone's overlap-add tile must hold.
struct ZoneTiles {
    int n = 0;
    int wo = 0, ho = 0;
};
ZoneTiles zone_tiles(int W, int H, int n) {
    ZoneTiles t;
    t.n = n;
    for (int z = 0; z < n; ++z) {
        int lo = 0, hi = 0;
        zone_span(W, n, z, &lo, &hi);
        t.wo = std::max(t.wo, hi - lo);
        zone_span(H, n, z, &lo, &hi);
        t.ho = std::max(t.ho, hi - lo);
    }
    return t;
}

struct PostEffects {
    bool resample = false;
    double scale = 1.0;   // working / source (ResolveLensDiffEffectWorkingScale)
    bool scatter = false;
    float scatter_radius = 0.0f;  // px
    float scatter_amount = 0.0f;
    float fringe = 0.0f;          // px; > 1e-6 when on
    bool any() const { return resample || scatter || fringe > 1e-6f; }
};

PostEffects post_effects(const ld_params& p) {
    PostEffects e;
    // LensDiffTypes.h:302-305; CpuReference.cpp:2091
    e.scale = static_cast<double>(optics_short_side(p)) / static_cast<double>(frame_short_side(p));
    e.resample = p.resolution_aware && std::abs(e.scale - 1.0) > 1e-6;
    // CpuReference.cpp:2181-2182
    const double radius = percent_to_px(p.scatter_radius, optics_short_side(p));
    e.scatter = p.scatter_amount > 1e-6 && radius > 0.25;
    e.scatter_radius = static_cast<float>(radius);
    e.scatter_amount = static_cast<float>(std::max(0.0, p.scatter_amount));
    // :2188-2190 with applyCreativeFringe's threshold (:1500)
    const float f = static_cast<float>(std::max(0.0, percent_to_px(p.creative_fringe, optics_short_side(p))));
    e.fringe = f > 1e-6f ? f : 0.0f;
    return e;
}

// Working frame size (CpuReference.cpp:2092-2093).
void working_size(const PostEffects& e, int W, int H, int* Ww, int* Hw) {
    *Ww = e.resample ? std::max(1, static_cast<int>(std::lround(W * e.scale))) : W;
    *Hw = e.resample ? std::max(1, static_cast<int>(std::lround(H * e.scale))) : H;
}
constexpr int kMaxWorkingSide = 32768;

// Debug views rendered from the frame's own images (renderDebugView,
// LensDiffCpuReference.cpp:1789-1824), as opposed to the lens's static views.
bool frame_debug_view(int v) {
    return v == LD_DEBUG_FINAL || v == LD_DEBUG_SELECTION || v == LD_DEBUG_CORE || v == LD_DEBUG_STRUCTURE ||
           v == LD_DEBUG_EFFECT || v == LD_DEBUG_CREATIVE_FRINGE || v == LD_DEBUG_SCATTER;
}

void validate_params(const ld_params& p) {
    if (p.debug_view < LD_DEBUG_FINAL || p.debug_view > LD_DEBUG_SCATTER) throw Fail{LD_ERR_ARG, "invalid-debug-view"};
    if (p.debug_view != LD_DEBUG_FINAL && frame_debug_view(p.debug_view) && p.fft_form == LD_FFT_CUFFT)
        throw Fail{LD_ERR_UNSUPPORTED, "unsupported-frame-debug-view-with-cufft-form"};
    if (p.look_mode != LD_LOOK_PHYSICAL && p.look_mode != LD_LOOK_SPLIT) throw Fail{LD_ERR_ARG, "invalid-look-mode"};
    if (p.look_mode == LD_LOOK_SPLIT && p.fft_form == LD_FFT_CUFFT)
        throw Fail{LD_ERR_UNSUPPORTED, "unsupported-split-look-with-cufft-form"};
    if (p.input_transfer != LD_TRANSFER_LINEAR && p.input_transfer != LD_TRANSFER_DAVINCI_INTERMEDIATE)
        throw Fail{LD_ERR_ARG, "invalid-input-transfer"};
    // Custom: the image the host decoded and handed over with ld_set_custom_aperture
    // (the reference's own loader is WIC / ImageIO only, LensDiffApertureImage.cpp)
    if (p.aperture_mode == LD_APERTURE_CUSTOM && (t_custom == nullptr || t_custom->img.p == nullptr))
        throw Fail{LD_ERR_ARG, "custom-aperture-image-not-set"};
    if (p.aperture_mode < LD_APERTURE_CIRCLE || p.aperture_mode > LD_APERTURE_SNOWFLAKE)
        throw Fail{LD_ERR_ARG, "invalid-aperture-mode"};
    if (p.apodization_mode < 0 || p.apodization_mode > 2) throw Fail{LD_ERR_ARG, "invalid-apodization-mode"};
    if (p.spectral_mode < 0 || p.spectral_mode > 3) throw Fail{LD_ERR_ARG, "invalid-spectral-mode"};
    if (p.field_grid != 0 && (p.field_grid < 2 || p.field_grid > kMaxFieldGrid))
        throw Fail{LD_ERR_ARG, "invalid-field-grid"};
    if (p.wavelength_count < 0 || p.wavelength_count > LD_MAX_WAVELENGTHS)
        throw Fail{LD_ERR_ARG, "invalid-wavelength-count"};
    if (p.vane_count > kMaxVanes) throw Fail{LD_ERR_UNSUPPORTED, "too-many-vanes"};
    if (p.fft_form != LD_FFT_OWN_FP32 && p.fft_form != LD_FFT_CUFFT && p.fft_form != LD_FFT_OWN_CHOSEN)
        throw Fail{LD_ERR_UNSUPPORTED, "unsupported-fft-form"};
    if (p.fft_form == LD_FFT_CUFFT && has_field_phase(p))
        throw Fail{LD_ERR_UNSUPPORTED, "unsupported-field-zones-with-cufft-form"};
    if (p.fft_form == LD_FFT_CUFFT && post_effects(p).any())
        throw Fail{LD_ERR_UNSUPPORTED, "unsupported-scatter-fringe-or-resolution-aware-with-cufft-form"};
}

size_t align256(size_t n) { return (n + 255) & ~static_cast<size_t>(255); }
size_t align1k(size_t n) { return (n + 1023) & ~static_cast<size_t>(1023); }

// Fills the pupil part of a bank argument block and launches the per-bank
// pupil pre-pass (amplitude, the λ-independent phase, the defocus term).
// Only pupil rows whose pixel centres lie within the outer radius of the
// (decentred) aperture can be non-zero; the row passes skip the others.
// The pupil's parameters, base phase and the rows that can be non-zero.
void pupil_geometry(PsfBankArgs& a, const ld_params& p, bool circle) {
    a.pupil = pupil_params(p, circle);
    a.base_phase = circle ? PhaseCoeffs{} : phase_for_wavelength(p, 550.0f);
    a.base_phase.c[4] = 0.0f;  // defocus is carried per wavelength
    const int n = a.pupil.size;
    int lo = n, hi = 0;
    for (int y = 0; y < n; ++y) {
        const float ny = ((static_cast<float>(y) + 0.5f) / static_cast<float>(n) - 0.5f) * 2.0f;
        if (std::abs(ny - a.pupil.decy) <= 0.8601f) {
            lo = std::min(lo, y);
            hi = std::max(hi, y + 1);
        }
    }
    if (hi <= lo) {
        lo = 0;
        hi = 1;
    }
    a.row_lo = lo;
    a.row_n = hi - lo;
}

// The pre-pass depends on the pupil's parameters and the λ-independent phase
// only, not on defocus, so the context's own pre-pass buffer keeps its
// contents for the next bank with the same key (a lens whose defocus alone
// changed skips the launch).  The key is recorded once the launch is
// enqueued; a failure before then leaves none.
void setup_pupil(ld_ctx* c, PsfBankArgs& a, const ld_params& p, bool circle, cudaStream_t s,
                 DevBuf* target = nullptr) {
    pupil_geometry(a, p, circle);
    const int n = a.pupil.size;
    const size_t bytes = static_cast<size_t>(n) * n * sizeof(float4);
    std::string key;
    if (!target) {
        const uint64_t custom = (a.pupil.custom && t_custom) ? t_custom->digest : 0;
        key = append_bytes(key, &a.pupil, sizeof(a.pupil));
        key = append_bytes(key, &a.base_phase, sizeof(a.base_phase));
        key = append_bytes(key, &custom, sizeof(custom));
        if (key == c->pupil_key && c->pupil_pre.bytes >= bytes) {
            a.pupil_pre = static_cast<float4*>(c->pupil_pre.p);
            return;
        }
        c->pupil_key.clear();
    }
    a.pupil_pre = static_cast<float4*>(ensure(c, target ? *target : c->pupil_pre, bytes));
    staged(c, LD_STAGE_PUPIL, s, [&] { launch_pupil_pre(a, s); });
    if (!target) {
        check_launch("pupil-pre");
        c->pupil_key = key;
    }
}

void dft_gemm_psf(ld_ctx* c, const PsfBankArgs& a, const std::vector<WavelengthInfo>& infos, cudaStream_t s);

// ---------------------------------------------------------------------------
// first-zero calibration of the clear circle (one host sync per (N_p, S))
// ---------------------------------------------------------------------------
// The first-zero radius is a function of (N_p, S) alone: every context of the
// process (a server's slots among them) shares it, so each pair is calibrated
// (and the host synchronised for it) once per process.
std::mutex g_r0_mu;
std::map<std::pair<int, int>, float> g_r0;

float first_zero(ld_ctx* c, int np, int S, cudaStream_t s) {
    auto key = std::make_pair(np, S);
    auto it = c->r0_cache.find(key);
    if (it != c->r0_cache.end()) return it->second;
    {
        std::lock_guard<std::mutex> lock(g_r0_mu);
        auto g = g_r0.find(key);
        if (g != g_r0.end()) {
            c->r0_cache[key] = g->second;
            return g->second;
        }
    }
    ld_params cp{};
    cp.pupil_resolution = np;
    PsfBankArgs a{};
    setup_pupil(c, a, cp, true, s);
    a.B = 1;
    a.S = S;
    a.half = S / 2;
    a.off = std::max(0, (S - np) / 2);
    a.win_stride = S;
    WavelengthInfo wi{};
    wi.win_x0 = 0;
    wi.win_n = S;
    const size_t rings = static_cast<size_t>(S / 2 + 1);
    // scratch layout, each part 256-byte aligned: wavelength info | scalars |
    // ring sums + profile (3 * rings doubles) | counts | total | r0
    const size_t o_sc = align256(sizeof(WavelengthInfo));
    const size_t o_sums = o_sc + align256(sizeof(PsfScalars));
    const size_t o_cnt = o_sums + align256(rings * 3 * sizeof(double));
    const size_t o_tot = o_cnt + align256(rings * sizeof(int));
    const size_t o_r0 = o_tot + 256;
    char* cal = static_cast<char*>(ensure(c, c->calib, o_r0 + 256));
    WavelengthInfo* dwl = reinterpret_cast<WavelengthInfo*>(cal);
    PsfScalars* dsc = reinterpret_cast<PsfScalars*>(cal + o_sc);
    double* sums = reinterpret_cast<double*>(cal + o_sums);
    int* counts = reinterpret_cast<int*>(cal + o_cnt);
    double* total = reinterpret_cast<double*>(cal + o_tot);
    float* r0d = reinterpret_cast<float*>(cal + o_r0);
    a.wl = dwl;
    a.scalars = dsc;
    float r0 = 0.0f;
    if (smooth(S)) {
        a.plan_s = make_plan(c, S, fft_family(S, 1) == kE25);
        a.rows = static_cast<float2*>(ensure(c, c->rows, static_cast<size_t>(a.row_n) * S * sizeof(float2)));
        a.win = static_cast<float*>(ensure(c, c->calib_psf, static_cast<size_t>(S) * S * sizeof(float)));
        check_cuda(cudaMemcpyAsync(dwl, &wi, sizeof(wi), cudaMemcpyHostToDevice, s), "calib-upload");
        check_cuda(cudaMemsetAsync(dsc, 0, sizeof(PsfScalars), s), "calib-memset");
        check_cuda(cudaMemsetAsync(cal + o_sums, 0, o_r0 + 256 - o_sums, s), "calib-memset");
        launch_psf_rows(a, s);
        launch_psf_cols(a, s);
        launch_first_zero(a.win, S, sums, counts, total, r0d, s);
        check_launch("first-zero-calibration");
        check_cuda(cudaMemcpyAsync(&r0, r0d, sizeof(float), cudaMemcpyDeviceToHost, s), "calib-readback");
        check_cuda(cudaStreamSynchronize(s), "calib-sync");
    } else {
        // S with a prime factor above 5 (the reference takes Bluestein's
        // transform, LensDiffCpuReference.cpp:234-275): the PSF window around
        // the centre by DFT-as-GEMM.  The rings that lie wholly inside the
        // window have the whole PSF's profile; the PSF's sum comes from the
        // pupil by Parseval.  The window spans about four first-zero radii; a
        // scan that finds no minimum in it is repeated over the whole PSF.
        const int ci = S / 2;
        const double airy = 1.22 * static_cast<double>(S) / (0.86 * static_cast<double>(np));
        int W = std::min(S / 2, std::max(64, static_cast<int>(std::ceil(4.0 * airy)) + 8));
        for (int attempt = 0; attempt < 2; ++attempt) {
            if (attempt == 1) W = S / 2;
            wi.win_x0 = std::max(0, ci - W);
            wi.win_n = std::min(S, ci + W + 1) - wi.win_x0;
            a.win_stride = wi.win_n;
            a.win = static_cast<float*>(
                ensure(c, c->calib_psf, static_cast<size_t>(wi.win_n) * wi.win_n * sizeof(float)));
            check_cuda(cudaMemcpyAsync(dwl, &wi, sizeof(wi), cudaMemcpyHostToDevice, s), "calib-upload");
            check_cuda(cudaMemsetAsync(dsc, 0, sizeof(PsfScalars), s), "calib-memset");
            check_cuda(cudaMemsetAsync(cal + o_sums, 0, o_r0 + 256 - o_sums, s), "calib-memset");
            dft_gemm_psf(c, a, std::vector<WavelengthInfo>{wi}, s);
            launch_pupil_energy(a, static_cast<double>(S) * static_cast<double>(S), total, s);
            const int rings = W >= S / 2 ? S / 2 + 1 : W;
            launch_first_zero_window(a.win, a.win_stride, wi.win_n, wi.win_x0, S, rings, sums, counts, total, false,
                                     r0d, s);
            check_launch("first-zero-calibration");
            check_cuda(cudaMemcpyAsync(&r0, r0d, sizeof(float), cudaMemcpyDeviceToHost, s), "calib-readback");
            check_cuda(cudaStreamSynchronize(s), "calib-sync");
            if (r0 >= 0.0f) break;
        }
    }
    c->launches += 5;
    c->r0_cache[key] = r0;
    {
        std::lock_guard<std::mutex> lock(g_r0_mu);
        g_r0[key] = r0;
    }
    return r0;
}

// ---------------------------------------------------------------------------
// PSF bank
// ---------------------------------------------------------------------------
void fill_wavelength_infos(const ld_params& p, const std::vector<float>& wl, float r0, int S, int R,
                           std::vector<WavelengthInfo>* out, int* win_stride) {
    const float r0f = std::max(1.0f, r0);
    const double diff_px = percent_to_px(p.diffraction_scale_px, optics_short_side(p));
    const float scale_base = static_cast<float>(std::max(1.0, diff_px)) / r0f;  // CpuReference.cpp:1715
    const float rc = (S % 2 == 0) ? static_cast<float>(S) * 0.5f : static_cast<float>(S - 1) * 0.5f;
    *win_stride = 0;
    out->clear();
    for (float w : wl) {
        WavelengthInfo wi{};
        wi.phase = phase_for_wavelength(p, w);
        const float off = (w - 550.0f) / 110.0f;
        const float chrom = std::max(0.25f, 1.0f + static_cast<float>(p.chromatic_spread) * off);
        const float scale = scale_base * (w / 550.0f) * chrom;  // CpuReference.cpp:1729-1730
        const float inv = 1.0f / std::max(scale, 0.05f);        // :1071
        wi.inv_scale = inv;
        if (inv <= 1.0f) {
            wi.taps = 0;
            wi.step = 0.0f;
        } else {  // :343-344
            wi.taps = std::min(std::max(static_cast<int>(std::ceil(inv)), 2), 6);
            wi.step = inv / static_cast<float>(wi.taps);
        }
        const double reach = static_cast<double>(R) * inv + (inv > 1.0f ? 0.5 * inv : 0.0);
        int lo = static_cast<int>(std::floor(rc - reach)) - 2;
        int hi = static_cast<int>(std::ceil(rc + reach)) + 3;
        lo = std::max(0, lo);
        hi = std::min(S, hi);
        wi.win_x0 = lo;
        wi.win_n = std::max(1, hi - lo);
        *win_stride = std::max(*win_stride, wi.win_n);
        out->push_back(wi);
    }
}

const int* ring_counts(ld_ctx* c, int R) {
    auto it = c->ring_counts.find(R);
    if (it != c->ring_counts.end()) return static_cast<const int*>(it->second.p);
    const int K = 2 * R + 1;
    std::vector<int> cnt(static_cast<size_t>(R + 1), 0);
    const float kc = static_cast<float>(K - 1) * 0.5f;
    for (int y = 0; y < K; ++y)
        for (int x = 0; x < K; ++x) {
            const float dx = static_cast<float>(x) - kc, dy = static_cast<float>(y) - kc;
            const int r = std::min(R, static_cast<int>(std::round(std::sqrt(dx * dx + dy * dy))));
            cnt[static_cast<size_t>(r)] += 1;
        }
    DevBuf b;
    ensure(c, b, cnt.size() * sizeof(int));
    check_cuda(cudaMemcpy(b.p, cnt.data(), cnt.size() * sizeof(int), cudaMemcpyHostToDevice), "ring-count-upload");
    c->ring_counts[R] = b;
    return static_cast<const int*>(b.p);
}

// Pupil pixels along one axis whose centres lie within the outer radius of
// the (decentred) aperture: only they can be non-zero.
void pupil_extent(int n, float dec, int* lo_out, int* n_out) {
    int lo = n, hi = 0;
    for (int i = 0; i < n; ++i) {
        const float v = ((static_cast<float>(i) + 0.5f) / static_cast<float>(n) - 0.5f) * 2.0f;
        if (std::abs(v - dec) <= 0.8601f) {
            lo = std::min(lo, i);
            hi = std::max(hi, i + 1);
        }
    }
    if (hi <= lo) {
        lo = 0;
        hi = 1;
    }
    *lo_out = lo;
    *n_out = hi - lo;
}

// Tiles of the chosen form's DFT-as-GEMM for the bank's windows: one union
// window origin, each wavelength's first computed column rounded down to a
// multiple of 4 (basis tiles then start on 8-row boundaries), and the operand
// image sizes (ld_dftgemm.cu).
DftPlan plan_dft(const PsfBankArgs& a, const std::vector<WavelengthInfo>& infos, std::vector<DftLambda>* lam) {
    DftPlan d{};
    pupil_extent(a.pupil.size, a.pupil.decx, &d.col_lo, &d.col_n);
    d.mt_rows = (a.row_n + 127) / 128;
    d.kc_rows = (d.col_n + 31) / 32;
    d.kc_cols = (a.row_n + 31) / 32;
    int x0 = a.S;
    for (const WavelengthInfo& w : infos) x0 = std::min(x0, w.win_x0);
    d.x0 = x0;
    int width = 0;
    lam->assign(infos.size(), DftLambda{});
    for (size_t i = 0; i < infos.size(); ++i) {
        DftLambda& l = (*lam)[i];
        l.n0 = (infos[i].win_x0 - x0) / 4 * 4;
        l.shift = infos[i].win_x0 - x0 - l.n0;
        l.nt = (l.shift + infos[i].win_n + 127) / 128;
        d.nt_max = std::max(d.nt_max, l.nt);
        width = std::max(width, l.n0 + l.nt * 128);
    }
    d.basis_rows = 2 * width;
    d.pf_slab = static_cast<size_t>(d.mt_rows) * 128 * 128;
    d.pf_lambda = d.pf_slab * d.kc_rows;
    d.dx_slab = static_cast<size_t>(d.basis_rows) * 128;
    d.dy_slab = d.dx_slab;
    d.yt_slab = static_cast<size_t>(d.nt_max) * 128 * 128;
    d.yt_lambda = d.yt_slab * d.mt_rows * 4;
    return d;
}


// Chosen form: the bank's |F|^2 windows by DFT-as-GEMM on the tensor cores
// in place of the row and column FFTs (ld_dftgemm.cu).
// Scratch bytes of one lens's DFT-as-GEMM operands (pupil fields and row-pass
// outputs of its B wavelengths), each image 1 KiB aligned.
size_t dft_lens_bytes(const DftPlan& d, int B) {
    return 2 * (align1k(static_cast<size_t>(B) * d.pf_lambda) + align1k(static_cast<size_t>(B) * d.yt_lambda));
}
size_t dft_basis_bytes(const DftPlan& d) {
    return 2 * (align1k(d.dx_slab * d.kc_rows) + align1k(d.dy_slab * d.kc_cols));
}

// The bank windows of several lenses (one PsfBankArgs and wavelength table
// each) in one launch per pass of the persistent tensor-core GEMM: every
// (lens, wavelength) pass is one problem of the work queue, whatever its
// pupil size, PSF size, window or wavelength count.  Lenses whose basis
// geometry matches (PSF size, pupil extent, union window: the field zones of
// one lens) share one pair of basis images; each keeps its own pupil fields.
void dft_gemm_psf_batch(ld_ctx* c, const std::vector<const PsfBankArgs*>& banks,
                        const std::vector<const std::vector<WavelengthInfo>*>& infos, cudaStream_t s) {
    const size_t Z = banks.size();
    std::vector<DftPlan> plan(Z);
    std::vector<std::vector<DftLambda>> lam(Z);
    std::vector<size_t> group(Z);  // index of the lens whose basis images this lens reads
    size_t P = 0, bytes = 1024;
    for (size_t z = 0; z < Z; ++z) {
        const PsfBankArgs& a = *banks[z];
        plan[z] = plan_dft(a, *infos[z], &lam[z]);
        const DftPlan& d = plan[z];
        group[z] = z;
        for (size_t k = 0; k < z; ++k) {
            const DftPlan& e = plan[k];
            const PsfBankArgs& b = *banks[k];
            if (group[k] == k && b.S == a.S && e.basis_rows == d.basis_rows && e.x0 == d.x0 &&
                e.kc_rows == d.kc_rows && e.col_n == d.col_n && b.off + e.col_lo == a.off + d.col_lo &&
                e.kc_cols == d.kc_cols && b.row_n == a.row_n && b.off + b.row_lo == a.off + a.row_lo) {
                group[z] = k;
                break;
            }
        }
        P += static_cast<size_t>(a.B);
        bytes += dft_lens_bytes(d, a.B) + (group[z] == z && Z > 1 ? dft_basis_bytes(d) : 0);
    }
    // one lens: its basis images live in the context's basis cache, rebuilt
    // only when the geometry changes
    bool basis_cached = false;
    std::vector<int> basis_key;
    if (Z == 1) {
        const PsfBankArgs& a = *banks[0];
        const DftPlan& d = plan[0];
        const std::vector<int> key{a.S,       d.basis_rows, d.x0,     d.kc_rows,         d.col_n,
                                   a.off + d.col_lo,        d.kc_cols, a.row_n, a.off + a.row_lo};
        const size_t rb = align1k(d.dx_slab * d.kc_rows), cb = align1k(d.dy_slab * d.kc_cols);
        basis_cached = c->basis_key == key && c->basis.bytes >= 2 * (rb + cb);
        // the key is recorded once both basis launches are enqueued: a build
        // that fails before then leaves no key for stale images to match
        if (!basis_cached) c->basis_key.clear();
        unsigned char* q = static_cast<unsigned char*>(ensure(c, c->basis, 2 * (rb + cb)));
        basis_key = key;
        plan[0].dx_hi = q;
        plan[0].dx_lo = q + rb;
        plan[0].dy_hi = q + 2 * rb;
        plan[0].dy_lo = q + 2 * rb + cb;
    }
    bytes += align1k(2 * P * sizeof(DftProblem)) + align1k((2 * P + 4) * sizeof(int));
    char* p = static_cast<char*>(ensure(c, c->dft, bytes));
    auto take = [&](size_t n) {
        char* q = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~static_cast<uintptr_t>(1023));
        p = q + n;
        return reinterpret_cast<unsigned char*>(q);
    };
    for (size_t z = 0; z < Z; ++z) {
        DftPlan& d = plan[z];
        const int B = banks[z]->B;
        d.pf_hi = take(B * d.pf_lambda);
        d.pf_lo = take(B * d.pf_lambda);
        d.yt_hi = take(B * d.yt_lambda);
        d.yt_lo = take(B * d.yt_lambda);
        if (group[z] == z) {
            if (Z == 1) continue;  // the basis cache's images
            d.dx_hi = take(d.dx_slab * d.kc_rows);
            d.dx_lo = take(d.dx_slab * d.kc_rows);
            d.dy_hi = take(d.dy_slab * d.kc_cols);
            d.dy_lo = take(d.dy_slab * d.kc_cols);
        } else {
            const DftPlan& g = plan[group[z]];
            d.dx_hi = g.dx_hi;
            d.dx_lo = g.dx_lo;
            d.dy_hi = g.dy_hi;
            d.dy_lo = g.dy_lo;
        }
    }
    // problem tables of the two passes (one problem per lens and wavelength),
    // their tile prefixes and the two work-queue counters
    std::vector<DftProblem> rows(P), cols(P);
    std::vector<int> rstart(P + 1, 0), cstart(P + 1, 0);
    size_t i = 0;
    for (size_t z = 0; z < Z; ++z) {
        const PsfBankArgs& a = *banks[z];
        const DftPlan& d = plan[z];
        for (int b = 0; b < a.B; ++b, ++i) {
            const DftLambda& l = lam[z][static_cast<size_t>(b)];
            DftProblem& r = rows[i];
            r.a_hi = d.pf_hi + b * d.pf_lambda;
            r.a_lo = d.pf_lo + b * d.pf_lambda;
            r.b_hi = d.dx_hi;
            r.b_lo = d.dx_lo;
            r.y_hi = d.yt_hi + b * d.yt_lambda;
            r.y_lo = d.yt_lo + b * d.yt_lambda;
            r.a_slab = static_cast<uint32_t>(d.pf_slab);
            r.b_slab = static_cast<uint32_t>(d.dx_slab);
            r.y_slab = static_cast<uint32_t>(d.yt_slab);
            r.kc = d.kc_rows;
            r.mt = d.mt_rows;
            r.nt = l.nt;
            r.n0 = l.n0;
            r.shift = l.shift;
            DftProblem& q = cols[i];
            q.a_hi = d.yt_hi + b * d.yt_lambda;
            q.a_lo = d.yt_lo + b * d.yt_lambda;
            q.b_hi = d.dy_hi;
            q.b_lo = d.dy_lo;
            q.win = a.win + static_cast<size_t>(b) * a.win_stride * a.win_stride;
            q.energy = a.want_energy ? &a.scalars[b].energy : nullptr;
            q.a_slab = static_cast<uint32_t>(d.yt_slab);
            q.b_slab = static_cast<uint32_t>(d.dy_slab);
            q.kc = d.kc_cols;
            q.mt = l.nt;
            q.nt = l.nt;
            q.n0 = l.n0;
            q.shift = l.shift;
            q.win_n = (*infos[z])[static_cast<size_t>(b)].win_n;
            q.win_stride = a.win_stride;
            rstart[i + 1] = rstart[i] + r.mt * r.nt;
            cstart[i + 1] = cstart[i] + q.mt * q.nt;
        }
    }
    // one block, one upload: the row and column problems, then the tile
    // prefixes and the two counters
    const int np = static_cast<int>(P);
    const size_t prob_bytes = (2 * P * sizeof(DftProblem) + 15) & ~static_cast<size_t>(15);
    std::vector<int> starts(rstart);
    starts.insert(starts.end(), cstart.begin(), cstart.end());
    starts.push_back(0);  // the two counters
    starts.push_back(0);
    const size_t table_bytes = prob_bytes + starts.size() * sizeof(int);
    unsigned char* dtab = take(table_bytes);
    DftProblem* drows = reinterpret_cast<DftProblem*>(dtab);
    DftProblem* dcols = drows + P;
    int* dstart = reinterpret_cast<int*>(dtab + prob_bytes);
    std::vector<unsigned char> table(table_bytes, 0);
    std::memcpy(table.data(), rows.data(), P * sizeof(DftProblem));
    std::memcpy(table.data() + P * sizeof(DftProblem), cols.data(), P * sizeof(DftProblem));
    std::memcpy(table.data() + prob_bytes, starts.data(), starts.size() * sizeof(int));
    upload_async(c, dtab, table.data(), table_bytes, s, "dft-upload");
    DftBatchArgs gr{drows, dstart, np, rstart.back(), kDftRows, dstart + 2 * (np + 1), c->err};
    DftBatchArgs gc{dcols, dstart + (np + 1), np, cstart.back(), kDftCols, dstart + 2 * (np + 1) + 1, c->err};
    auto basis = [&](const PsfBankArgs& a, const DftPlan& d, bool rows_pass) {
        return rows_pass ? DftBasisArgs{d.dx_hi, d.dx_lo, d.dx_slab, d.basis_rows, d.kc_rows, d.col_n,
                                        a.off + d.col_lo, d.x0, a.S / 2, a.S}
                         : DftBasisArgs{d.dy_hi, d.dy_lo, d.dy_slab, d.basis_rows, d.kc_cols, a.row_n,
                                        a.off + a.row_lo, d.x0, a.S / 2, a.S};
    };
    staged(c, LD_STAGE_PSF_ROWS, s, [&] {
        for (size_t z = 0; z < Z; ++z) {
            launch_pupil_field(*banks[z], plan[z], s);
            if (group[z] == z && !basis_cached) launch_dft_basis(basis(*banks[z], plan[z], true), s);
        }
    });
    staged(c, LD_STAGE_DFT_GEMM, s, [&] { launch_dft_gemm(gr, s); });
    if (!basis_cached) {
        staged(c, LD_STAGE_PSF_COLS, s, [&] {
            for (size_t z = 0; z < Z; ++z)
                if (group[z] == z) launch_dft_basis(basis(*banks[z], plan[z], false), s);
        });
        check_launch("dft-basis");
        if (Z == 1) c->basis_key = basis_key;
    }
    staged(c, LD_STAGE_DFT_GEMM, s, [&] { launch_dft_gemm(gc, s); });
    size_t groups = 0;  // the preparation stages launched Z + groups and groups kernels (Z without bases)
    for (size_t z = 0; z < Z; ++z) groups += group[z] == z;
    c->launches += basis_cached ? static_cast<int>(Z) - 1 : static_cast<int>(Z + 2 * groups) - 2;
    // a tile is a 128 x 256 x 64 real product per K-chunk, three times (hi.hi, hi.lo, lo.hi)
    double kt = 0.0;
    for (size_t k = 0; k < P; ++k)
        kt += static_cast<double>(rows[k].kc) * rows[k].mt * rows[k].nt + static_cast<double>(cols[k].kc) * cols[k].mt * cols[k].nt;
    c->tensor_flops += kt * 3.0 * 2.0 * 128.0 * 256.0 * 64.0;
}

void dft_gemm_psf(ld_ctx* c, const PsfBankArgs& a, const std::vector<WavelengthInfo>& infos, cudaStream_t s) {
    dft_gemm_psf_batch(c, {&a}, {&infos}, s);
}

// Bank windows computed ahead of the bank (several field zones' windows in
// one batched transform): the bank build takes them instead of synthesising.
struct PreWindows {
    float* win;
    WavelengthInfo* wl;  // device, the matching wavelength table
};

// The bank of `p`: the context's bank or a bank of the last lens set when
// one matches, else built into the context's bank.  With `into`, built into
// that entry unconditionally (lens sets).
BankEntry& ensure_bank(ld_ctx* c, const ld_params& p, cudaStream_t s, bool* rebuilt,
                       const PreWindows* pre = nullptr, BankEntry* into = nullptr) {
    const std::vector<float> wl = wavelengths_of(p);
    const std::string key = bank_key(p, wl);
    *rebuilt = false;
    if (!into) {
        if (c->bank.valid && c->bank.key == key) return c->bank;
        for (BankEntry& e : c->set_banks)
            if (e.valid && e.key == key) return e;
    }
    BankEntry& b = into ? *into : c->bank;
    b.valid = false;
    const int np = pupil_size(p);
    const int R = max_kernel_radius(p);
    const int S = raw_psf_size(np, R);
    const int K = 2 * R + 1;
    const int B = static_cast<int>(wl.size());
    if (B > kMaxBins) throw Fail{LD_ERR_ARG, "too-many-wavelengths"};
    const float r0 = first_zero(c, np, S, s);
    std::vector<WavelengthInfo> infos;
    int win_stride = 0;
    fill_wavelength_infos(p, wl, r0, S, R, &infos, &win_stride);

    PsfBankArgs& a = b.args;
    a = PsfBankArgs{};
    if (!pre) setup_pupil(c, a, p, false, s);
    a.B = B;
    a.S = S;
    a.half = S / 2;
    a.off = std::max(0, (S - np) / 2);
    a.win_stride = win_stride;
    a.raw_center = (S % 2 == 0) ? static_cast<float>(S) * 0.5f : static_cast<float>(S - 1) * 0.5f;
    a.R = R;
    a.K = K;
    a.gain = 1.0f + std::max(0.0f, static_cast<float>(p.anisotropy_emphasis)) * 4.0f;  // :1127
    // tensor-core DFT for the chosen form, and for S with a prime factor above
    // 5 (the reference's Bluestein sizes) in every own form
    const bool dft = p.fft_form == LD_FFT_OWN_CHOSEN || (p.fft_form == LD_FFT_OWN_FP32 && !smooth(S));
    if (!pre && !dft && p.fft_form != LD_FFT_CUFFT) {
        a.plan_s = make_plan(c, S, fft_family(S, 1) == kE25);
        a.rows = static_cast<float2*>(ensure(c, c->rows, static_cast<size_t>(B) * a.row_n * win_stride * sizeof(float2)));
    }
    a.win = pre ? pre->win
                : static_cast<float*>(ensure(c, c->win, static_cast<size_t>(B) * win_stride * win_stride * sizeof(float)));
    a.canvas = static_cast<float*>(ensure(c, b.canvas, static_cast<size_t>(B) * K * K * sizeof(float)));
    const size_t ringn = static_cast<size_t>(B) * (R + 1);
    a.ring_round = static_cast<double*>(ensure(c, b.ring_round, ringn * sizeof(double)));
    a.ring_ceil = static_cast<double*>(ensure(c, b.ring_ceil, ringn * sizeof(double)));
    a.ring_peak = static_cast<unsigned int*>(ensure(c, b.ring_peak, ringn * sizeof(unsigned int)));
    a.ring_mean = static_cast<float*>(ensure(c, b.ring_mean, ringn * sizeof(float)));
    a.scalars = static_cast<PsfScalars*>(ensure(c, b.scalars, static_cast<size_t>(B) * sizeof(PsfScalars)));
    WavelengthInfo* dwl =
        pre ? pre->wl : static_cast<WavelengthInfo*>(ensure(c, b.wl, static_cast<size_t>(B) * sizeof(WavelengthInfo)));
    a.wl = dwl;
    a.count_round = ring_counts(c, R);
    a.want_energy = 0;
    if (!pre) upload_async(c, dwl, infos.data(), infos.size() * sizeof(WavelengthInfo), s, "bank-upload");
    check_cuda(cudaMemsetAsync(a.ring_round, 0, ringn * sizeof(double), s), "bank-memset");
    check_cuda(cudaMemsetAsync(a.ring_ceil, 0, ringn * sizeof(double), s), "bank-memset");
    check_cuda(cudaMemsetAsync(a.ring_peak, 0, ringn * sizeof(unsigned int), s), "bank-memset");
    check_cuda(cudaMemsetAsync(a.scalars, 0, static_cast<size_t>(B) * sizeof(PsfScalars), s), "bank-memset");
    if (pre) {
        // windows already synthesised
    } else if (p.fft_form == LD_FFT_CUFFT) {
        float2* grid = static_cast<float2*>(
            ensure(c, c->cf_grid, cf_psf_chunk(S, B) * static_cast<size_t>(S) * S * sizeof(float2)));
        staged(c, LD_STAGE_PSF_ROWS, s, [&] { cf_psf_transform(a, grid, c->cufft, s); });
    } else if (dft) {
        dft_gemm_psf(c, a, infos, s);
    } else {
        staged(c, LD_STAGE_PSF_ROWS, s, [&] { launch_psf_rows(a, s); });
        staged(c, LD_STAGE_PSF_COLS, s, [&] { launch_psf_cols(a, s); });
    }
    const bool pairs = std::all_of(infos.begin(), infos.end(), [](const WavelengthInfo& w) { return w.taps == 0; });
    staged(c, LD_STAGE_RESAMPLE, s, [&] { launch_resample(a, pairs, s); });
    const bool fused = fused_shaping(a);
    if (!fused) staged(c, LD_STAGE_SHAPE_STATS, s, [&] { launch_shape_stats(a, s); });
    staged(c, LD_STAGE_SUPPORT, s, [&] { launch_support(a, s); });
    staged(c, LD_STAGE_CROP_SUM, s, [&] { launch_crop_sum(a, s); });
    check_launch("psf-bank");
    b.B = B;
    b.np = np;
    b.S = S;
    b.R = R;
    b.K = K;
    b.win_stride = win_stride;
    b.wavelengths = wl;
    b.cufft = p.fft_form == LD_FFT_CUFFT;
    b.h16 = chosen_h16(p);
    b.split_sums = false;
    b.ring_means = !fused;
    b.key = key;
    b.valid = true;
    if (!into) c->spectra.valid = false;
    *rebuilt = true;
    return b;
}

// ---------------------------------------------------------------------------
// spectral -> RGB combination (MapLensDiffSpectralBins, LensDiffSpectrum.cpp:462-497)
// ---------------------------------------------------------------------------
struct Combination {
    int mono = 0;
    int parts = 1;  // kernel sets: 1 (Physical: full) or 2 (Split: core, structure)
    int n_drv = 1, n_ker = 3, n_out = 3;
    int luma_lock = 0;
    float saturation = 1.0f;
    float coef[4][kMaxBins] = {};
};

void gaussian_matrix(const float* wl, int n, const float* center, float sigma, float* m) {
    for (int c = 0; c < 3; ++c) {
        double sum = 0.0;
        for (int b = 0; b < n; ++b) {
            const double t = (static_cast<double>(wl[b]) - center[c]) / sigma;
            sum += std::exp(-0.5 * t * t);
        }
        for (int b = 0; b < n; ++b) {
            const double t = (static_cast<double>(wl[b]) - center[c]) / sigma;
            m[c * n + b] = static_cast<float>(std::exp(-0.5 * t * t) / (sum > 0.0 ? sum : 1.0));
        }
    }
}

// Core and structure kernel sets are needed by the Split look and by the Core
// and Structure debug views (LensDiffCpuReference.cpp:2123-2157).
bool split_kernels(const ld_params& p) {
    return p.look_mode == LD_LOOK_SPLIT || p.debug_view == LD_DEBUG_CORE || p.debug_view == LD_DEBUG_STRUCTURE;
}

Combination make_combination(const ld_params& p, const std::vector<float>& wl) {
    Combination cb;
    const int B = static_cast<int>(wl.size());
    if (is_mono(p)) {  // convolveRgba, CpuReference.cpp:1195-1217
        cb.mono = 1;
        cb.parts = split_kernels(p) ? 2 : 1;
        cb.n_drv = 3;
        cb.n_ker = 1;
        cb.n_out = 3;
        cb.coef[0][0] = 1.0f;
        return cb;
    }
    std::vector<float> nat(static_cast<size_t>(3 * B)), sty(static_cast<size_t>(3 * B));
    if (B <= 1) {  // mulMatrix with binCount <= 1 replicates the bin (LensDiffSpectrum.cpp:365-367)
        for (int c = 0; c < 3; ++c) nat[c] = sty[c] = 1.0f;
    } else if (p.rgb_mode == LD_RGB_GAUSSIAN) {
        gaussian_matrix(wl.data(), B, p.rgb_gauss_center_nm, p.rgb_gauss_sigma_nm, nat.data());
        sty = nat;
    } else {
        for (int i = 0; i < 3 * B; ++i) {
            nat[static_cast<size_t>(i)] = p.natural_matrix[i];
            sty[static_cast<size_t>(i)] = p.style_matrix[i];
        }
        bool any = false;
        for (float v : nat) any |= v != 0.0f;
        if (!any) throw Fail{LD_ERR_ARG, "missing-spectral-matrix"};
    }
    const float force = std::min(std::max(static_cast<float>(p.spectrum_force), 0.0f), 1.0f);
    cb.saturation = static_cast<float>(std::max(0.0, p.spectrum_saturation));
    const float lw[3] = {0.2126f, 0.7152f, 0.0722f};
    bool lock_identity = true;
    for (int b = 0; b < B; ++b) {
        float ln = 0.0f, lm = 0.0f;
        for (int c = 0; c < 3; ++c) {
            const float n = nat[static_cast<size_t>(c * B + b)];
            const float m = n * (1.0f - force) + sty[static_cast<size_t>(c * B + b)] * force;
            cb.coef[c][b] = m;
            if (m < 0.0f) lock_identity = false;
            ln += lw[c] * n;
            lm += lw[c] * m;
        }
        cb.coef[3][b] = ln;
        if (std::abs(ln - lm) > 1e-6f * std::max(1.0f, std::abs(ln))) lock_identity = false;
    }
    cb.luma_lock = (!p.chromatic_affects_luma && !lock_identity) ? 1 : 0;
    cb.n_ker = cb.luma_lock ? 4 : 3;
    cb.n_out = cb.n_ker;
    cb.n_drv = 1;
    cb.parts = split_kernels(p) ? 2 : 1;
    return cb;
}

std::string spectra_key_for(const std::string& bank_key_s, const Combination& cb, const GridGeom& g) {
    std::string k = bank_key_s;
    k = append_bytes(k, &cb.parts, sizeof(int));
    k = append_bytes(k, &cb.n_ker, sizeof(int));
    k = append_bytes(k, cb.coef, sizeof(cb.coef));
    k = append_bytes(k, &g.Px, sizeof(int));
    k = append_bytes(k, &g.Py, sizeof(int));
    return k;
}

constexpr size_t kSmemBudget = 227 * 1024;

// Shared-memory passes of a transform of length n (its stage count), or a
// large number when n has no plan.
int fft_passes(int n, bool allow25) {
    std::vector<int> r;
    return factor_radices(n, allow25, &r) ? static_cast<int>(r.size()) : 1000;
}

// Cheapest 5-smooth length >= n (a multiple of `mult`) for up to C
// interleaved sequences: cost ~ m * (stages + 1.5), the stage passes plus the
// fill and drain, so a slightly longer length with fewer stages can win.
int choose_length(int n, int mult, int C) {
    int best = -1;
    double best_cost = 0.0;
    const int hi = n + std::max(64, n / 10);
    for (int m = std::max(n, 2); m <= hi; ++m) {
        if (m % mult != 0 || !smooth(m)) continue;
        const int fam = fft_family(m, C);
        if (fam == 0) continue;
        const double cost = static_cast<double>(m) * (fft_passes(m, fam == kE25) + 1.5);
        if (best < 0 || cost < best_cost) {
            best = m;
            best_cost = cost;
        }
    }
    return best;
}

// 5-smooth grid covering the linear convolution: Px = 2M with M the row
// transform length, Py even (16-byte bulk-copy sizes).  The reference pads to
// powers of two (LensDiffCpuReference.cpp:1172-1173); any grid of at least
// W+K-1 x H+K-1 gives the same linear convolution.  c_rows / c_cols: the
// most interleaved sequences any row / column kernel of the chain transforms
// (they pick the FFT family).
GridGeom make_geometry(ld_ctx* c, int W, int H, int K, int c_rows, int c_cols, int* req_w, int* req_h) {
    GridGeom g{};
    *req_w = W + K - 1;
    *req_h = H + K - 1;
    g.M = choose_length((*req_w + 1) / 2, 1, c_rows);
    g.Py = choose_length(*req_h, 4, c_cols);  // FP16 column bulk copies want Py * 3 * 4 bytes % 16 == 0
    if (g.M < 0 || g.Py < 0) throw Fail{LD_ERR_UNSUPPORTED, "frame-too-large-for-fft-grid"};
    g.Px = 2 * g.M;
    g.cols = g.M + 1;
    g.fam_m = fft_family(g.M, c_rows);
    g.fam_py = fft_family(g.Py, c_cols);
    const int Kp = K + (K & 1);
    if (frame_cols_smem(g.Py, c_cols) > kSmemBudget || kspec_cols_smem(g.Py, Kp, c_cols) > kSmemBudget)
        throw Fail{LD_ERR_UNSUPPORTED, "frame-too-large-for-column-pass"};
    g.plan_m = make_plan(c, g.M, g.fam_m == kE25);
    g.plan_py = make_plan(c, g.Py, g.fam_py == kE25);
    g.tw_px = twiddles(c, g.Px);
    return g;
}

// Layout of a kernel-spectra buffer: the parts' spectra (float2, or half2 in
// the chosen form) back to back, 256-byte aligned, then one float scale per
// column for each part (chosen form).
size_t ks_part_bytes(int n_ker, const GridGeom& g, bool h16) {
    return align256(static_cast<size_t>(n_ker) * g.cols * g.Py * (h16 ? 4 : 8));
}
const float2* ks_part(const void* base, int part, int n_ker, const GridGeom& g, bool h16) {
    return reinterpret_cast<const float2*>(static_cast<const char*>(base) + part * ks_part_bytes(n_ker, g, h16));
}
const float* ks_scale(const void* base, int part, int parts, int n_ker, const GridGeom& g, bool h16) {
    return reinterpret_cast<const float*>(static_cast<const char*>(base) + parts * ks_part_bytes(n_ker, g, h16)) +
           static_cast<size_t>(part) * g.cols;
}

// Kernel spectra of bank `b` into entry `e` (combination, row and column
// transforms), unless `e` already holds them.
SpectraEntry& ensure_spectra_in(ld_ctx* c, SpectraEntry& e, BankEntry& b, const Combination& cb, const GridGeom& g,
                                cudaStream_t s, bool* rebuilt) {
    const std::string key = spectra_key_for(b.key, cb, g);
    *rebuilt = false;
    if (e.valid && e.key == key) return e;
    e.valid = false;
    if (cb.parts == 2 && !b.ring_means) {
        staged(c, LD_STAGE_SHAPE_STATS, s, [&] { launch_ring_means(b.args, s); });
        b.ring_means = true;
    }
    if (cb.parts == 2 && !b.split_sums) {
        staged(c, LD_STAGE_CROP_SUM, s, [&] { launch_split_sums(b.args, s); });
        b.split_sums = true;
    }
    CombineArgs ca{};
    ca.bank = b.args;
    ca.n_ker = cb.n_ker;
    ca.split = cb.parts == 2 ? 1 : 0;
    std::memcpy(ca.coef, cb.coef, sizeof(ca.coef));
    const size_t kk = static_cast<size_t>(b.K) * b.K;
    ca.out = static_cast<float*>(ensure(c, c->combine_out, cb.parts * cb.n_ker * kk * sizeof(float)));
    staged(c, LD_STAGE_COMBINE, s, [&] { launch_combine(ca, s); });
    KernelSpectraArgs ka{};
    ka.g = g;
    ka.n_ker = cb.n_ker;
    ka.R = b.R;
    ka.K = b.K;
    ka.Kp = b.K + (b.K & 1);
    ka.rows = static_cast<float2*>(
        ensure(c, c->kspec_rows, static_cast<size_t>(cb.n_ker) * g.cols * ka.Kp * sizeof(float2)));
    const size_t part_bytes = ks_part_bytes(cb.n_ker, g, b.h16);
    char* ksbuf = static_cast<char*>(
        ensure(c, e.spectra, cb.parts * (part_bytes + static_cast<size_t>(g.cols) * sizeof(float))));
    ka.h16 = b.h16 ? 1 : 0;
    ka.scale = static_cast<float>(1.0 / (static_cast<double>(g.M) * static_cast<double>(g.Py)));
    ka.err = c->err;
    for (int part = 0; part < cb.parts; ++part) {
        ka.canvas = ca.out + static_cast<size_t>(part) * cb.n_ker * kk;
        ka.spectra = const_cast<float2*>(ks_part(ksbuf, part, cb.n_ker, g, b.h16));
        ka.kscale = const_cast<float*>(ks_scale(ksbuf, part, cb.parts, cb.n_ker, g, b.h16));
        if (b.cufft) {
            // cuFFT layout: KS [n_ker][Py][Px/2+1], the same size as the own layout
            float* planes = static_cast<float*>(
                ensure(c, c->cf_planes, static_cast<size_t>(cb.n_ker) * g.Px * g.Py * sizeof(float)));
            staged(c, LD_STAGE_KSPEC_COLS, s, [&] { cf_kernel_spectra(ka, planes, c->cufft, s); });
        } else {
            staged(c, LD_STAGE_KSPEC_ROWS, s, [&] { launch_kspec_rows(ka, s); });
            staged(c, LD_STAGE_KSPEC_COLS, s, [&] { launch_kspec_cols(ka, s); });
        }
    }
    check_launch("kernel-spectra");
    e.g = g;
    e.n_ker = cb.n_ker;
    e.key = key;
    e.valid = true;
    *rebuilt = true;
    return e;
}

// Three slots: one in use by the frame on the GPU, one being built on the bank
// stream, one for a recent lens; a stream of new lenses rotates through them,
// so its per-frame chains settle on three cached graphs.
constexpr size_t kSpectraCache = 3;

// Kernel spectra for (lens p, geometry g) from the context's LRU cache; the
// bank is built (or reused) only on a miss.
// Whether every kernel-spectra set a frame needs is cached already.
bool spectra_cached(ld_ctx* c, const ld_params& p, bool zones, int zn, const Combination& cb, const GridGeom& g) {
    const std::vector<float> wl = wavelengths_of(p);
    if (!zones) {
        const std::string key = spectra_key_for(bank_key(p, wl), cb, g);
        for (const auto& e : c->spectra_lru)
            if (e.valid && e.key == key) return true;
        return false;
    }
    if (static_cast<int>(c->zone_spectra.size()) != zn * zn) return false;
    for (int zy = 0; zy < zn; ++zy) {
        for (int zx = 0; zx < zn; ++zx) {
            const float nx = (2.0f * static_cast<float>(zx)) / static_cast<float>(zn - 1) - 1.0f;
            const float ny = (2.0f * static_cast<float>(zy)) / static_cast<float>(zn - 1) - 1.0f;
            const SpectraEntry& e = c->zone_spectra[static_cast<size_t>(zy) * zn + zx];
            if (!(e.valid && e.key == spectra_key_for(bank_key(zone_params(p, nx, ny), wl), cb, g))) return false;
        }
    }
    return true;
}

SpectraEntry& cached_spectra(ld_ctx* c, const ld_params& p, const Combination& cb, const GridGeom& g, cudaStream_t s,
                             bool* bank_rebuilt, bool* spectra_rebuilt) {
    const std::string key = spectra_key_for(bank_key(p, wavelengths_of(p)), cb, g);
    for (auto& e : c->spectra_lru) {
        if (e.valid && e.key == key) {
            e.last_use = ++c->spectra_clock;
            return e;
        }
    }
    if (c->spectra_lru.size() < kSpectraCache) c->spectra_lru.emplace_back();
    SpectraEntry* victim = &c->spectra_lru.front();
    for (auto& e : c->spectra_lru) {
        if (!e.valid) {
            victim = &e;
            break;
        }
        if (e.last_use < victim->last_use) victim = &e;
    }
    wait_free(*victim, s);
    BankEntry& b = ensure_bank(c, p, s, bank_rebuilt);
    ensure_spectra_in(c, *victim, b, cb, g, s, spectra_rebuilt);
    victim->last_use = ++c->spectra_clock;
    return *victim;
}

// Field zones: the kernel spectra of every zone of an n x n grid, in the
// reference's order (zy outer, zx inner, LensDiffCpuReference.cpp:1779-1783),
// each zone's bank built from its resolved parameters (makeFieldZoneCache,
// :1736-1756) only when that zone's spectra are not cached already.
std::vector<const SpectraEntry*> ensure_zone_spectra(ld_ctx* c, const ld_params& p, int n, const Combination& cb,
                                                     const GridGeom& g, cudaStream_t s, bool* bank_rebuilt,
                                                     bool* spectra_rebuilt) {
    if (static_cast<int>(c->zone_spectra.size()) != n * n) {
        for (auto& z : c->zone_spectra) free_buf(c, z.spectra);
        c->zone_spectra.clear();
        c->zone_spectra.resize(static_cast<size_t>(n) * n);
    }
    const std::vector<float> wl = wavelengths_of(p);
    const int nz = n * n;
    std::vector<ld_params> zps(static_cast<size_t>(nz));
    std::vector<std::string> keys(static_cast<size_t>(nz));
    std::vector<int> need;
    for (int z = 0; z < nz; ++z) {
        const float nx = (2.0f * static_cast<float>(z % n)) / static_cast<float>(n - 1) - 1.0f;
        const float ny = (2.0f * static_cast<float>(z / n)) / static_cast<float>(n - 1) - 1.0f;
        zps[static_cast<size_t>(z)] = zone_params(p, nx, ny);
        keys[static_cast<size_t>(z)] = spectra_key_for(bank_key(zps[static_cast<size_t>(z)], wl), cb, g);
        const SpectraEntry& e = c->zone_spectra[static_cast<size_t>(z)];
        if (!(e.valid && e.key == keys[static_cast<size_t>(z)])) need.push_back(z);
    }
    for (int z : need) wait_free(c->zone_spectra[static_cast<size_t>(z)], s);
    // The zones share the transform geometry: with the tensor-core DFT, every
    // zone's windows come from one batched launch per pass.
    const int np = pupil_size(p), R = max_kernel_radius(p), S = raw_psf_size(np, R);
    const bool dft = p.fft_form == LD_FFT_OWN_CHOSEN || (p.fft_form == LD_FFT_OWN_FP32 && !smooth(S));
    std::vector<PreWindows> pre(static_cast<size_t>(nz), PreWindows{nullptr, nullptr});
    if (dft && need.size() >= 2) {
        c->zone_pupil.resize(static_cast<size_t>(nz));
        c->zone_wl.resize(static_cast<size_t>(nz));
        c->zone_win.resize(static_cast<size_t>(nz));
        const float r0 = first_zero(c, np, S, s);
        std::vector<PsfBankArgs> args(need.size());
        std::vector<std::vector<WavelengthInfo>> infos(need.size());
        std::vector<const PsfBankArgs*> bp;
        std::vector<const std::vector<WavelengthInfo>*> ip;
        for (size_t k = 0; k < need.size(); ++k) {
            const int z = need[k];
            const ld_params& zp = zps[static_cast<size_t>(z)];
            int ws = 0;
            fill_wavelength_infos(zp, wl, r0, S, R, &infos[k], &ws);
            PsfBankArgs& a = args[k];
            setup_pupil(c, a, zp, false, s, &c->zone_pupil[static_cast<size_t>(z)]);
            a.B = static_cast<int>(wl.size());
            a.S = S;
            a.half = S / 2;
            a.off = std::max(0, (S - np) / 2);
            a.win_stride = ws;
            a.wl = static_cast<WavelengthInfo*>(
                ensure(c, c->zone_wl[static_cast<size_t>(z)], infos[k].size() * sizeof(WavelengthInfo)));
            a.win = static_cast<float*>(
                ensure(c, c->zone_win[static_cast<size_t>(z)], static_cast<size_t>(a.B) * ws * ws * sizeof(float)));
            upload_async(c, const_cast<WavelengthInfo*>(a.wl), infos[k].data(),
                         infos[k].size() * sizeof(WavelengthInfo), s, "zone-upload");
            pre[static_cast<size_t>(z)] = PreWindows{a.win, const_cast<WavelengthInfo*>(a.wl)};
            bp.push_back(&a);
            ip.push_back(&infos[k]);
        }
        dft_gemm_psf_batch(c, bp, ip, s);
    }
    std::vector<const SpectraEntry*> out;
    for (int zy = 0; zy < n; ++zy) {
        for (int zx = 0; zx < n; ++zx) {
            const int z = zy * n + zx;
            const ld_params& zp = zps[static_cast<size_t>(z)];
            SpectraEntry& e = c->zone_spectra[static_cast<size_t>(z)];
            const std::string& key = keys[static_cast<size_t>(z)];
            if (!(e.valid && e.key == key)) {
                bool rb = false, rs = false;
                const PreWindows& pw = pre[static_cast<size_t>(z)];
                BankEntry& b = ensure_bank(c, zp, s, &rb, pw.win ? &pw : nullptr);
                ensure_spectra_in(c, e, b, cb, g, s, &rs);
                *bank_rebuilt = *bank_rebuilt || rb;
                *spectra_rebuilt = *spectra_rebuilt || rs;
            }
            out.push_back(&e);
        }
    }
    return out;
}

// Scratch of one chunk of a lens set's batched transform (pupils, windows,
// DFT operand images): lenses join a chunk while its scratch stays within
// this, or a quarter of the context's HBM budget when that is smaller.
constexpr size_t kSetChunkBytes = size_t(32) << 30;

// The banks of `n` unrelated lenses (pupil size, PSF size, wavelengths and
// phase all free), each as EnsureLensDiffPsfBank builds one
// (LensDiffCpuReference.cpp:2068-2071).  Banks already built for the same
// lens at the same position are kept.  The lenses whose windows come from
// the tensor-core DFT have them computed together: one launch per transform
// pass of the persistent GEMM per chunk, every (lens, wavelength) pair a
// problem of its work queue.  The other lenses are built one by one.
void build_lens_set(ld_ctx* c, const ld_params* ps, size_t n, cudaStream_t s, int* rebuilt_count) {
    for (size_t i = n; i < c->set_banks.size(); ++i) {
        BankEntry& e = c->set_banks[i];
        for (DevBuf* b : {&e.canvas, &e.ring_round, &e.ring_ceil, &e.ring_peak, &e.ring_mean, &e.scalars, &e.wl})
            free_buf(c, *b);
    }
    c->set_banks.resize(n);
    struct Lens {
        size_t i;
        PsfBankArgs a;
        std::vector<WavelengthInfo> infos;
        size_t bytes;
    };
    std::vector<Lens> dft;
    std::vector<size_t> other;
    for (size_t i = 0; i < n; ++i) {
        const ld_params& p = ps[i];
        const std::vector<float> wl = wavelengths_of(p);
        BankEntry& e = c->set_banks[i];
        if (e.valid && e.key == bank_key(p, wl)) continue;
        e.valid = false;
        const int np = pupil_size(p), R = max_kernel_radius(p), S = raw_psf_size(np, R);
        if (static_cast<int>(wl.size()) > kMaxBins) throw Fail{LD_ERR_ARG, "too-many-wavelengths"};
        if (!(p.fft_form == LD_FFT_OWN_CHOSEN || (p.fft_form == LD_FFT_OWN_FP32 && !smooth(S)))) {
            other.push_back(i);
            continue;
        }
        // every calibration runs before the first chunk uses the DFT scratch
        const float r0 = first_zero(c, np, S, s);
        Lens l;
        l.i = i;
        l.a = PsfBankArgs{};
        int ws = 0;
        fill_wavelength_infos(p, wl, r0, S, R, &l.infos, &ws);
        pupil_geometry(l.a, p, false);
        l.a.B = static_cast<int>(wl.size());
        l.a.S = S;
        l.a.half = S / 2;
        l.a.off = std::max(0, (S - np) / 2);
        l.a.win_stride = ws;
        std::vector<DftLambda> lam;
        const DftPlan d = plan_dft(l.a, l.infos, &lam);
        l.bytes = static_cast<size_t>(np) * np * sizeof(float4) +
                  static_cast<size_t>(l.a.B) * ws * ws * sizeof(float) + dft_lens_bytes(d, l.a.B) +
                  dft_basis_bytes(d);
        dft.push_back(std::move(l));
    }
    const size_t budget = c->budget ? std::min(kSetChunkBytes, c->budget / 4) : kSetChunkBytes;
    for (size_t k = 0; k < dft.size();) {
        size_t m = k, used = 0;
        while (m < dft.size() && (m == k || used + dft[m].bytes <= budget)) used += dft[m++].bytes;
        if (c->set_pupil.size() < m - k) {
            c->set_pupil.resize(m - k);
            c->set_win.resize(m - k);
        }
        std::vector<const PsfBankArgs*> bp;
        std::vector<const std::vector<WavelengthInfo>*> ip;
        for (size_t j = k; j < m; ++j) {
            Lens& l = dft[j];
            BankEntry& e = c->set_banks[l.i];
            setup_pupil(c, l.a, ps[l.i], false, s, &c->set_pupil[j - k]);
            l.a.wl = static_cast<WavelengthInfo*>(ensure(c, e.wl, l.infos.size() * sizeof(WavelengthInfo)));
            l.a.win = static_cast<float*>(ensure(c, c->set_win[j - k], static_cast<size_t>(l.a.B) * l.a.win_stride *
                                                                           l.a.win_stride * sizeof(float)));
            upload_async(c, const_cast<WavelengthInfo*>(l.a.wl), l.infos.data(),
                         l.infos.size() * sizeof(WavelengthInfo), s, "set-upload");
            bp.push_back(&l.a);
            ip.push_back(&l.infos);
        }
        dft_gemm_psf_batch(c, bp, ip, s);
        for (size_t j = k; j < m; ++j) {
            const Lens& l = dft[j];
            BankEntry& e = c->set_banks[l.i];
            const PreWindows pre{l.a.win, const_cast<WavelengthInfo*>(l.a.wl)};
            bool rb = false;
            ensure_bank(c, ps[l.i], s, &rb, &pre, &e);
            e.args.win = nullptr;  // chunk scratch, reused by the next chunk
            ++*rebuilt_count;
        }
        k = m;
    }
    for (size_t i : other) {
        BankEntry& e = c->set_banks[i];
        bool rb = false;
        ensure_bank(c, ps[i], s, &rb, nullptr, &e);
        e.args.win = nullptr;  // the context's shared scratch
        e.args.rows = nullptr;
        ++*rebuilt_count;
    }
}

// Spectrum of the scatter kernel on grid g (one kernel, FP32 layout), built
// on the first frame with this (radius, grid).  The kernel is the reference's
// normalised Gaussian of radius ceil(max(.5, r)) and sigma max(.5, r / 2),
// evaluated in float (buildGaussianKernel, CpuReference.cpp:1680-1700).
const float2* scatter_spectrum(ld_ctx* c, float radius, const GridGeom& g, cudaStream_t s) {
    std::string key = append_bytes(std::string(), &radius, sizeof(radius));
    key = append_bytes(key, &g, sizeof(g));
    if (c->scatter_ks.p && c->scatter_key == key) return static_cast<const float2*>(c->scatter_ks.p);
    c->scatter_key.clear();
    const int R = std::max(1, static_cast<int>(std::ceil(std::max(0.5f, radius))));
    const int K = 2 * R + 1;
    const float sigma = std::max(0.5f, radius * 0.5f);
    std::vector<float> v(static_cast<size_t>(K) * K);
    float sum = 0.0f;
    for (int y = -R; y <= R; ++y) {
        for (int x = -R; x <= R; ++x) {
            const float e = std::exp(-(static_cast<float>(x * x + y * y) / (2.0f * sigma * sigma)));
            v[static_cast<size_t>(y + R) * K + (x + R)] = e;
            sum += e;
        }
    }
    if (sum > 0.0f)
        for (float& e : v) e /= sum;
    float* canvas = static_cast<float*>(ensure(c, c->scatter_canvas, v.size() * sizeof(float)));
    // pageable source: staged by the driver before the call returns
    check_cuda(cudaMemcpyAsync(canvas, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice, s),
               "scatter-kernel-upload");
    KernelSpectraArgs ka{};
    ka.g = g;
    ka.n_ker = 1;
    ka.R = R;
    ka.K = K;
    ka.Kp = K + (K & 1);
    ka.canvas = canvas;
    ka.rows = static_cast<float2*>(ensure(c, c->scatter_rows, static_cast<size_t>(g.cols) * ka.Kp * sizeof(float2)));
    const size_t part_bytes = ks_part_bytes(1, g, false);
    char* ks = static_cast<char*>(ensure(c, c->scatter_ks, part_bytes + static_cast<size_t>(g.cols) * sizeof(float)));
    ka.spectra = reinterpret_cast<float2*>(ks);
    ka.kscale = reinterpret_cast<float*>(ks + part_bytes);
    ka.h16 = 0;
    ka.scale = static_cast<float>(1.0 / (static_cast<double>(g.M) * static_cast<double>(g.Py)));
    ka.err = c->err;
    staged(c, LD_STAGE_KSPEC_ROWS, s, [&] { launch_kspec_rows(ka, s); });
    staged(c, LD_STAGE_KSPEC_COLS, s, [&] { launch_kspec_cols(ka, s); });
    check_launch("scatter-spectrum");
    c->scatter_key = key;
    return reinterpret_cast<const float2*>(ks);
}

void fill_sizes(ld_status* st, const ld_params& p) {
    if (!st) return;
    st->pupil_size = pupil_size(p);
    st->max_kernel_radius = max_kernel_radius(p);
    st->raw_psf_size = raw_psf_size(st->pupil_size, st->max_kernel_radius);
    st->wavelength_count = static_cast<int>(wavelengths_of(p).size());
}

SelectionParams selection_params(const ld_params& p) {  // CpuReference.cpp:1221-1223, :2096
    SelectionParams s{};
    const float soft = static_cast<float>(std::max(0.01, p.softness_stops));
    const float thr = static_cast<float>(p.threshold);
    s.luma = p.extraction_mode == LD_EXTRACT_LUMA;
    s.thr_stops = thr;
    s.edge0 = thr - soft * 0.5f;
    s.edge1 = thr + soft * 0.5f;
    s.thr_linear = 0.18f * std::pow(2.0f, thr);
    s.point_emphasis = static_cast<float>(p.point_emphasis);
    s.rscale = 1.0f - static_cast<float>(std::min(std::max(p.core_preserve, 0.0), 1.0));
    s.sig_zero = static_cast<float>(0.18 * std::exp2(static_cast<double>(s.edge0)) * 0.999);
    return s;
}

int run_guarded(ld_ctx* ctx, ld_status* st, const std::function<void()>& fn);

// The combination and frame grid of the kernel spectra that ld_render uses
// for a width x height source frame (the same resolution as the render's).
struct SpectraGeometry {
    Combination cb;
    GridGeom g;
    std::string key;
    size_t bytes;
};
SpectraGeometry spectra_geometry(ld_ctx* c, const ld_params& p, int W, int H) {
    validate_params(p);
    if (W <= 0 || H <= 0) throw Fail{LD_ERR_ARG, "invalid-frame-size"};
    if (has_field_phase(p)) throw Fail{LD_ERR_UNSUPPORTED, "unsupported-spectra-transfer-with-field-zones"};
    if (p.fft_form == LD_FFT_CUFFT) throw Fail{LD_ERR_UNSUPPORTED, "unsupported-spectra-transfer-with-cufft-form"};
    const std::vector<float> wl = wavelengths_of(p);
    SpectraGeometry sg{make_combination(p, wl), GridGeom{}, std::string(), 0};
    int Ww = W, Hw = H;
    working_size(post_effects(p), W, H, &Ww, &Hw);
    const int c_rows = std::max(std::max(sg.cb.n_drv == 1 ? 4 : 3, sg.cb.n_out), sg.cb.n_ker);
    const int c_cols = std::max(std::max(sg.cb.n_out, sg.cb.n_ker), sg.cb.n_drv);
    int rw = 0, rh = 0;
    sg.g = make_geometry(c, Ww, Hw, 2 * max_kernel_radius(p) + 1, c_rows, c_cols, &rw, &rh);
    sg.key = spectra_key_for(bank_key(p, wl), sg.cb, sg.g);
    const bool h16 = chosen_h16(p);
    sg.bytes = sg.cb.parts * (ks_part_bytes(sg.cb.n_ker, sg.g, h16) + static_cast<size_t>(sg.g.cols) * sizeof(float));
    return sg;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int ld_abi_version(void) { return LD_ABI_VERSION; }

int ld_create(ld_ctx** out, int device, size_t hbm_budget_bytes) {
    if (!out) return LD_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return LD_ERR_CUDA;
    }
    ld_ctx* c = new ld_ctx();
    c->device = device;
    c->budget = hbm_budget_bytes;
    {
        DeviceGuard g(device);
        configure_kernels();
        bool ok = cudaGetLastError() == cudaSuccess;
        if (ok) {
            try {
                c->err = static_cast<int*>(ensure(c, c->err_word, sizeof(int)));
                ok = cudaMemset(c->err, 0, sizeof(int)) == cudaSuccess;
            } catch (const Fail&) {
                ok = false;
            }
        }
        if (!ok) {
            delete c;
            return LD_ERR_CUDA;
        }
    }
    c->configured = true;
    *out = c;
    return LD_OK;
}

int ld_check_device_errors(ld_ctx* c, int32_t* error_word) {
    if (!c) return LD_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    DeviceGuard g(c->device);
    int v = 0;
    if (cudaMemcpy(&v, c->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return LD_ERR_CUDA;
    if (v != 0 && cudaMemset(c->err, 0, sizeof(int)) != cudaSuccess) return LD_ERR_CUDA;
    if (error_word) *error_word = v;
    return v == 0 ? LD_OK : LD_ERR_TIMEOUT;
}

void ld_destroy(ld_ctx* c) {
    if (!c) return;
    DeviceGuard g(c->device);
    for (auto& kv : c->twiddles) free_buf(c, kv.second);
    for (auto& kv : c->stage_twiddles) free_buf(c, kv.second);
    for (auto& kv : c->ring_counts) free_buf(c, kv.second);
    DevBuf* bufs[] = {&c->rows,   &c->win,     &c->combine_out, &c->kspec_rows, &c->frameA,    &c->frameB,
                      &c->calib,  &c->calib_psf, &c->err_word,  &c->pupil_pre,  &c->effect,    &c->cf_grid,
                      &c->cf_planes, &c->cf_sd,  &c->cf_prod,   &c->work,       &c->scatter_canvas,
                      &c->scatter_ks, &c->dft,  &c->basis,    &c->debug,    &c->selftest, &c->custom.img};
    c->cufft.release();
    for (DevBuf* b : bufs) free_buf(c, *b);
    for (cudaEvent_t e : c->event_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : c->stage_ev) cudaEventDestroy(e);
    if (c->fork_ev) cudaEventDestroy(c->fork_ev);
    if (c->join_ev) cudaEventDestroy(c->join_ev);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->bank_done) cudaEventDestroy(c->bank_done);
    if (c->bank_fence) cudaEventDestroy(c->bank_fence);
    if (c->bank_s) cudaStreamDestroy(c->bank_s);
    free_buf(c, c->scatter_rows);
    for (auto* v : {&c->zone_spectra, &c->spectra_lru})
        for (auto& e : *v)
            if (e.free_ev) cudaEventDestroy(e.free_ev);
    if (c->stage_host) cudaFreeHost(c->stage_host);
    for (auto& b : c->big_stage) {
        if (b.pending) cudaEventSynchronize(b.ev);
        if (b.host) cudaFreeHost(b.host);
        if (b.ev) cudaEventDestroy(b.ev);
    }
    DevBuf* bb[] = {&c->bank.canvas, &c->bank.ring_round, &c->bank.ring_ceil, &c->bank.ring_peak, &c->bank.ring_mean,
                    &c->bank.scalars, &c->bank.wl,        &c->spectra.spectra};
    for (DevBuf* b : bb) free_buf(c, *b);
    for (auto& z : c->zone_spectra) free_buf(c, z.spectra);
    for (auto& z : c->spectra_lru) free_buf(c, z.spectra);
    for (auto* v : {&c->zone_pupil, &c->zone_wl, &c->zone_win, &c->set_pupil, &c->set_win})
        for (auto& z : *v) free_buf(c, z);
    for (BankEntry& e : c->set_banks)
        for (DevBuf* b : {&e.canvas, &e.ring_round, &e.ring_ceil, &e.ring_peak, &e.ring_mean, &e.scalars, &e.wl})
            free_buf(c, *b);
    for (auto& g : c->graphs) cudaGraphExecDestroy(g.exec);
    delete c;
}

size_t ld_device_bytes(const ld_ctx* c) { return c ? c->held : 0; }

int ld_set_profiling(ld_ctx* c, int enable) {
    if (!c) return LD_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    c->profiling = enable != 0;
    return LD_OK;
}

int ld_profile_tensor_flops(ld_ctx* c, double* flops) {
    if (!c || !flops) return LD_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    *flops = c->tensor_flops;
    c->tensor_flops = 0.0;
    return LD_OK;
}

int ld_profile_collect(ld_ctx* c, double* ms, int32_t* launches, int32_t count) {
    if (!c || count < 0) return LD_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    DeviceGuard g(c->device);
    for (int i = 0; i < count; ++i) {
        if (ms) ms[i] = 0.0;
        if (launches) launches[i] = 0;
    }
    int rc = LD_OK;
    for (auto& m : c->marks) {
        if (cudaEventSynchronize(m.second.second) != cudaSuccess) {
            rc = LD_ERR_CUDA;
            continue;
        }
        float t = 0.0f;
        cudaEventElapsedTime(&t, m.second.first, m.second.second);
        if (m.first < count) {
            if (ms) ms[m.first] += t;
            if (launches) launches[m.first] += 1;
        }
    }
    c->marks.clear();
    c->events_used = 0;
    return rc;
}

void ld_clear_caches(ld_ctx* c) {
    if (!c) return;
    std::lock_guard<std::mutex> lock(c->mu);
    c->bank.valid = false;
    c->spectra.valid = false;
    for (auto& e : c->set_banks) e.valid = false;
    for (auto& z : c->zone_spectra) z.valid = false;
    for (auto& z : c->spectra_lru) z.valid = false;
    c->basis_key.clear();
    c->pupil_key.clear();
}

int ld_resolve_sizes(const ld_params* p, int32_t* np, int32_t* S, int32_t* R, int32_t* B) {
    if (!p) return LD_ERR_ARG;
    const int n = pupil_size(*p), r = max_kernel_radius(*p);
    if (np) *np = n;
    if (R) *R = r;
    if (S) *S = raw_psf_size(n, r);
    if (B) *B = static_cast<int32_t>(wavelengths_of(*p).size());
    return LD_OK;
}

int ld_gaussian_rgb_matrix(const float* wl, int32_t count, const float* center, float sigma, float* out) {
    if (!wl || !center || !out || count <= 0 || count > LD_MAX_WAVELENGTHS || !(sigma > 0.0f)) return LD_ERR_ARG;
    gaussian_matrix(wl, count, center, sigma, out);
    return LD_OK;
}

namespace {

constexpr size_t kGraphCache = 4;

// ---------------------------------------------------------------------------
// Autotuner of the fixed transform plans (ld_fxplans.h)
// ---------------------------------------------------------------------------
// Times launch(id, shape) for every compiled radix order of length n and
// every launch shape in [0, shapes) on stream s (one untimed launch, then
// kTuneReps between two events) and records the fastest as
// c->fixed_choice[n] = id | shape << 8.  A single candidate is recorded untimed.
void tune_length(ld_ctx* c, int n, const std::vector<int>& shapes, cudaStream_t s,
                 const std::function<void(int, int)>& launch) {
    int ids[8];
    const int k = fx_candidates(n, ids, 8);
    if (k == 0 || c->fixed_choice.count(n)) return;
    if (k == 1 && shapes.size() == 1) {
        c->fixed_choice[n] = ids[0];
        return;
    }
    constexpr int kTuneReps = 3;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    check_cuda(cudaEventCreate(&e0), "tune-event");
    check_cuda(cudaEventCreate(&e1), "tune-event");
    int best = ids[0];
    float best_ms = 0.0f;
    bool first = true;
    for (int i = 0; i < k; ++i) {
        for (const int sh : shapes) {
            launch(ids[i], sh);
            check_cuda(cudaEventRecord(e0, s), "tune-record");
            for (int r = 0; r < kTuneReps; ++r) launch(ids[i], sh);
            check_cuda(cudaEventRecord(e1, s), "tune-record");
            check_cuda(cudaEventSynchronize(e1), "tune-sync");
            float ms = 0.0f;
            check_cuda(cudaEventElapsedTime(&ms, e0, e1), "tune-elapsed");
            ms /= kTuneReps;
            if (first || ms < best_ms) {
                best = ids[i] | (sh << 8);
                best_ms = ms;
                first = false;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check_launch("autotune");
    c->fixed_choice[n] = best;
    c->fixed_ms[n] = best_ms;
}

// Tunes the row length (frame_rows + frame_inverse, which share its plan; eight
// launch shapes: the inverse pass at two CTAs-per-SM caps, the row pass and
// the inverse pass each with and without the L2 prefetch of the rows one
// resident generation later) and the column length (frame_cols, with and
// without its look-ahead prefetch) of a
// composite frame's grid, re-running the frame's own launches: each rewrites
// the results it wrote before.
void autotune_frame(ld_ctx* c, const FrameArgs& fa, cudaStream_t s) {
    if (c->autotune != 1 || fa.effect_mode != kEffectComposite) return;
    if (c->fixed_choice.count(fa.g.M) && c->fixed_choice.count(fa.g.Py)) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        return;
    }
    if (fa.g.fam_m == kE25) {
        // shape bits: inverse at one more CTA per SM; row pass, inverse pass
        // without their look-ahead prefetch
        tune_length(c, fa.g.M, {0, 1, 2, 3, 4, 5, 6, 7}, s, [&](int id, int shape) {
            FrameArgs a = fa;
            a.g.plan_m.fixed = id;
            a.g.plan_m.shape = shape;
            a.g.plan_m.stw = stage_twiddles(c, id);
            launch_frame_rows(a, s);
            launch_frame_inverse(a, s);
        });
    }
    if (fa.g.fam_py == kE25) {
        tune_length(c, fa.g.Py, {0, 2}, s, [&](int id, int shape) {  // shape 2: no look-ahead prefetch
            FrameArgs a = fa;
            a.g.plan_py.fixed = id;
            a.g.plan_py.shape = shape;
            a.g.plan_py.stw = stage_twiddles(c, id);
            launch_frame_cols(a, s);
        });
    }
}

// Issues a frame chain through a cached CUDA graph: on the first call with a
// given key the chain is captured (thread-local capture mode) and
// instantiated, later calls with the same key launch the graph.  The key is
// the bytes of every argument the chain's launches take, so a graph is only
// replayed for identical launches (buffer contents may differ: the kernels
// read them when the graph runs).  Direct launches when profiling (stage
// events), when graphs are off, or when the caller's stream is capturing.
void run_chain(ld_ctx* c, cudaStream_t s, const std::string& key, const std::function<void()>& chain) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (c->profiling || !c->graphs_enabled || cudaStreamIsCapturing(s, &cs) != cudaSuccess ||
        cs != cudaStreamCaptureStatusNone) {
        cudaGetLastError();
        chain();
        return;
    }
    for (auto& g : c->graphs) {
        if (g.exec && g.key == key) {
            g.last_use = ++c->graph_clock;
            c->launches += g.launches;
            check_cuda(cudaGraphLaunch(g.exec, s), "graph-launch");
            return;
        }
    }
    const int before = c->launches;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        chain();
        return;
    }
    try {
        chain();
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        throw;
    }
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const bool ok = cudaStreamEndCapture(s, &graph) == cudaSuccess && graph &&
                    cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    if (!ok) {  // not capturable here: launch directly
        cudaGetLastError();
        c->launches = before;
        chain();
        return;
    }
    ld_ctx::GraphEntry* slot = nullptr;
    if (c->graphs.size() < kGraphCache) {
        c->graphs.emplace_back();
        slot = &c->graphs.back();
    } else {
        slot = &c->graphs.front();
        for (auto& g : c->graphs)
            if (g.last_use < slot->last_use) slot = &g;
        cudaGraphExecDestroy(slot->exec);
    }
    slot->key = key;
    slot->exec = exec;
    slot->launches = c->launches - before;
    slot->last_use = ++c->graph_clock;
    check_cuda(cudaGraphLaunch(exec, s), "graph-launch");
}

}  // namespace

int ld_set_graphs(ld_ctx* c, int enable) {
    if (!c) return LD_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    c->graphs_enabled = enable != 0;
    return LD_OK;
}

int ld_export_kernel_spectra(ld_ctx* ctx, const ld_params* params, int32_t width, int32_t height, void* device_dst,
                             size_t capacity, size_t* bytes_out, void* stream, ld_status* st) {
    if (st) std::memset(st, 0, sizeof(*st));
    if (!ctx || !params || !bytes_out) {
        set_status(st, LD_ERR_ARG, "null-argument");
        return LD_ERR_ARG;
    }
    return run_guarded(ctx, st, [&]() {
        const ld_params& p = *params;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const SpectraGeometry sg = spectra_geometry(ctx, p, width, height);
        *bytes_out = sg.bytes;
        if (device_dst == nullptr) return;  // size query
        if (capacity < sg.bytes) throw Fail{LD_ERR_ARG, "spectra-buffer-too-small"};
        join_bank(ctx, s);
        bool bank_rebuilt = false, spectra_rebuilt = false;
        SpectraEntry& e = cached_spectra(ctx, p, sg.cb, sg.g, s, &bank_rebuilt, &spectra_rebuilt);
        check_cuda(cudaMemcpyAsync(device_dst, e.spectra.p, sg.bytes, cudaMemcpyDeviceToDevice, s), "spectra-export");
        mark_used(e, s);
        fence_bank(ctx, s);
        if (st) {
            st->bank_rebuilt = bank_rebuilt;
            st->spectra_rebuilt = spectra_rebuilt;
            st->grid_used_w = sg.g.Px;
            st->grid_used_h = sg.g.Py;
        }
    });
}

int ld_import_kernel_spectra(ld_ctx* ctx, const ld_params* params, int32_t width, int32_t height,
                             const void* device_src, size_t bytes, void* stream, ld_status* st) {
    if (st) std::memset(st, 0, sizeof(*st));
    if (!ctx || !params || !device_src) {
        set_status(st, LD_ERR_ARG, "null-argument");
        return LD_ERR_ARG;
    }
    return run_guarded(ctx, st, [&]() {
        const ld_params& p = *params;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const SpectraGeometry sg = spectra_geometry(ctx, p, width, height);
        if (bytes != sg.bytes) throw Fail{LD_ERR_ARG, "spectra-size-mismatch"};
        join_bank(ctx, s);
        SpectraEntry* slot = nullptr;
        for (auto& e : ctx->spectra_lru)
            if (e.valid && e.key == sg.key) slot = &e;
        if (slot == nullptr) {
            if (ctx->spectra_lru.size() < kSpectraCache) ctx->spectra_lru.emplace_back();
            slot = &ctx->spectra_lru.front();
            for (auto& e : ctx->spectra_lru) {
                if (!e.valid) {
                    slot = &e;
                    break;
                }
                if (e.last_use < slot->last_use) slot = &e;
            }
        }
        wait_free(*slot, s);
        slot->valid = false;
        ensure(ctx, slot->spectra, sg.bytes);
        check_cuda(cudaMemcpyAsync(slot->spectra.p, device_src, sg.bytes, cudaMemcpyDeviceToDevice, s),
                   "spectra-import");
        slot->g = sg.g;
        slot->n_ker = sg.cb.n_ker;
        slot->key = sg.key;
        slot->valid = true;
        slot->last_use = ++ctx->spectra_clock;
        fence_bank(ctx, s);
        if (st) {
            st->grid_used_w = sg.g.Px;
            st->grid_used_h = sg.g.Py;
        }
    });
}

int ld_set_custom_aperture(ld_ctx* c, const float* values, int32_t width, int32_t height, int32_t normalize,
                           int32_t invert) {
    if (!c) return LD_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    DeviceGuard g(c->device);
    if (values == nullptr) {  // clear
        free_buf(c, c->custom.img);
        c->custom = CustomAperture{};
        return LD_OK;
    }
    if (width <= 0 || height <= 0 || static_cast<int64_t>(width) * height > (int64_t(1) << 26)) return LD_ERR_ARG;
    // LoadLensDiffPreparedApertureImage (LensDiffApertureImage.cpp:367-399):
    // optional min/max normalisation clamped to [0, 1], then optional inversion
    std::vector<float> v(values, values + static_cast<size_t>(width) * height);
    float lo = v.front(), hi = v.front();
    for (float x : v) {
        lo = std::min(lo, x);
        hi = std::max(hi, x);
    }
    if (normalize && hi > lo) {
        const float scale = 1.0f / (hi - lo);
        for (float& x : v) x = std::min(std::max((x - lo) * scale, 0.0f), 1.0f);
    }
    if (invert)
        for (float& x : v) x = 1.0f - x;
    uint64_t h = 1469598103934665603ull;  // FNV-1a of the prepared values
    const unsigned char* b = reinterpret_cast<const unsigned char*>(v.data());
    for (size_t i = 0; i < v.size() * sizeof(float); ++i) h = (h ^ b[i]) * 1099511628211ull;
    try {
        float* d = static_cast<float*>(ensure(c, c->custom.img, v.size() * sizeof(float)));
        check_cuda(cudaMemcpy(d, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice), "custom-aperture-upload");
    } catch (const Fail& f) {
        return f.code;
    }
    c->custom.w = width;
    c->custom.h = height;
    c->custom.digest = h;
    return LD_OK;
}

int ld_inject_alloc_failure(ld_ctx* c, int32_t after) {
    if (!c) return LD_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    c->fail_alloc_after = after < 0 ? -1 : after;
    return LD_OK;
}

int ld_selftest_wait(ld_ctx* c, int32_t mode, int64_t budget_cycles, void* stream, int32_t* error_word) {
    if (!c || !error_word) return LD_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    DeviceGuard g(c->device);
    try {
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        int v = 0;
        check_cuda(cudaMemcpy(&v, c->err, sizeof(int), cudaMemcpyDeviceToHost), "selftest-read");
        if (v != 0) throw Fail{LD_ERR_ARG, "selftest-error-word-not-clear"};
        float4* scratch = static_cast<float4*>(ensure(c, c->selftest, 2 * 64 * sizeof(float4)));
        const int rc = launch_wait_selftest(mode, budget_cycles, scratch, c->err, s);
        if (rc != LD_OK) return rc;
        check_cuda(cudaStreamSynchronize(s), "selftest-sync");
        check_cuda(cudaMemcpy(&v, c->err, sizeof(int), cudaMemcpyDeviceToHost), "selftest-read");
        check_cuda(cudaMemset(c->err, 0, sizeof(int)), "selftest-clear");
        *error_word = v;
        return v == 0 ? LD_OK : LD_ERR_TIMEOUT;
    } catch (const Fail& f) {
        return f.code;
    }
}

int ld_set_autotune(ld_ctx* c, int enable) {
    if (!c) return LD_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    if (enable < -1 || enable > 9) return LD_ERR_ARG;
    c->autotune = enable;
    return LD_OK;
}

int ld_autotune_choice(ld_ctx* c, int32_t n, int32_t* radices_out, int32_t* shape_out, double* ms_out) {
    if (!c || !radices_out) return 0;
    std::lock_guard<std::mutex> lock(c->mu);
    auto it = c->fixed_choice.find(n);
    if (it == c->fixed_choice.end()) return 0;
    const FxPlanDesc* d = fx_plan(it->second & 255);
    if (d == nullptr) return 0;
    for (int i = 0; i < d->count; ++i) radices_out[i] = d->radix[i];
    if (shape_out) *shape_out = it->second >> 8;
    if (ms_out) {
        auto m = c->fixed_ms.find(n);
        *ms_out = m != c->fixed_ms.end() ? m->second : 0.0;
    }
    return d->count;
}

size_t ld_estimate_device_bytes(const ld_params* params, int32_t width, int32_t height) {
    if (!params || width <= 0 || height <= 0) return 0;
    try {
        const ld_params& p = *params;
        const size_t np = pupil_size(p), R = max_kernel_radius(p);
        const size_t S = raw_psf_size(static_cast<int>(np), static_cast<int>(R));
        const size_t K = 2 * R + 1, Kp = K + (K & 1);
        const size_t B = wavelengths_of(p).size();
        const Combination cb = make_combination(p, wavelengths_of(p));
        const int c_rows = std::max(std::max(cb.n_drv == 1 ? 4 : 3, cb.n_out), cb.n_ker);
        const int c_cols = std::max(std::max(cb.n_out, cb.n_ker), cb.n_drv);
        const PostEffects post = post_effects(p);
        working_size(post, width, height, &width, &height);  // the effect's frame
        const int M = choose_length((width + static_cast<int>(K) - 1 + 1) / 2, 1, c_rows);
        const int Py = choose_length(height + static_cast<int>(K) - 1, 2, c_cols);
        if (M < 0 || Py < 0) return 0;
        const size_t cols = static_cast<size_t>(M) + 1, Hp = (static_cast<size_t>(height) + 3) & ~size_t(3);
        const size_t zones = has_field_phase(p) ? static_cast<size_t>(p.field_grid > 0 ? p.field_grid : 3) *
                                                      (p.field_grid > 0 ? p.field_grid : 3)
                                                : 1;
        size_t t = 0;
        t += np * np * 16;                              // pupil pre-pass
        t += B * np * S * 8 + B * S * S * 4;            // row spectra + |F|^2 windows (window <= S)
        t += 2 * S * S * 4;                             // calibration PSF
        t += B * K * K * 4 + B * (R + 1) * 24;          // canvases + ring statistics
        t += static_cast<size_t>(cb.n_ker) * K * K * 4; // combined kernels
        t += static_cast<size_t>(cb.n_ker) * cols * Kp * 8;                 // kernel row spectra
        t += zones * static_cast<size_t>(cb.n_ker) * cols * Py * 8;         // kernel spectra
        size_t frame_ab = static_cast<size_t>(cb.n_drv + cb.n_out) * cols * Hp * 8;  // frame A, B
        if (post.scatter) {
            const size_t Rs = static_cast<size_t>(std::ceil(std::max(0.5f, post.scatter_radius)));
            const size_t Ks = 2 * Rs + 1;
            const int Ms = choose_length((width + static_cast<int>(Ks) - 1 + 1) / 2, 1, 3);
            const int Pys = choose_length(height + static_cast<int>(Ks) - 1, 2, 3);
            if (Ms < 0 || Pys < 0) return 0;
            const size_t cs = static_cast<size_t>(Ms) + 1;
            frame_ab = std::max(frame_ab, 6 * cs * Hp * 8);
            t += Ks * Ks * 4 + cs * (Ks + 1) * 8 + cs * Pys * 8;  // scatter canvas, rows, spectrum
        }
        t += frame_ab;
        if (zones > 1 || p.energy_mode == LD_ENERGY_PRESERVE || p.look_mode == LD_LOOK_SPLIT || post.any())
            t += static_cast<size_t>(width) * height * 16;            // stored effect
        if (post.resample) t += static_cast<size_t>(width) * height * 16;  // working source
        if (p.fft_form == LD_FFT_OWN_CHOSEN || (p.fft_form == LD_FFT_OWN_FP32 && !smooth(static_cast<int>(S)))) {
            // tensor-core DFT images, windows bounded by S
            const size_t mt = (np + 127) / 128, kc = (np + 31) / 32, nt = (S + 3 + 127) / 128 + 1;
            t += 2 * (B * (mt * 128 * 128 * kc + nt * 128 * 128 * mt * 4) + 2 * (2 * nt * 128) * 128 * kc);
        }
        if (p.fft_form == LD_FFT_CUFFT) {
            const size_t P = static_cast<size_t>(2 * M) * Py, half = static_cast<size_t>(Py) * (M + 1);
            t += cf_psf_chunk(static_cast<int>(S), static_cast<int>(B)) * S * S * 8;
            t += std::max(cb.n_drv, cb.n_out) * P * 4 + (cb.n_drv + cb.n_out) * half * 8;
        }
        return t + (size_t(16) << 20);  // twiddles, plans, scalars
    } catch (...) {
        return 0;
    }
}

namespace {
// The lens's static debug views (BuildLensDiffStaticDebugRgba,
// LensDiffCpuReference.cpp:1909-1970) into the render window of `o` (its
// source bounds give the frame the square is centred in).  The field-edge
// views take the last field zone, (1, 1), when field phase is on
// (cache.fieldZones.back()), else the lens itself.
void render_static_view(ld_ctx* c, const ld_params& p, const FrameArgs& o, cudaStream_t s, bool* bank_rebuilt) {
    const int dv = p.debug_view;
    const bool zones = has_field_phase(p);
    const bool edge = (dv == LD_DEBUG_PHASE_EDGE || dv == LD_DEBUG_FIELD_PSF) && zones;
    const ld_params q = edge ? zone_params(p, 1.0f, 1.0f) : p;
    if (dv == LD_DEBUG_PUPIL || dv == LD_DEBUG_PHASE || dv == LD_DEBUG_PHASE_EDGE) {
        const int n = pupil_size(q);
        const size_t nn = static_cast<size_t>(n) * n;
        char* buf = static_cast<char*>(ensure(c, c->debug, 256 + 2 * align256(nn * sizeof(float))));
        unsigned int* mx = reinterpret_cast<unsigned int*>(buf);
        float* amp = reinterpret_cast<float*>(buf + 256);
        float* phase = reinterpret_cast<float*>(buf + 256 + align256(nn * sizeof(float)));
        check_cuda(cudaMemsetAsync(mx, 0, 256, s), "debug-memset");
        launch_pupil_image(pupil_params(q, false), phase_for_wavelength(q, 550.0f), amp, phase, mx, mx + 1, s);
        if (dv == LD_DEBUG_PUPIL) launch_square_view(o, amp, nullptr, n, mx, false, 7, true, s);
        else launch_phase_view(o, amp, phase, n, mx + 1, s);
        check_launch("debug-view");
        return;
    }
    BankEntry& b = ensure_bank(c, q, s, bank_rebuilt);
    const size_t kk = static_cast<size_t>(b.K) * b.K;
    char* buf = static_cast<char*>(
        ensure(c, c->debug, 256 + 3 * align256(kk * sizeof(float)) + align256(kk * sizeof(double2))));
    unsigned int* mx = reinterpret_cast<unsigned int*>(buf);
    float* img[3];
    for (int i = 0; i < 3; ++i) img[i] = reinterpret_cast<float*>(buf + 256 + i * align256(kk * sizeof(float)));
    double2* tmp = reinterpret_cast<double2*>(buf + 256 + 3 * align256(kk * sizeof(float)));
    check_cuda(cudaMemsetAsync(mx, 0, 256, s), "debug-memset");
    const PsfScalars* sc = b.args.scalars;
    if (dv == LD_DEBUG_CHROMATIC_SPLIT) {  // red: last bin, green: middle, blue: first
        const int bins[3] = {b.B - 1, b.B / 2, 0};
        for (int ch = 0; ch < 3; ++ch) {
            launch_kernel_image(b.args, bins[ch], img[ch], mx + ch, s);
            launch_square_view(o, img[ch], sc + bins[ch], 0, mx + ch, true, 1 << ch, ch == 0, s);
        }
    } else {  // Psf, FieldPsf: bin 0; Otf: its transfer function
        launch_kernel_image(b.args, 0, img[0], mx, s);
        if (dv == LD_DEBUG_OTF) {
            launch_otf_image(img[0], sc, b.K, tmp, img[1], mx + 1, s);
            launch_square_view(o, img[1], sc, 0, mx + 1, true, 7, true, s);
        } else {
            launch_square_view(o, img[0], sc, 0, mx, true, 7, true, s);
        }
    }
    check_launch("debug-view");
}
}  // namespace

int ld_render(ld_ctx* ctx, const ld_render_request* rq, const ld_params* params, ld_status* st) {
    if (st) std::memset(st, 0, sizeof(*st));
    if (!ctx || !rq || !params) {
        set_status(st, LD_ERR_ARG, "null-argument");
        return LD_ERR_ARG;
    }
    // LensDiffCuda.cu:4646-4657
    if (!rq->host_enabled_cuda_render || rq->cuda_stream == nullptr) {
        set_status(st, LD_ERR_ARG, "cuda-render-not-enabled-by-host");
        return LD_ERR_ARG;
    }
    if (rq->src.data == nullptr || rq->dst.data == nullptr) {
        set_status(st, LD_ERR_ARG, "missing-source-or-destination-cuda-buffer");
        return LD_ERR_ARG;
    }
    return run_guarded(ctx, st, [&]() {
        const ld_params& p = *params;
        cudaStream_t s = static_cast<cudaStream_t>(rq->cuda_stream);
        const int W = rq->src.bounds.x2 - rq->src.bounds.x1;
        const int H = rq->src.bounds.y2 - rq->src.bounds.y1;
        if (W <= 0 || H <= 0) throw Fail{LD_ERR_ARG, "invalid-source-bounds"};
        if (rq->src.components != 4 || rq->src.bytes_per_component != 4 || rq->dst.components != 4 ||
            rq->dst.bytes_per_component != 4)
            throw Fail{LD_ERR_ARG, "unsupported-pixel-format"};
        validate_params(p);
        fill_sizes(st, p);
        ctx->launches = 0;
        bool bank_rebuilt = false, spectra_rebuilt = false;
        if (!frame_debug_view(p.debug_view)) {
            FrameArgs o;
            std::memset(&o, 0, sizeof(o));
            o.W = W;
            o.H = H;
            o.dst = static_cast<unsigned char*>(rq->dst.data);
            o.dst_pitch = rq->dst.row_bytes;
            o.src_x1 = rq->src.bounds.x1;
            o.src_y1 = rq->src.bounds.y1;
            o.dst_x1 = rq->dst.bounds.x1;
            o.dst_y1 = rq->dst.bounds.y1;
            o.out_x1 = std::max(rq->render_window.x1, rq->dst.bounds.x1);
            o.out_y1 = std::max(rq->render_window.y1, rq->dst.bounds.y1);
            o.out_x2 = std::max(o.out_x1, std::min(rq->render_window.x2, rq->dst.bounds.x2));
            o.out_y2 = std::max(o.out_y1, std::min(rq->render_window.y2, rq->dst.bounds.y2));
            const cudaStream_t vs = static_cast<cudaStream_t>(rq->cuda_stream);
            join_bank(ctx, vs);
            render_static_view(ctx, p, o, vs, &bank_rebuilt);
            fence_bank(ctx, vs);
            if (st) {
                st->bank_rebuilt = bank_rebuilt;
                st->kernel_launches = ctx->launches;
            }
            return;
        }
        const bool zones = has_field_phase(p);
        const int zn = p.field_grid > 0 ? p.field_grid : 3;
        const std::vector<float> wl = wavelengths_of(p);
        const Combination cb = make_combination(p, wl);
        const PostEffects post = post_effects(p);
        // the effect is computed on the working frame (the source frame unless
        // resolution-aware rendering resamples it, CpuReference.cpp:2089-2094)
        int Ww = W, Hw = H;
        working_size(post, W, H, &Ww, &Hw);
        if (Ww > kMaxWorkingSide || Hw > kMaxWorkingSide) throw Fail{LD_ERR_ARG, "invalid-working-frame-size"};
        int rw = 0, rh = 0;
        const int c_rows = std::max(std::max(cb.n_drv == 1 ? 4 : 3, cb.n_out), cb.n_ker);
        const int c_cols = std::max(std::max(cb.n_out, cb.n_ker), cb.n_drv);
        const int Kmax = 2 * max_kernel_radius(p) + 1;
        // Field zones: each zone's tent weight is non-zero only over its
        // neighbours' centres, so its convolution is needed only there.  With
        // overlap-add tiles every zone convolves just that window plus the
        // kernel's reach on a grid of its own size (one grid shared by every
        // zone) instead of the whole frame, when that grid is at most half
        // the frame's.
        const ZoneTiles zt = zones && p.fft_form != LD_FFT_CUFFT ? zone_tiles(Ww, Hw, zn) : ZoneTiles{};
        const bool tiled = zt.n > 0 && static_cast<double>(zt.wo + Kmax - 1) * (zt.ho + Kmax - 1) <=
                                           0.5 * static_cast<double>(Ww + Kmax - 1) * (Hw + Kmax - 1);
        const GridGeom g = tiled ? make_geometry(ctx, zt.wo, zt.ho, Kmax, c_rows, c_cols, &rw, &rh)
                                 : make_geometry(ctx, Ww, Hw, Kmax, c_rows, c_cols, &rw, &rh);
        // Spectra already cached (a warm frame)?  If not, the bank and kernel
        // spectra are built on s while the source's row transforms run on a
        // side stream: they do not depend on the lens.  (Tiles transform
        // their rows per zone, inside the chain.)
        const bool overlap_rows = p.fft_form != LD_FFT_CUFFT && p.debug_view != LD_DEBUG_SELECTION && !tiled &&
                                  !spectra_cached(ctx, p, zones, zn, cb, g);

        FrameArgs fa;
        std::memset(&fa, 0, sizeof(fa));  // padding too: the bytes key the frame graphs
        fa.g = g;
        fa.sel = selection_params(p);
        fa.W = W;
        fa.H = H;
        fa.src = static_cast<const unsigned char*>(rq->src.data);
        fa.src_pitch = rq->src.row_bytes;
        fa.dst = static_cast<unsigned char*>(rq->dst.data);
        fa.dst_pitch = rq->dst.row_bytes;
        fa.src_x1 = rq->src.bounds.x1;
        fa.src_y1 = rq->src.bounds.y1;
        fa.dst_x1 = rq->dst.bounds.x1;
        fa.dst_y1 = rq->dst.bounds.y1;
        // intersectRect(renderWindow, dst.bounds), CpuReference.cpp:116-125, :2235
        fa.out_x1 = std::max(rq->render_window.x1, rq->dst.bounds.x1);
        fa.out_y1 = std::max(rq->render_window.y1, rq->dst.bounds.y1);
        fa.out_x2 = std::max(fa.out_x1, std::min(rq->render_window.x2, rq->dst.bounds.x2));
        fa.out_y2 = std::max(fa.out_y1, std::min(rq->render_window.y2, rq->dst.bounds.y2));
        fa.n_drv = cb.n_drv;
        fa.n_out = cb.n_out;
        fa.n_ker = cb.n_ker;
        fa.mono = cb.mono;
        fa.saturation = cb.saturation;
        fa.luma_lock = cb.luma_lock;
        // effect gain and core compensation per energy mode (CpuReference.cpp:2104-2109)
        fa.preserve = p.energy_mode == LD_ENERGY_PRESERVE ? 1 : 0;
        if (fa.preserve) {
            fa.effect_gain = static_cast<float>(std::min(std::max(p.effect_gain, 0.0), 1.0));
            fa.core_comp = fa.effect_gain;
        } else {
            fa.effect_gain = static_cast<float>(std::max(0.0, p.effect_gain));
            fa.core_comp = static_cast<float>(std::max(0.0, p.core_compensation));
        }
        const float protect = std::max(0.2f, static_cast<float>(std::min(std::max(p.core_preserve, 0.0), 1.0)));
        fa.max_sub = fa.sel.rscale > 1e-6f ? (1.0f - protect) / fa.sel.rscale : 0.0f;
        fa.h16 = chosen_h16(p) ? 1 : 0;
        fa.err = ctx->err;
        const bool split = cb.parts == 2;
        const int dv = p.debug_view;
        const bool dv_parts = dv == LD_DEBUG_CORE || dv == LD_DEBUG_STRUCTURE;
        fa.effect_mode = (zones || split) ? kEffectAccumulate
                                          : ((fa.preserve || post.any() || dv != LD_DEBUG_FINAL) ? kEffectStore
                                                                                                  : kEffectComposite);
        fa.acc_gain = 1.0f;
        fa.acc_shoulder = 0.0f;
        fa.Ww = Ww;
        fa.Hw = Hw;
        fa.fringe_px = post.fringe;
        fa.transfer = p.input_transfer;
        // the chain's view of the working frame: the resampled source, or
        // the source itself
        FrameArgs fw = fa;
        if (post.resample) {
            fa.work = static_cast<float4*>(
                ensure(ctx, ctx->work, static_cast<size_t>(Ww) * Hw * sizeof(float4)));
            fw.src = reinterpret_cast<const unsigned char*>(fa.work);
            fw.src_pitch = static_cast<int64_t>(Ww) * sizeof(float4);
            fw.src_x1 = 0;
            fw.src_y1 = 0;
            fw.W = Ww;
            fw.H = Hw;
            fw.transfer = LD_TRANSFER_LINEAR;  // the working source is decoded already
        }
        // scatter: a Mono chain over the stored effect with one Gaussian kernel
        // on its own grid (CpuReference.cpp:2180-2186)
        FrameArgs fs;
        std::memset(&fs, 0, sizeof(fs));
        GridGeom gs{};
        if (post.scatter) {
            const int Ks = 2 * std::max(1, static_cast<int>(std::ceil(std::max(0.5f, post.scatter_radius)))) + 1;
            int srw = 0, srh = 0;
            gs = make_geometry(ctx, Ww, Hw, Ks, 3, 3, &srw, &srh);
        }
        // rows of the row spectra: the frame's, or a tile's input rows
        const int Hp = tiled ? ((zt.ho + Kmax - 1 + 3) & ~3) : ((Hw + 3) & ~3);
        // (the chosen form's half2 row spectra take half; their row exponents follow)
        const size_t a_bytes = align256(std::max(static_cast<size_t>(cb.n_drv) * g.cols,
                                                 post.scatter ? static_cast<size_t>(3) * gs.cols : size_t(0)) *
                                        Hp * sizeof(float2));
        // (the exponents go to shared memory in 16-byte units)
        float2* abuf = static_cast<float2*>(ensure(ctx, ctx->frameA, a_bytes + ((static_cast<size_t>(Hp) + 15) & ~size_t(15))));
        signed char* aexp = reinterpret_cast<signed char*>(abuf) + a_bytes;
        // column outputs in groups of four columns (ld_frame.cu b_index)
        auto b_bytes_of = [&](int n_out, const GridGeom& gg, bool h16) {
            const size_t bcols = (static_cast<size_t>(gg.cols) + 3) / 4 * 4;
            return align256(static_cast<size_t>(n_out) * bcols * Hp * (h16 ? 4 : 8));
        };
        const size_t b_main = b_bytes_of(cb.n_out, g, fa.h16) + static_cast<size_t>(g.cols) * sizeof(float);
        const size_t b_scatter = post.scatter ? b_bytes_of(3, gs, false) + static_cast<size_t>(gs.cols) * sizeof(float) : 0;
        char* bbuf = static_cast<char*>(ensure(ctx, ctx->frameB, std::max(b_main, b_scatter)));
        const float2* sks = post.scatter ? scatter_spectrum(ctx, post.scatter_radius, gs, s) : nullptr;
        float4* effect = nullptr;
        double* sums = nullptr;
        if (fa.effect_mode != kEffectComposite) {
            effect = static_cast<float4*>(
                ensure(ctx, ctx->effect, static_cast<size_t>(Ww) * Hw * sizeof(float4) + 4 * sizeof(double)));
            sums = reinterpret_cast<double*>(effect + static_cast<size_t>(Ww) * Hw);
        }
        for (FrameArgs* f : {&fa, &fw}) {
            f->Hp = Hp;
            f->acc_x0 = 0;
            f->acc_x1 = f->W;
            f->A = abuf;
            f->aexp = aexp;
            f->Bout = reinterpret_cast<float2*>(bbuf);
            f->bscale = reinterpret_cast<float*>(bbuf + b_bytes_of(cb.n_out, g, fa.h16));
            f->effect = effect;
            f->sums = sums;
            f->work = fa.work;
        }
        if (overlap_rows) {  // fork: working source and row transforms on the side stream
            cudaStream_t ws = side_stream(ctx);
            check_cuda(cudaEventRecord(ctx->fork_ev, s), "fork");
            check_cuda(cudaStreamWaitEvent(ws, ctx->fork_ev, 0), "fork");
            if (post.resample) staged(ctx, LD_STAGE_WORKING_SOURCE, ws, [&] { launch_resample_source(fa, ws); });
            staged(ctx, LD_STAGE_FRAME_ROWS, ws, [&] { launch_frame_rows(fw, ws); });
            check_cuda(cudaEventRecord(ctx->join_ev, ws), "fork");
        }
        // Bank and kernel spectra on the bank stream, so a cold frame's bank
        // overlaps the earlier frames' chains still running on s; s joins it
        // before this frame's chain.  Not while s is being captured (the bank
        // stream's work would sit outside the capture).
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        check_cuda(cudaStreamIsCapturing(s, &cap), "capture-status");
        const bool use_bs = cap == cudaStreamCaptureStatusNone && p.fft_form != LD_FFT_CUFFT;
        cudaStream_t bs = use_bs ? bank_stream(ctx) : s;
        if (!use_bs) join_bank(ctx, s);
        if (use_bs && ctx->fence_pending) {
            check_cuda(cudaStreamWaitEvent(bs, ctx->bank_fence, 0), "bank-fence");
            ctx->fence_pending = false;
        }
        std::vector<const SpectraEntry*> spectra;
        if (zones) {
            spectra = ensure_zone_spectra(ctx, p, zn, cb, g, bs, &bank_rebuilt, &spectra_rebuilt);
        } else {
            spectra.push_back(&cached_spectra(ctx, p, cb, g, bs, &bank_rebuilt, &spectra_rebuilt));
        }
        if (use_bs && (bank_rebuilt || spectra_rebuilt)) join_bank(ctx, s);
        if (!use_bs) fence_bank(ctx, s);
        const SpectraEntry& sp = *spectra.front();
        for (FrameArgs* f : {&fa, &fw}) {
            f->spectra = ks_part(sp.spectra.p, 0, cb.n_ker, g, fa.h16);
            f->kscale = ks_scale(sp.spectra.p, 0, cb.parts, cb.n_ker, g, fa.h16);
        }
        if (overlap_rows) check_cuda(cudaStreamWaitEvent(s, ctx->join_ev, 0), "join");
        if (post.scatter) {
            fs = fw;
            fs.g = gs;
            fs.n_drv = 3;
            fs.n_out = 3;
            fs.n_ker = 1;
            fs.mono = 1;
            fs.h16 = 0;
            fs.spectra = sks;
            fs.kscale = nullptr;
            fs.bscale = reinterpret_cast<float*>(bbuf + b_bytes_of(3, gs, false));
            fs.effect_mode = kEffectScatter;
            fs.drv_effect = 1;
            fs.scatter = post.scatter_amount;
            fs.scatter_replace = dv == LD_DEBUG_SCATTER ? 1 : 0;  // the view shows the convolution alone
        }
        // the scatter pass runs for the final frame and the views of the final effect
        const bool run_scatter = post.scatter && (dv == LD_DEBUG_FINAL || dv == LD_DEBUG_EFFECT ||
                                                  dv == LD_DEBUG_CREATIVE_FRINGE || dv == LD_DEBUG_SCATTER);
        if (!run_scatter) std::memset(&fs, 0, sizeof(fs));
        // the composite: source frame, stored effect (or a debug view of it)
        FrameArgs fin = fa;
        switch (dv) {
            case LD_DEBUG_SELECTION:
                fin.debug = kOutSelection;
                fin.mask_max = reinterpret_cast<unsigned int*>(sums + 2);
                break;
            case LD_DEBUG_EFFECT:
                fin.debug = kOutEffect;
                break;
            case LD_DEBUG_CORE:
            case LD_DEBUG_STRUCTURE:  // unscaled, unfringed (coreEffect, structureEffect)
                fin.debug = kOutEffect;
                fin.preserve = 0;
                fin.fringe_px = 0.0f;
                break;
            case LD_DEBUG_SCATTER:  // scatterPreview: zero when scatter is off
                fin.debug = run_scatter ? kOutEffect : kOutFringePreview;
                fin.fringe_px = 0.0f;
                break;
            case LD_DEBUG_CREATIVE_FRINGE:  // creativeFringePreview: zero when the fringe is off
                fin.debug = kOutFringePreview;
                break;
            default:
                break;
        }
        auto clear_effect = [&]() {
            if (fa.effect_mode == kEffectComposite) return;
            check_cuda(cudaMemsetAsync(fa.sums, 0, 2 * sizeof(double), s), "effect-memset");
            if (fa.effect_mode == kEffectAccumulate)
                check_cuda(cudaMemsetAsync(fa.effect, 0, static_cast<size_t>(Ww) * Hw * sizeof(float4), s),
                           "effect-memset");
        };
        if (p.fft_form == LD_FFT_CUFFT) {
            const size_t P = static_cast<size_t>(g.Px) * g.Py;
            const size_t half = static_cast<size_t>(g.Py) * (g.Px / 2 + 1);
            const int nc = std::max(cb.n_drv, cb.n_out);
            float* planes = static_cast<float*>(ensure(ctx, ctx->cf_planes, nc * P * sizeof(float)));
            float2* sd = static_cast<float2*>(ensure(ctx, ctx->cf_sd, cb.n_drv * half * sizeof(float2)));
            float2* prod = static_cast<float2*>(ensure(ctx, ctx->cf_prod, cb.n_out * half * sizeof(float2)));
            clear_effect();
            staged(ctx, LD_STAGE_FRAME_ROWS, s, [&] { cf_frame_forward(fa, planes, sd, ctx->cufft, s); });
            staged(ctx, LD_STAGE_FRAME_COLS, s, [&] { cf_frame_multiply(fa, sd, prod, s); });
            staged(ctx, LD_STAGE_FRAME_INVERSE, s, [&] { cf_frame_inverse(fa, prod, planes, ctx->cufft, s); });
            if (fa.effect_mode != kEffectComposite)
                staged(ctx, LD_STAGE_COMPOSITE, s, [&] { launch_composite(fa, s); });
            check_launch("frame-chain");
            for (const SpectraEntry* e : spectra) mark_used(const_cast<SpectraEntry&>(*e), s);
            if (st) {
                st->bank_rebuilt = bank_rebuilt;
                st->spectra_rebuilt = spectra_rebuilt;
                st->grid_requested_w = rw;
                st->grid_requested_h = rh;
                st->grid_used_w = g.Px;
                st->grid_used_h = g.Py;
                st->kernel_launches = ctx->launches;
            }
            return;
        }
        // graph key: the launch arguments (the zone loop derives the rest)
        std::string gkey(reinterpret_cast<const char*>(&fa), sizeof(fa));
        for (const SpectraEntry* e : spectra) gkey = append_bytes(gkey, &e->spectra.p, sizeof(void*));
        gkey = append_bytes(gkey, &zn, sizeof(zn));
        // Split look: core then structure, each with its gain and shoulder
        // (LensDiffCpuReference.cpp:2123-2146); Physical: the full kernels
        // Core / Structure views: that set alone, shouldered in the Split look,
        // without its gain (:2123-2157)
        const bool look_split = p.look_mode == LD_LOOK_SPLIT;
        const float gains[2] = {look_split && !dv_parts ? static_cast<float>(std::max(0.0, p.core_gain)) : 1.0f,
                                look_split && !dv_parts ? static_cast<float>(std::max(0.0, p.structure_gain)) : 1.0f};
        const float shoulders[2] = {look_split ? static_cast<float>(p.core_shoulder) : 0.0f,
                                    look_split ? static_cast<float>(p.structure_shoulder) : 0.0f};
        const int part_lo = dv == LD_DEBUG_STRUCTURE ? 1 : 0;
        const int part_hi = dv == LD_DEBUG_CORE ? 1 : cb.parts;
        gkey = append_bytes(gkey, gains, sizeof(gains));
        gkey = append_bytes(gkey, shoulders, sizeof(shoulders));
        gkey = append_bytes(gkey, &cb.parts, sizeof(cb.parts));
        gkey = append_bytes(gkey, &fw, sizeof(fw));
        gkey = append_bytes(gkey, &fs, sizeof(fs));
        gkey = append_bytes(gkey, &fin, sizeof(fin));
        gkey = append_bytes(gkey, &part_lo, sizeof(part_lo));
        gkey = append_bytes(gkey, &part_hi, sizeof(part_hi));
        gkey = append_bytes(gkey, &overlap_rows, sizeof(overlap_rows));
        auto chain = [&, fa = fw]() mutable {  // the loops below edit this copy
            if (dv == LD_DEBUG_SELECTION) {  // the mask alone: no convolution
                check_cuda(cudaMemsetAsync(fin.mask_max, 0, sizeof(unsigned int), s), "mask-memset");
                if (post.resample) staged(ctx, LD_STAGE_WORKING_SOURCE, s, [&] { launch_resample_source(fin, s); });
                staged(ctx, LD_STAGE_COMPOSITE, s, [&] { launch_composite(fin, s); });
                return;
            }
            clear_effect();
            if (!overlap_rows) {  // else already on the side stream
                if (post.resample) staged(ctx, LD_STAGE_WORKING_SOURCE, s, [&] { launch_resample_source(fin, s); });
                if (!tiled) staged(ctx, LD_STAGE_FRAME_ROWS, s, [&] { launch_frame_rows(fa, s); });
            }
            if (fa.effect_mode != kEffectAccumulate) {
                staged(ctx, LD_STAGE_FRAME_COLS, s, [&] { launch_frame_cols(fa, s); });
                staged(ctx, LD_STAGE_FRAME_INVERSE, s, [&] { launch_frame_inverse(fa, s); });
            } else {
                const int nz = zones ? zn * zn : 1;
                fa.zone_n = zones ? zn : 0;
                for (int z = 0; z < nz; ++z) {
                    const void* base = spectra[static_cast<size_t>(z)]->spectra.p;
                    int r0 = 0, r1 = Hw;
                    if (zones) {
                        fa.zone_x = z % zn;
                        fa.zone_y = z / zn;
                        // working rows whose tent weight can be non-zero (the kernel
                        // evaluates the weight itself; one row of margin each side)
                        zone_span(Hw, zn, fa.zone_y, &r0, &r1);
                    }
                    fa.row0 = r0;
                    if (tiled) {  // this zone's tile: its own row transforms, its columns only
                        int c0 = 0, c1 = Ww;
                        zone_span(Ww, zn, fa.zone_x, &c0, &c1);
                        fa.tile_x0 = c0 - Kmax / 2;
                        fa.tile_y0 = r0 - Kmax / 2;
                        fa.acc_x0 = c0;
                        fa.acc_x1 = c1;
                        staged(ctx, LD_STAGE_FRAME_ROWS, s, [&] { launch_frame_rows(fa, s); });
                    }
                    for (int part = part_lo; part < part_hi; ++part) {
                        fa.spectra = ks_part(base, part, cb.n_ker, g, fa.h16);
                        fa.kscale = ks_scale(base, part, cb.parts, cb.n_ker, g, fa.h16);
                        fa.acc_gain = gains[part];
                        fa.acc_shoulder = shoulders[part];
                        staged(ctx, LD_STAGE_FRAME_COLS, s, [&] { launch_frame_cols(fa, s); });
                        staged(ctx, LD_STAGE_FRAME_INVERSE, s, [&] { launch_frame_inverse_rows(fa, r1 - r0, s); });
                    }
                }
                if (fa.preserve) staged(ctx, LD_STAGE_COMPOSITE, s, [&] { launch_effect_sums(fa, s); });
            }
            if (run_scatter) {
                staged(ctx, LD_STAGE_SCATTER, s, [&] { launch_frame_rows(fs, s); });
                staged(ctx, LD_STAGE_SCATTER, s, [&] { launch_frame_cols(fs, s); });
                staged(ctx, LD_STAGE_SCATTER, s, [&] { launch_frame_inverse(fs, s); });
            }
            if (fa.effect_mode != kEffectComposite) staged(ctx, LD_STAGE_COMPOSITE, s, [&] { launch_composite(fin, s); });
        };
        run_chain(ctx, s, gkey, chain);
        // the first composite frame at this grid picks the transforms' radix orders
        if (!run_scatter && !zones && fa.effect_mode == kEffectComposite && dv == LD_DEBUG_FINAL)
            autotune_frame(ctx, fw, s);
        for (const SpectraEntry* e : spectra) mark_used(const_cast<SpectraEntry&>(*e), s);
        check_launch("frame-chain");
        if (st) {
            st->bank_rebuilt = bank_rebuilt;
            st->spectra_rebuilt = spectra_rebuilt;
            st->grid_requested_w = rw;
            st->grid_requested_h = rh;
            st->grid_used_w = g.Px;
            st->grid_used_h = g.Py;
            st->kernel_launches = ctx->launches;
        }
    });
}

int ld_build_psf_bank(ld_ctx* ctx, const ld_params* params, void* stream, ld_status* st) {
    if (st) std::memset(st, 0, sizeof(*st));
    if (!ctx || !params) {
        set_status(st, LD_ERR_ARG, "null-argument");
        return LD_ERR_ARG;
    }
    return run_guarded(ctx, st, [&]() {
        validate_params(*params);
        fill_sizes(st, *params);
        bool rebuilt = false;
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        ctx->launches = 0;
        join_bank(ctx, s);
        ensure_bank(ctx, *params, s, &rebuilt);
        fence_bank(ctx, s);
        if (st) {
            st->bank_rebuilt = rebuilt;
            st->kernel_launches = ctx->launches;
        }
    });
}

int ld_build_psf_banks(ld_ctx* ctx, const ld_params* params, int32_t count, void* stream, ld_status* st) {
    if (st) std::memset(st, 0, sizeof(*st));
    if (!ctx || !params) {
        set_status(st, LD_ERR_ARG, "null-argument");
        return LD_ERR_ARG;
    }
    if (count <= 0) {
        set_status(st, LD_ERR_ARG, "invalid-lens-count");
        return LD_ERR_ARG;
    }
    return run_guarded(ctx, st, [&]() {
        for (int32_t i = 0; i < count; ++i) validate_params(params[i]);
        fill_sizes(st, params[0]);
        int rebuilt = 0;
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        ctx->launches = 0;
        join_bank(ctx, s);
        build_lens_set(ctx, params, static_cast<size_t>(count), s, &rebuilt);
        fence_bank(ctx, s);
        if (st) {
            st->bank_rebuilt = rebuilt;
            st->kernel_launches = ctx->launches;
        }
    });
}

int ld_export_psf_bank(ld_ctx* ctx, const ld_params* params, void* stream, float* wl_out, int32_t* sizes,
                       int64_t* offsets, float* kernels_out, int64_t capacity, ld_status* st) {
    if (st) std::memset(st, 0, sizeof(*st));
    if (!ctx || !params || !sizes || !offsets || !kernels_out) {
        set_status(st, LD_ERR_ARG, "null-argument");
        return LD_ERR_ARG;
    }
    return run_guarded(ctx, st, [&]() {
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        validate_params(*params);
        fill_sizes(st, *params);
        bool rebuilt = false;
        join_bank(ctx, s);
        BankEntry& b = ensure_bank(ctx, *params, s, &rebuilt);
        fence_bank(ctx, s);
        std::vector<PsfScalars> sc(static_cast<size_t>(b.B));
        check_cuda(cudaMemcpyAsync(sc.data(), b.args.scalars, sc.size() * sizeof(PsfScalars), cudaMemcpyDeviceToHost, s),
                   "export-readback");
        check_cuda(cudaStreamSynchronize(s), "export-sync");
        int64_t total = 0;
        int support = 4;
        for (int i = 0; i < b.B; ++i) {
            const int side = 2 * sc[static_cast<size_t>(i)].radius + 1;
            sizes[i] = side;
            offsets[i] = total;
            total += static_cast<int64_t>(side) * side;
            support = std::max(support, sc[static_cast<size_t>(i)].radius);
            if (wl_out) wl_out[i] = b.wavelengths[static_cast<size_t>(i)];
        }
        if (total > capacity) throw Fail{LD_ERR_ARG, "export-capacity-too-small"};
        DevBuf off;
        DevBuf out;
        ensure(ctx, off, static_cast<size_t>(b.B) * sizeof(int64_t));
        ensure(ctx, out, static_cast<size_t>(total) * sizeof(float));
        check_cuda(cudaMemcpyAsync(off.p, offsets, static_cast<size_t>(b.B) * sizeof(int64_t), cudaMemcpyHostToDevice, s),
                   "export-upload");
        launch_export(b.args, static_cast<const int64_t*>(off.p), static_cast<float*>(out.p), s);
        check_launch("export");
        check_cuda(cudaMemcpyAsync(kernels_out, out.p, static_cast<size_t>(total) * sizeof(float), cudaMemcpyDeviceToHost, s),
                   "export-download");
        check_cuda(cudaStreamSynchronize(s), "export-sync");
        free_buf(ctx, off);
        free_buf(ctx, out);
        if (st) {
            st->bank_rebuilt = rebuilt;
            st->support_radius = support;
        }
    });
}

int ld_raw_psf(ld_ctx* ctx, const ld_params* params, int wavelength_index, float* psf_out, void* stream,
               ld_status* st) {
    if (st) std::memset(st, 0, sizeof(*st));
    if (!ctx || !params || !psf_out) {
        set_status(st, LD_ERR_ARG, "null-argument");
        return LD_ERR_ARG;
    }
    return run_guarded(ctx, st, [&]() {
        const ld_params& p = *params;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (p.aperture_mode == LD_APERTURE_CUSTOM && (t_custom == nullptr || t_custom->img.p == nullptr))
            throw Fail{LD_ERR_ARG, "custom-aperture-image-not-set"};
        if (p.aperture_mode < LD_APERTURE_CIRCLE || p.aperture_mode > LD_APERTURE_SNOWFLAKE)
            throw Fail{LD_ERR_ARG, "invalid-aperture-mode"};
        fill_sizes(st, p);
        const std::vector<float> wl = wavelengths_of(p);
        if (wavelength_index < 0 || wavelength_index >= static_cast<int>(wl.size()))
            throw Fail{LD_ERR_ARG, "invalid-wavelength-index"};
        const int np = pupil_size(p), R = max_kernel_radius(p), S = raw_psf_size(np, R);
        PsfBankArgs a{};
        join_bank(ctx, s);  // the pupil, calibration and transform buffers are the bank's
        setup_pupil(ctx, a, p, false, s);
        a.B = 1;
        a.S = S;
        a.half = S / 2;
        a.off = std::max(0, (S - np) / 2);
        a.win_stride = S;
        WavelengthInfo wi{};
        wi.phase = phase_for_wavelength(p, wl[static_cast<size_t>(wavelength_index)]);
        wi.win_x0 = 0;
        wi.win_n = S;
        char* cal = static_cast<char*>(ensure(ctx, ctx->calib, 2 * align256(sizeof(WavelengthInfo) + sizeof(PsfScalars))));
        WavelengthInfo* dwl = reinterpret_cast<WavelengthInfo*>(cal);
        PsfScalars* dsc = reinterpret_cast<PsfScalars*>(cal + align256(sizeof(WavelengthInfo)));
        a.wl = dwl;
        a.scalars = dsc;
        a.want_energy = 1;
        a.win = psf_out;
        check_cuda(cudaMemcpyAsync(dwl, &wi, sizeof(wi), cudaMemcpyHostToDevice, s), "rawpsf-upload");
        check_cuda(cudaMemsetAsync(dsc, 0, sizeof(PsfScalars), s), "rawpsf-memset");
        if (smooth(S)) {
            a.plan_s = make_plan(ctx, S, fft_family(S, 1) == kE25);
            a.rows = static_cast<float2*>(ensure(ctx, ctx->rows, static_cast<size_t>(a.row_n) * S * sizeof(float2)));
            launch_psf_rows(a, s);
            launch_psf_cols(a, s);
        } else {  // the reference's Bluestein sizes: the whole S x S window by DFT-as-GEMM
            dft_gemm_psf(ctx, a, std::vector<WavelengthInfo>{wi}, s);
        }
        launch_normalize_psf(psf_out, S * S, dsc, s);
        check_launch("raw-psf");
        fence_bank(ctx, s);
        // the upload above reads `wi` from the stack: finish before returning
        check_cuda(cudaStreamSynchronize(s), "rawpsf-sync");
    });
}

}  // extern "C"

namespace {
int run_guarded(ld_ctx* ctx, ld_status* st, const std::function<void()>& fn) {
    std::lock_guard<std::mutex> lock(ctx->mu);
    DeviceGuard g(ctx->device);
    CustomScope custom(&ctx->custom);
    try {
        fn();
    } catch (const Fail& f) {
        set_status(st, f.code, f.stage);
        return f.code;
    } catch (const CufftError& e) {
        set_status(st, LD_ERR_CUDA, std::string(e.what) + "-" + std::to_string(e.code));
        return LD_ERR_CUDA;
    } catch (const std::exception& e) {
        set_status(st, LD_ERR_CUDA, e.what());
        return LD_ERR_CUDA;
    }
    set_status(st, LD_OK, "ok");
    return LD_OK;
}
}  // namespace

// ---------------------------------------------------------------------------
// Parameter resolution shared with ld_noalloc.cu (same expressions as above).
// ---------------------------------------------------------------------------
namespace ld {
bool host_factor_plan(int n, bool allow25, FftPlan* plan) { return factor_plan(n, allow25, plan); }
PupilParams host_pupil_params(const ld_params& p) { return pupil_params(p, false); }
void host_pupil_geometry(PsfBankArgs& a, const ld_params& p) { pupil_geometry(a, p, false); }
PhaseCoeffs host_phase_for_wavelength(const ld_params& p, float wavelength) {
    return phase_for_wavelength(p, wavelength);
}
std::vector<float> host_wavelengths(const ld_params& p) { return wavelengths_of(p); }
void host_sizes(const ld_params& p, int* np, int* S, int* R) {
    *np = pupil_size(p);
    *R = max_kernel_radius(p);
    *S = raw_psf_size(*np, *R);
}
}  // namespace ld
