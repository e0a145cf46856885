// ld_frame_fx.cu — the frame chain's FFT kernels instantiated on the fixed
// plans of ld_fxplans.h (compile-time length and radix order, ld_fftx.cuh),
// their launchers, and the FP64 generation of the plans' stage twiddle tables.
//
// Each fx_launch_* returns false when no fixed instantiation covers the
// launch (another length, channel count or form); the caller then launches
// the runtime-planned kernel.  The fixed kernels run with exactly the thread
// count their transform was compiled for.
#include <cmath>
#include <vector>

#include "ld_frame_kernels.cuh"
#include "ld_fxplans.h"

namespace ld {
namespace {

// Fixed plan ID: its transform type, the passes it serves (kRowPlan: the
// frame's row transforms, length M; kColPlan: its column transforms, length
// Py) and the elements per thread E its kernels are compiled for (ld_fxplans.h).
constexpr int kRowPlan = 1, kColPlan = 2;
template <int ID>
struct FxType;
template <class F, int ROLE, int FAM>
struct FxTypeOf {
    using type = F;
    static constexpr int role = ROLE;
    static constexpr int E = FAM;
};
template <> struct FxType<1> : FxTypeOf<FixedFft<2500, 25, 25, 4>, kRowPlan, kE25> {};
template <> struct FxType<2> : FxTypeOf<FixedFft<2500, 25, 4, 25>, kRowPlan, kE25> {};
template <> struct FxType<3> : FxTypeOf<FixedFft<3200, 25, 16, 8>, kColPlan, kE25> {};
template <> struct FxType<4> : FxTypeOf<FixedFft<3200, 25, 8, 16>, kColPlan, kE25> {};
template <> struct FxType<5> : FxTypeOf<FixedFft<1250, 25, 25, 2>, kRowPlan, kE25> {};
template <> struct FxType<6> : FxTypeOf<FixedFft<1250, 25, 2, 25>, kRowPlan, kE25> {};
template <> struct FxType<7> : FxTypeOf<FixedFft<1600, 25, 16, 4>, kColPlan, kE25> {};
template <> struct FxType<8> : FxTypeOf<FixedFft<1600, 25, 4, 16>, kColPlan, kE25> {};
template <> struct FxType<9> : FxTypeOf<FixedFft<1280, 5, 16, 16>, kRowPlan, kE25> {};
template <> struct FxType<10> : FxTypeOf<FixedFft<1280, 16, 5, 16>, kRowPlan, kE25> {};
template <> struct FxType<11> : FxTypeOf<FixedFft<3200, 5, 5, 16, 8>, kColPlan, kE16> {};
template <> struct FxType<12> : FxTypeOf<FixedFft<1600, 5, 5, 16, 4>, kColPlan, kE16> {};

// Calls f(FxType<id>{}); false when there is no fixed plan `id`.
template <class F>
bool fx_visit(int id, F&& f) {
    switch (id) {
        case 1: f(FxType<1>{}); return true;
        case 2: f(FxType<2>{}); return true;
        case 3: f(FxType<3>{}); return true;
        case 4: f(FxType<4>{}); return true;
        case 5: f(FxType<5>{}); return true;
        case 6: f(FxType<6>{}); return true;
        case 7: f(FxType<7>{}); return true;
        case 8: f(FxType<8>{}); return true;
        case 9: f(FxType<9>{}); return true;
        case 10: f(FxType<10>{}); return true;
        case 11: f(FxType<11>{}); return true;
        case 12: f(FxType<12>{}); return true;
        default: return false;
    }
}

// Thread counts and CTAs per SM of the fixed kernels (register caps follow
// from __launch_bounds__(T, MINB)).
constexpr int rows_c(int n) { return fft_threads(n, 2, kE25) <= 224 ? 2 : 4; }
constexpr int minb_for(int t) { return t <= 128 ? 4 : (t <= 224 ? 3 : 2); }
// column passes: as many CTAs per SM as the column's working set (four
// sequences of n complex values) fits in shared memory, at most four
constexpr int cols_minb(int n) {
    return kMaxSmem / (32 * n + 1024) >= 4 ? 4 : (kMaxSmem / (32 * n + 1024) >= 3 ? 3 : 2);
}

template <class FFT>
void rows_fixed(const FrameArgs& a, cudaStream_t s) {
    constexpr int N = FFT::n;
    constexpr int C = rows_c(N);
    constexpr int T = fft_threads(N, C, kE25);
    const size_t sm = rows_smem(N, C);
    FrameArgs b = a;
    auto f = frame_rows_kernel<kE25, C, 1, T, minb_for(T), false, FFT>;
    b.ahead = resident_ctas(f, T, sm);
    f<<<a.Hp / C, T, sm, s>>>(b);
}

template <class D, bool H16>
void cols_fixed(FrameArgs a, cudaStream_t s) {
    using FFT = typename D::type;
    constexpr int N = FFT::n;
    constexpr int T = fft_threads(N, 3, D::E);
    const size_t sm = frame_cols_smem(N, 3);
    auto f = frame_cols_kernel<D::E, 3, T, cols_minb(N), H16, FFT>;
    a.ahead = resident_ctas(f, T, sm);
    f<<<a.g.cols, T, sm, s>>>(a);
}

template <class FFT, bool H16, int MINB>
void inverse_fixed_m(const FrameArgs& a, int rows, cudaStream_t s) {
    constexpr int N = FFT::n;
    constexpr int T = fft_threads(N, 3, kE25);
    const size_t sm = static_cast<size_t>(N) * 3 * sizeof(float2);
    FrameArgs b = a;
    auto f = frame_inverse_kernel<kE25, 3, T, MINB, H16, FFT>;
    b.ahead = resident_ctas(f, T, sm);
    f<<<rows, T, sm, s>>>(b);
}

// shape bit 0 clear: minb_for(T) CTAs per SM; set: one more (tighter
// register cap).  (Bit 1 is the row pass's prefetch, frame_rows_kernel.)
template <class FFT, bool H16>
void inverse_fixed(const FrameArgs& a, int rows, cudaStream_t s) {
    constexpr int T = fft_threads(FFT::n, 3, kE25);
    if (a.g.plan_m.shape & 1) inverse_fixed_m<FFT, H16, minb_for(T) + 1>(a, rows, s);
    else inverse_fixed_m<FFT, H16, minb_for(T)>(a, rows, s);
}

template <class D, bool H16>
void kspec_cols_fixed(KernelSpectraArgs a, cudaStream_t s) {
    using FFT = typename D::type;
    constexpr int N = FFT::n;
    constexpr int T = fft_threads(N, 3, D::E);
    const size_t sm = kspec_cols_smem(N, a.Kp, 3);
    auto f = kspec_cols_kernel<D::E, 3, T, cols_minb(N), H16, FFT>;
    a.ahead = resident_ctas(f, T, sm);
    f<<<a.g.cols, T, sm, s>>>(a);
}

template <class FFT>
void kspec_rows_fixed(const KernelSpectraArgs& a, cudaStream_t s) {
    constexpr int T = fft_threads(FFT::n, 3, kE25);
    const size_t sm = static_cast<size_t>(FFT::n) * 3 * sizeof(float2);
    kspec_rows_kernel<kE25, 3, T, minb_for(T) + 1, FFT><<<a.Kp, T, sm, s>>>(a);
}

template <class D>
void configure_fixed() {
    using FFT = typename D::type;
    constexpr int N = FFT::n;
    if constexpr (D::role == kRowPlan) {
        constexpr int C = rows_c(N);
        constexpr int TR = fft_threads(N, C, kE25);
        constexpr int T3 = fft_threads(N, 3, kE25);
        set_smem(frame_rows_kernel<kE25, C, 1, TR, minb_for(TR), false, FFT>);
        set_smem(frame_inverse_kernel<kE25, 3, T3, minb_for(T3), false, FFT>);
        set_smem(frame_inverse_kernel<kE25, 3, T3, minb_for(T3), true, FFT>);
        set_smem(frame_inverse_kernel<kE25, 3, T3, minb_for(T3) + 1, false, FFT>);
        set_smem(frame_inverse_kernel<kE25, 3, T3, minb_for(T3) + 1, true, FFT>);
        set_smem(kspec_rows_kernel<kE25, 3, T3, minb_for(T3) + 1, FFT>);
    } else {
        constexpr int T3 = fft_threads(N, 3, D::E);
        set_smem(frame_cols_kernel<D::E, 3, T3, cols_minb(N), false, FFT>);
        set_smem(frame_cols_kernel<D::E, 3, T3, cols_minb(N), true, FFT>);
        set_smem(kspec_cols_kernel<D::E, 3, T3, cols_minb(N), false, FFT>);
        set_smem(kspec_cols_kernel<D::E, 3, T3, cols_minb(N), true, FFT>);
    }
}

}  // namespace

bool fx_launch_frame_rows(const FrameArgs& a, cudaStream_t s) {
    if (a.n_drv != 1 || a.drv_effect || a.g.fam_m != kE25) return false;
    bool done = false;
    fx_visit(a.g.plan_m.fixed, [&](auto d) {
        using D = decltype(d);
        if constexpr (D::role == kRowPlan) {
            rows_fixed<typename D::type>(a, s);
            done = true;
        }
    });
    return done;
}

bool fx_launch_frame_cols(const FrameArgs& a, cudaStream_t s) {
    if (a.n_drv != 1 || a.n_out != 3 || a.g.fam_py != kE25) return false;
    bool done = false;
    fx_visit(a.g.plan_py.fixed, [&](auto d) {
        using D = decltype(d);
        if constexpr (D::role == kColPlan) {
            if (a.h16) cols_fixed<D, true>(a, s);
            else cols_fixed<D, false>(a, s);
            done = true;
        }
    });
    return done;
}

bool fx_launch_frame_inverse(const FrameArgs& a, int rows, cudaStream_t s) {
    if (a.n_out != 3 || a.g.fam_m != kE25) return false;
    bool done = false;
    fx_visit(a.g.plan_m.fixed, [&](auto d) {
        using D = decltype(d);
        if constexpr (D::role == kRowPlan) {
            if (a.h16) inverse_fixed<typename D::type, true>(a, rows, s);
            else inverse_fixed<typename D::type, false>(a, rows, s);
            done = true;
        }
    });
    return done;
}

bool fx_launch_kspec_rows(const KernelSpectraArgs& a, cudaStream_t s) {
    if (a.n_ker != 3 || a.g.fam_m != kE25) return false;
    bool done = false;
    fx_visit(a.g.plan_m.fixed, [&](auto d) {
        using D = decltype(d);
        if constexpr (D::role == kRowPlan) {
            kspec_rows_fixed<typename D::type>(a, s);
            done = true;
        }
    });
    return done;
}

bool fx_launch_kspec_cols(const KernelSpectraArgs& a, cudaStream_t s) {
    if (a.n_ker != 3 || a.g.fam_py != kE25) return false;
    bool done = false;
    fx_visit(a.g.plan_py.fixed, [&](auto d) {
        using D = decltype(d);
        if constexpr (D::role == kColPlan) {
            if (a.h16) kspec_cols_fixed<D, true>(a, s);
            else kspec_cols_fixed<D, false>(a, s);
            done = true;
        }
    });
    return done;
}

void fx_configure() {
    for (int id = 1; id <= kFxPlanCount; ++id) fx_visit(id, [](auto d) { configure_fixed<decltype(d)>(); });
}

// Stage twiddle tables of fixed plan `id`: for every stage after the first,
// NS x RP entries w^(k r), w = exp(-2 pi i / (NS R)), k < NS, r < R (zero for
// r >= R), RP = R rounded up to even, as RP / 2 rows of NS pairs
// (w^(k 2q), w^(k (2q+1))): pair q of butterfly span k at q * NS + k, so
// the threads of a warp (consecutive k) read consecutive 16-byte pairs;
// evaluated in FP64.
std::vector<float2> fx_stage_table(int id) {
    std::vector<float2> out;
    const FxPlanDesc* d = fx_plan(id);
    if (d == nullptr) return out;
    int ns = 1;
    for (int st = 0; st < d->count; ++st) {
        const int R = d->radix[st];
        const int RP = (R + 1) & ~1;
        if (ns > 1) {
            for (int q = 0; q < RP / 2; ++q) {
                for (int k = 0; k < ns; ++k) {
                    for (int r = 2 * q; r < 2 * q + 2; ++r) {
                        if (r >= R) {
                            out.push_back(make_float2(0.0f, 0.0f));
                            continue;
                        }
                        const long long e = static_cast<long long>(k) * r;
                        const double ang = -2.0 * M_PI * static_cast<double>(e) / static_cast<double>(ns * R);
                        out.push_back(make_float2(static_cast<float>(std::cos(ang)), static_cast<float>(std::sin(ang))));
                    }
                }
            }
        }
        ns *= R;
    }
    return out;
}

}  // namespace ld
