// ld_fxplans.h — the transform lengths and radix orders compiled as fixed
// plans (ld_fftx.cuh), shared by the host (planning, twiddle tables, the
// autotuner's candidate lists) and the fixed-plan launchers (ld_frame_fx.cu).
//
// The lengths are those of the frame grids the cost model picks for the
// benchmarked frame sizes: 3840x2160 with kernels up to 1025 px (grid
// 5000 x 3200: rows of M = 2500 bins, columns of 3200) and 1920x1080 or
// 2048x1080 with kernels up to 513 px (rows of 1250 / 1280, columns of 1600).
// Each length has several radix orders; the autotuner times them on first
// use and keeps the fastest (the first is the default).  Odd radices lead:
// their strided first-stage stores spread over the shared-memory banks.
// `fam` is the elements per thread the plan's kernels are compiled for:
// 25 (every stage holds up to 25 complex values per thread) or 16 (more
// threads per transform, 16 values each, so fewer registers per thread and
// more warps per SM, at the cost of no radix-25 stage: one more pass).
#pragma once

namespace ld {

struct FxPlanDesc {
    int id;         // 1-based; 0 means "no fixed plan"
    int n;          // transform length
    int count;      // stages
    int radix[4];   // radix of each stage, first stage first
    int fam;        // elements per thread (25 or 16)
};

constexpr int kFxPlanCount = 12;
constexpr FxPlanDesc kFxPlans[kFxPlanCount] = {
    {1, 2500, 3, {25, 25, 4, 0}, 25},
    {2, 2500, 3, {25, 4, 25, 0}, 25},
    {3, 3200, 3, {25, 16, 8, 0}, 25},
    {4, 3200, 3, {25, 8, 16, 0}, 25},
    {5, 1250, 3, {25, 25, 2, 0}, 25},
    {6, 1250, 3, {25, 2, 25, 0}, 25},
    {7, 1600, 3, {25, 16, 4, 0}, 25},
    {8, 1600, 3, {25, 4, 16, 0}, 25},
    {9, 1280, 3, {5, 16, 16, 0}, 25},
    {10, 1280, 3, {16, 5, 16, 0}, 25},
    {11, 3200, 4, {5, 5, 16, 8}, 16},
    {12, 1600, 4, {5, 5, 16, 4}, 16},
};

inline const FxPlanDesc* fx_plan(int id) {
    return id >= 1 && id <= kFxPlanCount ? &kFxPlans[id - 1] : nullptr;
}

// Fixed plans of length n, in preference order; returns how many (<= max).
inline int fx_candidates(int n, int* ids, int max) {
    int k = 0;
    for (int i = 0; i < kFxPlanCount && k < max; ++i)
        if (kFxPlans[i].n == n) ids[k++] = kFxPlans[i].id;
    return k;
}

}  // namespace ld
