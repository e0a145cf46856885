// ld_dftgemm.cu — the chosen form's pupil-to-PSF transform as DFT-as-GEMM on
// the 5th-generation tensor cores: tcgen05.mma with BF16 operands in a 3-way
// split and FP32 accumulators in tensor memory (TMEM).
//
// The raw PSF of wavelength b is |DFT_S(pupil field embedded at offset
// `off`)|^2, fftshifted, of which the λ-rescale reads one window
// (buildShiftedRawPsf, LensDiffCpuReference.cpp:831-859).  Only the pupil's
// non-zero rows m and columns x, and only the window's frequencies, enter:
//
//   row pass     Y_b[m][n] = sum_x F_b[m][x] D[x][n]
//   column pass  Z_b[n][r] = sum_m Y_b[m][n] D'[m][r]
//   window       win_b[r][n] = |Z_b[n][r]|^2
//
// D[x][n]  = exp(-2 pi i ((col_lo + x + off) * u_n mod S) / S),
// D'[m][r] = exp(-2 pi i ((row_lo + m + off) * u_r mod S) / S),
// u_n = (x0 + n + S/2) mod S, the unshifted frequency of shifted column x0 + n.
//
// Complex products run as real GEMMs over an interleaved K: an operand row
// holds (re, im) pairs, and output column 2n (2n+1) of the real GEMM is the
// real (imaginary) part of complex output n when the basis row 2n holds
// (d_r, -d_i) and row 2n+1 holds (d_i, d_r) for each K pair.
//
// BF16 3-way split: every FP32 operand value v is stored as hi = bf16(v) and
// lo = bf16(v - hi), and each product accumulates hi*hi + hi*lo + lo*hi in
// FP32 (the lo*lo term is below the FP32 accumulation error), about 16
// significant bits per product.
//
// Operands are written by their producers directly in the layout the tensor
// core reads from shared memory ("images"): K-major, 128-byte swizzle, 64
// BF16 per row and K-chunk (32 complex values).  For each K-chunk an operand
// keeps all its rows contiguous (row r at (r / 8) * 1024 + (r % 8) * 128,
// 16-byte units XOR-ed with r % 8), so any 8-aligned run of rows is one
// contiguous block that a single bulk copy (cp.async.bulk) brings into shared
// memory.  No tensor map is needed.
#include <algorithm>

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "ld_async.cuh"
#include "ld_internal.h"

namespace ld {
namespace {

constexpr int kTileM = 128;                   // UMMA M (TMEM lanes)
constexpr int kTileN = 256;                   // UMMA N: 128 complex outputs
constexpr int kChunkK = 64;                   // BF16 per row and K-chunk (128 bytes)
constexpr uint32_t kImgA = kTileM * 128;      // 16 KB
constexpr uint32_t kImgB = kTileN * 128;      // 32 KB
constexpr uint32_t kStageBytes = 2 * kImgA + 2 * kImgB;
constexpr int kStages = 2;
constexpr uint32_t kTmemCols = 256;

// Byte offset of BF16 element k (0..63) of row `row` inside one K-chunk.
__host__ __device__ __forceinline__ uint32_t img_byte(int row, int k) {
    return static_cast<uint32_t>((row >> 3) * 1024 + (row & 7) * 128 + ((((k >> 3) ^ row) & 7) << 4) + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t bf16_pair(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);  // .x = a (low half)
    return *reinterpret_cast<const uint32_t*>(&v);
}

// hi and lo BF16 pairs of (a, b).
__device__ __forceinline__ void split_pair(float a, float b, uint32_t* hi, uint32_t* lo) {
    const __nv_bfloat16 ah = __float2bfloat16_rn(a), bh = __float2bfloat16_rn(b);
    *hi = bf16_pair(__bfloat162float(ah), __bfloat162float(bh));
    *lo = bf16_pair(a - __bfloat162float(ah), b - __bfloat162float(bh));
}

// ---- tcgen05 (tensor core, tensor memory) ---------------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {  // one full warp
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(cols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {  // one full warp
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, both K-major; one thread issues.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}

// Arrives once on `bar` when every tcgen05.mma this thread issued has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(bar))
                 : "memory");
}

// 32 consecutive 32-bit TMEM columns of this warp's 32 lanes.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Shared-memory matrix descriptor of a K-major, 128-byte-swizzled operand
// tile at `addr` (1024-byte aligned): 8-row core groups 1024 bytes apart.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu)  // start address
           | (static_cast<uint64_t>(1) << 16)            // leading byte offset (unused when swizzled)
           | (static_cast<uint64_t>(1024 >> 4) << 32)    // stride byte offset
           | (static_cast<uint64_t>(1) << 46)            // descriptor version (tcgen05)
           | (static_cast<uint64_t>(2) << 61);           // 128-byte swizzle
}

// Instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128, N = 256.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(kTileN >> 3) << 17) |
                            (static_cast<uint32_t>(kTileM >> 4) << 24);

// ---- operand producers --------------------------------------------------------------
// DFT basis images: row j (2n: real, 2n+1: imaginary output column n) over
// K-chunk c; element pair q is spatial index x = 32 c + q, angle
// 2 pi ((x + koff) * u_n mod S) / S with u_n = (x0 + n + S/2) mod S, the
// exponential evaluated in FP64.  Pairs with x >= k_valid are zero.
__global__ void __launch_bounds__(256) dft_basis_kernel(DftBasisArgs a) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t per_chunk = static_cast<int64_t>(a.rows) * 32;
    if (i >= per_chunk * a.kc) return;
    const int c = static_cast<int>(i / per_chunk);
    const int rem = static_cast<int>(i - static_cast<int64_t>(c) * per_chunk);
    const int j = rem >> 5, q = rem & 31;
    const int x = c * 32 + q;
    float pr = 0.0f, pi = 0.0f;
    if (x < a.k_valid) {
        const int n = j >> 1;
        const int64_t u = (static_cast<int64_t>(a.x0) + n + a.half) % a.S;
        const int64_t t = ((static_cast<int64_t>(x) + a.koff) * u) % a.S;
        double sd, cd;
        sincospi(2.0 * static_cast<double>(t) / static_cast<double>(a.S), &sd, &cd);
        const float cs = static_cast<float>(cd), sn = static_cast<float>(sd);
        // d = cos - i sin: real row (d_r, -d_i) = (cos, sin); imaginary row (d_i, d_r) = (-sin, cos)
        if ((j & 1) == 0) {
            pr = cs;
            pi = sn;
        } else {
            pr = -sn;
            pi = cs;
        }
    }
    uint32_t hi, lo;
    split_pair(pr, pi, &hi, &lo);
    const size_t off = static_cast<size_t>(c) * a.slab + img_byte(j, 2 * q);
    *reinterpret_cast<uint32_t*>(a.hi + off) = hi;
    *reinterpret_cast<uint32_t*>(a.lo + off) = lo;
}

// Pupil field images of every wavelength: row m (pupil row row_lo + m)
// over K-chunk c (pupil column col_lo + 32 c + q), the field
// amplitude * exp(i 2 pi phase) as the row transform embeds it
// (psf_rows_kernel; LensDiffCpuReference.cpp:831-845).
// grid (mt_rows * 128 / 8, kc_rows), block (32, 8): lane q of warp row m
// of K-chunk c (one 128-byte image row per warp), looping over the
// wavelengths.
__global__ void __launch_bounds__(256) pupil_field_kernel(PsfBankArgs a, DftPlan d) {
    const int c = blockIdx.y;
    const int m = blockIdx.x * 8 + threadIdx.y, q = threadIdx.x;
    const int np = a.pupil.size;
    const int y = a.row_lo + m, x = d.col_lo + c * 32 + q;
    // the pupil pre-pass of this pixel is read once and serves every
    // wavelength (their fields differ only in the defocus term)
    float4 p = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (m < a.row_n && c * 32 + q < d.col_n && x < np && y < np) p = a.pupil_pre[static_cast<size_t>(y) * np + x];
    const size_t off0 = static_cast<size_t>(c) * d.pf_slab + img_byte(m, 2 * q);
#pragma unroll 2
    for (int b = 0; b < a.B; ++b) {
        float fr = 0.0f, fi = 0.0f;
        if (p.x > 0.0f) {
            const WavelengthInfo* w = a.wl + b;
            const float ph = (w->phase.enabled && p.w != 0.0f) ? p.y + w->phase.c[4] * p.z : 0.0f;
            if (ph == 0.0f) {
                fr = p.x;
            } else {
                float sn, cs;
                sincospif(2.0f * ph, &sn, &cs);  // exp(i 2 pi phase), phase in waves
                fr = p.x * cs;
                fi = p.x * sn;
            }
        }
        uint32_t hi, lo;
        split_pair(fr, fi, &hi, &lo);
        const size_t off = static_cast<size_t>(b) * d.pf_lambda + off0;
        *reinterpret_cast<uint32_t*>(d.pf_hi + off) = hi;
        *reinterpret_cast<uint32_t*>(d.pf_lo + off) = lo;
    }
}

// ---- the GEMM --------------------------------------------------------------------------
// Persistent work queue over a table of transform problems (each one pass of
// one wavelength of one lens, with its own operands, sizes and window): one
// CTA per SM, tensor memory allocated once, three warp roles that run ahead
// of one another as far as their buffers allow:
//   warp 0 (one thread), producer: takes the next 128 x 128-complex output
//     tile from a global counter, publishes it in a four-entry tile ring,
//     and streams the tile's K-chunks (hi and lo tiles of A and B) into a
//     two-stage shared-memory ring with bulk copies;
//   warp 1 (one thread), MMA issuer: per tile, waits for one of the two
//     256-column accumulators in tensor memory to be drained, issues the
//     tensor-core MMAs of every K-chunk into it (three per 16-wide K step:
//     hi*hi, hi*lo, lo*hi), commits each stage back to the producer and the
//     finished accumulator to the epilogue;
//   warps 2-5, epilogue: read the accumulator out of tensor memory (warp w
//     owns lanes 32 (w % 4) .. + 31) while the next tile's MMAs run in the
//     other accumulator:
//       kDftRows: Y as the column pass's A images (row n, K pair m);
//       kDftCols: |Z|^2 into the PSF window (and its sum when asked).
// A tile index past the last tile ends every role.  Every wait is bounded; a
// wait that gives up records the error, its role stops, and the other roles'
// waits on it give up in turn; the CTA then releases its tensor memory.
constexpr int kTileRing = 4;
constexpr uint32_t kAccCols = 2 * kTmemCols;  // two accumulators
constexpr int kGemmThreads = 192;

struct TileSlot {
    int prob;    // problem of the tile; -1: no more tiles
    int tm, tn;  // its M and N tile within the problem
};

__device__ __forceinline__ TileSlot next_tile(const DftBatchArgs& g) {
    TileSlot ts{-1, 0, 0};
    const int t = atomicAdd(g.counter, 1);
    if (t >= g.tiles) return ts;
    // the problem of tile t: the last p with tile_start[p] <= t
    int lo = 0, hi = g.problems - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&g.tile_start[mid]) <= t) lo = mid;
        else hi = mid - 1;
    }
    const int local = t - __ldg(&g.tile_start[lo]);
    const int mt = g.probs[lo].mt;
    ts.prob = lo;
    ts.tm = local % mt;
    ts.tn = local / mt;
    return ts;
}

__global__ void __launch_bounds__(kGemmThreads, 1) dft_gemm_kernel(DftBatchArgs g) {
    extern __shared__ __align__(1024) unsigned char smraw[];
    __shared__ uint64_t full[kStages], empty[kStages];
    __shared__ uint64_t acc_full[2], acc_empty[2];
    __shared__ uint64_t tq_full[kTileRing], tq_empty[kTileRing];
    __shared__ uint64_t drained;
    __shared__ TileSlot tq[kTileRing];
    __shared__ uint32_t tmem_slot;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* base =
        smraw + ((1024u - (smem_addr(smraw) & 1023u)) & 1023u);  // 1024-byte aligned stages
    if (warp == 1) {
        tmem_alloc(&tmem_slot, kAccCols);
        tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 4);   // the four bulk copies of a stage
            mbar_init(&empty[s], 1);  // the MMA issuer's commit
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);   // the MMA issuer's commit
            mbar_init(&acc_empty[b], 4);  // one arrive per epilogue warp
        }
        for (int d = 0; d < kTileRing; ++d) {
            mbar_init(&tq_full[d], 1);   // the producer
            mbar_init(&tq_empty[d], 5);  // the MMA issuer and the four epilogue warps
        }
        mbar_init(&drained, 1);
        mbar_init_fence();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    if (warp == 0) {
        if (lane == 0) {  // producer
            uint32_t gc = 0;  // K-chunks streamed: ring stage and barrier phases
            for (uint32_t i = 0;; ++i) {
                const int d = static_cast<int>(i % kTileRing);
                const uint32_t use = i / kTileRing;
                if (use > 0 && !mbar_wait(&tq_empty[d], (use - 1) & 1, g.err)) break;
                const TileSlot ts = next_tile(g);
                tq[d] = ts;
                mbar_arrive(&tq_full[d]);  // release: the slot is visible to its waiters
                if (ts.prob < 0) break;
                const DftProblem& pr = g.probs[ts.prob];
                const int kc = pr.kc;
                const unsigned char* a_hi = pr.a_hi + static_cast<size_t>(ts.tm) * kImgA;
                const unsigned char* a_lo = pr.a_lo + static_cast<size_t>(ts.tm) * kImgA;
                const size_t b_row0 = static_cast<size_t>(2) * (pr.n0 + ts.tn * (kTileN / 2));  // multiple of 8
                const unsigned char* b_hi = pr.b_hi + (b_row0 >> 3) * 1024;
                const unsigned char* b_lo = pr.b_lo + (b_row0 >> 3) * 1024;
                bool ok = true;
                for (int c = 0; c < kc; ++c, ++gc) {
                    const int s = static_cast<int>(gc % kStages);
                    const uint32_t su = gc / kStages;
                    if (su > 0 && !mbar_wait(&empty[s], (su - 1) & 1, g.err)) {
                        ok = false;
                        break;
                    }
                    unsigned char* st = base + s * kStageBytes;
                    bulk_load_checked(st, a_hi + static_cast<size_t>(c) * pr.a_slab, kImgA, &full[s], smraw, g.err);
                    bulk_load_checked(st + kImgA, a_lo + static_cast<size_t>(c) * pr.a_slab, kImgA, &full[s], smraw,
                                      g.err);
                    bulk_load_checked(st + 2 * kImgA, b_hi + static_cast<size_t>(c) * pr.b_slab, kImgB, &full[s],
                                      smraw, g.err);
                    bulk_load_checked(st + 2 * kImgA + kImgB, b_lo + static_cast<size_t>(c) * pr.b_slab, kImgB,
                                      &full[s], smraw, g.err);
                }
                if (!ok) break;
            }
            // the copies still in flight land before the CTA exits: wait
            // (bounded) for the last use of each stage (gc: chunks issued)
            for (int s = 0; s < kStages; ++s) {
                const uint32_t issued = (gc + kStages - 1 - s) / kStages;  // uses of stage s
                if (issued > 0) mbar_wait(&full[s], (issued - 1) & 1, g.err);
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {  // MMA issuer
            uint32_t gc = 0;
            for (uint32_t i = 0;; ++i) {
                const int d = static_cast<int>(i % kTileRing);
                if (!mbar_wait(&tq_full[d], (i / kTileRing) & 1, g.err)) break;
                const TileSlot ts = tq[d];
                mbar_arrive(&tq_empty[d]);
                if (ts.prob < 0) break;
                const int kc = g.probs[ts.prob].kc;
                const int buf = static_cast<int>(i & 1);
                const uint32_t au = i >> 1;  // earlier uses of this accumulator
                if (au > 0 && !mbar_wait(&acc_empty[buf], (au - 1) & 1, g.err)) break;
                tc_fence_after();
                const uint32_t acc = tmem + static_cast<uint32_t>(buf) * kTmemCols;
                bool ok = true;
                for (int c = 0; c < kc; ++c, ++gc) {
                    const int s = static_cast<int>(gc % kStages);
                    if (!mbar_wait(&full[s], (gc / kStages) & 1, g.err)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t st = smem_addr(base + s * kStageBytes);
                    const uint64_t ah = smem_desc(st), al = smem_desc(st + kImgA);
                    const uint64_t bh = smem_desc(st + 2 * kImgA), bl = smem_desc(st + 2 * kImgA + kImgB);
#pragma unroll
                    for (int kk = 0; kk < kChunkK / 16; ++kk) {
                        const uint64_t dk = static_cast<uint64_t>(kk * 2);  // 32 bytes, in 16-byte units
                        mma_bf16(acc, ah + dk, bh + dk, kIdesc, (c | kk) != 0 ? 1u : 0u);
                        mma_bf16(acc, ah + dk, bl + dk, kIdesc, 1u);
                        mma_bf16(acc, al + dk, bh + dk, kIdesc, 1u);
                    }
                    mma_commit(&empty[s]);
                }
                if (!ok) break;
                mma_commit(&acc_full[buf]);
            }
            // every MMA this thread issued has completed before tensor
            // memory is released (the commit arrives at once if none is left)
            mma_commit(&drained);
            mbar_wait(&drained, 0, g.err);
        }
        __syncwarp();
    } else {  // epilogue, warps 2-5
        const int quarter = warp & 3;  // the TMEM lanes this warp may read
        const uint32_t lane_base = static_cast<uint32_t>(quarter * 32) << 16;
        for (uint32_t i = 0;; ++i) {
            const int d = static_cast<int>(i % kTileRing);
            if (!__all_sync(0xffffffffu, mbar_wait(&tq_full[d], (i / kTileRing) & 1, g.err))) break;
            const TileSlot ts = tq[d];
            __syncwarp();
            if (lane == 0) mbar_arrive(&tq_empty[d]);
            if (ts.prob < 0) break;
            const int buf = static_cast<int>(i & 1);
            const bool ready = __all_sync(0xffffffffu, mbar_wait(&acc_full[buf], (i >> 1) & 1, g.err));
            tc_fence_after();
            if (!ready) break;
            const DftProblem& pr = g.probs[ts.prob];
            float esum = 0.0f;  // kDftCols: this thread's window pixels
            const uint32_t lane_addr = tmem + static_cast<uint32_t>(buf) * kTmemCols + lane_base;
            const int row = ts.tm * kTileM + quarter * 32 + lane;  // M index of this thread
            for (int q = 0; q < static_cast<int>(kTmemCols) / 32; ++q) {
                uint32_t v[32];
                tmem_ld32(lane_addr + static_cast<uint32_t>(q * 32), v);
                const int n_first = ts.tn * (kTileN / 2) + q * 16;  // complex column of v[0], v[1]
                if (g.mode == kDftRows) {
                    // Y[m = row][n]: the column pass's A image row n, K pair m
                    const size_t chunk_off = static_cast<size_t>(row >> 5) * pr.y_slab;
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        const float re = __uint_as_float(v[2 * e]), im = __uint_as_float(v[2 * e + 1]);
                        uint32_t hi2, lo2;
                        split_pair(re, im, &hi2, &lo2);
                        const size_t off = chunk_off + img_byte(n_first + e, 2 * (row & 31));
                        *reinterpret_cast<uint32_t*>(pr.y_hi + off) = hi2;
                        *reinterpret_cast<uint32_t*>(pr.y_lo + off) = lo2;
                    }
                } else {
                    // Z[n = row][r]: window pixel (wy, wx) = (r, n) - shift
                    const int wx = row - pr.shift;
                    if (wx >= 0 && wx < pr.win_n) {
                        float* out = pr.win + wx;
#pragma unroll
                        for (int e = 0; e < 16; ++e) {
                            const int wy = n_first + e - pr.shift;
                            const float re = __uint_as_float(v[2 * e]), im = __uint_as_float(v[2 * e + 1]);
                            if (wy >= 0 && wy < pr.win_n) {
                                const float I = re * re + im * im;
                                out[static_cast<size_t>(wy) * pr.win_stride] = I;
                                esum += I;
                            }
                        }
                    }
                }
            }
            // this warp's reads of the accumulator are complete: hand it back
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[buf]);
            if (pr.energy) {  // uniform
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) esum += __shfl_xor_sync(0xffffffffu, esum, o);
                if (lane == 0 && esum != 0.0f) atomicAdd(pr.energy, static_cast<double>(esum));
            }
        }
    }
    // every role is done with tensor memory before it is released
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmem, kAccCols);
}

}  // namespace

size_t dft_gemm_smem() { return static_cast<size_t>(kStages) * kStageBytes + 1024; }

void launch_dft_basis(const DftBasisArgs& a, cudaStream_t s) {
    const int64_t total = static_cast<int64_t>(a.rows) * 32 * a.kc;
    if (total <= 0) return;
    dft_basis_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(a);
}

void launch_pupil_field(const PsfBankArgs& a, const DftPlan& d, cudaStream_t s) {
    if (d.mt_rows <= 0 || d.kc_rows <= 0) return;
    pupil_field_kernel<<<dim3(static_cast<unsigned>(d.mt_rows * kTileM / 8), static_cast<unsigned>(d.kc_rows), 1),
                         dim3(32, 8), 0, s>>>(a, d);
}

void launch_dft_gemm(const DftBatchArgs& g, cudaStream_t s) {
    if (g.tiles <= 0 || g.problems <= 0) return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    dft_gemm_kernel<<<static_cast<unsigned>(std::min(g.tiles, sms)), kGemmThreads, dft_gemm_smem(), s>>>(g);
}

void configure_dft_kernels() {
    cudaFuncSetAttribute(dft_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(dft_gemm_smem()));
}

}  // namespace ld
