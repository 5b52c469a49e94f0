// Whitening apply on the 5th-generation tensor cores (tcgen05, TMEM).
//
// y_t = W^T x_t for every timepoint (p_whiten.cpp:174-183: out[m1] +=
// in[m2] * W[m1*M + m2]), then the reference's 1e-4 rounding and optional
// int16 scaling.  As a GEMM: OUT[t][m1] = sum_m2 X[t][m2] * Wt[m1][m2] with
// Wt[m1][m2] = W[m1*M + m2]; X (rows of M channels) and Wt are both K-major.
//
// Precision: three TF32 products per term, accumulated in FP32 in TMEM:
//     x w ~= x_hi w_hi + x_hi w_lo + x_lo w_hi
// x_hi is x truncated to TF32 (what the tensor core reads from the raw FP32
// tile that TMA delivers), x_lo = rna_tf32(x - x_hi) is computed in shared
// memory by a converter warpgroup; w_hi = rna_tf32(w), w_lo = rna_tf32(w - w_hi)
// are prepared once per call.  The representation error is ~2^-22 of each
// term, the same order as the reference's own float accumulation.
//
// A persistent CTA per SM walks 128 (timepoints) x 128 (channels) output tiles:
//   warp 0      TMA producer: X, Wt_hi, Wt_lo K-blocks of 32 into an
//               S-stage ring (128-byte swizzle, the UMMA canonical layout),
//               streaming continuously across the CTA's tiles
//   warp 1      TMEM allocation; one thread issues 3 MMAs per K=8 step and
//               commits each stage back to the producer
//   warps 2..3  convert X to X_lo per stage
//   warps 4..7  drain the accumulators (tcgen05.ld), round, store
// Every mbarrier wait is bounded (tc::mbar_wait); a timeout raises *err.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <mutex>

#include "common.cuh"
#include "ms3gpu.h"
#include "tc_sm100.cuh"
#include "whiten.h"

namespace ms3gpu {

namespace {

constexpr int kTM = 128;       // timepoints per tile (MMA M)
constexpr int kKB = 32;        // K elements per stage (one 128-byte row)

template <int BN, bool DRAIN>
struct TcCfg {
    static constexpr int kStages = 3;
    static constexpr int kABytes = kTM * 128;  // 16 KB
    static constexpr int kBBytes = BN * 128;
    static constexpr int kStageBytes = 2 * kABytes + 2 * kBBytes;  // X, X_lo, W_hi, W_lo
    // DRAIN: two per-K-block accumulators plus two tile sums (alternate
    // tiles); mixed: two tile accumulators (alternate tiles)
    static constexpr int kUsedCols = DRAIN ? 4 * BN : 2 * BN;
    static constexpr int kTmemCols = (kUsedCols <= 32) ? 32 : (kUsedCols <= 64) ? 64 : (kUsedCols <= 128) ? 128
                                     : (kUsedCols <= 256) ? 256 : 512;
    // DRAIN adds a warpgroup that rounds and stores finished tiles
    static constexpr int kThreads = DRAIN ? 384 : 256;
    // output staging: two 32 x 32 float buffers per storing warp (128-byte swizzle)
    static constexpr int kStagingBytes = 4 * 2 * 32 * 128;
    static constexpr size_t kSmemBytes =
        (size_t)kStages * kStageBytes + kStagingBytes + 1024 /*align*/ + 256 /*barriers*/;
};

// The reference's 1e-4 rounding, floor(x / 1e-4 + 0.5) * 1e-4 in double
// (p_whiten.cpp:185-189), for 32 values in place.  x * 10000 stands in for
// the division: for a float x it is exact in double and the quotient rounds
// to the same double (it lies within 0.43 ulp of it).  As a guard, values
// within 1e-6 of a rounding boundary are redone with the division in a
// second loop, so the main loop has no branch and its 32 chains interleave.
__device__ __forceinline__ void quantize_1e4_x32(float (&y)[32]) {
#pragma unroll
    for (int h = 0; h < 32; h += 16) {  // two halves keep the live registers down
        uint32_t redo = 0;
        float q[16];
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const double t = __dadd_rn(__dmul_rn((double)y[h + j], 10000.0), 0.5);
            const double f = floor(t);
            redo |= (uint32_t)((t - f < 1e-6) | (f + 1.0 - t < 1e-6)) << j;
            q[j] = (float)__dmul_rn(f, 0.0001);
        }
        if (redo) {
#pragma unroll
            for (int j = 0; j < 16; j++) {
                if ((redo >> j) & 1) {
                    const double f = floor(__dadd_rn(__ddiv_rn((double)y[h + j], 0.0001), 0.5));
                    q[j] = (float)__dmul_rn(f, 0.0001);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < 16; j++) y[h + j] = q[j];
    }
}

// x - trunc_tf32(x), rounded to TF32 (nearest, ties away from zero) and
// returned as its 32-bit pattern: the same value cvt.rna.tf32.f32 gives.
__device__ __forceinline__ uint32_t x_lo_tf32(uint32_t xb) {
    const float lo = __uint_as_float(xb) - __uint_as_float(xb & 0xFFFFE000u);
    return (__float_as_uint(lo) + 0x1000u) & 0xFFFFE000u;
}

// Stores 32 consecutive output channels of one timepoint, already rounded
// to 1e-4; int16 output is scaled by the quantization unit as the reference
// does ((int)(x / q + 0.5) truncated to 16 bits).
__device__ __forceinline__ void store_row32(const float (&y)[32], int64_t t, int64_t nbase, int64_t M, double qunit,
                                            void* __restrict__ out) {
    if (qunit > 0) {
        int16_t* o16 = static_cast<int16_t*>(out) + t * M;
#pragma unroll
        for (int j = 0; j < 32; j++) {
            if (nbase + j >= M) break;
            const int32_t iv = x86_double_to_int32(__dadd_rn(__ddiv_rn((double)y[j], qunit), 0.5));
            o16[nbase + j] = x86_float_to_int16((float)iv);
        }
        return;
    }
    float* of = static_cast<float*>(out) + t * M + nbase;
    if (nbase + 32 <= M && ((reinterpret_cast<uintptr_t>(of) & 15) == 0)) {
#pragma unroll
        for (int j = 0; j < 32; j += 4) *reinterpret_cast<float4*>(of + j) = make_float4(y[j], y[j + 1], y[j + 2], y[j + 3]);
    } else {
#pragma unroll
        for (int j = 0; j < 32; j++) {
            if (nbase + j >= M) break;
            of[j] = y[j];
        }
    }
}

// Rounds 32 values of one timepoint to 1e-4 (unless round_1e4 is 0) and writes them: float output
// through the warp's swizzled staging buffer and one TMA store of the warp's
// 32 x 32 block (full 128-byte lines), int16 output directly.
__device__ __forceinline__ void emit_row32(float (&y)[32], int lane, uint8_t* staging_warp, int& sbuf,
                                           const CUtensorMap* tmOut, int out_tma, int64_t t, int64_t trow0, int n,
                                           int64_t M, int64_t N, double qunit, int round_1e4,
                                           void* __restrict__ out) {
    // a float block that starts beyond the last row or column would be clipped
    // whole: nothing is staged or stored, and the staging ring does not turn
    // (its bulk-group accounting counts only issued stores)
    if (out_tma && (n >= M || trow0 >= N)) return;
    if (round_1e4) quantize_1e4_x32(y);
    if (out_tma) {
        uint8_t* stg = staging_warp + (size_t)sbuf * (32 * 128);
        if (lane == 0) tc::bulk_wait_group_read<1>();  // its previous store has read it
        __syncwarp();
#pragma unroll
        for (int jj = 0; jj < 8; jj++) {
            const float4 v = make_float4(y[4 * jj], y[4 * jj + 1], y[4 * jj + 2], y[4 * jj + 3]);
            *reinterpret_cast<float4*>(stg + lane * 128 + ((jj ^ (lane & 7)) << 4)) = v;
        }
        tc::fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0 && MS3_IN_BOUNDS(n, M, 301) && MS3_IN_BOUNDS(trow0, N, 302)) {
            tc::tma_store_2d(tmOut, stg, n, (int)trow0);
            tc::bulk_commit_group();
        }
        sbuf ^= 1;
    } else if (t < N) {
        store_row32(y, t, n, M, qunit, out);
    }
}

// Persistent: each CTA walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ...
// with column blocks of one time tile adjacent in tile order, so the CTAs
// running at any moment share their X tiles through L2.  The producer and
// converter stream K-blocks continuously across tiles (a global K-block
// counter g drives the stage ring), so the next tile's loads overlap the
// current tile's last MMAs and epilogue.
//
// DRAIN = false (mixed form): all three products accumulate over the whole K
// range in a tile accumulator; two alternate by tile parity so a tile's
// epilogue (warps 4-7) overlaps the next tile's MMAs.
// DRAIN = true (plain form): the tensor core's FP32 accumulation rounds
// toward zero, so long accumulations drift.  Each K-block's three products go
// to a fresh accumulator (two alternate) that warps 4-7 add into
// round-to-nearest FP32 sums kept in TMEM while the next K-block runs; warps
// 8-11 round and store a finished tile's sums during the next tile (the
// sums alternate between two TMEM buffers by tile parity).
template <int BN, bool DRAIN>
__global__ void __launch_bounds__(TcCfg<BN, DRAIN>::kThreads, 1)
    apply_tc_kernel(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmWhi,
                    const __grid_constant__ CUtensorMap tmWlo, const __grid_constant__ CUtensorMap tmOut, int out_tma,
                    int64_t M, int64_t N, int ncb, int64_t ntiles, double qunit, int round_1e4,
                    void* __restrict__ out, int* __restrict__ err) {
    using C = TcCfg<BN, DRAIN>;
    constexpr int S = C::kStages;
    constexpr int R = 2;  // accumulator ring (K-blocks when DRAIN, tiles when mixed)
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* staging = smem + (size_t)S * C::kStageBytes;  // 1024-byte aligned
    uint64_t* bars = reinterpret_cast<uint64_t*>(staging + C::kStagingBytes);
    uint64_t* full = bars;                // [S] TMA bytes landed
    uint64_t* conv = bars + S;            // [S] X_lo written
    uint64_t* empty = bars + 2 * S;       // [S] MMAs done reading the stage
    uint64_t* acc_full = bars + 3 * S;      // [2] accumulator complete (K-block, or tile when mixed)
    uint64_t* acc_free = bars + 3 * S + 2;  // [2] accumulator read back
    uint64_t* y_full = bars + 3 * S + 4;    // [2] DRAIN: a tile's sums complete in TMEM
    uint64_t* y_free = bars + 3 * S + 6;    // [2] DRAIN: a tile's sums read by the storing warps
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 3 * S + 8);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nkb = (int)((M + kKB - 1) / kKB);
    const int64_t my_tiles = (blockIdx.x < ntiles) ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    auto stageA = [&](int s) { return smem + (size_t)s * C::kStageBytes; };
    auto stageAlo = [&](int s) { return smem + (size_t)s * C::kStageBytes + C::kABytes; };
    auto stageBhi = [&](int s) { return smem + (size_t)s * C::kStageBytes + 2 * C::kABytes; };
    auto stageBlo = [&](int s) { return smem + (size_t)s * C::kStageBytes + 2 * C::kABytes + C::kBBytes; };
    auto tile_of = [&](int64_t i, int64_t& t0, int& n0) {
        const int64_t tile = blockIdx.x + i * gridDim.x;
        t0 = (tile / ncb) * kTM;
        n0 = (int)(tile % ncb) * BN;
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; s++) {
            tc::mbar_init(&full[s], 1);
            tc::mbar_init(&conv[s], 64);
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            tc::mbar_init(&acc_full[b], 1);
            tc::mbar_init(&acc_free[b], 128);
            tc::mbar_init(&y_full[b], 128);
            tc::mbar_init(&y_free[b], 128);
        }
        tc::fence_mbar_init();
    }
    if (warp == 1) tc::tmem_alloc(tmem_slot, C::kTmemCols);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t taddr = *tmem_slot;
    // TMEM columns: accumulator b at b * BN; DRAIN keeps tile sums at (2 + tp) * BN
    const uint32_t ysum[2] = {taddr + 2u * BN, taddr + 3u * BN};
    const int64_t total_kb = my_tiles * nkb;

    if (warp == 0) {
        if (lane == 0) {
            // indices advance incrementally: a 64-bit division here would sit on
            // the stage ring's critical path
            int64_t issued = 0, t0 = 0;
            int n0 = 0, kb = 0, s = 0;
            uint32_t phase = 0;  // parity of the previous use of stage s
            if (my_tiles > 0) tile_of(0, t0, n0);
            for (int64_t g = 0, i = 0; g < total_kb; g++) {
                if (g >= S && !tc::mbar_wait(&empty[s], phase, err)) break;
                tc::mbar_expect_tx(&full[s], C::kABytes + 2 * C::kBBytes);
                tc::tma_load_2d(stageA(s), &tmX, &full[s], kb * kKB, (int)t0);
                tc::tma_load_2d(stageBhi(s), &tmWhi, &full[s], kb * kKB, n0);
                tc::tma_load_2d(stageBlo(s), &tmWlo, &full[s], kb * kKB, n0);
                issued = g + 1;
                if (++s == S) {
                    s = 0;
                    if (g + 1 > S) phase ^= 1;
                }
                if (++kb == nkb) {
                    kb = 0;
                    if (++i < my_tiles) tile_of(i, t0, n0);
                }
            }
            // no copy may still be landing in shared memory when the CTA exits
            for (int64_t g = (issued > S ? issued - S : 0); g < issued; g++)
                tc::mbar_wait(&full[g % S], (uint32_t)((g / S) & 1), err);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = tc::instr_desc(2u /*TF32*/, kTM, BN);
            bool ok = true;
            for (int64_t i = 0; i < my_tiles && ok; i++) {
                const int tp = (int)(i & 1);
                // mixed: the tile accumulator must have been read back (tile i - 2)
                if (!DRAIN && i >= 2) ok = tc::mbar_wait(&acc_free[tp], (uint32_t)(((i >> 1) - 1) & 1), err);
                for (int kb = 0; kb < nkb && ok; kb++) {
                    const int64_t g = i * nkb + kb;
                    const int s = (int)(g % S);
                    const int b = DRAIN ? (int)(g % R) : tp;
                    ok = tc::mbar_wait(&full[s], (uint32_t)((g / S) & 1), err) &&
                         tc::mbar_wait(&conv[s], (uint32_t)((g / S) & 1), err);
                    if (ok && DRAIN && g >= R) ok = tc::mbar_wait(&acc_free[b], (uint32_t)(((g / R) - 1) & 1), err);
                    if (!ok) break;
                    tc::tc_fence_after();
                    const uint32_t acc = taddr + (uint32_t)(b * BN);
                    const uint32_t a = tc::smem_u32(stageA(s)), al = tc::smem_u32(stageAlo(s));
                    const uint32_t bh = tc::smem_u32(stageBhi(s)), bl = tc::smem_u32(stageBlo(s));
#pragma unroll
                    for (int ks = 0; ks < kKB / 8; ks++) {
                        const uint32_t off = ks * 32;  // 8 TF32 = 32 bytes along K inside the swizzle atom
                        const uint64_t da = tc::smem_desc_k_sw128(a + off), dal = tc::smem_desc_k_sw128(al + off);
                        const uint64_t dbh = tc::smem_desc_k_sw128(bh + off), dbl = tc::smem_desc_k_sw128(bl + off);
                        tc::mma_tf32(acc, da, dbh, idesc, DRAIN ? (ks != 0) : ((kb | ks) != 0));
                        tc::mma_tf32(acc, da, dbl, idesc, 1);
                        tc::mma_tf32(acc, dal, dbh, idesc, 1);
                    }
                    tc::mma_commit(&empty[s]);
                    if (DRAIN) tc::mma_commit(&acc_full[b]);
                }
                if (!DRAIN && ok) tc::mma_commit(&acc_full[tp]);
            }
            // mixed: no MMA may still be writing TMEM when it is freed
            for (int64_t i = (my_tiles > 2 ? my_tiles - 2 : 0); !DRAIN && i < my_tiles && ok; i++)
                ok = tc::mbar_wait(&acc_free[i & 1], (uint32_t)((i >> 1) & 1), err);
        }
    } else if (warp < 4) {
        // warps 2-3: X_lo = rna_tf32(x - trunc_tf32(x)), same swizzled layout as X.
        // x - trunc_tf32(x) is exact in FP32; its round-to-nearest-away TF32
        // value is the integer round-half-up of its magnitude bits at bit 13
        // (sign-magnitude encoding), which keeps the conversion on the
        // full-rate integer pipe.  Eight 16-byte loads per thread are in flight at once.
        const int ct = threadIdx.x - 64;
        for (int64_t g = 0; g < total_kb; g++) {
            const int s = (int)(g % S);
            if (!tc::mbar_wait(&full[s], (uint32_t)((g / S) & 1), err)) break;
            const uint4* src = reinterpret_cast<const uint4*>(stageA(s));
            uint4* dst = reinterpret_cast<uint4*>(stageAlo(s));
            constexpr int kPer = kTM * kKB / 4 / 64;
#pragma unroll
            for (int h = 0; h < kPer; h += 8) {
                uint4 v[8];
#pragma unroll
                for (int k = 0; k < 8; k++) v[k] = src[ct + 64 * (h + k)];
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    uint4 r;
                    r.x = x_lo_tf32(v[k].x);
                    r.y = x_lo_tf32(v[k].y);
                    r.z = x_lo_tf32(v[k].z);
                    r.w = x_lo_tf32(v[k].w);
                    dst[ct + 64 * (h + k)] = r;
                }
            }
            tc::fence_proxy_async_smem();
            tc::mbar_arrive(&conv[s]);
        }
    } else if (warp < 8) {
        // warps 4-7; warp q reads TMEM lanes 32q..32q+31 (timepoints of the tile)
        const int q = warp & 3;
        const uint32_t lane_base = (uint32_t)(q * 32) << 16;
        uint8_t* stg = staging + (size_t)q * 2 * (32 * 128);
        int sbuf = 0;
        bool ok = true;
        for (int64_t i = 0; i < my_tiles && ok; i++) {
            int64_t t0;
            int n0;
            tile_of(i, t0, n0);
            if (DRAIN) {
                // running round-to-nearest sums live in TMEM (ysum[tp]); the
                // storing warps must have read this buffer's previous tile
                const int tp = (int)(i & 1);
                if (i >= 2) ok = tc::mbar_wait(&y_free[tp], (uint32_t)(((i >> 1) - 1) & 1), err);
                if (!__all_sync(0xffffffffu, ok)) break;
                for (int kb = 0; kb < nkb; kb++) {
                    const int64_t g = i * nkb + kb;
                    const int b = (int)(g & 1);
                    ok = tc::mbar_wait(&acc_full[b], (uint32_t)((g >> 1) & 1), err);
                    if (!__all_sync(0xffffffffu, ok)) {
                        ok = false;
                        break;
                    }
                    tc::tc_fence_after();
#pragma unroll
                    for (int c0 = 0; c0 < BN; c0 += 32) {
                        uint32_t r[32];
                        tc::tmem_ld_32x32b_x32(taddr + (uint32_t)(b * BN) + lane_base + (uint32_t)c0, r);
                        if (kb != 0) {
                            uint32_t u[32];
                            tc::tmem_ld_32x32b_x32(ysum[tp] + lane_base + (uint32_t)c0, u);
#pragma unroll
                            for (int j = 0; j < 32; j++)
                                r[j] = __float_as_uint(__fadd_rn(__uint_as_float(u[j]), __uint_as_float(r[j])));
                        }
                        tc::tmem_st_32x32b_x32(ysum[tp] + lane_base + (uint32_t)c0, r);
                    }
                    tc::tmem_st_wait();
                    tc::tc_fence_before();
                    tc::mbar_arrive(&acc_free[b]);
                }
                if (!ok) break;
                tc::mbar_arrive(&y_full[tp]);
            } else {
                const int tp = (int)(i & 1);
                ok = tc::mbar_wait(&acc_full[tp], (uint32_t)((i >> 1) & 1), err);
                if (!__all_sync(0xffffffffu, ok)) break;
                tc::tc_fence_after();
                const int64_t t = t0 + q * 32 + lane;
#pragma unroll 1
                for (int c0 = 0; c0 < BN; c0 += 32) {
                    uint32_t r[32];
                    tc::tmem_ld_32x32b_x32(taddr + (uint32_t)(tp * BN) + lane_base + (uint32_t)c0, r);
                    float y[32];
#pragma unroll
                    for (int j = 0; j < 32; j++) y[j] = __uint_as_float(r[j]);
                    emit_row32(y, lane, stg, sbuf, &tmOut, out_tma, t, t0 + q * 32, n0 + c0, M, N, qunit, round_1e4, out);
                }
                tc::tc_fence_before();
                tc::mbar_arrive(&acc_free[tp]);
            }
        }
        if (!DRAIN && out_tma && lane == 0) tc::bulk_wait_group<0>();  // stores complete before the CTA exits
    } else if (DRAIN) {
        // warps 8-11: round and store each tile's sums
        const int q = warp & 3;
        const uint32_t lane_base = (uint32_t)(q * 32) << 16;
        uint8_t* stg = staging + (size_t)q * 2 * (32 * 128);
        int sbuf = 0;
        for (int64_t i = 0; i < my_tiles; i++) {
            int64_t t0;
            int n0;
            tile_of(i, t0, n0);
            const int tp = (int)(i & 1);
            const bool ok = tc::mbar_wait(&y_full[tp], (uint32_t)((i >> 1) & 1), err);
            if (!__all_sync(0xffffffffu, ok)) break;
            tc::tc_fence_after();
            const int64_t t = t0 + q * 32 + lane;
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 32) {
                uint32_t r[32];
                tc::tmem_ld_32x32b_x32(ysum[tp] + lane_base + (uint32_t)c0, r);
                if (c0 + 32 == BN) {  // every sum of the tile is read
                    tc::tc_fence_before();
                    tc::mbar_arrive(&y_free[tp]);
                }
                float y[32];
#pragma unroll
                for (int j = 0; j < 32; j++) y[j] = __uint_as_float(r[j]);
                emit_row32(y, lane, stg, sbuf, &tmOut, out_tma, t, t0 + q * 32, n0 + c0, M, N, qunit, round_1e4, out);
            }
        }
        if (out_tma && lane == 0) tc::bulk_wait_group<0>();  // stores complete before the CTA exits
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc::tc_fence_after();
        tc::tmem_dealloc(taddr, C::kTmemCols);
    }
}

// w_hi = rna_tf32(w), w_lo = rna_tf32(w - w_hi) of Wt[m1][m2] = W[m1*M + m2].
__global__ void w_split_tf32(const double* __restrict__ W, int64_t MM, float* __restrict__ hi, float* __restrict__ lo) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MM) return;
    const double w = W[i];
    const float h = __uint_as_float(tc::cvt_rna_tf32((float)w));
    hi[i] = h;
    lo[i] = __uint_as_float(tc::cvt_rna_tf32((float)(w - (double)h)));
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static cudaError_t status = cudaSuccess;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        status = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (status == cudaSuccess && q == cudaDriverEntryPointSuccess) fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    if (!fn) throw_unsupported("cuTensorMapEncodeTiled is not available from the driver");
    return fn;
}

// Row-major [rows][cols] float32 matrix, tiles of box_rows x 32 columns, 128-byte swizzle.
CUtensorMap make_map(const void* base, uint64_t cols, uint64_t rows, uint32_t box_rows) {
    CUtensorMap m;
    const cuuint64_t dims[2] = {cols, rows};
    const cuuint64_t strides[1] = {cols * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)kKB, box_rows};
    const cuuint32_t es[2] = {1, 1};
    const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(base), dims, strides, box,
                                   es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw_unsupported("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return m;
}

template <int BN, bool DRAIN>
void launch_apply_tc(const float* X, int64_t M, int64_t N, const float* whi, const float* wlo, double qunit,
                     int round_1e4, void* out, int* err, cudaStream_t stream) {
    using C = TcCfg<BN, DRAIN>;
    MS3_CUDA(cudaFuncSetAttribute(apply_tc_kernel<BN, DRAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)C::kSmemBytes));
    const CUtensorMap mx = make_map(X, (uint64_t)M, (uint64_t)N, kTM);
    const CUtensorMap mh = make_map(whi, (uint64_t)M, (uint64_t)M, BN);
    const CUtensorMap ml = make_map(wlo, (uint64_t)M, (uint64_t)M, BN);
    // float output goes out through TMA stores of 32 x 32 blocks
    const int out_tma = (qunit <= 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0) ? 1 : 0;
    const CUtensorMap mo = out_tma ? make_map(out, (uint64_t)M, (uint64_t)N, 32) : mx;
    const int ncb = (int)ceil_div(M, BN);
    const int64_t ntiles = ceil_div(N, kTM) * ncb;
    int dev = 0, nsm = 0;
    MS3_CUDA(cudaGetDevice(&dev));
    MS3_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int64_t grid = std::min<int64_t>(ntiles, nsm);  // one persistent CTA per SM
    apply_tc_kernel<BN, DRAIN><<<(unsigned)grid, C::kThreads, C::kSmemBytes, stream>>>(mx, mh, ml, mo, out_tma, M, N, ncb,
                                                                                     ntiles, qunit, round_1e4,
                                                                                     out, err);
    MS3_LAUNCH_CHECK();
}

}  // namespace

bool apply_tc_supported(const float* X, int64_t M, int64_t N, const void* out) {
    if (M < 4 || M % 4 != 0 || M > 65536 || N < 1) return false;  // TMA: 16-byte row strides
    if ((reinterpret_cast<uintptr_t>(X) & 15) != 0) return false;
    (void)out;
    return true;
}

void apply_whitening_tc(const float* X, int64_t M, int64_t N, const double* W, double quantization_unit,
                        bool drain, void* out, cudaStream_t stream, int* ext_err, bool round_1e4) {
    DevBuf wbuf(sizeof(float) * (size_t)(2 * M * M) + 256, stream);
    float* whi = wbuf.as<float>();
    float* wlo = whi + M * M;
    int* err = ext_err ? ext_err : reinterpret_cast<int*>(wlo + M * M);
    if (!ext_err) MS3_CUDA(cudaMemsetAsync(err, 0, sizeof(int), stream));
    w_split_tf32<<<(unsigned)ceil_div(M * M, 256), 256, 0, stream>>>(W, M * M, whi, wlo);
    MS3_LAUNCH_CHECK();
    if (drain)
        launch_apply_tc<128, true>(X, M, N, whi, wlo, quantization_unit, round_1e4 ? 1 : 0, out, err, stream);
    else
        launch_apply_tc<128, false>(X, M, N, whi, wlo, quantization_unit, round_1e4 ? 1 : 0, out, err, stream);
    if (ext_err) return;  // the caller checks the flag once for many calls
    int herr = 0;
    MS3_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, stream));
    MS3_CUDA(cudaStreamSynchronize(stream));
    if (herr) throw Error(MS3GPU_ERR_CUDA, "tensor-core apply: pipeline wait timed out");
}

int bounds_site_apply(cudaStream_t s) {
#ifdef MS3GPU_BOUNDS_CHECK
    return take_bounds_site(s);
#else
    (void)s;
    return 0;
#endif
}

}  // namespace ms3gpu
