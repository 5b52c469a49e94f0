// Channel covariance (whiten pass 1, p_whiten.cpp:64-118) on the
// 5th-generation tensor cores with exact integer arithmetic.
//
// XXt = sum_t x_t x_t^T.  The reference multiplies float by float (rounded
// to float) and sums in double.  Here each value is turned into a 30-bit
// fixed-point integer relative to its channel's largest magnitude within a
// run of R timepoints,
//     v = rint(x * 2^(30 - e)),   2^e > max |x| over the run   (|v| < 2^30),
// and v is written as four signed 8-bit digits
//     v = d0 2^24 + d1 2^16 + d2 2^8 + d3,   d1..d3 in [-128, 127], |d0| <= 64.
// The products of digits are summed exactly by tcgen05.mma kind::i8 (int32
// accumulation) in four weight classes, kept in TMEM for a whole run:
//     A0 = sum d0 d0'                             (weight 2^48)
//     A1 = sum d0 d1' + d1 d0'                    (2^40)
//     A2 = sum d0 d2' + d2 d0' + d1 d1'           (2^32)
//     A3 = sum d0 d3' + d3 d0' + d1 d2' + d2 d1'  (2^24)
// (ten MMAs per 32 timepoints, seven for a diagonal block pair, whose
// classes 1 and 3 are computed one half at a time, d0 d1' instead of d0 d1' +
// d1 d0' = d0 d1' + (d0 d1')^T, the transpose added when the tile is reduced;
// int32 cannot overflow for R <= 32768).  The
// classes below 2^24 are dropped; their only non-zero-mean part, the d2 d2
// term on the diagonal, is added back from per-channel sums of d2^2 kept by
// the converter threads.  At the end of a run the classes are combined in
// FP64 and scaled by 2^(e_i + e_j - 36), one partial tile per (run, tile
// pair); the reduction sums the runs in order.  Relative to the exact sum
// the result is within ~5e-9 (the reference's own float products are within
// ~1e-9), and it does not depend on how the runs are grouped into CTAs or
// slabs, so a recording streamed in slabs of whole runs gives the same bits.
//
// Work items are (run, pair of 128-channel blocks with bi <= bj); a
// persistent CTA per SM walks items r * P + p so CTAs running at the same
// time share the run's rows through L2.  Per CTA:
//   warp 0      TMA: fp32 tiles of 32 timepoints x 128 channels (blocks bi,
//               bj) into a 3-stage ring
//   warp 1      TMEM allocation (512 columns: four 128 x 128 int32
//               accumulators); one thread issues the ten MMAs per stage
//   warps 2-17  convert fp32 tiles to the four digit planes in the UMMA
//               MN-major 128-byte-swizzle layout (3-stage ring)
//   warps 18-21 at the end of each run: read the accumulators, combine,
//               scale, store the run's FP64 partial tile
// Every mbarrier wait is bounded (tc::mbar_wait); a timeout sets
// g_cov_timeout, which the host checks after the call.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <string>

#include "common.cuh"
#include "ms3gpu.h"
#include "tc_sm100.cuh"
#include "whiten.h"

namespace ms3gpu {

__device__ int g_cov_timeout;  // set when a pipeline wait gave up (checked by the host)

namespace {

constexpr int kB = 128;                       // channels per block (MMA M and N)
constexpr int kKT = 32;                       // timepoints per stage (one MMA K step for 8-bit digits)
constexpr int kS1 = 3;                        // fp32 ring stages
constexpr int kS2 = 3;                        // digit-plane ring stages
constexpr int kF32Bytes = kKT * kB * 4;       // 16 KB: one block's fp32 tile
constexpr int kPlaneBytes = kKT * kB;         // 4 KB: one digit plane of one block
constexpr int kF32Stage = 2 * kF32Bytes;      // blocks bi and bj
constexpr int kPlaneStage = 2 * 4 * kPlaneBytes;
constexpr int kConvWarps = 16;
constexpr int kThreads = (2 + kConvWarps + 4) * 32;  // 704
static_assert(kKT == 2 * kConvWarps, "each converter thread takes two rows of a stage");
static_assert(kS1 == kS2, "the converters walk both rings with one stage counter");
constexpr int kSentinel = 1000;               // scale exponent of a channel whose run holds inf / NaN
constexpr size_t kSmemBytes = (size_t)kS1 * kF32Stage + (size_t)kS2 * kPlaneStage + 2 * kB * sizeof(int) +
                              1024 /*align*/ + 256 /*barriers*/;

// (bi, bj), bi <= bj, of pair index p in row order over nb blocks.
__host__ __device__ inline void pair_blocks(int p, int nb, int& bi, int& bj) {
    bi = 0;
    while (p >= nb - bi) {
        p -= nb - bi;
        bi++;
    }
    bj = bi + p;
}

// 2^k as a double (k within the normal range).
__device__ __forceinline__ double pow2d(int k) { return __longlong_as_double((long long)(1023 + k) << 52); }

// maxbits[r * Mp + m] = the bit pattern of max |x(m, t)| over run r (the
// IEEE patterns of non-negative floats order like their values, so atomicMax
// on them is a max of the magnitudes; inf / NaN patterns lie above every
// finite one).  The table must be zero on entry.  Block: 32 channel quads x 8
// time phases over `seg` rows (seg divides the run length); grid (row
// segments, channel blocks of 128).
__global__ void __launch_bounds__(256) cov_run_maxbits(const float* __restrict__ X, int64_t M, int64_t rows,
                                                       int64_t R, int64_t seg, int64_t Mp,
                                                       unsigned int* __restrict__ maxbits) {
    __shared__ unsigned int red[8][kB];
    const int q = threadIdx.x & 31, ph = threadIdx.x >> 5;
    const int64_t t0 = (int64_t)blockIdx.x * seg, t1 = min(rows, t0 + seg);
    const int64_t c0 = (int64_t)blockIdx.y * kB + 4 * q;
    unsigned int mx[4] = {0u, 0u, 0u, 0u};
    if (c0 < M) {
        const float* p = X + c0;
#pragma unroll 8
        for (int64_t t = t0 + ph; t < t1; t += 8) {
            const float4 v = __ldg(reinterpret_cast<const float4*>(p + t * M));
            mx[0] = max(mx[0], __float_as_uint(v.x) & 0x7FFFFFFFu);
            mx[1] = max(mx[1], __float_as_uint(v.y) & 0x7FFFFFFFu);
            mx[2] = max(mx[2], __float_as_uint(v.z) & 0x7FFFFFFFu);
            mx[3] = max(mx[3], __float_as_uint(v.w) & 0x7FFFFFFFu);
        }
    }
#pragma unroll
    for (int i = 0; i < 4; i++) red[ph][4 * q + i] = mx[i];
    __syncthreads();
    if (threadIdx.x < kB) {
        unsigned int m = red[0][threadIdx.x];
        for (int k = 1; k < 8; k++) m = max(m, red[k][threadIdx.x]);
        const int64_t c = (int64_t)blockIdx.y * kB + threadIdx.x;
        if (m != 0u && c < Mp && MS3_IN_BOUNDS((t0 / R) * Mp + c, ((rows + R - 1) / R) * Mp, 402))
            atomicMax(maxbits + (t0 / R) * Mp + c, m);
    }
}

// The run's scale exponent of a channel from its max-magnitude bits: the
// smallest e with 2^e > max |x| (frexp's exponent), at least -96 so that
// 2^(30 - e) stays a normal float; 0 for an all-zero run; kSentinel when the
// run holds inf / NaN.
__device__ __forceinline__ int run_exponent(unsigned int m) {
    if (m >= 0x7F800000u) return kSentinel;
    if (m == 0u) return 0;
    return max((int)(m >> 23) - 126, -96);
}

// Digits of 4 values, with m8 = 2^(22 - e) and m = 2^(30 - e) (xs = x m):
// w[i] = bits of (rint(xs / 256) + 1.5 * 2^23) minus 0x3F7F80, whose bytes 2,
// 1, 0 are d0, d1 ^ 0x80, d2 ^ 0x80; lo[i] = bits of (rint(xs - 256 rint(xs /
// 256)) + 1.5 * 2^23), whose byte 0 is d3.  The remainder lies in [-128, 128];
// it is held at 127 from above (v moves by at most one unit): large values
// are multiples of their float spacing, so xs / 256 often falls exactly on
// a half, where rounding to even leaves a remainder of +128, which a byte
// cannot hold.
__device__ __forceinline__ void digits4(const float4 x, const float (&m8)[4], const float (&m)[4], uint32_t (&w)[4],
                                        uint32_t (&lo)[4]) {
    const float xv[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float y1 = __fmaf_rn(xv[i], m8[i], 12582912.0f);  // rint(xs / 256) + 1.5 * 2^23 (one rounding)
        const float vh = __fsub_rn(y1, 12582912.0f);
        const float rem = fminf(__fmaf_rn(vh, -256.0f, __fmul_rn(xv[i], m[i])), 127.0f);  // exact, then held
        const float y2 = __fadd_rn(rem, 12582912.0f);
        w[i] = __float_as_uint(y1) - 0x3F7F80u;  // + 0x8080 (balanced d1, d2), - 0x400000 (d0 in byte 2)
        lo[i] = __float_as_uint(y2);
    }
}

// byte K of each of four words, packed low to high
template <int K>
__device__ __forceinline__ uint32_t gather_byte(const uint32_t (&v)[4]) {
    const uint32_t a = __byte_perm(v[0], v[1], K | ((K + 4) << 4));
    const uint32_t b = __byte_perm(v[2], v[3], K | ((K + 4) << 4));
    return __byte_perm(a, b, 0x5410);
}

// 32 lanes x 8 consecutive 32-bit TMEM columns (thread i: row lane base + i).
__device__ __forceinline__ void tmem_ld_32x32b_x8(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ int sext8(uint32_t b) { return (int)(int8_t)(uint8_t)(b & 0xFFu); }

// Shared-memory descriptor of one digit plane: MN-major, 128-byte swizzle,
// 128 channels (one 128-byte row) x 32 timepoints, 8-row groups 1024 bytes
// apart (stride byte offset); the leading byte offset (the next 128 channels)
// is not reached when the MN extent is one swizzle row.
__device__ __forceinline__ uint64_t plane_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)(kPlaneBytes >> 4) << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// kind::i8 instruction descriptor: S32 accumulator (2), both operands signed
// 8-bit (1) and MN-major, M = N = 128.
constexpr uint32_t kIdescI8 = (2u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) |
                              ((uint32_t)(kB >> 3) << 17) | ((uint32_t)(kB >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %3, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %4, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(accumulate), "r"(kIdescI8)
        : "memory");
}

// One stage of the converter warps: thread (tg, q) turns rows tg and tg + 16
// of each block's fp32 tile (channels 4q .. 4q + 3) into the four digit
// planes; all its loads are issued before the arithmetic.  DIAG: one block
// (bi == bj), whose d2^2 sums go to dsum.
template <int NBLK, bool DIAG>
__device__ __forceinline__ void convert_stage(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int tg,
                                              int q, const float (&m8)[2][4], const float (&mult)[2][4],
                                              int (&dsum)[4]) {
    float4 x[NBLK][2];
#pragma unroll
    for (int b = 0; b < NBLK; b++)
#pragma unroll
        for (int h = 0; h < 2; h++)
            x[b][h] = *reinterpret_cast<const float4*>(src + (size_t)b * kF32Bytes + (tg + 16 * h) * (kB * 4) + q * 16);
#pragma unroll
    for (int b = 0; b < NBLK; b++) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int t = tg + 16 * h;
            uint32_t w[4], lo[4];
            digits4(x[b][h], m8[b], mult[b], w, lo);
            const uint32_t p0 = gather_byte<2>(w);
            const uint32_t p1 = gather_byte<1>(w) ^ 0x80808080u;
            const uint32_t p2 = gather_byte<0>(w) ^ 0x80808080u;
            const uint32_t p3 = gather_byte<0>(lo);
            if (DIAG) {
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const int d2 = sext8(p2 >> (8 * c));
                    dsum[c] += d2 * d2;
                }
            }
            const int r8 = t & 7;
            const size_t off = (size_t)(t >> 3) * 1024 + r8 * 128 + (((q >> 2) ^ r8) << 4) + ((q & 3) << 2);
            uint8_t* pl = dst + (size_t)b * 4 * kPlaneBytes + off;
            *reinterpret_cast<uint32_t*>(pl) = p0;
            *reinterpret_cast<uint32_t*>(pl + kPlaneBytes) = p1;
            *reinterpret_cast<uint32_t*>(pl + 2 * kPlaneBytes) = p2;
            *reinterpret_cast<uint32_t*>(pl + 3 * kPlaneBytes) = p3;
        }
    }
}

struct Item {
    int64_t r;   // run
    int p;       // block pair
    int bi, bj;  // channel blocks
    int nkb;     // K blocks (32 timepoints) in the run
};

__global__ void __launch_bounds__(kThreads, 1)
    cov_i8_kernel(const __grid_constant__ CUtensorMap tmX, int64_t rows, int64_t R, int64_t nruns, int nb, int P,
                  int64_t Mp, const unsigned int* __restrict__ mb, double* __restrict__ partials) {
    int* err = &g_cov_timeout;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* planes = smem;                                             // [kS2][kPlaneStage], 1024-aligned
    uint8_t* f32 = planes + (size_t)kS2 * kPlaneStage;                  // [kS1][kF32Stage]
    int* corr = reinterpret_cast<int*>(f32 + (size_t)kS1 * kF32Stage);  // [2][kB]
    uint64_t* bars = reinterpret_cast<uint64_t*>(corr + 2 * kB);
    uint64_t* f_full = bars;               // [kS1] TMA bytes landed
    uint64_t* f_empty = bars + kS1;        // [kS1] converters done reading
    uint64_t* p_full = bars + 2 * kS1;     // [kS2] planes written
    uint64_t* p_empty = p_full + kS2;      // [kS2] MMAs done reading
    uint64_t* acc_full = p_empty + kS2;    // the run's MMAs complete
    uint64_t* acc_free = acc_full + 1;     // accumulators read back
    uint64_t* corr_ready = acc_free + 1;   // [2] diagonal sums of an item complete
    uint64_t* corr_free = corr_ready + 2;  // [2] diagonal sums read and cleared
    uint64_t* mma_done = corr_free + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t nitems = nruns * P;
    const int64_t my_items = (blockIdx.x < nitems) ? (nitems - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    if (my_items == 0) return;
    auto item_of = [&](int64_t i) {
        Item it;
        const int64_t w = blockIdx.x + i * gridDim.x;
        it.r = w / P;
        it.p = (int)(w % P);
        pair_blocks(it.p, nb, it.bi, it.bj);
        const int64_t len = min(R, rows - it.r * R);
        it.nkb = (int)((len + kKT - 1) / kKT);
        return it;
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < kS1; s++) {
            tc::mbar_init(&f_full[s], 1);
            tc::mbar_init(&f_empty[s], kConvWarps);
        }
        for (int s = 0; s < kS2; s++) {
            tc::mbar_init(&p_full[s], kConvWarps);
            tc::mbar_init(&p_empty[s], 1);
        }
        tc::mbar_init(acc_full, 1);
        tc::mbar_init(acc_free, 4);
        for (int b = 0; b < 2; b++) {
            tc::mbar_init(&corr_ready[b], kConvWarps);
            tc::mbar_init(&corr_free[b], 4);
        }
        tc::mbar_init(mma_done, 1);
        tc::fence_mbar_init();
    }
    for (int k = threadIdx.x; k < 2 * kB; k += blockDim.x) corr[k] = 0;
    if (warp == 1) tc::tmem_alloc(tmem_slot, 512);
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t taddr = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            int64_t g = 0;
            int gs = 0;        // g % kS1
            uint32_t gph = 0;  // (g / kS1) & 1
            bool ok = true;
            for (int64_t i = 0; i < my_items && ok; i++) {
                const Item it = item_of(i);
                const bool diag = it.bi == it.bj;
                for (int kb = 0; kb < it.nkb; kb++, g++) {
                    const int s = gs;
                    if (g >= kS1 && !(ok = tc::mbar_wait(&f_empty[s], gph ^ 1u, err))) break;
                    if (++gs == kS1) {
                        gs = 0;
                        gph ^= 1u;
                    }
                    uint8_t* dst = f32 + (size_t)s * kF32Stage;
                    const int y = (int)(it.r * R + (int64_t)kb * kKT);
                    tc::mbar_expect_tx(&f_full[s], diag ? kF32Bytes : 2 * kF32Bytes);
                    tc::tma_load_2d(dst, &tmX, &f_full[s], it.bi * kB, y);
                    if (!diag) tc::tma_load_2d(dst + kF32Bytes, &tmX, &f_full[s], it.bj * kB, y);
                }
            }
            // no copy may still be landing in shared memory when the CTA exits
            for (int64_t h = (g > kS1 ? g - kS1 : 0); h < g; h++)
                tc::mbar_wait(&f_full[h % kS1], (uint32_t)((h / kS1) & 1), err);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int64_t g = 0;
            int gs = 0;        // g % kS2
            uint32_t gph = 0;  // (g / kS2) & 1
            bool ok = true;
            for (int64_t i = 0; i < my_items && ok; i++) {
                const Item it = item_of(i);
                const bool diag = it.bi == it.bj;
                if (i > 0 && !(ok = tc::mbar_wait(acc_free, (uint32_t)((i - 1) & 1), err))) break;
                tc::tc_fence_after();
                for (int kb = 0; kb < it.nkb; kb++, g++) {
                    const int s = gs;
                    if (!(ok = tc::mbar_wait(&p_full[s], gph, err))) break;
                    if (++gs == kS2) {
                        gs = 0;
                        gph ^= 1u;
                    }
                    tc::tc_fence_after();
                    const uint32_t pa = tc::smem_u32(planes + (size_t)s * kPlaneStage);
                    const uint32_t pb = diag ? pa : pa + 4 * kPlaneBytes;
                    uint64_t a[4], b[4];
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        a[k] = plane_desc(pa + k * kPlaneBytes);
                        b[k] = plane_desc(pb + k * kPlaneBytes);
                    }
                    const uint32_t acc0 = (kb != 0);
                    // a diagonal pair (b = a) skips the transposed halves of
                    // classes 1 and 3 (d1 d0' = (d0 d1')^T, ...): seven MMAs; the
                    // drain and the reduction add the transposes back
                    mma_i8(taddr + 0 * kB, a[0], b[0], acc0);
                    mma_i8(taddr + 1 * kB, a[0], b[1], acc0);
                    if (!diag) mma_i8(taddr + 1 * kB, a[1], b[0], 1);
                    mma_i8(taddr + 2 * kB, a[0], b[2], acc0);
                    mma_i8(taddr + 2 * kB, a[2], b[0], 1);
                    mma_i8(taddr + 2 * kB, a[1], b[1], 1);
                    mma_i8(taddr + 3 * kB, a[0], b[3], acc0);
                    if (!diag) mma_i8(taddr + 3 * kB, a[3], b[0], 1);
                    mma_i8(taddr + 3 * kB, a[1], b[2], 1);
                    if (!diag) mma_i8(taddr + 3 * kB, a[2], b[1], 1);
                    tc::mma_commit(&p_empty[s]);
                }
                if (ok) tc::mma_commit(acc_full);
            }
            // no MMA may still be writing TMEM when it is freed
            tc::mma_commit(mma_done);
            tc::mbar_wait(mma_done, 0, err);
        }
    } else if (warp < 2 + kConvWarps) {
        const int tid = threadIdx.x - 64;
        const int q = tid & 31;   // channel quad within a block: channels 4q .. 4q+3
        const int tg = tid >> 5;  // rows tg and tg + 16 of each stage
        int64_t g = 0;
        int gs = 0;         // g % kS1 (= g % kS2)
        uint32_t gph = 0;   // (g / kS1) & 1
        bool ok = true;
        for (int64_t i = 0; i < my_items && ok; i++) {
            const Item it = item_of(i);
            const bool diag = it.bi == it.bj;
            float mult[2][4], m8[2][4];
#pragma unroll
            for (int b = 0; b < 2; b++) {
                const int64_t c0 = (int64_t)(b ? it.bj : it.bi) * kB + 4 * q;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const int64_t mi = it.r * Mp + c0 + k;
                    int e = MS3_IN_BOUNDS(mi, nruns * Mp, 403) ? run_exponent(__ldg(mb + mi)) : kSentinel;
                    if (e == kSentinel) e = 0;  // digits are garbage; the drain writes NaN for the channel
                    mult[b][k] = __uint_as_float((uint32_t)(157 - e) << 23);  // 2^(30 - e)
                    m8[b][k] = __uint_as_float((uint32_t)(149 - e) << 23);    // 2^(22 - e)
                }
            }
            int dsum[4] = {0, 0, 0, 0};  // sums of d2^2 per channel (diagonal items)
            for (int kb = 0; kb < it.nkb; kb++, g++) {
                const int s1 = gs, s2 = gs;
                ok = tc::mbar_wait(&f_full[s1], gph, err);
                if (ok && g >= kS2) ok = tc::mbar_wait(&p_empty[s2], gph ^ 1u, err);
                if (!__all_sync(0xffffffffu, ok)) {
                    ok = false;
                    break;
                }
                if (++gs == kS1) {  // stage and phase of K-block g + 1
                    gs = 0;
                    gph ^= 1u;
                }
                const uint8_t* src = f32 + (size_t)s1 * kF32Stage;
                uint8_t* dst = planes + (size_t)s2 * kPlaneStage;
                if (diag)
                    convert_stage<1, true>(src, dst, tg, q, m8, mult, dsum);
                else
                    convert_stage<2, false>(src, dst, tg, q, m8, mult, dsum);
                tc::fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) {
                    tc::mbar_arrive(&f_empty[s1]);
                    tc::mbar_arrive(&p_full[s2]);
                }
            }
            if (!ok) break;
            // the item's diagonal sums; corr[i & 1] must have been read for item i - 2
            const int par = (int)(i & 1);
            if (i >= 2) ok = tc::mbar_wait(&corr_free[par], (uint32_t)(((i >> 1) - 1) & 1), err);
            if (!__all_sync(0xffffffffu, ok)) break;
            if (diag) {
#pragma unroll
                for (int c = 0; c < 4; c++) atomicAdd(&corr[par * kB + 4 * q + c], dsum[c]);
            }
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&corr_ready[par]);
        }
    } else {
        // warps 18-21: warp w reads TMEM lanes 32 (w % 4) .. +31 (rows of the tile)
        const int quad = warp & 3;
        const int row = quad * 32 + lane;
        const uint32_t lane_base = (uint32_t)(quad * 32) << 16;
        for (int64_t i = 0; i < my_items; i++) {
            const Item it = item_of(i);
            const int par = (int)(i & 1);
            const bool ok = tc::mbar_wait(acc_full, (uint32_t)(i & 1), err) &&
                            tc::mbar_wait(&corr_ready[par], (uint32_t)((i >> 1) & 1), err);
            if (!__all_sync(0xffffffffu, ok)) break;
            tc::tc_fence_after();
            const int ei = run_exponent(__ldg(mb + it.r * Mp + (int64_t)it.bi * kB + row));
            const bool diag = it.bi == it.bj;
            const int dcorr = corr[par * kB + row];
            corr[par * kB + row] = 0;
            const unsigned int* mbj = mb + it.r * Mp + (int64_t)it.bj * kB;
            double* dst = partials + ((size_t)it.r * P + it.p) * (kB * kB) + (size_t)row * kB;
#pragma unroll 1
            for (int j0 = 0; j0 < kB; j0 += 8) {
                uint32_t a0[8], a1[8], a2[8], a3[8];
                tmem_ld_32x32b_x8(taddr + 0 * kB + lane_base + j0, a0);
                tmem_ld_32x32b_x8(taddr + 1 * kB + lane_base + j0, a1);
                tmem_ld_32x32b_x8(taddr + 2 * kB + lane_base + j0, a2);
                tmem_ld_32x32b_x8(taddr + 3 * kB + lane_base + j0, a3);
#pragma unroll
                for (int jj = 0; jj < 8; jj += 2) {
                    double v[2];
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const int j = j0 + jj + h;
                        const int ej = run_exponent(__ldg(mbj + j));
                        double acc;
                        if (!diag) {
                            acc = (double)(int)a0[jj + h] * 16777216.0 + (double)(int)a1[jj + h] * 65536.0;
                            acc += (double)(int)a2[jj + h] * 256.0 + (double)(int)a3[jj + h];
                        } else {
                            // symmetric classes 0 and 2 (and the d2^2 correction) on and
                            // above the diagonal; the half classes 1 and 3 everywhere, the
                            // diagonal's twice: the reduction adds tile(c, r) to tile(r, c)
                            const double half = (double)(int)a1[jj + h] * 65536.0 + (double)(int)a3[jj + h];
                            double sym = (double)(int)a0[jj + h] * 16777216.0 + (double)(int)a2[jj + h] * 256.0;
                            if (j == row) sym += (double)dcorr * 0.00390625;
                            acc = j > row ? sym + half : (j == row ? sym + 2.0 * half : half);
                        }
                        v[h] = (ei == kSentinel || ej == kSentinel) ? __longlong_as_double(0x7FF8000000000000LL)
                                                                  : acc * pow2d(ei + ej - 36);
                    }
                    if (MS3_IN_BOUNDS((((int64_t)it.r * P + it.p) * (kB * kB) + (int64_t)row * kB + j0 + jj + 1),
                                      nruns * P * (kB * kB), 401))
                        *reinterpret_cast<double2*>(dst + j0 + jj) = make_double2(v[0], v[1]);
                }
            }
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                tc::mbar_arrive(acc_free);
                tc::mbar_arrive(&corr_free[par]);
            }
        }
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc::tc_fence_after();
        tc::tmem_dealloc(taddr, 512);
    }
}

// XXt[i + M j] = XXt[j + M i] = sum over the runs (in order) of the pair's
// tile element, divided by N - 1 when N > 1.
__global__ void cov_i8_reduce(const double* __restrict__ partials, int64_t S, int P, int nb, int64_t M, int64_t N,
                              double* __restrict__ XXt) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)P * kB * kB) return;
    const int p = (int)(idx / (kB * kB));
    const int e = (int)(idx % (kB * kB));
    const int r = e / kB, c = e % kB;
    int bi, bj;
    pair_blocks(p, nb, bi, bj);
    const int64_t i = (int64_t)bi * kB + r, j = (int64_t)bj * kB + c;
    if (i >= M || j >= M) return;
    if (bi == bj && c < r) return;  // the diagonal tile's lower half mirrors its upper half
    double s = 0.0;
    if (bi == bj && c > r) {  // the half classes of the diagonal pair: tile(r, c) + tile(c, r)
        const int et = c * kB + r;
        for (int64_t k = 0; k < S; k++) {
            const double* t = partials + ((size_t)k * P + p) * (kB * kB);
            s += t[e] + t[et];
        }
    } else {
        for (int64_t k = 0; k < S; k++) s += partials[((size_t)k * P + p) * (kB * kB) + e];
    }
    if (N > 1) s /= (double)(N - 1);
    XXt[i + M * j] = s;
    XXt[j + M * i] = s;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn_cov() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    if (!fn) throw_unsupported("cuTensorMapEncodeTiled is not available from the driver");
    return fn;
}

int sm_count_cov() {
    int dev = 0, n = 0;
    MS3_CUDA(cudaGetDevice(&dev));
    MS3_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    return n;
}

}  // namespace

int cov_i8_pairs(int64_t M) {
    const int nb = (int)ceil_div(M, kB);
    return nb * (nb + 1) / 2;
}

int64_t cov_i8_run_length(int64_t M, int64_t rows) {
    // runs of 32768 timepoints (the int32 accumulators cannot overflow), down
    // to 8192 for short recordings so that the items still fill the GPU
    const int64_t P = cov_i8_pairs(M);
    const int64_t sms = sm_count_cov();
    int64_t R = 32768;
    while (R > 8192 && ceil_div(rows, R) * P < sms) R >>= 1;
    return std::max<int64_t>(kKT, std::min<int64_t>(R, ceil_div(std::max<int64_t>(rows, 1), kKT) * kKT));
}

size_t cov_i8_partials_bytes(int64_t M, int64_t runs) {
    return (size_t)runs * cov_i8_pairs(M) * kB * kB * sizeof(double);
}

void cov_i8_partials(const float* X, int64_t M, int64_t r0, int64_t r1, int64_t R, double* partials,
                     cudaStream_t stream) {
    const int64_t rows = r1 - r0;
    if (rows <= 0 || M <= 0) return;
    if (R <= 0 || R % kKT != 0 || R > 32768)
        throw_invalid("covariance run length must be a multiple of 32, at most 32768");
    const float* Xr = X + r0 * M;
    if (M % 4 != 0 || (reinterpret_cast<uintptr_t>(Xr) & 15) != 0)
        throw_invalid("tensor-core covariance needs M % 4 == 0 and 16-byte aligned rows");
    if (rows > 0x7fffffffLL) throw_unsupported("tensor-core covariance: more than 2^31 rows in one call");
    const int nb = (int)ceil_div(M, kB);
    const int P = nb * (nb + 1) / 2;
    const int64_t nruns = ceil_div(rows, R);
    const int64_t Mp = (int64_t)nb * kB;
    DevBuf maxbits(sizeof(unsigned int) * (size_t)(nruns * Mp), stream);
    MS3_CUDA(cudaMemsetAsync(maxbits.get(), 0, sizeof(unsigned int) * (size_t)(nruns * Mp), stream));
    int64_t seg = 1024;  // rows per block of the max pass: a divisor of R
    while (R % seg != 0) seg >>= 1;
    cov_run_maxbits<<<dim3((unsigned)ceil_div(rows, seg), (unsigned)nb), 256, 0, stream>>>(
        Xr, M, rows, R, seg, Mp, maxbits.as<unsigned int>());
    MS3_LAUNCH_CHECK();
    CUtensorMap map;
    const cuuint64_t dims[2] = {(cuuint64_t)M, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)M * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)kB, (cuuint32_t)kKT};
    const cuuint32_t es[2] = {1, 1};
    const CUresult cr = encode_fn_cov()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(Xr), dims,
                                        strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) throw_unsupported("cuTensorMapEncodeTiled failed (" + std::to_string((int)cr) + ")");
    MS3_CUDA(cudaFuncSetAttribute(cov_i8_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes));
    const int64_t nitems = nruns * P;
    const int sms = sm_count_cov();
    // a multiple of P CTAs keeps each CTA on one block pair
    int64_t grid = (P <= sms) ? (int64_t)(sms / P) * P : sms;
    grid = std::min<int64_t>(grid, nitems);
    cov_i8_kernel<<<(unsigned)grid, kThreads, kSmemBytes, stream>>>(map, rows, R, nruns, nb, P, Mp,
                                                                 maxbits.as<unsigned int>(), partials);
    MS3_LAUNCH_CHECK();
}

void cov_i8_finish(const double* partials, int64_t runs, int64_t M, int64_t N, double* XXt, cudaStream_t stream) {
    if (runs == 0) {
        MS3_CUDA(cudaMemsetAsync(XXt, 0, sizeof(double) * (size_t)(M * M), stream));
        return;
    }
    const int nb = (int)ceil_div(M, kB);
    const int P = nb * (nb + 1) / 2;
    const int64_t total = (int64_t)P * kB * kB;
    cov_i8_reduce<<<(unsigned)ceil_div(total, 256), 256, 0, stream>>>(partials, runs, P, nb, M, N, XXt);
    MS3_LAUNCH_CHECK();
}

void covariance_check_timeout(cudaStream_t stream) {
    int h = 0;
    MS3_CUDA(cudaMemcpyFromSymbolAsync(&h, g_cov_timeout, sizeof(int), 0, cudaMemcpyDeviceToHost, stream));
    MS3_CUDA(cudaStreamSynchronize(stream));
    if (h) {
        const int zero = 0;
        MS3_CUDA(cudaMemcpyToSymbolAsync(g_cov_timeout, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, stream));
        MS3_CUDA(cudaStreamSynchronize(stream));
        throw Error(MS3GPU_ERR_CUDA, "tensor-core covariance: pipeline wait timed out");
    }
    whitening_check_timeout(stream);
}

int bounds_site_cov(cudaStream_t s) {
#ifdef MS3GPU_BOUNDS_CHECK
    return take_bounds_site(s);
#else
    (void)s;
    return 0;
#endif
}

}  // namespace ms3gpu
