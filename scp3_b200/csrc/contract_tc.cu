// Split-precision contraction on the 5th-generation tensor cores (tcgen05).
//
//   M_ij += sum_s Phi_i(s) V_s Phi_j(s)       (the -G accumulation,
//                                              ScaledMatrixElements.cpp:951-971)
//
// Operand.  X_i(s) = sqrt|V_s| Phi_i(s), so that X_i X_j = |V_s| Phi_i Phi_j and
// one operand array serves as both A (a 128-row panel) and B (two consecutive
// panels).  Within every 4096-sample block the samples are stably partitioned
// by the sign of V (positive first), each sign group padded to a multiple of
// 16, so a whole K=16 MMA step has one sign; negative steps set the negate-A
// bit of the instruction descriptor.  X is stored split, X = hi + lo in BF16
// (hi = bf16(x), lo = bf16(x - hi)) or FP16 (scaled by 2^6), and every product
// is formed as hi*hi + hi*lo + lo*hi: three kind::f16 MMAs of M = 128, N = 256,
// K = 16 into one FP32 TMEM accumulator.
//
// Operand layout.  The expansion writes X in boxes of 128 rows x 32 K slots
// (8 KB), each already in the 64-byte-swizzled order the MMA descriptors read
// (16-byte chunk c of row r at chunk c ^ ((r >> 1) & 3)), the hi and lo boxes
// of a (row block, k-block) next to each other: [row block][k-block][hi, lo].
// A pipeline stage is five bulk copies (A hi+lo, then B hi and lo of each of
// the two panels), and the expansion's stores are sequential.
//
// Accumulation: see the 128 x 256 kernel below.  Why the FP32 runs are short:
// the tensor core's FP32 accumulation error grows with the number of additions
// into one accumulator, and V carries the cluster's binding energy (~ -0.07 Eh)
// into every element; on the hexamer, 4096-sample FP32 runs in one accumulator
// put ~0.45 cm^-1 into the levels.
//
// Warp roles (320 threads): warp 0 lane 0 issues the bulk copies, warp 1 owns
// TMEM (512 columns) and lane 0 issues the MMAs and commits, warps 2..9 drain
// the accumulator.  Every mbarrier wait is bounded (4 s of %globaltimer); on
// expiry the CTA records an error, stops issuing, waits (bounded) for its own
// loads and MMAs, frees TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "tc.h"

namespace scp3 {
namespace tc {

namespace {

constexpr int kThreads = 320;
constexpr int kEpiWarps = 8;
constexpr unsigned long long kWaitNs = 4000000000ull;

// FP16 operands are stored as 2^6 x; products carry 2^12
constexpr float kF16Scale = 64.0f;
constexpr double kF16Unscale = 1.0 / 4096.0;

#include "tc_ptx.cuh"

// ---------------------------------------------------------------------------
// The single build's contraction: 128 x 256 tiles, one M=128, N=256, K=16 MMA
// per product.  An MMA costs about the same time for N = 128 and N = 256, so
// the wider tile doubles the work per instruction.
//
// Operand: 32-slot boxes in the 64-byte swizzle, [row block][k-block32][hi, lo]
// [128 x 32] (16-byte chunk c of row r at c ^ ((r >> 1) & 3)).  A stage holds
// 32 K slots: A (one row panel, hi + lo, 16 KB) and B (two consecutive panels,
// hi then lo, 32 KB); four stages are in flight.
//
// Tiles: (first A row, first B row, offset of the cluster's sign-group table);
// every needed upper 128 x 128 block is owned by one tile (the tiling and which
// half of a tile owns which block are the host's; a tile may own one half only).  Work unit u = split * ntiles + tile takes the
// tile over k-blocks [split * nkb_pass / nsplit, (split + 1) * nkb_pass /
// nsplit) of the pass (so a shorter pass has shorter units, not fewer); a
// launch covers units [u_begin, u_end), CTA b running
// u_begin + b, u_begin + b + gridDim.x, ... .  Units of one
// wave share k-ranges, so L2 serves the panels they have in common.
//
// Accumulation.  One FP32 TMEM accumulator per tile takes all three products
// (256 columns; two alternate, so a drain overlaps the next run's MMAs).  It is
// drained every 12 k-blocks (384 K slots, 72 MMAs) into FP32 registers of the
// epilogue threads (one row and 128 columns each), which are added into the
// unit's own FP64 partial at the unit's end, and every 256 drains (98304 K slots)
// within longer units.  Longer TMEM runs cost accuracy (the hexamer's 10 lowest
// levels against FP64: 0.049 cm^-1 at 4 k-blocks, 0.054 at 8, 0.063 at 12, 0.073
// at 16) and save drain hand-offs (contraction time -6 % at 8, -9 % at 12).  Each write-back is a read-modify-write of the unit's
// 256 KB partial in HBM, so the fewer the better: at one per unit the hexamer
// pass moves ~0.2 GB of partials per 2^17 samples instead of ~0.5 GB at one per
// 32 drains, with no measurable change in the levels (the FP32 register sums
// of up to 256 runs stay well inside the products' own BF16x3 error).
// (A 128 x 256 tile's FP64 state would not fit beside the operand stages.)
constexpr int kBK2 = 32;
constexpr int kStages2 = 4;
constexpr int kBox2 = kTile * kBK2 * 2;            // 8 KB: one half of one panel
constexpr int kStageBytes2 = 6 * kBox2;            // A hi, A lo, B hi x2, B lo x2
constexpr int kKB2PerFlush = kSlotsPerFlush / kBK2;   // 130
constexpr int kDrain2 = 12;                         // k-blocks per FP32 TMEM run
constexpr int kL2Drains = 256;                      // runs per FP64 flush (at most)
constexpr int kSmemBytes2 = kStages2 * kStageBytes2 + 1024 + 256;
constexpr int kN2 = 2 * kTile;
constexpr uint32_t kIdesc2 = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kN2 >> 3) << 17) |
                             ((uint32_t)(kTile >> 4) << 24);
constexpr uint32_t kIdesc2NegA = kIdesc2 | (1u << 13);
constexpr uint32_t kIdesc2F16 = kIdesc2 & ~((7u << 7) | (7u << 10));
constexpr uint32_t kIdesc2F16NegA = kIdesc2F16 | (1u << 13);

__global__ void __launch_bounds__(kThreads, 1)
    contract_n256_kernel(const uint16_t* __restrict__ xop, long long nkb_alloc, const int4* __restrict__ tiles,
                         int ntiles, int nsplit, int nkb_pass, int u_begin, int u_end,
                         const int* __restrict__ neg_group,
                         int f16, double* __restrict__ partial, int* __restrict__ err_flag)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kStages2 * kStageBytes2);
    uint64_t* full = bars;
    uint64_t* empty = bars + kStages2;
    uint64_t* acc_full = bars + 2 * kStages2;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* drain = acc_empty + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
    volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // k-blocks [lo, hi) of unit u in this pass
    auto krange = [&](int u, int& lo, int& hi) {
        const int split = u / ntiles;
        lo = (int)((long long)split * nkb_pass / nsplit);
        hi = (int)((long long)(split + 1) * nkb_pass / nsplit);
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages2; s++) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(acc_full + a, 1);
            mbar_init(acc_empty + a, kEpiWarps);
        }
        mbar_init(drain, 1);
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    constexpr int kBoxElems = kTile * kBK2;           // 4096 16-bit values per half box

    if (warp == 0) {
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int issued[kStages2] = {0, 0, 0, 0};
            uint32_t issued_phase[kStages2] = {0, 0, 0, 0};
            bool ok = true;
            for (int u = u_begin + blockIdx.x; u < u_end && ok; u += gridDim.x) {
                int lo, hi;
                krange(u, lo, hi);
                const int4 ti = tiles[u % ntiles];
                const uint16_t* pa = xop + (size_t)(ti.x / kTile) * nkb_alloc * (2 * kBoxElems);
                const uint16_t* pb0 = xop + (size_t)(ti.y / kTile) * nkb_alloc * (2 * kBoxElems);
                const uint16_t* pb1 = xop + (size_t)(ti.w / kTile) * nkb_alloc * (2 * kBoxElems);
                for (int kb = lo; kb < hi; kb++) {
                    if (!mbar_wait(empty + stage, phase ^ 1, abort)) {
                        ok = false;
                        break;
                    }
                    uint8_t* st = smem + stage * kStageBytes2;
                    mbar_expect_tx(full + stage, kStageBytes2);
                    const size_t o = (size_t)kb * (2 * kBoxElems);
                    bulk_load(st, pa + o, 2 * kBox2, full + stage);                      // A hi, lo
                    bulk_load(st + 2 * kBox2, pb0 + o, kBox2, full + stage);             // B hi rows 0..127
                    bulk_load(st + 3 * kBox2, pb1 + o, kBox2, full + stage);             // B hi rows 128..255
                    bulk_load(st + 4 * kBox2, pb0 + o + kBoxElems, kBox2, full + stage); // B lo rows 0..127
                    bulk_load(st + 5 * kBox2, pb1 + o + kBoxElems, kBox2, full + stage); // B lo rows 128..255
                    issued[stage] = 1;
                    issued_phase[stage] = phase;
                    if (++stage == kStages2) {
                        stage = 0;
                        phase ^= 1;
                    }
                }
            }
            if (*abort) {
                for (int s = 0; s < kStages2; s++)
                    if (issued[s]) {
                        volatile int never = 0;
                        mbar_wait(full + s, issued_phase[s], &never);
                    }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int stage = 0, use = 0;
            uint32_t phase = 0;
            bool ok = true;
            for (int u = u_begin + blockIdx.x; u < u_end && ok; u += gridDim.x) {
                int lo, hi;
                krange(u, lo, hi);
                const int neg_off = tiles[u % ntiles].z;
                for (int k0 = lo; k0 < hi && ok; k0 += kDrain2, use++) {
                    const int a = use & 1;
                    if (!mbar_wait(acc_empty + a, ((use >> 1) & 1) ^ 1, abort)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d = tmem + (uint32_t)(a * kN2);
                    const int k1 = min(hi, k0 + kDrain2);
                    for (int kb = k0; kb < k1; kb++) {
                        if (!mbar_wait(full + stage, phase, abort)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        uint8_t* st = smem + stage * kStageBytes2;
                        const uint64_t ahi = smem_desc64(st), alo = smem_desc64(st + kBox2);
                        const uint64_t bhi = smem_desc64(st + 2 * kBox2), blo = smem_desc64(st + 4 * kBox2);
                        const int f = kb / kKB2PerFlush;
                        const int neg0 = neg_group[neg_off + f];
                        const int ks0 = (kb - f * kKB2PerFlush) * (kBK2 / 16);
#pragma unroll
                        for (int kk = 0; kk < kBK2 / 16; kk++) {
                            const bool neg = ks0 + kk >= neg0;
                            const uint32_t idesc =
                                f16 ? (neg ? kIdesc2F16NegA : kIdesc2F16) : (neg ? kIdesc2NegA : kIdesc2);
                            const uint64_t adv = (uint64_t)(kk * 2);    // 32 B along K inside the 64 B atom
                            const uint32_t acc = (kb != k0) | (kk != 0);
                            mma_bf16(d, ahi + adv, bhi + adv, idesc, acc);
                            mma_bf16(d, ahi + adv, blo + adv, idesc, 1);
                            mma_bf16(d, alo + adv, bhi + adv, idesc, 1);
                        }
                        mma_commit(empty + stage);
                        if (++stage == kStages2) {
                            stage = 0;
                            phase ^= 1;
                        }
                    }
                    if (ok) mma_commit(acc_full + a);
                }
            }
            mma_commit(drain);
            volatile int never = 0;
            mbar_wait(drain, 0, &never);
        }
    } else {
        // epilogue: warp w reads TMEM lane quadrant w % 4 and column half (w - 2) / 4
        const int quad = warp & 3, half = (warp - 2) >> 2;
        const int row = quad * 32 + lane;
        const double unscale = f16 ? kF16Unscale : 1.0;
        float l2[kTile];
#pragma unroll
        for (int j = 0; j < kTile; j++) l2[j] = 0.f;
        int use = 0;
        bool ok = true;
        for (int u = u_begin + blockIdx.x; u < u_end && ok; u += gridDim.x) {
            int lo, hi;
            krange(u, lo, hi);
            const int nruns = (hi - lo + kDrain2 - 1) / kDrain2;
            double* P = partial + (size_t)u * (size_t)(kTile * kN2);
            for (int k = 0; k < nruns; k++, use++) {
                const int a = use & 1;
                if (!mbar_wait(acc_full + a, (use >> 1) & 1, abort)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t base = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(a * kN2 + half * kTile);
#pragma unroll
                for (int c0 = 0; c0 < kTile; c0 += 32) {
                    float v[32];
                    tmem_ld32(base + c0, v);
#pragma unroll
                    for (int j = 0; j < 32; j++) l2[c0 + j] += v[j];
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(acc_empty + a);
                if (k % kL2Drains == kL2Drains - 1 || k == nruns - 1) {
#pragma unroll
                    for (int j = 0; j < kTile; j++) {
                        P[(size_t)(half * kTile + j) * kTile + row] += (double)l2[j] * unscale;
                        l2[j] = 0.f;
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && *abort) atomicExch(err_flag, 1);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
    }
}

// Dense column-major nb x nb from the 128 x 256 tiles' unit partials: element
// (r <= c) lies in block (r / 128, c / 128), owned by tile t at column half h,
// as itself or transposed (block_owner = 4 t + 2 transposed + h); its value is
// the sum over the splits, in order, of unit (split * ntiles + t) at row
// r % 128 and column 128 h + c % 128 (transposed: row c % 128, column
// 128 h + r % 128).
__global__ void unpack_n256_kernel(const double* __restrict__ partial, const int* __restrict__ block_owner, int nt,
                                   int ntiles, int nsplit, int nb, double divisor, const double* __restrict__ diag,
                                   double zpe, double* __restrict__ M, int64_t ld)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)nb * nb) return;
    const int j = (int)(e / nb), i = (int)(e - (int64_t)j * nb);
    const int r = min(i, j), c = max(i, j);
    const int ti = r / kTile, tj = c / kTile;
    const int own = block_owner[ti * nt + tj];
    const int t = own >> 2, h = own & 1;
    const int rr = r - ti * kTile, cc = c - tj * kTile;
    const size_t off = (own & 2) ? (size_t)(h * kTile + rr) * kTile + cc : (size_t)(h * kTile + cc) * kTile + rr;
    double val = 0.0;
    for (int s = 0; s < nsplit; s++) val += partial[((size_t)s * ntiles + t) * (size_t)(kTile * kN2) + off];
    val = val / divisor;
    if (diag && i == j) val = (val + diag[i]) + zpe;
    M[(size_t)j * ld + i] = val;
}

// One CTA of 1024 threads per 4096-sample block (4 samples per thread): stable
// partition of its samples by the sign of V into K slots; writes slot -> sample
// (-1 = zero padding) and the first negative 16-group of the block.
__global__ void __launch_bounds__(1024) partition_kernel(const double* __restrict__ v, int* __restrict__ sample_of_slot,
                                                         int* __restrict__ neg_group, int64_t v_stride,
                                                         int64_t slot_stride, int neg_stride)
{
    static_assert(kFlush == 4096, "four samples per thread");
    __shared__ int wpos[32], tot;
    const int b = blockIdx.x, t = threadIdx.x, lane = t & 31, w = t >> 5;
    v += blockIdx.y * v_stride;              // cluster blockIdx.y of a batch
    sample_of_slot += blockIdx.y * slot_stride;
    neg_group += blockIdx.y * neg_stride;
    const int64_t s0 = (int64_t)b * kFlush + 4 * t;
    int flags = 0, np = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const bool pos = !(v[s0 + k] < 0.0);
        flags |= (int)pos << k;
        np += pos;
    }
    int incl = np;     // inclusive warp scan of positives
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wpos[w] = incl;
    __syncthreads();
    if (w == 0) {
        const int c = wpos[lane];
        int x = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        wpos[lane] = x - c;      // exclusive
        if (lane == 31) tot = x;
    }
    __syncthreads();
    const int P = tot, P16 = (P + 15) & ~15, N = kFlush - P;
    int op = wpos[w] + incl - np;           // positives before this thread's samples
    int on = 4 * t - op;                    // negatives before them
    int* out = sample_of_slot + (size_t)b * kSlotsPerFlush;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if ((flags >> k) & 1) out[op++] = (int)(s0 + k);
        else out[P16 + on++] = (int)(s0 + k);
    }
    for (int sl = t; sl < kSlotsPerFlush; sl += 1024)
        if ((sl >= P && sl < P16) || sl >= P16 + N) out[sl] = -1;
    if (t == 0) neg_group[b] = P16 / 16;
}

// Expansion into the split operand X = sqrt|V| Phi (hi + lo halves).
//
// Work unit: one k-block (64 K slots) x one chunk of kExpChunk basis rows of one
// cluster.  Units are numbered cluster by cluster, k-block-major, and a
// persistent grid (as many CTAs as the SMs hold at once) gives each CTA one
// contiguous, balanced range of them, so there is no tail wave and a CTA
// rebuilds its table only when its k-block changes.
//
// Per k-block the CTA tabulates, per slot, [1, h1(q_m), h2(q_m), h3(q_m)] for
// all modes in shared memory; every basis value is then the product of three
// table entries (basis_factor_table).  Thread (g, r) handles slots 8g..8g+7 of
// rows 4r..4r+3, 4r+128..4r+131, ...: two 16-byte table reads per factor (the
// table's columns are permuted so these are conflict-free; a first factor shared
// with the previous row is not read again) and one 16-byte store per half, so
// the 8 threads of a row write its 128 contiguous bytes.  While a
// k-block's rows are written, its successor's q rows and V values are already
// in flight into a staging area (cp.async), so the table build that follows
// does not wait on the gathers; when the staging area does not fit next to the
// table (very many modes) the gathers are made at build time instead.
constexpr int kExpSlots = 64, kExpChunk = 256, kExpThreads = 256;

// x = hi + lo for two values, each half packed in one 32-bit word (the first
// value in the low 16 bits): hi = round(x), lo = round(x - hi), round-to-nearest.
template <bool F16>
__device__ __forceinline__ void split2(float x0, float x1, uint32_t& hi, uint32_t& lo)
{
    if (F16) {
        const __half2 h = __floats2half2_rn(x0, x1);
        const float2 hf = __half22float2(h);
        const __half2 l = __floats2half2_rn(x0 - hf.x, x1 - hf.y);
        hi = *reinterpret_cast<const uint32_t*>(&h);
        lo = *reinterpret_cast<const uint32_t*>(&l);
    } else {
        const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
        const float2 hf = __bfloat1622float2(h);
        const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
        hi = *reinterpret_cast<const uint32_t*>(&h);
        lo = *reinterpret_cast<const uint32_t*>(&l);
    }
}

// Table column of K slot l (0..63): slots 8g..8g+3 at columns 4g..4g+3 and slots
// 8g+4..8g+7 at 32+4g..32+4g+3, so the 8 threads of a row, thread g taking
// slots 8g..8g+7, read two contiguous 128-byte spans (no bank conflict).
__device__ __forceinline__ int tab_col(int l) { return ((l >> 3) << 2) | (l & 3) | ((l & 4) << 3); }
__device__ __forceinline__ int tab_slot(int c) { return (((c & 31) >> 2) << 3) | (c & 3) | ((c >> 5) << 2); }

__device__ __forceinline__ void cp_async(void* dst, const void* src, int bytes, bool valid)
{
    // zero-filled (nothing read) when !valid; src is then any mapped address
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    const int n = valid ? bytes : 0;
    if (bytes == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
    else if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Shared memory of the expansion (floats): table [3nm+1][64], sqrt|V| [64], and
// when staged, q [nm][64] (in 4-mode groups when nm % 4 == 0) and V [64] (doubles).
__host__ __device__ inline size_t expand_smem(int nm, bool staged)
{
    size_t f = (size_t)(3 * nm + 1) * kExpSlots + kExpSlots;
    if (staged) f += (size_t)nm * kExpSlots + 2 * kExpSlots;
    return f * sizeof(float);
}

// The operand is written as 32-slot boxes in the 64-byte swizzle (nkb counts
// 32-slot k-blocks per row block).
template <bool F16>
__global__ void __launch_bounds__(kExpThreads, 3) expand_split_kernel(const ExpandDesc* __restrict__ descs, int ncl,
                                                                    int64_t nkbp, int64_t nkb, int staged,
                                                                    uint16_t* __restrict__ xop)
{
    extern __shared__ __align__(16) float smem_f[];
    const int t = threadIdx.x;
    // units of the whole launch and this CTA's range
    int64_t utot = 0;
    for (int z = 0; z < ncl; z++) utot += nkbp * ((descs[z].nb_pad + kExpChunk - 1) / kExpChunk);
    const int64_t u0 = utot * blockIdx.x / gridDim.x, u1 = utot * (blockIdx.x + 1) / gridDim.x;
    if (u0 >= u1) return;
    int max_nm = 0;
    for (int z = 0; z < ncl; z++) max_nm = max(max_nm, descs[z].nm);
    float* tab = smem_f;                                         // [3 nm + 1][64]
    float* sv = tab + (size_t)(3 * max_nm + 1) * kExpSlots;     // [64]
    float* stq = sv + kExpSlots;                                 // [nm][64] staged q
    double* stv = reinterpret_cast<double*>(stq + (size_t)max_nm * kExpSlots);   // [64] staged V

    // Group: the units of one (cluster, k-block) inside [u0, u1).
    struct Group {
        int z;
        int64_t kb;
        int r0, r1;     // basis rows [r0, r1) of the cluster
    };
    int zc = 0;
    int64_t pre = 0;    // first unit of cluster zc
    auto group_at = [&](int64_t u) {
        for (;;) {
            const int64_t nu = nkbp * ((descs[zc].nb_pad + kExpChunk - 1) / kExpChunk);
            if (u < pre + nu) break;
            pre += nu;
            zc++;
        }
        const int nrc = (descs[zc].nb_pad + kExpChunk - 1) / kExpChunk;
        const int64_t w = u - pre;
        Group g;
        g.z = zc;
        g.kb = w / nrc;
        const int rc = (int)(w - g.kb * nrc);
        const int64_t gend = min(u1, pre + (g.kb + 1) * nrc);      // first unit after the group
        g.r0 = rc * kExpChunk;
        g.r1 = min((int)(rc + (gend - u)) * kExpChunk, descs[zc].nb_pad);
        return g;
    };
    // gathers of a group's q rows and V into the staging area
    auto issue = [&](const Group& g) {
        const ExpandDesc d = descs[g.z];
        const int64_t slot0 = g.kb * kExpSlots;
        const bool vec = (d.nm & 3) == 0;
        const int nv = vec ? d.nm >> 2 : d.nm;
        for (int e = t; e < (nv + 1) * kExpSlots; e += kExpThreads) {
            const int l = e & (kExpSlots - 1), k = e >> 6;
            const int s = d.slot_of[slot0 + l];
            if (k == nv) cp_async(stv + l, d.v + (s >= 0 ? s : 0), 8, s >= 0);
            else if (vec) cp_async(stq + (size_t)e * 4, d.q + (int64_t)(s >= 0 ? s : 0) * d.nm + 4 * k, 16, s >= 0);
            else cp_async(stq + e, d.q + (int64_t)(s >= 0 ? s : 0) * d.nm + k, 4, s >= 0);
        }
    };
    // the table of a group: from the staging area, or (unstaged) gathered here;
    // slot l goes to table column tab_col(l)
    auto build = [&](const Group& g) {
        const ExpandDesc d = descs[g.z];
        const int nm = d.nm;
        const int64_t slot0 = g.kb * kExpSlots;
        auto put = [&](int c, int m, float y) {
            tab[(1 + m) * kExpSlots + c] = 1.41421356f * y;                                  // ho1
            tab[(1 + nm + m) * kExpSlots + c] = (2.0f * y * y - 1.0f) * 0.70710678f;          // ho2
            tab[(1 + 2 * nm + m) * kExpSlots + c] = (2.0f * y * y - 3.0f) * y * 0.57735027f;  // ho3
        };
        for (int c = t; c < kExpSlots; c += kExpThreads) {
            const int l = tab_slot(c);
            tab[c] = 1.0f;
            double vv;
            if (staged) {
                vv = stv[l];
            } else {
                const int s = d.slot_of[slot0 + l];
                vv = s >= 0 ? d.v[s] : 0.0;
            }
            sv[c] = (float)sqrt(fabs(vv)) * (F16 ? kF16Scale : 1.0f);
        }
        if ((nm & 3) == 0) {
            const int n4 = nm >> 2;
            for (int e = t; e < n4 * kExpSlots; e += kExpThreads) {
                const int c = e & (kExpSlots - 1), m4 = e >> 6, l = tab_slot(c);
                float4 y;
                if (staged) {
                    y = reinterpret_cast<const float4*>(stq)[m4 * kExpSlots + l];
                } else {
                    const int s = d.slot_of[slot0 + l];
                    y = s >= 0 ? reinterpret_cast<const float4*>(d.q + (int64_t)s * nm)[m4]
                               : make_float4(0.f, 0.f, 0.f, 0.f);
                }
                put(c, 4 * m4, y.x), put(c, 4 * m4 + 1, y.y), put(c, 4 * m4 + 2, y.z), put(c, 4 * m4 + 3, y.w);
            }
        } else {
            for (int e = t; e < nm * kExpSlots; e += kExpThreads) {
                const int c = e & (kExpSlots - 1), m = e >> 6, l = tab_slot(c);
                float y;
                if (staged) {
                    y = stq[m * kExpSlots + l];
                } else {
                    const int s = d.slot_of[slot0 + l];
                    y = s >= 0 ? d.q[(int64_t)s * nm + m] : 0.0f;
                }
                put(c, m, y);
            }
        }
    };

    const int g8 = t & 7, rl = t >> 3;
    constexpr int kStep = kExpThreads / 8;                 // rows per trip of the CTA
    constexpr uint32_t kNone = 0xffffffffu;                // rows beyond nb (zero padding); real factors < 2^30
    Group cur = group_at(u0);
    if (staged) {
        issue(cur);
        cp_async_wait_all();
        __syncthreads();
    }
    build(cur);
    __syncthreads();
    for (;;) {
        const int64_t nxt_u = pre + (cur.kb + 1) * ((descs[cur.z].nb_pad + kExpChunk - 1) / kExpChunk);
        const bool more = nxt_u < u1;
        Group nxt{};
        if (more) {
            nxt = group_at(nxt_u);
            if (staged) issue(nxt);
        }
        // rows [r0, r1) of (cluster, k-block)
        {
            const uint32_t* __restrict__ factors = descs[cur.z].factors;
            const int nb = descs[cur.z].nb, row0 = descs[cur.z].row0;
            const float4* tab4 = reinterpret_cast<const float4*>(tab);
            const float4 w0 = reinterpret_cast<const float4*>(sv)[g8];
            const float4 w1 = reinterpret_cast<const float4*>(sv)[g8 + 8];
            // rows past nb stay as the operand's allocation zeroed them
            const int rend = min(cur.r1, nb);
            // thread rl takes 4 consecutive rows per trip: consecutive rows mostly share
            // their first factor (pairs (m, n), (m, n + 1), ...), read once
            for (int r = cur.r0 + 4 * rl; r < rend; r += 4 * kStep) {
                uint32_t f[4];
#pragma unroll
                for (int u = 0; u < 4; u++) f[u] = r + u < rend ? __ldg(factors + r + u) : kNone;
                uint32_t pia = 0xffffffffu;
                float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = a0;
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int rr = r + u;
                    if (rr >= rend) break;
                    uint4 hi = make_uint4(0, 0, 0, 0), lo = hi;
                    if (f[u] != kNone) {
                        // factor 0 is the constant 1: not read (most rows have one or two)
                        const uint32_t ia = f[u] & 1023u, ib = (f[u] >> 10) & 1023u, ic = f[u] >> 20;
                        if (ia != pia) {
                            a0 = tab4[ia * (kExpSlots / 4) + g8];
                            a1 = tab4[ia * (kExpSlots / 4) + g8 + 8];
                            pia = ia;
                        }
                        const float4 one = make_float4(1.f, 1.f, 1.f, 1.f);
                        float4 b0 = one, b1 = one, c0 = one, c1 = one;
                        if (ib) b0 = tab4[ib * (kExpSlots / 4) + g8], b1 = tab4[ib * (kExpSlots / 4) + g8 + 8];
                        if (ic) c0 = tab4[ic * (kExpSlots / 4) + g8], c1 = tab4[ic * (kExpSlots / 4) + g8 + 8];
                        split2<F16>(w0.x * (a0.x * b0.x * c0.x), w0.y * (a0.y * b0.y * c0.y), hi.x, lo.x);
                        split2<F16>(w0.z * (a0.z * b0.z * c0.z), w0.w * (a0.w * b0.w * c0.w), hi.y, lo.y);
                        split2<F16>(w1.x * (a1.x * b1.x * c1.x), w1.y * (a1.y * b1.y * c1.y), hi.z, lo.z);
                        split2<F16>(w1.z * (a1.z * b1.z * c1.z), w1.w * (a1.w * b1.w * c1.w), hi.w, lo.w);
                    }
                    // 32-slot box (row block, 2 k-block + g8 / 4): chunk c of row rin at c ^ ((rin >> 1) & 3)
                    const int row = row0 + rr, rin = row & (kTile - 1), c = g8 & 3;
                    uint16_t* box = xop + ((size_t)(row / kTile) * nkb + 2 * cur.kb + (g8 >> 2)) * (2 * kTile * kBK2);
                    const int off = rin * kBK2 + ((c ^ ((rin >> 1) & 3)) << 3);
                    *reinterpret_cast<uint4*>(box + off) = hi;
                    *reinterpret_cast<uint4*>(box + kTile * kBK2 + off) = lo;
                }
            }
        }
        if (!more) break;
        if (staged) cp_async_wait_all();
        __syncthreads();          // every row of cur written: the table is free
        build(nxt);
        __syncthreads();
        cur = nxt;
    }
}

void record(std::vector<cudaEvent_t>* pev, std::vector<int>* pkind, int kind, cudaStream_t s)
{
    if (!pev) return;
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    cudaEventRecord(e, s);
    pev->push_back(e);
    pkind->push_back(kind);
}

}  // namespace

// The 128 x 256 tiling of a cluster's upper block triangle: blocks
// {ti, tj} of 128 x 128, ti <= tj < nt_need, each needed once.  A tile is one A
// panel p against two B panels (q, r) and yields blocks (p, q) and (p, r); a
// block (p, q) with q < p is the transpose of the needed block (q, p), so the
// read-out takes it transposed.  Which panel plays A for block {i, j} is an
// orientation of the complete graph on the panels (with a loop per panel):
// panel i starts with the blocks j >= i (nt_need - i of them), panels with an
// odd count are paired in order and each pair's block moves to the later
// panel, so at most one panel keeps an odd count.  Each panel's blocks, in
// column order, pair up into tiles; an odd one out makes a one-half tile (both
// B panels the same).  That is ceil(nt_need (nt_need + 1) / 4) tiles, the
// fewest that cover the triangle (55 blocks on 10 panels: 28 tiles, where
// aligned column pairs need 30).  Tiles come in 12-row x 6-pair groups so that
// a wave of CTAs shares panels.
void add_cluster_tiles(std::vector<BaseTile>& base, int cluster, int nt, int nt_need, int row0, int neg_off)
{
    (void)nt;
    const int n = nt_need;
    std::vector<std::vector<int>> cols(n);       // B panels of A panel p; negative = transposed, ~q
    for (int i = 0; i < n; i++)
        for (int j = i; j < n; j++) cols[i].push_back(j);
    int odd = -1;
    for (int i = 0; i < n; i++) {
        if ((n - i) % 2 == 0) continue;
        if (odd < 0) {
            odd = i;
            continue;
        }
        // block {odd, i}: from panel odd's list to panel i's, transposed
        std::vector<int>& a = cols[odd];
        a.erase(std::find(a.begin(), a.end(), i));
        std::vector<int>& b = cols[i];
        b.insert(std::lower_bound(b.begin(), b.end(), odd,
                                  [](int x, int v) { return (x < 0 ? ~x : x) < v; }),
                 ~odd);
        odd = -1;
    }
    const int R = 12, C = 6;
    int maxp = 0;
    for (int i = 0; i < n; i++) maxp = std::max(maxp, (int)(cols[i].size() + 1) / 2);
    for (int r0 = 0; r0 < n; r0 += R)
        for (int c0 = 0; c0 < maxp; c0 += C)
            for (int ti = r0; ti < std::min(r0 + R, n); ti++)
                for (int k = c0; k < std::min(c0 + C, maxp); k++) {
                    const std::vector<int>& l = cols[ti];
                    if (2 * k >= (int)l.size()) continue;
                    const int a = l[2 * k];
                    const bool two = 2 * k + 1 < (int)l.size();
                    const int b = two ? l[2 * k + 1] : a;
                    BaseTile t;
                    t.cluster = cluster;
                    t.ti = ti;
                    t.s0 = a < 0 ? ~a : a;
                    t.s1 = b < 0 ? ~b : b;
                    t.halves = two ? 3 : 1;
                    t.tr = (a < 0 ? 1 : 0) | (two && b < 0 ? 2 : 0);
                    t.row0 = row0;
                    t.neg_off = neg_off;
                    base.push_back(t);
                }
}

// Chooses the number of tiles (the base tiling, with some pairs split into two
// one-half tiles) and of splits, minimising waves / splits -- the contraction
// time in units of one whole-pass tile -- over at most 16 splits and 4 GB of
// partials; emits the tiles and, per cluster, owner[ti * nt + tj] (ti <= tj) =
// 4 tile + 2 transposed + half.
void finish_tiling(const std::vector<BaseTile>& base, const std::vector<int>& cluster_nt, int sms,
                   std::vector<int4>& tiles, std::vector<std::vector<int>>& owner, int& nsplit)
{
    const int tmin = (int)base.size();
    int pairs = 0;
    for (const BaseTile& t : base) pairs += t.halves == 3;
    double best = 1e30;
    int bestT = tmin, bestM = 1;
    long long bestU = 0;
    for (int m = 1; m <= 16; m++)
        for (int T = tmin; T <= tmin + pairs; T++) {
            const long long units = (long long)T * m;
            if (units * (long long)(kTile * kN2) * 8 > (4ll << 30)) continue;
            const double cost = (double)((units + sms - 1) / sms) / m;
            if (cost < best - 1e-12 || (cost < best + 1e-12 && units < bestU)) {
                best = cost;
                bestT = T;
                bestM = m;
                bestU = units;
            }
        }
    tiles.clear();
    owner.assign(cluster_nt.size(), {});
    for (size_t c = 0; c < cluster_nt.size(); c++) owner[c].assign((size_t)cluster_nt[c] * cluster_nt[c], -1);
    // the block that half h of tile `index` yields, owned by that tile
    auto own = [&](const BaseTile& t, int h, int index, int half_in_tile) {
        const int nt = cluster_nt[t.cluster];
        const int s = h ? t.s1 : t.s0;
        const int tr = (t.tr >> h) & 1;
        const int r = tr ? s : t.ti, c = tr ? t.ti : s;
        owner[t.cluster][(size_t)r * nt + c] = 4 * index + 2 * tr + half_in_tile;
    };
    int extra = bestT - tmin;
    for (const BaseTile& t : base) {
        const int a = t.row0 + t.ti * kTile;
        if (t.halves == 3 && extra > 0) {
            extra--;
            for (int h = 0; h < 2; h++) {
                const int b = t.row0 + (h ? t.s1 : t.s0) * kTile;
                own(t, h, (int)tiles.size(), 0);
                tiles.push_back(make_int4(a, b, t.neg_off, b));
            }
            continue;
        }
        for (int h = 0; h < 2; h++)
            if (t.halves & (1 << h)) own(t, h, (int)tiles.size(), h);
        tiles.push_back(make_int4(a, t.row0 + t.s0 * kTile, t.neg_off, t.row0 + t.s1 * kTile));
    }
    nsplit = bestM;
}

int launch_contract(const uint16_t* x, int64_t nkb_alloc, const int4* tiles, int ntiles, int nsplit, int nkb_pass,
                    const int* neg, bool f16, double* partial, int* err_flag, int grid, cudaStream_t s,
                    int u_begin, int u_end)
{
    if (u_end < 0) u_end = ntiles * nsplit;
    if (ntiles <= 0 || nsplit <= 0 || grid <= 0 || u_end <= u_begin) return SCP3GPU_OK;
    SCP3_CUDA(cudaFuncSetAttribute(contract_n256_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes2));
    contract_n256_kernel<<<grid, kThreads, kSmemBytes2, s>>>(x, (long long)nkb_alloc, tiles, ntiles, nsplit, nkb_pass,
                                                             u_begin, u_end, neg, (int)f16, partial,
                                                             err_flag);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

int launch_unpack(const double* partial, const int* owner, int nt, int ntiles, int nsplit, int nb, double divisor,
                   const double* diag, double zpe, double* M, int64_t ld, cudaStream_t s)
{
    const int64_t total = (int64_t)nb * nb;
    if (total <= 0) return SCP3GPU_OK;
    unpack_n256_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(partial, owner, nt, ntiles, nsplit, nb, divisor,
                                                                      diag, zpe, M, ld);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

int create(Plan& p, int nb, int nm, int n2_for_factors, int n3_for_factors, int chunk_req, int sms, bool f16)
{
    const int nm_for_factors = nm;
    p.f16 = f16;
    p.nb = nb;
    p.nm = nm;
    p.nb_pad = (nb + kN2 - 1) / kN2 * kN2;         // whole 256-row panel pairs
    p.nt = p.nb_pad / kTile;
    // 2^18 samples per pass by default: each work unit ends with a read-modify-write
    // of its FP64 partial, so longer passes spread that over more samples
    int64_t chunk = chunk_req > 0 ? chunk_req : (int64_t)kFlush * 64;
    // the split operand of one pass stays under ~6 GB
    while (chunk > kFlush && (int64_t)p.nb_pad * (chunk / kFlush) * kSlotsPerFlush * 4 > (6ll << 30)) chunk /= 2;
    chunk = chunk / kFlush * kFlush;
    p.chunk = chunk;
    const int nflush = (int)(chunk / kFlush);
    p.slots = (int64_t)nflush * kSlotsPerFlush;
    std::vector<BaseTile> base;
    add_cluster_tiles(base, 0, p.nt, (nb + kTile - 1) / kTile, 0, 0);
    std::vector<int4> tiles;
    std::vector<std::vector<int>> owners;
    finish_tiling(base, std::vector<int>{p.nt}, sms, tiles, owners, p.nsplit);
    const std::vector<int>& owner = owners[0];
    p.ntiles = (int)tiles.size();
    p.grid = (int)std::min<long long>((long long)p.ntiles * p.nsplit, sms);
    for (int b = 0; b < 2; b++) {
        SCP3_CUDA(cudaMalloc(&p.x[b], sizeof(uint16_t) * 2 * (size_t)p.nb_pad * p.slots));
        // padding rows (nb..nb_pad) are never written by the expansion: zero once
        SCP3_CUDA(cudaMemset(p.x[b], 0, sizeof(uint16_t) * 2 * (size_t)p.nb_pad * p.slots));
        SCP3_CUDA(cudaMalloc(&p.slot_of[b], sizeof(int) * (size_t)p.slots));
        SCP3_CUDA(cudaMalloc(&p.group_meta[b], sizeof(int) * nflush));
    }
    SCP3_CUDA(cudaMalloc(&p.tiles2, sizeof(int4) * tiles.size()));
    SCP3_CUDA(cudaMemcpy(p.tiles2, tiles.data(), sizeof(int4) * tiles.size(), cudaMemcpyHostToDevice));
    const std::vector<uint32_t> fac = basis_factor_table(nm_for_factors, n2_for_factors, n3_for_factors);
    SCP3_CUDA(cudaMalloc(&p.factors, sizeof(uint32_t) * fac.size()));
    SCP3_CUDA(cudaMemcpy(p.factors, fac.data(), sizeof(uint32_t) * fac.size(), cudaMemcpyHostToDevice));
    SCP3_CUDA(cudaMalloc(&p.desc_dev, sizeof(ExpandDesc) * 2));
    SCP3_CUDA(cudaMalloc(&p.tile_index, sizeof(int) * owner.size()));
    SCP3_CUDA(cudaMemcpy(p.tile_index, owner.data(), sizeof(int) * owner.size(), cudaMemcpyHostToDevice));
    SCP3_CUDA(cudaMalloc(&p.partial, sizeof(double) * (size_t)p.nsplit * p.ntiles * kTile * kN2));
    SCP3_CUDA(cudaMalloc(&p.err_flag, sizeof(int)));
    SCP3_CUDA(cudaMemset(p.err_flag, 0, sizeof(int)));
    SCP3_CUDA(cudaFuncSetAttribute(contract_n256_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes2));
    return SCP3GPU_OK;
}

void destroy(Plan& p)
{
    void* ptrs[] = {p.x[0], p.x[1], p.slot_of[0], p.slot_of[1], p.group_meta[0],
                    p.group_meta[1], p.tiles2, p.tile_index, p.factors, p.partial, p.err_flag, p.desc_dev};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    p = Plan{};
}

int64_t pass_samples(const Plan& p, int64_t nvalid)
{
    (void)p;
    return (nvalid + kFlush - 1) / kFlush * kFlush;
}

int zero(Plan& p, cudaStream_t s)
{
    SCP3_CUDA(cudaMemsetAsync(p.partial, 0, sizeof(double) * (size_t)p.nsplit * p.ntiles * kTile * kN2, s));
    SCP3_CUDA(cudaMemsetAsync(p.err_flag, 0, sizeof(int), s));
    return SCP3GPU_OK;
}

int launch_partition(const double* v, int64_t v_stride, int* slot_of, int64_t slot_stride, int* neg, int neg_stride,
                     int nflush, int nclusters, cudaStream_t s)
{
    partition_kernel<<<dim3(nflush, nclusters), 1024, 0, s>>>(v, slot_of, neg, v_stride, slot_stride, neg_stride);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

int launch_expand(const ExpandDesc* descs_dev, int nclusters, int max_nb_pad, int max_nm, int64_t slots, int64_t nkb,
                  uint16_t* x, bool f16, cudaStream_t s)
{
    constexpr size_t kMaxSmem = 227 * 1024;
    const bool staged = expand_smem(max_nm, true) <= kMaxSmem;
    const size_t sm = expand_smem(max_nm, staged);
    auto kern = f16 ? expand_split_kernel<true> : expand_split_kernel<false>;
    if (sm > 48 * 1024) SCP3_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int dev = 0, sms = 148, per = 0;
    SCP3_CUDA(cudaGetDevice(&dev));
    SCP3_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    SCP3_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kExpThreads, sm));
    const int64_t nkbp = slots / kExpSlots;
    const int64_t units_max = nkbp * nclusters * ((max_nb_pad + kExpChunk - 1) / kExpChunk);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)std::max(per, 1) * sms, units_max));
    kern<<<grid, kExpThreads, sm, s>>>(descs_dev, nclusters, nkbp, nkb, staged ? 1 : 0, x);
    SCP3_CUDA(cudaGetLastError());
    return SCP3GPU_OK;
}

int prepare(Plan& p, int buf, int nb, int nm, const float* q32, const double* v, int64_t n, cudaStream_t s,
            std::vector<cudaEvent_t>* pev, std::vector<int>* pkind)
{
    if (n % kFlush != 0 || n > p.chunk || buf < 0 || buf > 1)
        return fail(SCP3GPU_ERR_ARG, "tc pass: sample count not in flush blocks");
    const int nflush = (int)(n / kFlush);
    const int64_t slots = (int64_t)nflush * kSlotsPerFlush;
    record(pev, pkind, 1, s);
    int rc = launch_partition(v, 0, p.slot_of[buf], 0, p.group_meta[buf], 0, nflush, 1, s);
    if (rc) return rc;
    const ExpandDesc d{p.factors, nb, p.nb_pad, nm, 0, q32, v, p.slot_of[buf]};
    if (std::memcmp(&d, &p.desc_host[buf], sizeof(d)) != 0) {
        // pageable source: the copy has read it when the call returns
        SCP3_CUDA(cudaMemcpyAsync(p.desc_dev + buf, &d, sizeof(d), cudaMemcpyHostToDevice, s));
        p.desc_host[buf] = d;
    }
    rc = launch_expand(p.desc_dev + buf, 1, p.nb_pad, nm, slots, p.slots / kBK2, p.x[buf], p.f16, s);
    if (rc) return rc;
    record(pev, pkind, 1, s);
    return SCP3GPU_OK;
}

int contract(Plan& p, int buf, int64_t n, cudaStream_t s, std::vector<cudaEvent_t>* pev, std::vector<int>* pkind,
             cudaEvent_t head_done)
{
    const int nflush = (int)(n / kFlush);
    const int units = p.ntiles * p.nsplit;
    // whole waves first, then the partial last wave as its own launch, so that
    // work queued behind head_done can use the SMs that last wave leaves idle
    const int head = units > p.grid && units % p.grid ? units / p.grid * p.grid : units;
    for (int part = 0; part < 2; part++) {
        const int u0 = part ? head : 0, u1 = part ? units : head;
        if (u1 <= u0) continue;
        record(pev, pkind, 2, s);
        const int rc = launch_contract(p.x[buf], p.slots / kBK2, p.tiles2, p.ntiles, p.nsplit, nflush * kKB2PerFlush,
                                       p.group_meta[buf], p.f16, p.partial, p.err_flag,
                                       std::min(p.grid, u1 - u0), s, u0, u1);
        if (rc) return rc;
        record(pev, pkind, 2, s);
        if (part == 0 && head_done) SCP3_CUDA(cudaEventRecord(head_done, s));
    }
    return SCP3GPU_OK;
}

int accumulate_pass(Plan& p, const uint32_t* desc, int nb, int nm, const float* q32, const double* v, int64_t n,
                    cudaStream_t s, std::vector<cudaEvent_t>* pev, std::vector<int>* pkind)
{
    (void)desc;
    int rc = prepare(p, 0, nb, nm, q32, v, n, s, pev, pkind);
    return rc ? rc : contract(p, 0, n, s, pev, pkind);
}

int unpack(Plan& p, int nb, double divisor, const double* diag, double zpe, double* M, int64_t ld, cudaStream_t s)
{
    int err = 0;
    SCP3_CUDA(cudaMemcpyAsync(&err, p.err_flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    SCP3_CUDA(cudaStreamSynchronize(s));
    if (err) return fail(SCP3GPU_ERR_TIMEOUT, "tensor-core contraction: a bounded pipeline wait expired");
    return launch_unpack(p.partial, p.tile_index, p.nt, p.ntiles, p.nsplit, nb, divisor, diag, zpe, M, ld, s);
}

}  // namespace tc
}  // namespace scp3

// Host-only view of the 128 x 256 tiling of one cluster with nt_need 128-row
// panels on `sms` SMs, for tests: the tile count, splits, and per tile (A
// panel, B panel 0, B panel 1), and owner[ti * nt + tj] for nt = nt_need
// rounded up to even.  tiles may be null (counts only).
extern "C" int scp3gpu_internal_tiling(int nt_need, int sms, int* ntiles, int* nsplit, int* tiles, int max_tiles,
                                       int* owner)
{
    using namespace scp3::tc;
    if (nt_need < 1 || sms < 1 || !ntiles || !nsplit) return SCP3GPU_ERR_ARG;
    const int nt = (nt_need + 1) / 2 * 2;
    std::vector<BaseTile> base;
    add_cluster_tiles(base, 0, nt, nt_need, 0, 0);
    std::vector<int4> t;
    std::vector<std::vector<int>> own;
    finish_tiling(base, std::vector<int>{nt}, sms, t, own, *nsplit);
    *ntiles = (int)t.size();
    if (tiles) {
        if ((int)t.size() > max_tiles) return SCP3GPU_ERR_ARG;
        for (size_t i = 0; i < t.size(); i++) {
            tiles[3 * i] = t[i].x / kTile;
            tiles[3 * i + 1] = t[i].y / kTile;
            tiles[3 * i + 2] = t[i].w / kTile;
        }
    }
    if (owner) std::copy(own[0].begin(), own[0].end(), owner);
    return SCP3GPU_OK;
}
