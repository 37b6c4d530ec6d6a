// dpmm_tc.cu -- Gaussian label phase on the 5th-generation tensor cores (tcgen05 + TMEM).
//
// For a tile of 128 points and every cluster k the whitened residual
//     z_k = W_k^T x - b_k,   b_k = W_k^T (mu_k - shift),   inv_sigma_k = W_k W_k^T
// is one GEMM row block: C[p, (k, j)] = sum_i X[p, i] W_k(i, j).  It runs as split BF16
// (x = x_hi + x_lo, W = W_hi + W_lo; C = X_hi W_hi + X_lo W_hi + X_hi W_lo, FP32 accumulation
// in TMEM), which keeps the residual at FP32 accuracy.  The N x (K*D) product never leaves the
// SM: the epilogue reads each 64-column cluster block from TMEM, forms
//     r_k = c_k - 0.5 * sum_j (C[p, (k, j)] - b_kj)^2
// into a shared-memory table, and finishes with the softmax + Walker alias draw (or argmax)
// of the reference (cudaKernel.cu:374-424, 27-124) in a second kernel, one thread per point.
//
// CTA roles (608 threads, persistent over 256-point super-tiles): warp 0 streams the A tiles
// (points, packed at upload) and the B tiles (2 clusters = 128 columns, hi + lo, 32 KB, stored
// pre-swizzled) with cp.async.bulk; warp 1 allocates TMEM; warps 1-2 each issue the 12
// tcgen05.mma (M=128, N=128, K=16) of one 128-point half per N tile into 2 accumulator pairs;
// warps 3-18 drain the accumulators into r.
// Every mbarrier wait is bounded: on timeout the CTA records an error code, stops issuing work,
// drains what it issued (bounded) and frees its TMEM.
//
// Operand layout: K-major, 128-byte swizzle (8-row x 128-byte atoms, 16-byte chunk c of row r
// stored at chunk c ^ (r % 8)), descriptor SBO = 1024 B; a K-step of 16 elements advances the
// descriptor start address by 32 bytes.  The padded dimension must be 32 or 64 (zero-filled
// to 64).
#include <cuda_bf16.h>

#include <algorithm>

#include "dpmm_device.cuh"

namespace dpmm {
namespace tc {

constexpr int BM = 128;                    // points per tile (TMEM lanes)
constexpr int KD = 64;                     // contraction length (one 128-byte bf16 row)
constexpr int CPT = 2;                     // clusters per N tile
constexpr int BN = CPT * KD;               // 128 accumulator columns per N tile
constexpr int A_BYTES = BM * KD * 2;       // 16 KB (one of hi / lo)
constexpr int B_BYTES = BN * KD * 2;       // 16 KB (one of hi / lo)
constexpr int STAGE_BYTES = 2 * B_BYTES;   // 32 KB: hi then lo
constexpr int A_TILE = 2 * A_BYTES;        // 32 KB: hi then lo
constexpr uint32_t TMEM_COLS = 512;        // 2 accumulator pairs: 2 halves x 128 columns each
constexpr int NPAIR = 2;                   // accumulator pairs (N tiles in flight)
constexpr int HALVES = 2;                  // point tiles per super-tile (M = 2 x 128 per B tile)
constexpr int A_SLOT = HALVES * 2 * A_BYTES;   // 64 KB: tile 0 hi, lo, tile 1 hi, lo
constexpr int MAX_BSTAGES = 4;
constexpr int BIAS_REC = 528;              // per N tile: b (2 x 64 floats), c (2 floats), pad
constexpr int BIAS_SLOTS = 8;              // bias ring depth
constexpr int MMA_WARPS = 2;               // one MMA issuer per 128-point half
constexpr int DRAIN_WARPS = 16;            // (lane quarter, cluster of the N tile, half)
constexpr int WARP_MMA0 = 1, WARP_DRAIN0 = WARP_MMA0 + MMA_WARPS;
constexpr int THREADS = 32 * (1 + MMA_WARPS + DRAIN_WARPS);

enum : int {
    ERR_TIMEOUT_FULL = 1, ERR_TIMEOUT_EMPTY = 2, ERR_TIMEOUT_TFULL = 3, ERR_TIMEOUT_TEMPTY = 4,
    ERR_TIMEOUT_AFULL = 5, ERR_TIMEOUT_AEMPTY = 6, ERR_TIMEOUT_BFULL = 9, ERR_TIMEOUT_BEMPTY = 10
};

__host__ __device__ constexpr uint32_t sw128_offset(int row, int k)
{
    return (uint32_t)((row >> 3) * 1024 + (row & 7) * 128 + ((((k >> 3) ^ (row & 7)) & 7) << 4) + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

constexpr uint64_t WAIT_LIMIT_NS = 2000000000ull;   // 2 s: legitimate waits here are microseconds

// Non-blocking probe of a phase (no suspend).
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Potentially blocking probe: the thread may sleep until the phase completes, for at most about
// `ns` nanoseconds (the suspend-time hint), instead of returning at once and spinning.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, uint32_t parity, uint32_t ns)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
        : "memory");
    return ok != 0;
}

// Single-thread bounded wait.  Gives up after WAIT_LIMIT_NS, or early when another CTA of the
// launch has already reported an error (gerr != nullptr).  Between non-blocking probes the thread
// backs off with nanosleep (32 ns growing to 256 ns), so that waiting warps do not fill the issue
// slots and the barrier / timer pipes that the working warps need.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, const volatile int32_t* gerr)
{
    if (mbar_test_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    uint32_t sleep = 32;
    for (uint32_t i = 1;; ++i) {
        __nanosleep(sleep);
        if (mbar_test_wait(bar, parity)) return true;
        if (sleep < 256) sleep <<= 1;
        if ((i & 63) == 0) {
            if (global_ns() - t0 > WAIT_LIMIT_NS) return false;
            if (gerr && *gerr) return false;
        }
    }
}

// Warp-uniform bounded wait: lane 0 polls (one barrier operation per poll instead of 32) and
// the outcome is broadcast; __syncwarp orders the other lanes after lane 0's acquire.  All lanes
// take the same decision (the epilogue's tcgen05.ld is warp-collective).
__device__ __forceinline__ bool warp_wait_bounded(uint64_t* bar, uint32_t parity, const volatile int32_t* gerr)
{
    int ok = 1;
    if ((threadIdx.x & 31) == 0) ok = mbar_wait_bounded(bar, parity, gerr) ? 1 : 0;
    ok = __shfl_sync(0xffffffffu, ok, 0);
    __syncwarp();
    return ok != 0;
}

// One arrival per warp: every lane's prior work is ordered before lane 0's release by __syncwarp.
__device__ __forceinline__ void warp_arrive(uint64_t* bar)
{
    __syncwarp();
    if ((threadIdx.x & 31) == 0) mbar_arrive(bar);
}

__device__ __forceinline__ void bulk_copy_g2s(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);   // start address
    d |= (uint64_t)1 << 16;                      // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;            // stride byte offset: 8-row atoms 1024 B apart
    d |= (uint64_t)1 << 46;                      // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;                      // 128-byte swizzle
    return d;
}

// kind::f16 instruction descriptor: F32 accumulator, BF16 A and B, both K-major, M=128, N=128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accum)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accum)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive accumulator columns of this thread's TMEM lane (warp-collective)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void bf16_split(float v, __nv_bfloat16& hi, __nv_bfloat16& lo)
{
    hi = __float2bfloat16_rn(v);
    lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

__device__ __forceinline__ uint32_t bf16x2_bits(__nv_bfloat162 v)
{
    return (uint32_t)__bfloat16_as_ushort(v.x) | ((uint32_t)__bfloat16_as_ushort(v.y) << 16);
}

// bf16_split of four values, packed: hi and lo as 4 x BF16 (8 bytes) each
__device__ __forceinline__ void bf16_split4(float a, float b, float c, float d, uint2& hi, uint2& lo)
{
    const __nv_bfloat162 h01 = __floats2bfloat162_rn(a, b), h23 = __floats2bfloat162_rn(c, d);
    const float2 f01 = __bfloat1622float2(h01), f23 = __bfloat1622float2(h23);
    hi = make_uint2(bf16x2_bits(h01), bf16x2_bits(h23));
    lo = make_uint2(bf16x2_bits(__floats2bfloat162_rn(a - f01.x, b - f01.y)),
                    bf16x2_bits(__floats2bfloat162_rn(c - f23.x, d - f23.y)));
}

// ------------------------------------------------------------------------- B packing
// Bpack[t] = 32 KB: hi (16 KB) then lo (16 KB) of the 128 x 64 K-major swizzled tile holding
// rows n = (c, j) -> W_{2t+c}(i, j) over i (zero outside the K clusters / the dimension).
// sub = 1: tile t holds instead the two sub-cluster factors of cluster t (slots 3t+1, 3t+2),
// the B operand of the sub-label contraction.
__global__ void k_pack_b(const float* __restrict__ Wt, int K, int Dp, int NT, int sub, uint8_t* __restrict__ Bpack)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;   // (t, n, chunk)
    if (e >= NT * BN * 8) return;
    const int t = e / (BN * 8);
    const int n = (e / 8) % BN;
    const int ch = e % 8;
    const int half = n / KD;
    const bool valid = sub ? t < K : CPT * t + half < K;
    const int slot = sub ? 3 * t + 1 + half : 3 * (CPT * t + half);
    const int j = n % KD;
    __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int i = ch * 8 + q;
        float w = 0.f;
        if (valid && j < Dp && i < Dp) w = Wt[((size_t)slot * Dp + j) * Dp + i];
        bf16_split(w, hi[q], lo[q]);
    }
    uint8_t* base = Bpack + (size_t)t * STAGE_BYTES;
    const uint32_t off = sw128_offset(n, ch * 8);
    *reinterpret_cast<uint4*>(base + off) = *reinterpret_cast<const uint4*>(hi);
    *reinterpret_cast<uint4*>(base + B_BYTES + off) = *reinterpret_cast<const uint4*>(lo);
}

// Bias records: per N tile t, b of clusters 2t and 2t+1 (64 floats each, zero past Dp / K) and
// their constants c (slot 3k of cvec), so the drain reads them from shared memory.
__global__ void k_pack_bias(const float* __restrict__ bvec, const float* __restrict__ cvec, int K, int Dp, int NT,
                            uint8_t* __restrict__ Bbias)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;   // (t, i)
    if (e >= NT * (BIAS_REC / 4)) return;
    const int t = e / (BIAS_REC / 4), i = e % (BIAS_REC / 4);
    float v = 0.f;
    if (i < 2 * KD) {
        const int k = CPT * t + i / KD, j = i % KD;
        if (k < K && j < Dp) v = bvec[(size_t)3 * k * Dp + j];
    } else if (i < 2 * KD + CPT) {
        const int k = CPT * t + (i - 2 * KD);
        if (k < K) v = cvec[3 * k];
    }
    reinterpret_cast<float*>(Bbias + (size_t)t * BIAS_REC)[i] = v;
}

// ------------------------------------------------------------------------- A packing
// Apack[t] = 32 KB: hi (16 KB) then lo (16 KB) of the 128 x 64 K-major swizzled tile holding the
// points 128t .. 128t+127 (zero rows past N, zero columns past Dp).  The points never change
// during a run, so the split is done once at upload.
__global__ void k_pack_a(const float* __restrict__ x, int64_t N, int Dp, int64_t ntiles, uint8_t* __restrict__ Apack)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;   // (tile, row, chunk)
    if (e >= ntiles * BM * 8) return;
    const int64_t t = e / (BM * 8);
    const int row = (int)((e / 8) % BM), ch = (int)(e % 8);
    const int64_t pt = t * BM + row;
    float v[8];
    if (pt < N && ch * 8 < Dp) {
        const float4* src = reinterpret_cast<const float4*>(x + pt * Dp + ch * 8);
        const float4 a = src[0], b = src[1];
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
        v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = 0.f;
    }
    __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) bf16_split(v[q], hi[q], lo[q]);
    uint8_t* base = Apack + (size_t)t * A_TILE;
    const uint32_t off = sw128_offset(row, ch * 8);
    *reinterpret_cast<uint4*>(base + off) = *reinterpret_cast<const uint4*>(hi);
    *reinterpret_cast<uint4*>(base + A_BYTES + off) = *reinterpret_cast<const uint4*>(lo);
}

// ------------------------------------------------------------------------- label kernel
// Persistent: one CTA per SM walks the super-tiles blockIdx.x, blockIdx.x + gridDim.x, ... of
// 256 points (two 128-point tiles sharing every B tile, which halves the B traffic and the MMA
// issue overhead per point).
//
//   warp 0      producer: A super-tile (64 KB, with an L2 prefetch of the next one), B tiles
//               (32 KB) into a B ring, bias records into a bias ring
//   warps 1-2   MMA issuers: per N tile 12 tcgen05.mma each (one per half) into pair g % 2
//   warps 3-18  drain: TMEM accumulator -> r = c - |z|^2 / 2 for one (lane quarter, cluster,
//               half) per warp, written cluster-major to rbuf[k][point] (32 points per store),
//               with a running max / sum of exp (or the first maximum, final mode) per point and
//               cluster parity, written to part at the end of the super-tile
//
// The softmax + alias draw runs in k_draw_labels at full occupancy.
struct SmemLayout {
    int bstages;
    size_t a, b, bias, bar, total;
};

// mbarrier slots: B ring (full, empty), A slot (afull, aempty), accumulator pairs (tfull,
// tempty), bias ring (bfull, bempty)
constexpr int BAR_FULL = 0, BAR_EMPTY = BAR_FULL + MAX_BSTAGES, BAR_AFULL = BAR_EMPTY + MAX_BSTAGES,
              BAR_AEMPTY = BAR_AFULL + 1, BAR_TFULL = BAR_AEMPTY + 1, BAR_TEMPTY = BAR_TFULL + NPAIR,
              BAR_BFULL = BAR_TEMPTY + NPAIR, BAR_BEMPTY = BAR_BFULL + BIAS_SLOTS, NBARS = BAR_BEMPTY + BIAS_SLOTS;
static_assert(NBARS == 30, "barrier slots");

__host__ __device__ inline SmemLayout smem_layout(int bstages)
{
    SmemLayout L;
    L.bstages = bstages;
    L.a = 0;                                            // one 64 KB A slot (1024-aligned)
    L.b = (size_t)A_SLOT;                               // bstages x 32 KB
    L.bias = L.b + (size_t)bstages * STAGE_BYTES;       // BIAS_SLOTS x BIAS_REC
    L.bar = L.bias + (size_t)BIAS_SLOTS * BIAS_REC;
    L.total = L.bar + NBARS * 8 + 16 + 1024;            // barriers, tmem slot + flag, alignment slack
    return L;
}

__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

__global__ void __launch_bounds__(THREADS, 1) k_gauss_labels_tc(
    const uint8_t* __restrict__ Apack, int64_t N, int ntiles, const uint8_t* __restrict__ Bpack,
    const uint8_t* __restrict__ Bbias, int Dp, int K, int bstages, int final_, float* __restrict__ rbuf,
    float* __restrict__ part, float* __restrict__ r_out, int32_t* __restrict__ err, int stall)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const SmemLayout L = smem_layout(bstages);
    uint8_t* sA = smem + L.a;
    uint8_t* sB = smem + L.b;
    uint8_t* sBias = smem + L.bias;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.bar);
    uint64_t* full = bars + BAR_FULL;       // [bstages]   B tile landed
    uint64_t* empty = bars + BAR_EMPTY;     // [bstages]   B tile consumed by the MMAs
    uint64_t* afull = bars + BAR_AFULL;     // A super-tile landed
    uint64_t* aempty = bars + BAR_AEMPTY;   // A super-tile consumed
    uint64_t* tfull = bars + BAR_TFULL;     // [NPAIR]     accumulator pair ready
    uint64_t* tempty = bars + BAR_TEMPTY;   // [NPAIR]     accumulator pair drained
    uint64_t* bfull = bars + BAR_BFULL;     // [BIAS_SLOTS] bias record landed
    uint64_t* bempty = bars + BAR_BEMPTY;   // [BIAS_SLOTS] bias record read by every drain warp
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + NBARS);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int NT = (K + CPT - 1) / CPT;
    const int nst = (ntiles + HALVES - 1) / HALVES;
    const volatile int32_t* gerr = err;

    if (tid == 0) {
        *abort_flag = *gerr ? 1 : 0;
        for (int s = 0; s < bstages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], MMA_WARPS);
        }
        mbar_init(afull, 1);
        mbar_init(aempty, MMA_WARPS);
        for (int t = 0; t < NPAIR; ++t) {
            mbar_init(&tfull[t], MMA_WARPS);
            mbar_init(&tempty[t], DRAIN_WARPS);
        }
        for (int s = 0; s < BIAS_SLOTS; ++s) {
            mbar_init(&bfull[s], 1);
            mbar_init(&bempty[s], DRAIN_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (*abort_flag) return;   // a CTA that starts after another one reported an error does nothing
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        // ---------------- producer
        if (lane == 0) {
            int gb = 0, la = 0;
            for (int st = blockIdx.x; st < nst && !*abort_flag; st += gridDim.x, ++la) {
                if (!mbar_wait_bounded(aempty, (la & 1) ^ 1, gerr)) {
                    atomicCAS(err, 0, ERR_TIMEOUT_AEMPTY);
                    *abort_flag = 1;
                    break;
                }
                const int tiles = min(HALVES, ntiles - HALVES * st);
                const uint32_t abytes = (uint32_t)tiles * A_TILE;
                mbar_arrive_expect_tx(afull, abytes);
                bulk_copy_g2s(sA, Apack + (size_t)HALVES * st * A_TILE, abytes, afull);
                const int nx = st + gridDim.x;   // this CTA's next super-tile: warm L2 for it
                if (nx < nst)
                    prefetch_l2(Apack + (size_t)HALVES * nx * A_TILE, (uint32_t)min(HALVES, ntiles - HALVES * nx) * A_TILE);
                bool ok = true;
                for (int nt = 0; nt < NT; ++nt, ++gb) {
                    const int s = gb % bstages, sb = gb % BIAS_SLOTS;
                    if (!mbar_wait_bounded(&empty[s], ((gb / bstages) & 1) ^ 1, gerr)) {
                        atomicCAS(err, 0, ERR_TIMEOUT_EMPTY);
                        ok = false;   // gb stays the count of B copies issued
                        break;
                    }
                    if (!mbar_wait_bounded(&bempty[sb], ((gb / BIAS_SLOTS) & 1) ^ 1, gerr)) {
                        atomicCAS(err, 0, ERR_TIMEOUT_BEMPTY);
                        ok = false;
                        break;
                    }
                    mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
                    bulk_copy_g2s(sB + (size_t)s * STAGE_BYTES, Bpack + (size_t)nt * STAGE_BYTES, STAGE_BYTES,
                                  &full[s]);
                    mbar_arrive_expect_tx(&bfull[sb], BIAS_REC);
                    bulk_copy_g2s(sBias + (size_t)sb * BIAS_REC, Bbias + (size_t)nt * BIAS_REC, BIAS_REC, &bfull[sb]);
                }
                if (!ok) {
                    *abort_flag = 1;
                    ++la;   // this super-tile's A copy was issued
                    break;
                }
            }
            // drain: every copy issued has landed before shared memory is released
            if (la > 0) mbar_wait_bounded(afull, (la - 1) & 1, nullptr);
            for (int q = gb > bstages ? gb - bstages : 0; q < gb; ++q)
                mbar_wait_bounded(&full[q % bstages], (q / bstages) & 1, nullptr);
            for (int q = gb > BIAS_SLOTS ? gb - BIAS_SLOTS : 0; q < gb; ++q)
                mbar_wait_bounded(&bfull[q % BIAS_SLOTS], (q / BIAS_SLOTS) & 1, nullptr);
        }
    } else if (warp < WARP_DRAIN0) {
        // ---------------- MMA issuers: warp WARP_MMA0 + h issues the half-h MMAs of every N tile
        // into accumulator 2t + h and commits to the shared barriers (count MMA_WARPS); while one
        // issuer waits or commits, the other's MMAs keep the tensor pipe fed.  stall (test seam):
        // no product is issued, so the waits for them run out and report ERR_TIMEOUT_*
        if (lane == 0 && !stall) {
            const int h = warp - WARP_MMA0;
            int g = 0, la = 0, issued = 0;
            const uint64_t dah = sw128_desc(smem_u32(sA + (size_t)h * A_TILE));
            const uint64_t dal = sw128_desc(smem_u32(sA + (size_t)h * A_TILE + A_BYTES));
            for (int st = blockIdx.x; st < nst && !*abort_flag; st += gridDim.x, ++la) {
                if (!mbar_wait_bounded(afull, la & 1, gerr)) {
                    atomicCAS(err, 0, ERR_TIMEOUT_AFULL);
                    *abort_flag = 1;
                    break;
                }
                bool ok = true;
                for (int nt = 0; nt < NT; ++nt, ++g) {
                    const int s = g % bstages, t = g % NPAIR;
                    if (!mbar_wait_bounded(&full[s], (g / bstages) & 1, gerr)) {
                        atomicCAS(err, 0, ERR_TIMEOUT_FULL);
                        ok = false;
                        break;
                    }
                    if (!mbar_wait_bounded(&tempty[t], ((g / NPAIR) & 1) ^ 1, gerr)) {
                        atomicCAS(err, 0, ERR_TIMEOUT_TEMPTY);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t b_hi = smem_u32(sB + (size_t)s * STAGE_BYTES), b_lo = b_hi + B_BYTES;
                    // descriptors: a K step of 16 elements (32 bytes) adds 2 to the start-address field
                    const uint64_t dbh = sw128_desc(b_hi), dbl = sw128_desc(b_lo);
                    const uint32_t d = tmem_base + (uint32_t)((HALVES * t + h) * BN);
#pragma unroll
                    for (int ks = 0; ks < KD / 16; ++ks) umma_bf16(d, dah + 2 * ks, dbh + 2 * ks, ks != 0 ? 1u : 0u);
#pragma unroll
                    for (int ks = 0; ks < KD / 16; ++ks) umma_bf16(d, dal + 2 * ks, dbh + 2 * ks, 1u);
#pragma unroll
                    for (int ks = 0; ks < KD / 16; ++ks) umma_bf16(d, dah + 2 * ks, dbl + 2 * ks, 1u);
                    umma_commit(&empty[s]);
                    umma_commit(&tfull[t]);
                    issued = g + 1;
                }
                umma_commit(aempty);   // the A slot is free once this super-tile's MMAs complete
                if (!ok) {
                    *abort_flag = 1;
                    break;
                }
            }
            // drain: the last MMAs issued have completed before TMEM is freed (the phase completes
            // once both issuers' commits have arrived; bounded if the other one stopped early)
            if (issued > 0) mbar_wait_bounded(&tfull[(issued - 1) % NPAIR], ((issued - 1) / NPAIR) & 1, nullptr);
        }
    } else {
        // ---------------- drain: (lane quarter, cluster c of the N tile, half h) per warp
        const int quarter = warp & 3;
        const int idx = (warp - WARP_DRAIN0) >> 2;
        const int c = idx & 1, h = idx >> 1;
        const int p = quarter * 32 + lane;
        const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
        int g = 0;
        for (int st = blockIdx.x; st < nst; st += gridDim.x) {
            if (__any_sync(0xffffffffu, *abort_flag != 0)) break;
            const int64_t pt = ((int64_t)HALVES * st + h) * BM + p;
            const bool valid = pt < N;
            float m = -INFINITY, sum = 0.f;   // running max and sum of exp(r - max); final: best, arg
            int arg = -1;
            bool ok = true;
            for (int nt = 0; nt < NT; ++nt, ++g) {
                const int t = g % NPAIR, sb = g % BIAS_SLOTS;
                if (!warp_wait_bounded(&tfull[t], (g / NPAIR) & 1, gerr)) {
                    if (lane == 0) atomicCAS(err, 0, ERR_TIMEOUT_TFULL);
                    ok = false;
                    break;
                }
                if (!warp_wait_bounded(&bfull[sb], (g / BIAS_SLOTS) & 1, gerr)) {
                    if (lane == 0) atomicCAS(err, 0, ERR_TIMEOUT_BFULL);
                    ok = false;
                    break;
                }
                tc_fence_after();
                const int k = nt * CPT + c;
                const float* rec = reinterpret_cast<const float*>(sBias + (size_t)sb * BIAS_REC);
                const float* bk = rec + c * KD;   // b of cluster k; its constant c_k is rec[2 * KD + c]
                if (k < K) {
                    // z_j = C[p, j] - b_j over the cluster's 64 columns, in two halves of 32
                    float q0 = 0.f, q1 = 0.f, q2 = 0.f, q3 = 0.f;
#pragma unroll
                    for (int hh = 0; hh < 2; ++hh) {
                        if (hh == 1 && Dp <= 32) break;   // columns past Dp are zero
                        uint32_t v[32];
                        tmem_ld32(tmem_base + lane_addr + (uint32_t)((HALVES * t + h) * BN + c * KD + 32 * hh), v);
                        const float4* b4p = reinterpret_cast<const float4*>(bk + 32 * hh);
#pragma unroll
                        for (int j4 = 0; j4 < 8; ++j4) {
                            const float4 b4 = b4p[j4];
                            const float z0 = __uint_as_float(v[4 * j4 + 0]) - b4.x;
                            const float z1 = __uint_as_float(v[4 * j4 + 1]) - b4.y;
                            const float z2 = __uint_as_float(v[4 * j4 + 2]) - b4.z;
                            const float z3 = __uint_as_float(v[4 * j4 + 3]) - b4.w;
                            q0 = fmaf(z0, z0, q0);
                            q1 = fmaf(z1, z1, q1);
                            q2 = fmaf(z2, z2, q2);
                            q3 = fmaf(z3, z3, q3);
                        }
                    }
                    const float r = rec[2 * KD + c] - 0.5f * ((q0 + q1) + (q2 + q3));
                    if (final_) {
                        if (arg < 0 || m < r) { m = r; arg = k; }   // first maximum in cluster order
                    } else {
                        if (r > m) {
                            sum = sum * __expf(m - r) + 1.f;
                            m = r;
                        } else {
                            sum += __expf(r - m);
                        }
                        if (valid) rbuf[(size_t)k * N + pt] = r;
                    }
                    if (r_out && valid) r_out[pt * K + k] = r;
                }
                tc_fence_before();
                warp_arrive(&tempty[t]);
                if (lane == 0) mbar_arrive(&bempty[sb]);
            }
            if (!ok) {
                *abort_flag = 1;
                break;
            }
            if (valid) {
                part[(size_t)(2 * c) * N + pt] = m;
                part[(size_t)(2 * c + 1) * N + pt] = final_ ? __int_as_float(arg) : sum;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS));
    }
}

// Softmax + alias draw (or argmax) per point from the label kernel's r (cluster-major) and the
// two halves' partials: build_log_likelihood_array_kernel + sample_by_probability
// (cudaKernel.cu:374-403, 27-124) or update_labels_by_max_index_kernel (:405-424).
__global__ void __launch_bounds__(256) k_draw_labels(const float* __restrict__ rbuf, const float* __restrict__ part,
                                                     int64_t N, int K, int final_, RngArgs rng,
                                                     int32_t* __restrict__ labels)
{
    const int64_t pt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pt >= N) return;
    const float m0 = part[pt], x0 = part[N + pt], m1 = part[2 * N + pt], x1 = part[3 * N + pt];
    if (final_) {
        // first maximum wins: half 0 holds the even clusters, half 1 the odd ones
        const int a0 = __float_as_int(x0), a1 = __float_as_int(x1);
        int arg = a0;
        if (a1 >= 0 && (a0 < 0 || m0 < m1 || (m1 == m0 && a1 < a0))) arg = a1;
        labels[pt] = arg + 1;
        return;
    }
    const float mx = fmaxf(m0, m1);
    const float sum = x0 * __expf(m0 - mx) + x1 * __expf(m1 - mx);
    const float inv = 1.0f / sum, fk = (float)K;
    const float* rp = rbuf + pt;
    auto y = [=](int i) -> float { return (__expf(__ldg(rp + (size_t)i * N) - mx) * inv) * fk; };
    // y < 1  <=>  r < max + log(sum / K): one compare per cluster for the small/large split
    const float thr = mx + __logf(sum / fk);
    auto is_small = [=](int i) -> bool { return __ldg(rp + (size_t)i * N) < thr; };
    float u1, u2;
    draw_uniform2(rng, pt, u1, u2);
    labels[pt] = alias_draw_y(y, is_small, K, u1, u2);
}

// ------------------------------------------------------------------------- sub-label kernel
// Sub-cluster labels of the points of one chunk (one cluster, in label order; cudaKernel.cu
// create_subclusters_labels, :1299-1398): per tile of 128 points the A operand (split BF16,
// swizzled) is built in shared memory from the gathered rows, and 12 tcgen05.mma against the
// cluster's B tile [W_l | W_r] give z for both sub-clusters.  8 warps drain
// r_s = c_s - |z_s - b_s|^2 / 2 (warp w: lane quarter w % 4, side w / 4); one thread per point then
// adds log lr_weights, normalises and draws with the two-category alias (cudaKernel.cu:352-372).
// Every wait is bounded and decided block-uniformly.
struct SubSmem {
    static constexpr size_t b = 0;                        // 32 KB B tile (hi, lo)
    static constexpr size_t a = STAGE_BYTES;              // 32 KB A tile (hi, lo)
    static constexpr size_t q = a + A_TILE;               // r of both sides [2][BM] floats
    static constexpr size_t bias = q + 2 * BM * 4;        // b_l, b_r [2][KD] floats
    static constexpr size_t pidx = bias + 2 * KD * 4;     // the tile's permutation entries [2][BM] ints
    static constexpr size_t bar = pidx + 2 * BM * 4;      // mbarrier, tmem slot, flag
    static constexpr size_t total = bar + 32 + 1024;      // + alignment slack
};

template <int DP>
__global__ void __launch_bounds__(256, 2) k_sub_labels_tc(
    const float* __restrict__ x, const int32_t* __restrict__ perm, const int32_t* __restrict__ chunk,
    const int32_t* __restrict__ nchunks, const uint8_t* __restrict__ Bsub, const float* __restrict__ bvec,
    const float* __restrict__ cvec, const float* __restrict__ lrw, RngArgs rng, int32_t* __restrict__ sub,
    float* __restrict__ r_out, int32_t* __restrict__ err, int stall)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* sB = smem + SubSmem::b;
    uint8_t* sA = smem + SubSmem::a;
    float* sq = reinterpret_cast<float*>(smem + SubSmem::q);
    float* sbias = reinterpret_cast<float*>(smem + SubSmem::bias);
    int32_t* spidx = reinterpret_cast<int32_t*>(smem + SubSmem::pidx);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + SubSmem::bar);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
    volatile int* flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int ch = blockIdx.x;
    if (ch >= *nchunks) return;
    const int k = chunk[3 * ch], start = chunk[3 * ch + 1], len = chunk[3 * ch + 2];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const volatile int32_t* gerr = err;

    // B tile of cluster k and the two sub-cluster biases
    {
        const uint4* src = reinterpret_cast<const uint4*>(Bsub + (size_t)k * STAGE_BYTES);
        uint4* dst = reinterpret_cast<uint4*>(sB);
        for (int e = tid; e < STAGE_BYTES / 16; e += 256) dst[e] = src[e];
        if (tid < 2 * KD) {
            const int side = tid / KD, j = tid % KD;
            sbias[tid] = j < DP ? bvec[(size_t)(3 * k + 1 + side) * DP + j] : 0.f;
        }
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        *flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"((uint32_t)BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const float cl = cvec[3 * k + 1], cr = cvec[3 * k + 2];
    const float wl = lrw[2 * k], wr = lrw[2 * k + 1];

    // gathered rows: item u of this thread is (row tid / 8 + 32 u, 8-float chunk tid % 8); a tile's
    // permutation entries load one tile ahead of its rows
    float4 pf[4][2];
    int pq[4], pcur[4];   // entries of the tile after the loaded one / of the loaded one
    auto load_perm = [&](int t0) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int row = (tid >> 3) + 32 * u;
            pq[u] = t0 + row < len ? __ldg(perm + start + t0 + row) : -1;
        }
    };
    auto load_rows = [&]() {   // rows of the tile whose entries pq holds
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int c8 = tid & 7;
            pcur[u] = pq[u];
            pf[u][0] = make_float4(0.f, 0.f, 0.f, 0.f);
            pf[u][1] = pf[u][0];
            if (pq[u] >= 0 && c8 * 8 < DP) {
                const float4* src = reinterpret_cast<const float4*>(x + (size_t)pq[u] * DP + c8 * 8);
                pf[u][0] = __ldg(src);
                pf[u][1] = __ldg(src + 1);
            }
        }
    };
    load_perm(0);
    load_rows();
    load_perm(BM);
    uint32_t phase = 0;
    bool failed = false;
    const uint64_t da_h = sw128_desc(smem_u32(sA)), da_l = sw128_desc(smem_u32(sA + A_BYTES));
    const uint64_t db_h = sw128_desc(smem_u32(sB)), db_l = sw128_desc(smem_u32(sB + B_BYTES));
    for (int t0 = 0; t0 < len && !failed; t0 += BM) {
        const int nt = min(BM, len - t0);
        // A tile: split BF16, 128-byte swizzle
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int row = (tid >> 3) + 32 * u, c8 = tid & 7;
            const float v[8] = {pf[u][0].x, pf[u][0].y, pf[u][0].z, pf[u][0].w,
                                pf[u][1].x, pf[u][1].y, pf[u][1].z, pf[u][1].w};
            __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) bf16_split(v[q], hi[q], lo[q]);
            const uint32_t off = sw128_offset(row, c8 * 8);
            *reinterpret_cast<uint4*>(sA + off) = *reinterpret_cast<const uint4*>(hi);
            *reinterpret_cast<uint4*>(sA + A_BYTES + off) = *reinterpret_cast<const uint4*>(lo);
            if (c8 == 0) spidx[((t0 / BM) & 1) * BM + row] = pcur[u];   // for the draw, two tiles apart
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        if (tid == 0 && !stall) {   // stall: the wait-test seam issues nothing
            tc_fence_after();
#pragma unroll
            for (int ks = 0; ks < KD / 16; ++ks) umma_bf16(tmem_base, da_h + 2 * ks, db_h + 2 * ks, ks != 0 ? 1u : 0u);
#pragma unroll
            for (int ks = 0; ks < KD / 16; ++ks) umma_bf16(tmem_base, da_l + 2 * ks, db_h + 2 * ks, 1u);
#pragma unroll
            for (int ks = 0; ks < KD / 16; ++ks) umma_bf16(tmem_base, da_h + 2 * ks, db_l + 2 * ks, 1u);
            umma_commit(bar);
        }
        if (t0 + BM < len) {   // the next tile's rows load while the MMAs run
            load_rows();
            load_perm(t0 + 2 * BM);
        }
        if (tid == 0) {
            if (!mbar_wait_bounded(bar, phase & 1, gerr)) {
                atomicCAS(err, 0, ERR_TIMEOUT_TFULL);
                *flag = 1;
            }
        }
        ++phase;
        __syncthreads();
        if (*flag) { failed = true; break; }
        tc_fence_after();
        {
            const int quarter = warp & 3, side = warp >> 2;
            const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
            const float* bs = sbias + side * KD;
            float q0 = 0.f, q1 = 0.f, q2 = 0.f, q3 = 0.f;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (h == 1 && DP <= 32) break;   // columns past DP are zero
                uint32_t v[32];
                tmem_ld32(tmem_base + lane_addr + (uint32_t)(side * KD + 32 * h), v);
#pragma unroll
                for (int j4 = 0; j4 < 8; ++j4) {
                    const float4 b4 = *reinterpret_cast<const float4*>(bs + 32 * h + 4 * j4);
                    const float z0 = __uint_as_float(v[4 * j4 + 0]) - b4.x;
                    const float z1 = __uint_as_float(v[4 * j4 + 1]) - b4.y;
                    const float z2 = __uint_as_float(v[4 * j4 + 2]) - b4.z;
                    const float z3 = __uint_as_float(v[4 * j4 + 3]) - b4.w;
                    q0 = fmaf(z0, z0, q0);
                    q1 = fmaf(z1, z1, q1);
                    q2 = fmaf(z2, z2, q2);
                    q3 = fmaf(z3, z3, q3);
                }
            }
            sq[side * BM + quarter * 32 + lane] = (side ? cr : cl) - 0.5f * ((q0 + q1) + (q2 + q3));
        }
        tc_fence_before();
        __syncthreads();
        if (tid < nt) {
            const int64_t pt = spidx[((t0 / BM) & 1) * BM + tid];
            float rl = sq[tid], rr = sq[BM + tid];
            if (r_out) { r_out[2 * pt] = rl; r_out[2 * pt + 1] = rr; }
            rl += wl;
            rr += wr;
            const float mx = fmaxf(rl, rr);
            const float el = __expf(rl - mx), er = __expf(rr - mx);
            const float s = el + er;
            float u1, u2;
            draw_uniform2(rng, pt, u1, u2);
            sub[pt] = alias_draw2(el / s, er / s, u1, u2);
        }
    }
    if (failed && tid == 0 && !stall) mbar_wait_bounded(bar, (phase - 1) & 1, nullptr);   // nothing in flight at dealloc
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"((uint32_t)BN));
    }
}

// ------------------------------------------------------------------------- pruned-phase scan
// Pass 1 of the pruned label phase (the bounds are stated at k_prune_scan, dpmm_kernels.cu) on the
// tensor cores, one CTA per chunk of cluster h:
//   phase 1  per 128-point tile, the gathered rows (split BF16, swizzled) times the dense phase's
//            packed B tile h / 2 give z_h in accumulator columns (h % 2) * 64 ..; 8 warps drain
//            r_h = c_h - |z_h - b_h|^2 / 2 (the dense tensor-core phase's r of the point's own
//            cluster, from the same operands); |x - mu_h|^2 comes from the FP32 rows;
//   chunk    with the CTA's r_min and radius R the chunk bound leaves out clusters; the others
//            (ascending) become the rows of a candidate B operand [v_hk] (split BF16, 1-2 tiles);
//   phase 2  per tile the rows again times the candidate operand give v_hk^T x, and candidate k is
//            kept when c_k - (v_hk^T x - beta_hk)^2 / 2 >= r_h - margin at some point of the chunk.
// Shared memory below (about 102 KB: two CTAs per SM); 256 TMEM columns.
constexpr int kScanMaxK = 256;
struct ScanSmem {
    static constexpr size_t a = 0;                               // 32 KB A tile (hi, lo)
    static constexpr size_t b = a + A_TILE;                      // 64 KB: h's B tile, then candidate tiles
    static constexpr size_t sq = b + 2 * STAGE_BYTES;            // [2][BM] partial |z - b|^2
    static constexpr size_t bias = sq + 2 * BM * 4;              // b_h, mu_h: [2][KD] floats
    static constexpr size_t cb = bias + 2 * KD * 4;              // beta, c of the candidates: [2][kScanMaxK]
    static constexpr size_t ck = cb + 2 * kScanMaxK * 4;         // candidate clusters [kScanMaxK] ints
    static constexpr size_t bits = ck + kScanMaxK * 4;           // kept bits [8], warp r_min / R^2 [16], counts [8]
    static constexpr size_t bar = bits + 32 * 4;                 // mbarrier, tmem slot, flag
    static constexpr size_t total = bar + 32 + 1024;             // + alignment slack
};
static_assert(ScanSmem::bar % 8 == 0, "mbarrier alignment");
constexpr uint32_t SCAN_TMEM_COLS = 2 * BN;

template <int DP>
__global__ void __launch_bounds__(256, 2) k_prune_scan_tc(
    const float* __restrict__ x, const int32_t* __restrict__ perm, const int32_t* __restrict__ chunk,
    const int32_t* __restrict__ nchunks, const uint8_t* __restrict__ Btc, const float* __restrict__ bvec,
    const float* __restrict__ cvec, const float* __restrict__ mu, const float* __restrict__ lam,
    const float* __restrict__ M, const float* __restrict__ V, const float* __restrict__ beta, int K, float margin,
    float* __restrict__ rh, int32_t* __restrict__ cand, unsigned long long* __restrict__ cnt,
    int32_t* __restrict__ err, int stall)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* sA = smem + ScanSmem::a;
    uint8_t* sB = smem + ScanSmem::b;
    float* sq = reinterpret_cast<float*>(smem + ScanSmem::sq);
    float* sbias = reinterpret_cast<float*>(smem + ScanSmem::bias);
    float* sbeta = reinterpret_cast<float*>(smem + ScanSmem::cb);
    float* sck = sbeta + kScanMaxK;
    int32_t* sk = reinterpret_cast<int32_t*>(smem + ScanSmem::ck);
    uint32_t* kbits = reinterpret_cast<uint32_t*>(smem + ScanSmem::bits);
    float* wred = reinterpret_cast<float*>(kbits + kScanMaxK / 32);
    int32_t* wcnt = reinterpret_cast<int32_t*>(wred + 16);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + ScanSmem::bar);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
    volatile int* flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int q = blockIdx.x;
    if (q >= *nchunks) return;
    const int h = chunk[3 * q], start = chunk[3 * q + 1], len = chunk[3 * q + 2];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const volatile int32_t* gerr = err;

    {
        const uint4* src = reinterpret_cast<const uint4*>(Btc + (size_t)(h / CPT) * STAGE_BYTES);
        uint4* dst = reinterpret_cast<uint4*>(sB);
        for (int e = tid; e < STAGE_BYTES / 16; e += 256) dst[e] = src[e];
        if (tid < 2 * KD) {
            const int side = tid / KD, j = tid % KD;
            sbias[tid] = j < DP ? (side ? mu : bvec)[(size_t)3 * h * DP + j] : 0.f;
        }
        if (tid < kScanMaxK / 32) kbits[tid] = 0u;
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        *flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(SCAN_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const uint32_t lane_addr = (uint32_t)((warp & 3) * 32) << 16;
    const float ch = cvec[3 * h];

    // gathered rows: item u of this thread is (row tid / 8 + 32 u, 8-float chunk tid % 8); a tile's
    // permutation entries load one tile ahead of its rows
    float4 pf[4][2];
    int pq[4];
    auto load_perm = [&](int t0) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int row = (tid >> 3) + 32 * u;
            pq[u] = t0 + row < len ? __ldg(perm + start + t0 + row) : -1;
        }
    };
    auto load_rows = [&]() {   // rows of the tile whose entries pq holds
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int c8 = tid & 7;
            pf[u][0] = make_float4(0.f, 0.f, 0.f, 0.f);
            pf[u][1] = pf[u][0];
            if (pq[u] >= 0 && c8 * 8 < DP) {
                const float4* src = reinterpret_cast<const float4*>(x + (size_t)pq[u] * DP + c8 * 8);
                pf[u][0] = __ldg(src);
                pf[u][1] = __ldg(src + 1);
            }
        }
    };
    // A tile (split BF16, 128-byte swizzle) from the rows; with want_r2, the largest |x - mu_h|^2
    auto build_a = [&](int ntn, bool want_r2, float& r2max) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int row = (tid >> 3) + 32 * u, c8 = tid & 7;
            const float v[8] = {pf[u][0].x, pf[u][0].y, pf[u][0].z, pf[u][0].w,
                                pf[u][1].x, pf[u][1].y, pf[u][1].z, pf[u][1].w};
            __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) bf16_split(v[e], hi[e], lo[e]);
            const uint32_t off = sw128_offset(row, c8 * 8);
            *reinterpret_cast<uint4*>(sA + off) = *reinterpret_cast<const uint4*>(hi);
            *reinterpret_cast<uint4*>(sA + A_BYTES + off) = *reinterpret_cast<const uint4*>(lo);
            if (want_r2) {
                float d2 = 0.f;
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const float t = v[e] - sbias[KD + c8 * 8 + e];
                    d2 = fmaf(t, t, d2);
                }
                d2 += __shfl_xor_sync(0xffffffffu, d2, 1);
                d2 += __shfl_xor_sync(0xffffffffu, d2, 2);
                d2 += __shfl_xor_sync(0xffffffffu, d2, 4);
                if (row < ntn) r2max = fmaxf(r2max, d2);
            }
        }
    };
    // one tile's MMAs (12 per 128-column B tile) and the bounded wait for them; block-uniform result
    uint32_t phase = 0;
    const uint64_t da_h = sw128_desc(smem_u32(sA)), da_l = sw128_desc(smem_u32(sA + A_BYTES));
    auto mma_tile = [&](int nbt) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        if (tid == 0 && !stall) {   // stall: the wait-test seam issues nothing
            tc_fence_after();
            for (int nb = 0; nb < nbt; ++nb) {
                const uint8_t* bt = sB + (size_t)nb * STAGE_BYTES;
                const uint64_t db_h = sw128_desc(smem_u32(bt)), db_l = sw128_desc(smem_u32(bt + B_BYTES));
                const uint32_t td = tmem_base + (uint32_t)(nb * BN);
#pragma unroll
                for (int ks = 0; ks < KD / 16; ++ks) umma_bf16(td, da_h + 2 * ks, db_h + 2 * ks, ks != 0 ? 1u : 0u);
#pragma unroll
                for (int ks = 0; ks < KD / 16; ++ks) umma_bf16(td, da_l + 2 * ks, db_h + 2 * ks, 1u);
#pragma unroll
                for (int ks = 0; ks < KD / 16; ++ks) umma_bf16(td, da_h + 2 * ks, db_l + 2 * ks, 1u);
            }
            umma_commit(bar);
        }
    };
    auto mma_wait = [&]() -> bool {
        if (tid == 0) {
            if (!mbar_wait_bounded(bar, phase & 1, gerr)) {
                atomicCAS(err, 0, ERR_TIMEOUT_TFULL);
                *flag = 1;
            }
        }
        ++phase;
        __syncthreads();
        if (*flag) return false;
        tc_fence_after();
        return true;
    };

    bool failed = false;
    // phase 1: r_h, r_min, radius
    float tmin = INFINITY, r2max = 0.f;
    load_perm(0);
    load_rows();
    load_perm(BM);
    for (int t0 = 0; t0 < len; t0 += BM) {
        const int ntn = min(BM, len - t0);
        build_a(ntn, true, r2max);
        mma_tile(1);
        if (t0 + BM < len) {   // the next tile's rows load while the MMAs run
            load_rows();
            load_perm(t0 + 2 * BM);
        }
        if (!mma_wait()) { failed = true; break; }
        {
            const int part = warp >> 2;
            float qs = 0.f;
            if (DP > 32 || part == 0) {
                uint32_t v[32];
                tmem_ld32(tmem_base + lane_addr + (uint32_t)((h % CPT) * KD + 32 * part), v);
                const float* bs = sbias + 32 * part;
                float q1 = 0.f;
#pragma unroll
                for (int j = 0; j < 32; j += 2) {
                    const float z0 = __uint_as_float(v[j]) - bs[j];
                    const float z1 = __uint_as_float(v[j + 1]) - bs[j + 1];
                    qs = fmaf(z0, z0, qs);
                    q1 = fmaf(z1, z1, q1);
                }
                qs += q1;
            }
            sq[part * BM + (warp & 3) * 32 + lane] = qs;
        }
        tc_fence_before();
        __syncthreads();
        if (tid < ntn) {
            const float r = ch - 0.5f * (sq[tid] + sq[BM + tid]);
            rh[start + t0 + tid] = r;
            tmin = fminf(tmin, r);
        }
    }
    int nt = 0;
    if (!failed) {
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            tmin = fminf(tmin, __shfl_xor_sync(0xffffffffu, tmin, o));
            r2max = fmaxf(r2max, __shfl_xor_sync(0xffffffffu, r2max, o));
        }
        if (lane == 0) {
            wred[warp] = tmin;
            wred[8 + warp] = r2max;
        }
        __syncthreads();
        float rmin = wred[0], r2 = wred[8];
        for (int w = 1; w < 8; ++w) {
            rmin = fminf(rmin, wred[w]);
            r2 = fmaxf(r2, wred[8 + w]);
        }
        const float R = sqrtf(r2) * 1.0001f + 1e-4f;
        // chunk bound, thread k: surviving clusters listed in ascending order
        bool keep_k = false;
        if (tid < K && tid != h) {
            const float d = M[(size_t)h * K + tid] - lam[tid] * R;
            const float ub = cvec[3 * tid] - 0.5f * (d > 0.f ? d * d : 0.f);
            keep_k = !(ub < rmin - margin);
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep_k);
        if (lane == 0) wcnt[warp] = __popc(bal);
        __syncthreads();
        int off = 0;
        for (int w = 0; w < 8; ++w) {
            const int cw = wcnt[w];
            off += w < warp ? cw : 0;
            nt += cw;
        }
        if (keep_k) sk[off + __popc(bal & ((1u << lane) - 1u))] = tid;
        __syncthreads();
        if (nt > 0) {
            // candidate operand: row a = v_{h, sk[a]} (split BF16), zero rows up to the tile edge
            const int nbt = (nt + BN - 1) / BN;
            for (int e = tid; e < nbt * BN * 8; e += 256) {
                const int n = e / 8, c8 = e % 8;
                float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                if (n < nt && c8 * 8 < DP) {
                    const float4* src = reinterpret_cast<const float4*>(V + ((size_t)h * K + sk[n]) * DP + c8 * 8);
                    const float4 a = src[0], b = src[1];
                    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
                    v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
                }
                __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) bf16_split(v[j], hi[j], lo[j]);
                uint8_t* base = sB + (size_t)(n / BN) * STAGE_BYTES;
                const uint32_t o = sw128_offset(n % BN, c8 * 8);
                *reinterpret_cast<uint4*>(base + o) = *reinterpret_cast<const uint4*>(hi);
                *reinterpret_cast<uint4*>(base + B_BYTES + o) = *reinterpret_cast<const uint4*>(lo);
            }
            for (int a = tid; a < nt; a += 256) {
                sbeta[a] = beta[(size_t)h * K + sk[a]];
                sck[a] = cvec[3 * sk[a]];
            }
            // phase 2: point bound
            load_perm(0);
            load_rows();
            load_perm(BM);
            for (int t0 = 0; t0 < len; t0 += BM) {
                const int ntn = min(BM, len - t0);
                float unused = 0.f;
                build_a(ntn, false, unused);
                mma_tile(nbt);
                if (t0 + BM < len) {
                    load_rows();
                    load_perm(t0 + 2 * BM);
                }
                const int row = (warp & 3) * 32 + lane;
                const bool valid = row < ntn;
                const float lim = valid ? rh[start + t0 + row] - margin : 0.f;
                if (!mma_wait()) { failed = true; break; }
                const int part = warp >> 2;
                for (int nb = 0; nb < nbt; ++nb) {
#pragma unroll
                    for (int s = 0; s < 2; ++s) {
                        const int a0 = nb * BN + 64 * part + 32 * s;
                        if (a0 >= nt) continue;   // warp-uniform
                        uint32_t v[32];
                        tmem_ld32(tmem_base + lane_addr + (uint32_t)a0, v);
                        uint32_t m = 0u;
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            const int a = a0 + j;
                            if (a < nt) {
                                const float p = __uint_as_float(v[j]) - sbeta[a];
                                const float ub = sck[a] - 0.5f * p * p;
                                if (!(ub < lim)) m |= 1u << j;
                            }
                        }
                        if (!valid) m = 0u;
                        m = __reduce_or_sync(0xffffffffu, m);
                        if (lane == 0 && m) atomicOr(&kbits[a0 >> 5], m);
                    }
                }
                tc_fence_before();
                __syncthreads();
            }
        }
    }
    __syncthreads();
    if (!failed && tid == 0) {
        int n = 0;
        int32_t* cq = cand + (size_t)q * (kPrMaxCand + 1);
        for (int a = 0; a < nt; ++a)
            if ((kbits[a >> 5] >> (a & 31)) & 1u) {
                if (n < kPrMaxCand) cq[1 + n] = sk[a];
                ++n;
            }
        cq[0] = n;
        atomicAdd(&cnt[0], (unsigned long long)n * (unsigned long long)len);
        if (n > kPrMaxCand) atomicAdd(&cnt[1], 1ull);
    }
    if (failed && tid == 0 && !stall) mbar_wait_bounded(bar, (phase - 1) & 1, nullptr);   // nothing in flight at dealloc
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(SCAN_TMEM_COLS));
    }
}


// Single-pass form of the same scan for K - 1 <= kScan1MaxCand: B = [W_h | v_h,k for every k != h]
// (h's 64 rows copied from the dense phase's packed tile, then one row per other cluster, ascending),
// so one gather and one group of MMAs per 128-point tile give r_h and every projection.  The drain
// records, per cluster, whether the point bound keeps it at some point of the chunk; after the last
// tile the chunk bound (r_min and radius of the whole chunk) is applied to those, which is the same
// kept set as the two-pass form (chunk bound first, point bound on its survivors).
constexpr int kScan1MaxCand = 2 * BN - KD;   // 192 other clusters
template <int DP>
__global__ void __launch_bounds__(256, 2) k_prune_scan1_tc(
    const float* __restrict__ x, const int32_t* __restrict__ perm, const int32_t* __restrict__ chunk,
    const int32_t* __restrict__ nchunks, const uint8_t* __restrict__ Btc, const float* __restrict__ bvec,
    const float* __restrict__ cvec, const float* __restrict__ mu, const float* __restrict__ lam,
    const float* __restrict__ M, const float* __restrict__ V, const float* __restrict__ beta, int K, float margin,
    float* __restrict__ rh, int32_t* __restrict__ cand, unsigned long long* __restrict__ cnt,
    int32_t* __restrict__ err, int stall)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* sA = smem + ScanSmem::a;
    uint8_t* sB = smem + ScanSmem::b;
    float* sq = reinterpret_cast<float*>(smem + ScanSmem::sq);
    float* sbias = reinterpret_cast<float*>(smem + ScanSmem::bias);
    float* sbeta = reinterpret_cast<float*>(smem + ScanSmem::cb);
    float* sck = sbeta + kScanMaxK;
    int32_t* skeep = reinterpret_cast<int32_t*>(smem + ScanSmem::ck);   // chunk-bound verdict per candidate
    uint32_t* kbits = reinterpret_cast<uint32_t*>(smem + ScanSmem::bits);
    float* wred = reinterpret_cast<float*>(kbits + kScanMaxK / 32);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + ScanSmem::bar);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
    volatile int* flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int q = blockIdx.x;
    if (q >= *nchunks) return;
    const int h = chunk[3 * q], start = chunk[3 * q + 1], len = chunk[3 * q + 2];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const volatile int32_t* gerr = err;
    const int nt = K - 1;                                   // candidate a is cluster a + (a >= h)
    const int nbt = (KD + nt + BN - 1) / BN;                // B tiles (1 or 2)
    auto cand_k = [&](int a) { return a + (a >= h ? 1 : 0); };

    {
        // rows 0..63: cluster h's rows of its packed pair tile (same swizzle phase: 64 is a multiple of 8)
        const uint8_t* tile = Btc + (size_t)(h / CPT) * STAGE_BYTES + (size_t)(h % CPT) * KD * 128;
        for (int e = tid; e < 2 * KD * 128 / 16; e += 256) {
            const int half = e / (KD * 8), o = e % (KD * 8);
            reinterpret_cast<uint4*>(sB + half * B_BYTES)[o] = reinterpret_cast<const uint4*>(tile + half * B_BYTES)[o];
        }
        // rows 64 .. : v_h,k of every other cluster (split BF16), zero up to the tile edge
        for (int e = tid; e < (nbt * BN - KD) * 8; e += 256) {
            const int a = e / 8, c8 = e % 8, n = KD + a;
            float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            if (a < nt && c8 * 8 < DP) {
                const float4* src = reinterpret_cast<const float4*>(V + ((size_t)h * K + cand_k(a)) * DP + c8 * 8);
                const float4 u0 = src[0], u1 = src[1];
                v[0] = u0.x; v[1] = u0.y; v[2] = u0.z; v[3] = u0.w;
                v[4] = u1.x; v[5] = u1.y; v[6] = u1.z; v[7] = u1.w;
            }
            __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) bf16_split(v[j], hi[j], lo[j]);
            uint8_t* base = sB + (size_t)(n / BN) * STAGE_BYTES;
            const uint32_t o = sw128_offset(n % BN, c8 * 8);
            *reinterpret_cast<uint4*>(base + o) = *reinterpret_cast<const uint4*>(hi);
            *reinterpret_cast<uint4*>(base + B_BYTES + o) = *reinterpret_cast<const uint4*>(lo);
        }
        for (int a = tid; a < nt; a += 256) {
            const int k = cand_k(a);
            sbeta[a] = beta[(size_t)h * K + k];
            sck[a] = cvec[3 * k];
        }
        if (tid < 2 * KD) {
            const int side = tid / KD, j = tid % KD;
            sbias[tid] = j < DP ? (side ? mu : bvec)[(size_t)3 * h * DP + j] : 0.f;
        }
        if (tid < kScanMaxK / 32) kbits[tid] = 0u;
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        *flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(SCAN_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const uint32_t lane_addr = (uint32_t)((warp & 3) * 32) << 16;
    const float ch = cvec[3 * h];

    // gathered rows: item u of this thread is (row tid / 8 + 32 u, 8-float chunk tid % 8); a tile's
    // permutation entries load one tile ahead of its rows
    float4 pf[4][2];
    int pq[4];
    auto load_perm = [&](int t0) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int row = (tid >> 3) + 32 * u;
            pq[u] = t0 + row < len ? __ldg(perm + start + t0 + row) : -1;
        }
    };
    auto load_rows = [&]() {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int c8 = tid & 7;
            pf[u][0] = make_float4(0.f, 0.f, 0.f, 0.f);
            pf[u][1] = pf[u][0];
            if (pq[u] >= 0 && c8 * 8 < DP) {
                const float4* src = reinterpret_cast<const float4*>(x + (size_t)pq[u] * DP + c8 * 8);
                pf[u][0] = __ldg(src);
                pf[u][1] = __ldg(src + 1);
            }
        }
    };

    uint32_t phase = 0;
    bool failed = false;
    float tmin = INFINITY, r2max = 0.f;
    const uint64_t da_h = sw128_desc(smem_u32(sA)), da_l = sw128_desc(smem_u32(sA + A_BYTES));
    load_perm(0);
    load_rows();
    load_perm(BM);
    for (int t0 = 0; t0 < len; t0 += BM) {
        const int ntn = min(BM, len - t0);
        // A tile from the rows, and the largest |x - mu_h|^2
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int row = (tid >> 3) + 32 * u, c8 = tid & 7;
            const float v[8] = {pf[u][0].x, pf[u][0].y, pf[u][0].z, pf[u][0].w,
                                pf[u][1].x, pf[u][1].y, pf[u][1].z, pf[u][1].w};
            __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) bf16_split(v[e], hi[e], lo[e]);
            const uint32_t off = sw128_offset(row, c8 * 8);
            *reinterpret_cast<uint4*>(sA + off) = *reinterpret_cast<const uint4*>(hi);
            *reinterpret_cast<uint4*>(sA + A_BYTES + off) = *reinterpret_cast<const uint4*>(lo);
            float d2 = 0.f;
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const float tt = v[e] - sbias[KD + c8 * 8 + e];
                d2 = fmaf(tt, tt, d2);
            }
            d2 += __shfl_xor_sync(0xffffffffu, d2, 1);
            d2 += __shfl_xor_sync(0xffffffffu, d2, 2);
            d2 += __shfl_xor_sync(0xffffffffu, d2, 4);
            if (row < ntn) r2max = fmaxf(r2max, d2);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        if (tid == 0 && !stall) {   // stall: the wait-test seam issues nothing
            tc_fence_after();
            for (int nb = 0; nb < nbt; ++nb) {
                const uint8_t* bt = sB + (size_t)nb * STAGE_BYTES;
                const uint64_t db_h = sw128_desc(smem_u32(bt)), db_l = sw128_desc(smem_u32(bt + B_BYTES));
                const uint32_t td = tmem_base + (uint32_t)(nb * BN);
#pragma unroll
                for (int ks = 0; ks < KD / 16; ++ks) umma_bf16(td, da_h + 2 * ks, db_h + 2 * ks, ks != 0 ? 1u : 0u);
#pragma unroll
                for (int ks = 0; ks < KD / 16; ++ks) umma_bf16(td, da_l + 2 * ks, db_h + 2 * ks, 1u);
#pragma unroll
                for (int ks = 0; ks < KD / 16; ++ks) umma_bf16(td, da_h + 2 * ks, db_l + 2 * ks, 1u);
            }
            umma_commit(bar);
        }
        if (t0 + BM < len) {   // the next tile's rows load while the MMAs run
            load_rows();
            load_perm(t0 + 2 * BM);
        }
        if (tid == 0 && !mbar_wait_bounded(bar, phase & 1, gerr)) {
            atomicCAS(err, 0, ERR_TIMEOUT_TFULL);
            *flag = 1;
        }
        ++phase;
        __syncthreads();
        if (*flag) { failed = true; break; }
        tc_fence_after();
        const int part = warp >> 2, row = (warp & 3) * 32 + lane;
        {   // r_h from columns 0..63
            float qs = 0.f;
            if (DP > 32 || part == 0) {
                uint32_t v[32];
                tmem_ld32(tmem_base + lane_addr + (uint32_t)(32 * part), v);
                const float* bs = sbias + 32 * part;
                float q1 = 0.f;
#pragma unroll
                for (int j = 0; j < 32; j += 2) {
                    const float z0 = __uint_as_float(v[j]) - bs[j];
                    const float z1 = __uint_as_float(v[j + 1]) - bs[j + 1];
                    qs = fmaf(z0, z0, qs);
                    q1 = fmaf(z1, z1, q1);
                }
                qs += q1;
            }
            sq[part * BM + row] = qs;
        }
        __syncthreads();
        float r_row = 0.f;
        if (tid < BM) r_row = ch - 0.5f * (sq[tid] + sq[BM + tid]);
        __syncthreads();
        if (tid < BM) {
            sq[tid] = r_row;
            if (tid < ntn) {
                rh[start + t0 + tid] = r_row;
                tmin = fminf(tmin, r_row);
            }
        }
        __syncthreads();
        {   // point bound of every candidate: columns 64 + a
            const bool valid = row < ntn;
            const float lim = valid ? sq[row] - margin : 0.f;
            for (int g = 2 + part; 32 * (g - 2) < nt; g += 2) {   // warp-uniform
                uint32_t v[32];
                tmem_ld32(tmem_base + lane_addr + (uint32_t)(32 * g), v);
                const int a0 = 32 * (g - 2);
                uint32_t m = 0u;
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int a = a0 + j;
                    if (a < nt) {
                        const float p = __uint_as_float(v[j]) - sbeta[a];
                        const float ub = sck[a] - 0.5f * p * p;
                        if (!(ub < lim)) m |= 1u << j;
                    }
                }
                if (!valid) m = 0u;
                m = __reduce_or_sync(0xffffffffu, m);
                if (lane == 0 && m) atomicOr(&kbits[g - 2], m);
            }
        }
        tc_fence_before();
        __syncthreads();
    }
    if (!failed) {
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            tmin = fminf(tmin, __shfl_xor_sync(0xffffffffu, tmin, o));
            r2max = fmaxf(r2max, __shfl_xor_sync(0xffffffffu, r2max, o));
        }
        if (lane == 0) {
            wred[warp] = tmin;
            wred[8 + warp] = r2max;
        }
        __syncthreads();
        float rmin = wred[0], r2 = wred[8];
        for (int w = 1; w < 8; ++w) {
            rmin = fminf(rmin, wred[w]);
            r2 = fmaxf(r2, wred[8 + w]);
        }
        const float R = sqrtf(r2) * 1.0001f + 1e-4f;
        for (int a = tid; a < nt; a += 256) {   // chunk bound
            const int k = cand_k(a);
            const float d = M[(size_t)h * K + k] - lam[k] * R;
            const float ub = cvec[3 * k] - 0.5f * (d > 0.f ? d * d : 0.f);
            skeep[a] = !(ub < rmin - margin);
        }
    }
    __syncthreads();
    if (!failed && tid == 0) {
        int n = 0;
        int32_t* cq = cand + (size_t)q * (kPrMaxCand + 1);
        for (int a = 0; a < nt; ++a)
            if (skeep[a] && ((kbits[a >> 5] >> (a & 31)) & 1u)) {
                if (n < kPrMaxCand) cq[1 + n] = cand_k(a);
                ++n;
            }
        cq[0] = n;
        atomicAdd(&cnt[0], (unsigned long long)n * (unsigned long long)len);
        if (n > kPrMaxCand) atomicAdd(&cnt[1], 1ull);
    }
    if (failed && tid == 0 && !stall) mbar_wait_bounded(bar, (phase - 1) & 1, nullptr);   // nothing in flight at dealloc
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(SCAN_TMEM_COLS));
    }
}

// ------------------------------------------------------------------------- slot statistics
// Statistics of the two sub-clusters of one chunk (cluster k, sub-labels given) on the tensor
// cores, Dp = 32 or 64: count, sum c and the upper triangle of sum c c^T over each sub-cluster's
// points, c = x - mu_k (mu_k the cluster's mean parameter), the partial records of
// k_gauss_slot_stats (dpmm_kernels.cu).  Per tile of 32 points (the contraction dimension K):
//   A (M = 128 x K, MN-major TF32)   column 64 s + i, point p: c_i(p) where p's sub-label is s + 1,
//                                    else 0 (columns Dp .. 63 of each half stay 0)
//   B (N = Dp + 32 x K, MN-major)    column j < Dp: c_j(p); column Dp: 1; the rest 0
//   D = A B^T                        D[64 s + i][j] = sum c_i c_j, D[64 s + i][Dp] = sum c_i
// MN-major means the operand is stored point by point: each point's row is its features, in
// 128-byte rows of 32 features.  TF32 MN-major operands take the 128-byte swizzle with 32-byte
// atomicity (the one MN-major layout the tensor cores accept for TF32): an atom is 4 points x 128 B,
// its 32-byte pieces XOR-permuted by the point's row (0..3); atoms along M / N at 512 B, groups of 4
// points at 4 x 512 B for A and (Dp + 32) / 32 x 512 B for B.  A row is built from the staged FP32
// row with 16-byte stores.  The ones column lives in B's last atom, written once.
// The operands are split TF32 (hi = rna(c), lo = rna(c - hi), |c - hi - lo| <= 2^-22 |c|) and
// D = A_hi B_hi + A_lo B_hi + A_hi B_lo (12 tcgen05.mma of K = 8).  The accumulator runs over a
// group of ST_G tiles (FP32 over 256 points: 96 accumulator roundings) and is then added into FP64
// registers; two accumulators in TMEM alternate by group.  The products are centred at the mean a
// of the chunk's first tile (within a cluster's spread of every point, wherever mu_k lies) and the
// totals moved to mu_k in FP64 at the end:
//   sum (x-mu)(x-mu)^T = S_a + d S1^T + S1 d^T + n d d^T,  sum (x-mu) = S1 + n d,  d = a - mu.
// Pipeline: tile t + 3's rows and sub-labels (gathered through permutation entries that were
// staged three tiles earlier, all by cp.async) are in flight while tile t is split into the
// operands; a group's accumulator is drained while the next group's MMAs run.  Every wait is
// bounded.
constexpr int ST_P = 32;                   // points per tile (K of the contraction)
constexpr int ST_STAGES = 4;               // staged tiles of rows (3 in flight)
constexpr int ST_PERM = 8;                 // staged tiles of permutation entries
constexpr int ST_G = 8;                    // tiles per accumulation group
constexpr uint32_t ST_TMEM_COLS = 256;     // two accumulators, at columns 0 and 128

template <int DP>
struct StatSmem {
    static constexpr int NA = DP / 32 + 1;                              // B atoms: features, then ones
    static constexpr int N = NA * 32;                                   // B columns (N of the MMA)
    static constexpr int SX = DP + 4;                                   // staged row stride (floats)
    static constexpr size_t a_hi = 0;                                   // 4 groups x 4 atoms x 1 KB
    static constexpr size_t a_lo = a_hi + 16384;
    static constexpr size_t b_hi = a_lo + 16384;                        // 4 groups x NA atoms x 1 KB
    static constexpr size_t b_lo = b_hi + (size_t)NA * 4096;
    static constexpr size_t stage = b_lo + (size_t)NA * 4096;           // [ST_STAGES][ST_P][SX] floats
    static constexpr size_t ssub = stage + (size_t)ST_STAGES * ST_P * SX * 4;   // [ST_STAGES][ST_P] ints
    static constexpr size_t sperm = ssub + (size_t)ST_STAGES * ST_P * 4;        // [ST_PERM][ST_P] ints
    static constexpr size_t shift = sperm + (size_t)ST_PERM * ST_P * 4;         // [DP] floats
    static constexpr size_t bar = shift + (size_t)DP * 4;               // mbarrier, tmem slot, flag
    static constexpr size_t total = bar + 32 + 1024;                    // + alignment slack
};

// Shared-memory descriptor of an MN-major TF32 operand with the 128-byte swizzle of 32-byte atomicity:
// atoms of 4 rows (K) x 128 B (32 elements of M / N) 512 B apart along M / N (leading byte offset),
// groups of 4 rows sbo bytes apart along K (stride byte offset).
__device__ __forceinline__ uint64_t sw128b32_mn_desc(uint32_t saddr, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)(512 >> 4) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)1 << 61;   // 128-byte swizzle, 32-byte atomicity
    return d;
}

// byte offset of the 16-byte piece j4 (elements 4 j4 .. 4 j4 + 3 of M / N) of row p (K) in such an
// operand whose groups of 4 rows hold `atoms` atoms; the piece's atom is (j4 >> 3) + atom0
__device__ __forceinline__ uint32_t mn32_offset(int p, int j4, int atom0, int atoms)
{
    const int r = p & 3;
    return (uint32_t)((p >> 2) * atoms * 512 + ((j4 >> 3) + atom0) * 512 + r * 128 + ((((j4 & 7) >> 1) ^ r) << 5) +
                      ((j4 & 1) << 4));
}

// round to TF32 (10 explicit mantissa bits), nearest with ties away from zero: add half of the
// dropped 13-bit field to the magnitude and clear it (finite inputs; integer pipe)
__device__ __forceinline__ float tf32_rna(float v)
{
    return __uint_as_float((__float_as_uint(v) + 0x1000u) & 0xFFFFE000u);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accum)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
        : "memory");
}

__device__ __forceinline__ void tmem_ld1(uint32_t taddr, uint32_t& r)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src, uint32_t src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}

__device__ __forceinline__ void cp_async4(void* dst, const void* src, uint32_t src_bytes)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// the barrier receives one arrival once every cp.async this thread issued so far has landed (its
// expected count includes these arrivals)
__device__ __forceinline__ void cp_async_mbar_arrive(uint64_t* bar)
{
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <int DP>
__global__ void __launch_bounds__(256, 2) k_slot_stats_tc(
    const float* __restrict__ x, const int32_t* __restrict__ perm, const int32_t* __restrict__ chunk,
    const int32_t* __restrict__ nchunks, const float* __restrict__ muv, const int32_t* __restrict__ sub,
    double* __restrict__ part, const uint8_t* __restrict__ mask, int32_t* __restrict__ err, int stall)
{
    using L = StatSmem<DP>;
    constexpr int N = L::N, NA = L::NA, SX = L::SX;
    constexpr int SL = 1 + DP + tri(DP);
    constexpr int C4 = DP / 4;                     // float4 per row
    constexpr int ITEMS = ST_P * C4 / 256;         // row pieces per thread per tile
    static_assert(ITEMS >= 1 && ST_P * C4 % 256 == 0 && 256 % C4 == 0, "tile shape");
    // F32 accumulator, TF32 A and B, both MN-major, M = 128
    constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | (1u << 15) | (1u << 16) |
                               ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    constexpr uint32_t A_GROUP = 4096, B_GROUP = NA * 1024;   // bytes per 8 points (two groups of 4)
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    float* stage = reinterpret_cast<float*>(smem + L::stage);
    int32_t* ssub = reinterpret_cast<int32_t*>(smem + L::ssub);
    int32_t* sperm = reinterpret_cast<int32_t*>(smem + L::sperm);
    float* sshift = reinterpret_cast<float*>(smem + L::shift);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L::bar);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
    volatile int* flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int ch = blockIdx.x;
    if (ch >= *nchunks) return;
    const int k = chunk[3 * ch], start = chunk[3 * ch + 1], len = chunk[3 * ch + 2];
    if (mask && !mask[k]) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const volatile int32_t* gerr = err;
    const int ntiles = (len + ST_P - 1) / ST_P;

    // operands zeroed once (rows past Dp stay zero), then the ones row of B
    for (int e = tid; e < (int)(L::stage / 16); e += 256) reinterpret_cast<uint4*>(smem)[e] = make_uint4(0u, 0u, 0u, 0u);
    if (tid == 0) {
        mbar_init(bar, 1);
        *flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(ST_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    if (tid < ST_P)   // the ones column: element 0 of B's last atom in every point's row (hi part)
        *reinterpret_cast<float*>(smem + L::b_hi + mn32_offset(tid, 0, NA - 1, NA)) = 1.0f;

    // loader pieces (cp.async; the caller commits)
    auto issue_perm = [&](int t) {   // permutation entries of tile t (threads 0..31; 0 past the chunk)
        if (t < ntiles && tid < ST_P) {
            const int i = t * ST_P + tid;
            const bool ok = i < len;
            cp_async4(sperm + (t % ST_PERM) * ST_P + tid, ok ? perm + start + i : perm, ok ? 4u : 0u);
        }
    };
    auto issue_rows = [&](int t) {   // rows and sub-labels of tile t (zero past the chunk)
        if (t >= ntiles) return;
        float* sb = stage + (size_t)(t % ST_STAGES) * ST_P * SX;
        int32_t* sbs = ssub + (t % ST_STAGES) * ST_P;
        const int32_t* pp = sperm + (t % ST_PERM) * ST_P;
#pragma unroll
        for (int u = 0; u < ITEMS; ++u) {
            const int e = tid + 256 * u, row = e / C4, c4 = e % C4;
            const bool ok = t * ST_P + row < len;
            const int64_t pt = ok ? pp[row] : 0;
            cp_async16(sb + row * SX + 4 * c4, x + (size_t)pt * DP + 4 * c4, ok ? 16u : 0u);
            if (c4 == 0) cp_async4(sbs + row, sub + pt, ok ? 4u : 0u);
        }
    };
    // prologue: entries of tiles 0..2 (waited), then per tile j < 3 its rows and tile j + 3's entries
    for (int t = 0; t < 3; ++t) issue_perm(t);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
#pragma unroll 1
    for (int j = 0; j < 3; ++j) {
        issue_rows(j);
        issue_perm(j + 3);
        cp_async_commit();
    }

    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const uint64_t da_h = sw128b32_mn_desc(smem_u32(smem + L::a_hi), A_GROUP / 2);
    const uint64_t da_l = sw128b32_mn_desc(smem_u32(smem + L::a_lo), A_GROUP / 2);
    const uint64_t db_h = sw128b32_mn_desc(smem_u32(smem + L::b_hi), B_GROUP / 2);
    const uint64_t db_l = sw128b32_mn_desc(smem_u32(smem + L::b_lo), B_GROUP / 2);
    // operand pieces of this thread: point tid / C4 + (256 / C4) u, features 4 (tid % C4) ..; their
    // offsets in the operands (side l's half of A, then + 1024 for side r; B) for u = 0, and the step
    // to the next u (whole groups of 4 points)
    const int j4 = tid % C4;
    const uint32_t a_off0 = mn32_offset(tid / C4, j4, 0, 4), b_off0 = mn32_offset(tid / C4, j4, 0, NA);
    constexpr uint32_t A_STEP = (256 / C4) / 4 * 4 * 512, B_STEP = (256 / C4) / 4 * NA * 512;
    float4 s4 = make_float4(0.f, 0.f, 0.f, 0.f);   // its four centre coordinates (set at tile 0)

    // drain role: TMEM lane quarter q (accumulator rows 32 q ..), column half hc
    const int q = warp & 3, hc = warp >> 2;
    const int slot = q >> 1, fi = (q & 1) * 32 + lane;   // sub-cluster, feature i of this lane's row
    const bool row_live = (q & 1) * 32 < DP;            // warp-uniform
    const bool do_s = row_live && (DP > 32 ? (q & 1) <= hc : hc == 0);
    const bool do_sum = row_live && hc == 0;
    double acc[32];
#pragma unroll
    for (int m = 0; m < 32; ++m) acc[m] = 0.0;
    double sacc = 0.0;
    int cnt_l = 0, cnt_r = 0;
    auto drain = [&](int g) {   // accumulator of group g (its MMAs complete)
        const uint32_t base = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)((g & 1) * 128);
        if (do_s) {
            uint32_t v[32];
            tmem_ld32(base + (uint32_t)(32 * hc), v);
#pragma unroll
            for (int m = 0; m < 32; ++m) acc[m] += (double)__uint_as_float(v[m]);
        }
        if (do_sum) {
            uint32_t v1;
            tmem_ld1(base + (uint32_t)DP, v1);
            sacc += (double)__uint_as_float(v1);
        }
    };
    // block-uniform: tile t's MMAs (the t-th commit) complete
    auto wait_mma = [&](int t) -> bool {
        if (tid == 0 && !mbar_wait_bounded(bar, (uint32_t)(t & 1), gerr)) {
            atomicCAS(err, 0, ERR_TIMEOUT_TFULL);
            *flag = 1;
        }
        __syncthreads();
        return *flag == 0;
    };

    bool failed = false;
    int pending = -1;   // tile whose MMAs were issued and not yet seen complete
#pragma unroll 1
    for (int t = 0; t < ntiles; ++t) {
        cp_async_wait<2>();   // this thread's rows of tile t and entries of tile t + 3 have landed
        if (t > 0) {
            if (!wait_mma(t - 1)) { failed = true; break; }
            pending = -1;
        } else {
            __syncthreads();
            if (tid < DP) {   // centre: mean of the first tile's points
                const int nv = min(ST_P, len);
                float a = 0.f;
                for (int r = 0; r < nv; ++r) a += stage[r * SX + tid];
                sshift[tid] = a / (float)nv;
            }
            __syncthreads();
            s4 = *reinterpret_cast<const float4*>(sshift + 4 * j4);
        }
        tc_fence_after();
        issue_rows(t + 3);
        issue_perm(t + 6);
        cp_async_commit();
        {
            const float* sb = stage + (size_t)(t % ST_STAGES) * ST_P * SX;
            const int32_t* sbs = ssub + (t % ST_STAGES) * ST_P;
            if (warp == 0) {
                const int sv = sbs[lane];
                const unsigned bl = __ballot_sync(0xffffffffu, sv == 1), br = __ballot_sync(0xffffffffu, sv == 2);
                cnt_l += __popc(bl);
                cnt_r += __popc(br);
            }
            // one 16-byte piece of a point's row per item: split, then stored into the side's half of
            // A (zeros into the other half) and into B; a point past the chunk (sub-label 0) is all zero
#pragma unroll
            for (int u = 0; u < ITEMS; ++u) {
                const int p = tid / C4 + (256 / C4) * u;
                const int sv = sbs[p];
                const float4 v4 = *reinterpret_cast<const float4*>(sb + p * SX + 4 * j4);
                const float cv[4] = {v4.x - s4.x, v4.y - s4.y, v4.z - s4.z, v4.w - s4.w};
                float hi[4], lo[4];
                const bool live = sv == 1 || sv == 2;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    hi[e] = tf32_rna(cv[e]);
                    lo[e] = tf32_rna(cv[e] - hi[e]);
                    if (!live) hi[e] = lo[e] = 0.f;
                }
                const uint32_t a0 = a_off0 + A_STEP * u, b_o = b_off0 + B_STEP * u;
                const uint32_t a_c = sv == 2 ? a0 + 1024 : a0, a_z = sv == 2 ? a0 : a0 + 1024;
                const uint4 h4 = make_uint4(__float_as_uint(hi[0]), __float_as_uint(hi[1]), __float_as_uint(hi[2]),
                                            __float_as_uint(hi[3]));
                const uint4 l4 = make_uint4(__float_as_uint(lo[0]), __float_as_uint(lo[1]), __float_as_uint(lo[2]),
                                            __float_as_uint(lo[3]));
                const uint4 z4 = make_uint4(0u, 0u, 0u, 0u);
                *reinterpret_cast<uint4*>(smem + L::a_hi + a_c) = h4;
                *reinterpret_cast<uint4*>(smem + L::a_lo + a_c) = l4;
                *reinterpret_cast<uint4*>(smem + L::a_hi + a_z) = z4;
                *reinterpret_cast<uint4*>(smem + L::a_lo + a_z) = z4;
                *reinterpret_cast<uint4*>(smem + L::b_hi + b_o) = h4;
                *reinterpret_cast<uint4*>(smem + L::b_lo + b_o) = l4;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        const int grp = t / ST_G;
        if (tid == 0 && !stall) {   // stall: the wait-test seam issues nothing
            tc_fence_after();
            const uint32_t td = tmem_base + (uint32_t)((grp & 1) * 128);
            const uint32_t first = (t % ST_G) == 0 ? 0u : 1u;   // a fresh accumulator per group
#pragma unroll
            for (int ks = 0; ks < ST_P / 8; ++ks)   // one group of 8 points per MMA (K = 8)
                umma_tf32(td, da_h + (A_GROUP >> 4) * ks, db_h + (B_GROUP >> 4) * ks, IDESC, ks != 0 ? 1u : first);
#pragma unroll
            for (int ks = 0; ks < ST_P / 8; ++ks)
                umma_tf32(td, da_l + (A_GROUP >> 4) * ks, db_h + (B_GROUP >> 4) * ks, IDESC, 1u);
#pragma unroll
            for (int ks = 0; ks < ST_P / 8; ++ks)
                umma_tf32(td, da_h + (A_GROUP >> 4) * ks, db_l + (B_GROUP >> 4) * ks, IDESC, 1u);
            umma_commit(bar);
        }
        pending = t;
        // the previous group's last MMAs completed (waited above): drain it while this group runs
        if (t % ST_G == 0 && grp > 0) drain(grp - 1);
        tc_fence_before();
    }
    if (!failed && ntiles > 0) {
        if (wait_mma(ntiles - 1)) {
            pending = -1;
            tc_fence_after();
            drain((ntiles - 1) / ST_G);
        } else {
            failed = true;
        }
    }
    cp_async_wait<0>();
    __syncthreads();   // the stage area now holds the sums, counts and d for the move to mu_k
    double* xs = reinterpret_cast<double*>(smem + L::stage);   // [2][DP] sums S1
    double* xd = xs + 2 * DP;                                  // [DP] d = a - mu_k
    double* xn = xd + DP;                                      // [2] counts
    if (!failed) {
        if (do_sum) xs[slot * DP + fi] = sacc;
        if (tid < DP) xd[tid] = ntiles > 0 ? (double)sshift[tid] - (double)muv[(size_t)3 * k * DP + tid] : 0.0;
        if (tid == 0) {
            xn[0] = (double)cnt_l;
            xn[1] = (double)cnt_r;
        }
    }
    __syncthreads();
    if (!failed) {
        double* out = part + (size_t)ch * 2 * SL;
        if (tid < 2) out[(size_t)tid * SL] = xn[tid];
        const double n = xn[slot];
        if (do_s) {
            double* po = out + (size_t)slot * SL + 1 + DP;
            const double di = xd[fi], si = xs[slot * DP + fi];
#pragma unroll
            for (int m = 0; m < 32; ++m) {
                const int j = 32 * hc + m;
                if (fi <= j && j < DP) {
                    const double dj = xd[j], sj = xs[slot * DP + j];
                    po[tri_index(DP, fi, j)] = acc[m] + di * sj + si * dj + n * di * dj;
                }
            }
        }
        if (do_sum) out[(size_t)slot * SL + 1 + fi] = sacc + n * xd[fi];
    }
    if (failed && tid == 0 && pending >= 0 && !stall)   // nothing in flight at dealloc
        mbar_wait_bounded(bar, (uint32_t)(pending & 1), nullptr);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(ST_TMEM_COLS));
    }
}


// ------------------------------------------------------------------------- fused sub-labels + statistics
// One pass over the points of a chunk (cluster k, label order) for both steps that follow the label
// phase: the sub-cluster labels (cudaKernel.cu create_subclusters_labels, :1299-1398) and then the
// sub-cluster statistics of the drawn labels (niw::create_sufficient_statistics per slot); each point's
// row is gathered from HBM once.  Per super-tile of 128 points:
//   sub-labels   the rows (split BF16, K-major, a point per row) times the cluster's [W_l | W_r] tile
//                give z for both sub-clusters (the 12 tcgen05.mma of k_sub_labels_tc); one thread per
//                point drains r_l and r_r and draws its sub-label;
//   statistics   8 tiles of 16 points feed the split-TF32 Gram products of k_slot_stats_tc
//                (MN-major operands, 6 tcgen05.mma of K = 8 per tile) into an FP32 accumulator of
//                256 points, added into FP64 registers per group.
// Warp roles (320 threads; the shared memory holds one CTA per SM), three chains that overlap:
//   warp 0       loader: the permutation entries, then the rows into a three-slot stage by 16-byte
//                cp.async (a warp instruction copies whole rows; per-row bulk copies measured several
//                times slower for 256-byte rows); the cluster's B tile once per chunk;
//   warp 1       MMA issuer (one thread): sub-label products of super-tile T + 1, then the
//                statistics tiles of T, the order in which the two groups produce their operands;
//   warps 2..5   sub-label group (a thread per point): the row -> the sub-label operand, then r and
//                the draw; it runs up to two super-tiles ahead of
//   warps 6..9   statistics group: the operand tiles of a super-tile whose sub-labels are drawn, from
//                the same staged rows; it frees the stage slot.
// Both groups drain the accumulation groups into FP64 (32 values per thread each).  Every wait is
// bounded; on a failure every role stops, waits (bounded) for the copies or products it issued, and
// the tensor memory is freed.  Output: the partial record per chunk of k_slot_stats_tc; sub[].
constexpr int SS_T = 128;                        // points per super-tile (M of the sub-label products)
constexpr int SS_SLOTS = 3;                      // staged super-tiles of rows (and of drawn sub-labels)
constexpr int SS_PIDX = 4;                       // staged super-tiles of permutation entries
constexpr int SS_KT = 16;                        // points per statistics tile (two groups of 8)
constexpr int SS_TPS = SS_T / SS_KT;             // statistics tiles per super-tile
constexpr int SS_G = 16;                         // statistics tiles per accumulation group (256 points)
constexpr int SS_THREADS = 320;
constexpr uint32_t SS_TMEM_COLS = 512;           // statistics accumulators at 0 and 128, sub-labels at 256
constexpr uint32_t SS_SUBC = 256;

enum : int {
    SB_BFULL = 0, SB_FULL = 1, SB_EMPTY = SB_FULL + SS_SLOTS, SB_SUBREADY = SB_EMPTY + SS_SLOTS,
    SB_AFULL = SB_SUBREADY + SS_SLOTS, SB_SUBDONE = SB_AFULL + 1, SB_STFULL = SB_SUBDONE + 1,
    SB_STFREE = SB_STFULL + 2, SB_GRPDONE = SB_STFREE + 2, SB_ACCEMPTY = SB_GRPDONE + 2, SB_COUNT = SB_ACCEMPTY + 2
};

template <int DP>
struct SubStatSmem {
    static constexpr int NA = DP / 32 + 1;                     // statistics B atoms: features, then ones
    static constexpr uint32_t A_GROUP = 4096, B_GROUP = NA * 1024;   // bytes per 8 points (two groups of 4)
    static constexpr uint32_t OP_AH = 0, OP_AL = 2 * A_GROUP, OP_BH = 4 * A_GROUP, OP_BL = OP_BH + 2 * B_GROUP;
    static constexpr uint32_t OP_BYTES = OP_BL + 2 * B_GROUP;        // one statistics operand buffer
    static constexpr size_t sb = 0;                                  // 32 KB sub-label B tile (hi, lo)
    static constexpr size_t sa = sb + STAGE_BYTES;                   // 32 KB sub-label A tile (hi, lo)
    static constexpr size_t op = sa + A_TILE;                        // 2 statistics operand buffers
    static constexpr size_t stage = op + 2 * (size_t)OP_BYTES;       // [SS_SLOTS][SS_T][DP] floats
    static constexpr size_t pidx = stage + (size_t)SS_SLOTS * SS_T * DP * 4;   // [SS_PIDX][SS_T] ints
    static constexpr size_t ssub = pidx + (size_t)SS_PIDX * SS_T * 4;          // [SS_SLOTS][SS_T] ints
    static constexpr size_t bias = ssub + (size_t)SS_SLOTS * SS_T * 4;         // [2][KD] floats
    static constexpr size_t shift = bias + (size_t)2 * KD * 4;                 // [64] floats
    static constexpr size_t misc = shift + 64 * 4;                             // counts [2], abort flag
    static constexpr size_t bar = misc + 16;
    static constexpr size_t total = bar + SB_COUNT * 8 + 16 + 1024;           // + tmem slot, alignment
    static_assert(stage % 1024 == 0 && OP_BH % 512 == 0 && OP_BL % 512 == 0 && OP_BYTES % 1024 == 0, "atoms");
    static_assert(total <= 227 * 1024, "shared memory");
};

template <int DP>
__global__ void __launch_bounds__(SS_THREADS, 1) k_sub_stats_tc(
    const float* __restrict__ x, const int32_t* __restrict__ perm, const int32_t* __restrict__ chunk,
    const int32_t* __restrict__ nchunks, const uint8_t* __restrict__ Bsub, const float* __restrict__ bvec,
    const float* __restrict__ cvec, const float* __restrict__ lrw, const float* __restrict__ muv, RngArgs rng,
    int32_t* __restrict__ sub, float* __restrict__ r_out, double* __restrict__ part, int32_t* __restrict__ err,
    int stall)
{
    using L = SubStatSmem<DP>;
    constexpr int NA = L::NA, N = NA * 32, C4 = DP / 4;
    constexpr int SL = 1 + DP + tri(DP);
    constexpr uint32_t A_GROUP = L::A_GROUP, B_GROUP = L::B_GROUP;
    // F32 accumulator, TF32 A and B, both MN-major, M = 128, N = Dp + 32
    constexpr uint32_t IDESC_ST = (1u << 4) | (2u << 7) | (2u << 10) | (1u << 15) | (1u << 16) |
                                  ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* sB = smem + L::sb;
    uint8_t* sA = smem + L::sa;
    uint8_t* sop = smem + L::op;
    float* stage = reinterpret_cast<float*>(smem + L::stage);
    int32_t* spidx = reinterpret_cast<int32_t*>(smem + L::pidx);
    int32_t* ssub = reinterpret_cast<int32_t*>(smem + L::ssub);
    float* sbias = reinterpret_cast<float*>(smem + L::bias);
    float* sshift = reinterpret_cast<float*>(smem + L::shift);
    int* scnt = reinterpret_cast<int*>(smem + L::misc);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(scnt + 2);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::bar);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + SB_COUNT);

    const int ch = blockIdx.x;
    if (ch >= *nchunks) return;
    const int k = chunk[3 * ch], start = chunk[3 * ch + 1], len = chunk[3 * ch + 2];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const volatile int32_t* gerr = err;
    const int nst = (len + SS_T - 1) / SS_T;     // super-tiles
    const int ntt = (len + SS_KT - 1) / SS_KT;   // statistics tiles
    const int ngr = (ntt + SS_G - 1) / SS_G;     // accumulation groups

    // statistics operands zeroed once: A's halves past Dp and B's ones atom rely on it
    for (int e = tid; e < (int)(2 * L::OP_BYTES / 16); e += SS_THREADS)
        reinterpret_cast<uint4*>(sop)[e] = make_uint4(0u, 0u, 0u, 0u);
    if (tid < 2 * KD) {
        const int side = tid / KD, j = tid % KD;
        sbias[tid] = j < DP ? bvec[(size_t)(3 * k + 1 + side) * DP + j] : 0.f;
    }
    if (tid == 0) {
        *abort_flag = *gerr ? 1 : 0;
        scnt[0] = scnt[1] = 0;
        mbar_init(&bars[SB_BFULL], 1);
        for (int s = 0; s < SS_SLOTS; ++s) {
            mbar_init(&bars[SB_FULL + s], 33);    // the loader's 32 lanes' copies, then its lane 0
            mbar_init(&bars[SB_EMPTY + s], 4);    // the statistics group
            mbar_init(&bars[SB_SUBREADY + s], 4); // the sub-label group
        }
        mbar_init(&bars[SB_AFULL], 4);
        mbar_init(&bars[SB_SUBDONE], 1);
        for (int b = 0; b < 2; ++b) {
            mbar_init(&bars[SB_STFULL + b], 4);
            mbar_init(&bars[SB_STFREE + b], 1);
            mbar_init(&bars[SB_GRPDONE + b], 1);
            mbar_init(&bars[SB_ACCEMPTY + b], 8);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(SS_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    if (tid < 2 * SS_KT)   // the ones column: element 0 of B's last atom in every row, both buffers (hi part)
        *reinterpret_cast<float*>(sop + (tid / SS_KT) * L::OP_BYTES + L::OP_BH + mn32_offset(tid % SS_KT, 0, NA - 1, NA)) =
            1.0f;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;
    const bool run = *abort_flag == 0;

    // group drain role of warps 2..9: TMEM lane quarter q, column half hc (0: sub-label group)
    const int q = warp & 3, hc = (warp - 2) >> 2;
    const int dslot = q >> 1, fi = (q & 1) * 32 + lane;   // sub-cluster, feature i of this lane's row
    const bool row_live = (q & 1) * 32 < DP;
    const bool do_s = row_live && (DP > 32 ? (q & 1) <= hc : hc == 0);
    const bool do_sum = row_live && hc == 0;
    double acc[32];
#pragma unroll
    for (int m = 0; m < 32; ++m) acc[m] = 0.0;
    double sacc = 0.0;
    int cnt_l = 0, cnt_r = 0;
    auto drain_group = [&](int g) -> bool {   // warps 2..9, each group once (both halves of the columns)
        if (!warp_wait_bounded(&bars[SB_GRPDONE + (g & 1)], (uint32_t)((g >> 1) & 1), gerr)) {
            if (lane == 0) atomicCAS(err, 0, ERR_TIMEOUT_TFULL);
            return false;
        }
        tc_fence_after();
        const uint32_t base = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)((g & 1) * 128);
        if (do_s) {
            uint32_t v[32];
            tmem_ld32(base + (uint32_t)(32 * hc), v);
#pragma unroll
            for (int i = 0; i < 32; ++i) acc[i] += (double)__uint_as_float(v[i]);
        }
        if (do_sum) {
            uint32_t v1;
            tmem_ld1(base + (uint32_t)DP, v1);
            sacc += (double)__uint_as_float(v1);
        }
        tc_fence_before();
        warp_arrive(&bars[SB_ACCEMPTY + (g & 1)]);
        return true;
    };

    if (warp == 0) {
        // ---------------- loader
        if (run) {
            if (lane == 0) {
                mbar_arrive_expect_tx(&bars[SB_BFULL], STAGE_BYTES);
                bulk_copy_g2s(sB, Bsub + (size_t)k * STAGE_BYTES, STAGE_BYTES, &bars[SB_BFULL]);
            }
            int pe[4];
            auto load_pe = [&](int T) {
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const int row = T * SS_T + 4 * lane + r;
                    pe[r] = row < len ? __ldg(perm + start + row) : -1;
                }
            };
            load_pe(0);
            int issued = 0;
            for (int T = 0; T < nst; ++T) {
                const int slot = T % SS_SLOTS;
                if (T >= SS_SLOTS &&
                    !warp_wait_bounded(&bars[SB_EMPTY + slot], (uint32_t)((T / SS_SLOTS - 1) & 1), gerr)) {
                    if (lane == 0) {
                        atomicCAS(err, 0, ERR_TIMEOUT_EMPTY);
                        *abort_flag = 1;
                    }
                    break;
                }
                if (__any_sync(0xffffffffu, *abort_flag != 0)) break;
                const int nv = min(SS_T, len - T * SS_T);
                int32_t* pix = spidx + (T % SS_PIDX) * SS_T;
#pragma unroll
                for (int r = 0; r < 4; ++r) pix[4 * lane + r] = pe[r];
                __syncwarp();
                // a warp instruction copies 32 / (Dp / 4) whole rows, 16 bytes per lane (zero past the chunk)
                constexpr int RPI = 32 / C4;
                float* sl = stage + (size_t)slot * SS_T * DP;
                const int pc = lane % C4, pr = lane / C4;
#pragma unroll 4
                for (int i = 0; i < SS_T / RPI; ++i) {
                    const int row = RPI * i + pr;
                    const bool live = row < nv;
                    cp_async16(sl + row * DP + 4 * pc, x + (size_t)(live ? pix[row] : 0) * DP + 4 * pc, live ? 16u : 0u);
                }
                cp_async_mbar_arrive(&bars[SB_FULL + slot]);
                __syncwarp();
                if (lane == 0) mbar_arrive(&bars[SB_FULL + slot]);   // orders the entries written above
                ++issued;
                if (T + 1 < nst) load_pe(T + 1);
            }
            // every copy issued has landed before the shared memory is released
            if (lane == 0) {
                mbar_wait_bounded(&bars[SB_BFULL], 0, nullptr);
                for (int t = issued > SS_SLOTS ? issued - SS_SLOTS : 0; t < issued; ++t)
                    mbar_wait_bounded(&bars[SB_FULL + t % SS_SLOTS], (uint32_t)((t / SS_SLOTS) & 1), nullptr);
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer.  stall (test seam): nothing is issued, so the groups' waits run out
        if (run && lane == 0 && !stall) {
            uint64_t* last = nullptr;   // the barrier of the last commit and its phase parity
            uint32_t last_par = 0;
            bool ok = mbar_wait_bounded(&bars[SB_BFULL], 0, gerr);
            if (!ok) atomicCAS(err, 0, ERR_TIMEOUT_BFULL);
            const uint64_t da_h = sw128_desc(smem_u32(sA)), da_l = sw128_desc(smem_u32(sA + A_BYTES));
            const uint64_t db_h = sw128_desc(smem_u32(sB)), db_l = sw128_desc(smem_u32(sB + B_BYTES));
            // issue order: sub(0), then per super-tile T: sub(T + 1), the statistics tiles of T -- the
            // order in which the groups produce them (the sub-label group runs ahead); every wait sleeps
            auto issue_sub = [&](int ts) -> bool {
                if (!mbar_wait_bounded(&bars[SB_AFULL], (uint32_t)(ts & 1), gerr)) {
                    atomicCAS(err, 0, ERR_TIMEOUT_AFULL);
                    return false;
                }
                tc_fence_after();
                const uint32_t dsub = tmem_base + SS_SUBC;
#pragma unroll
                for (int ks = 0; ks < KD / 16; ++ks) umma_bf16(dsub, da_h + 2 * ks, db_h + 2 * ks, ks != 0 ? 1u : 0u);
#pragma unroll
                for (int ks = 0; ks < KD / 16; ++ks) umma_bf16(dsub, da_l + 2 * ks, db_h + 2 * ks, 1u);
#pragma unroll
                for (int ks = 0; ks < KD / 16; ++ks) umma_bf16(dsub, da_h + 2 * ks, db_l + 2 * ks, 1u);
                umma_commit(&bars[SB_SUBDONE]);
                last = &bars[SB_SUBDONE];
                last_par = (uint32_t)(ts & 1);
                return true;
            };
            auto issue_tile = [&](int ti) -> bool {
                const int b = ti & 1, g = ti / SS_G;
                if (ti % SS_G == 0 && g >= 2 &&
                    !mbar_wait_bounded(&bars[SB_ACCEMPTY + (g & 1)], (uint32_t)(((g >> 1) - 1) & 1), gerr)) {
                    atomicCAS(err, 0, ERR_TIMEOUT_TEMPTY);
                    return false;
                }
                if (!mbar_wait_bounded(&bars[SB_STFULL + b], (uint32_t)((ti >> 1) & 1), gerr)) {
                    atomicCAS(err, 0, ERR_TIMEOUT_FULL);
                    return false;
                }
                tc_fence_after();
                const uint32_t td = tmem_base + (uint32_t)((g & 1) * 128);
                const uint32_t ob = smem_u32(sop + (size_t)b * L::OP_BYTES);
#pragma unroll
                for (int kg = 0; kg < SS_KT / 8; ++kg) {   // one group of 8 points per product (K = 8)
                    const uint64_t adh = sw128b32_mn_desc(ob + L::OP_AH + kg * A_GROUP, A_GROUP / 2);
                    const uint64_t adl = sw128b32_mn_desc(ob + L::OP_AL + kg * A_GROUP, A_GROUP / 2);
                    const uint64_t bdh = sw128b32_mn_desc(ob + L::OP_BH + kg * B_GROUP, B_GROUP / 2);
                    const uint64_t bdl = sw128b32_mn_desc(ob + L::OP_BL + kg * B_GROUP, B_GROUP / 2);
                    umma_tf32(td, adh, bdh, IDESC_ST, (ti % SS_G == 0 && kg == 0) ? 0u : 1u);
                    umma_tf32(td, adl, bdh, IDESC_ST, 1u);
                    umma_tf32(td, adh, bdl, IDESC_ST, 1u);
                }
                umma_commit(&bars[SB_STFREE + b]);
                last = &bars[SB_STFREE + b];
                last_par = (uint32_t)((ti >> 1) & 1);
                if (ti % SS_G == SS_G - 1 || ti == ntt - 1) {
                    umma_commit(&bars[SB_GRPDONE + (g & 1)]);
                    last = &bars[SB_GRPDONE + (g & 1)];
                    last_par = (uint32_t)((g >> 1) & 1);
                }
                return true;
            };
            if (ok) ok = issue_sub(0);
            for (int T = 0; T < nst && ok; ++T) {
                if (*abort_flag) { ok = false; break; }
                if (T + 1 < nst && !issue_sub(T + 1)) { ok = false; break; }
                const int nj = min(SS_TPS, ntt - T * SS_TPS);
                for (int j = 0; j < nj && ok; ++j) ok = issue_tile(T * SS_TPS + j);
            }
            if (!ok) *abort_flag = 1;
            // the products issued have completed before the tensor memory is freed (a commit tracks
            // every earlier product of this thread)
            if (last) mbar_wait_bounded(last, last_par, nullptr);
        }
    } else if (warp < 6) {
        // ---------------- sub-label group: point p of every super-tile
        const int p = q * 32 + lane;
        const float cl = cvec[3 * k + 1], cr = cvec[3 * k + 2], wl = lrw[2 * k], wr = lrw[2 * k + 1];
        bool ok = run;
        int drained = 0;   // accumulation groups drained (this group's half)
        for (int T = 0; T < nst && ok; ++T) {
            if (__any_sync(0xffffffffu, *abort_flag != 0)) { ok = false; break; }
            // the accumulation group that ended two super-tiles ago (its products completed long since)
            if ((T & 1) == 0 && T >= 4) {
                if (!drain_group(T / 2 - 2)) { ok = false; break; }
                drained = T / 2 - 1;
            }
            const int slot = T % SS_SLOTS, nv = min(SS_T, len - T * SS_T);
            if (!warp_wait_bounded(&bars[SB_FULL + slot], (uint32_t)((T / SS_SLOTS) & 1), gerr)) {
                if (lane == 0) atomicCAS(err, 0, ERR_TIMEOUT_FULL);
                ok = false;
                break;
            }
            const float* row = stage + ((size_t)slot * SS_T + p) * DP;
            if (T == 0 && p < DP) {   // centre of the statistics: mean of the chunk's first 32 points
                const int n0 = min(32, len);
                float a = 0.f;
                for (int r = 0; r < n0; ++r) a += stage[(size_t)r * DP + p];
                sshift[p] = a / (float)n0;
            }
            // the sub-label operand: this point's row split into BF16 hi / lo (zero past Dp and past the
            // chunk: the stage's rows past the chunk are zero-filled); the lanes visit the 16 pieces in
            // rotated order so that neither the row reads nor the operand stores share banks
#pragma unroll 4
            for (int i = 0; i < 16; ++i) {
                const int c = (i + lane) & 15;   // features 4 c .. 4 c + 3
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (4 * c < DP) v = *reinterpret_cast<const float4*>(row + 4 * c);
                uint2 hi, lo;
                bf16_split4(v.x, v.y, v.z, v.w, hi, lo);
                const uint32_t off = sw128_offset(p, 4 * c);
                *reinterpret_cast<uint2*>(sA + off) = hi;
                *reinterpret_cast<uint2*>(sA + A_BYTES + off) = lo;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            warp_arrive(&bars[SB_AFULL]);
            // r of both sub-clusters for this point (its TMEM lane), then the draw (cudaKernel.cu:352-372)
            if (!warp_wait_bounded(&bars[SB_SUBDONE], (uint32_t)(T & 1), gerr)) {
                if (lane == 0) atomicCAS(err, 0, ERR_TIMEOUT_TFULL);
                ok = false;
                break;
            }
            tc_fence_after();
            float rs[2];
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const float* bs = sbias + side * KD;
                float q0 = 0.f, q1 = 0.f, q2 = 0.f, q3 = 0.f;
#pragma unroll
                for (int hh = 0; hh < 2; ++hh) {
                    if (hh == 1 && DP <= 32) break;   // columns past Dp are zero
                    uint32_t v[32];
                    tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + SS_SUBC + (uint32_t)(side * KD + 32 * hh), v);
#pragma unroll
                    for (int j4 = 0; j4 < 8; ++j4) {
                        const float4 b4 = *reinterpret_cast<const float4*>(bs + 32 * hh + 4 * j4);
                        const float z0 = __uint_as_float(v[4 * j4 + 0]) - b4.x;
                        const float z1 = __uint_as_float(v[4 * j4 + 1]) - b4.y;
                        const float z2 = __uint_as_float(v[4 * j4 + 2]) - b4.z;
                        const float z3 = __uint_as_float(v[4 * j4 + 3]) - b4.w;
                        q0 = fmaf(z0, z0, q0);
                        q1 = fmaf(z1, z1, q1);
                        q2 = fmaf(z2, z2, q2);
                        q3 = fmaf(z3, z3, q3);
                    }
                }
                rs[side] = (side ? cr : cl) - 0.5f * ((q0 + q1) + (q2 + q3));
            }
            tc_fence_before();   // the accumulator is read: the next super-tile's products may overwrite it
            int lab = 0;
            if (p < nv) {
                const int64_t pt = spidx[(T % SS_PIDX) * SS_T + p];
                float rl = rs[0], rr = rs[1];
                if (r_out) {
                    r_out[2 * pt] = rl;
                    r_out[2 * pt + 1] = rr;
                }
                rl += wl;
                rr += wr;
                const float mx = fmaxf(rl, rr);
                const float el = __expf(rl - mx), er = __expf(rr - mx);
                const float s = el + er;
                float u1, u2;
                draw_uniform2(rng, pt, u1, u2);
                lab = alias_draw2(el / s, er / s, u1, u2);
                sub[pt] = lab;
            }
            ssub[slot * SS_T + p] = lab;
            const unsigned bl = __ballot_sync(0xffffffffu, lab == 1), br = __ballot_sync(0xffffffffu, lab == 2);
            cnt_l += __popc(bl);
            cnt_r += __popc(br);
            warp_arrive(&bars[SB_SUBREADY + slot]);
        }
        if (ok)
            for (int g = drained; g < ngr && ok; ++g) ok = drain_group(g);
        if (!ok) *abort_flag = 1;
        if (lane == 0) {
            atomicAdd(&scnt[0], cnt_l);
            atomicAdd(&scnt[1], cnt_r);
        }
    } else {
        // ---------------- statistics group: 16-point tiles of the super-tiles whose sub-labels are drawn
        const int gt = tid - 192;                  // 0 .. 127
        constexpr int ITEMS = SS_KT * C4 / 128;    // 16-byte pieces per thread per tile (2 or 1)
        const int j4 = gt % C4;                    // the thread's piece of every row: features 4 j4 ..
        // offsets of its pieces in an operand buffer (side l's half of A, + 1024 for side r; B) for
        // item 0, and the step to the next item (whole groups of 4 points)
        const uint32_t a_off0 = mn32_offset(gt / C4, j4, 0, 4), b_off0 = mn32_offset(gt / C4, j4, 0, NA);
        constexpr uint32_t A_STEP = (128 / C4) / 4 * 4 * 512, B_STEP = (128 / C4) / 4 * NA * 512;
        bool ok = run;
        int drained = 0;
        float4 s4 = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int T = 0; T < nst && ok; ++T) {
            if (__any_sync(0xffffffffu, *abort_flag != 0)) { ok = false; break; }
            const int slot = T % SS_SLOTS;
            if (!warp_wait_bounded(&bars[SB_SUBREADY + slot], (uint32_t)((T / SS_SLOTS) & 1), gerr)) {
                if (lane == 0) atomicCAS(err, 0, ERR_TIMEOUT_AFULL);
                ok = false;
                break;
            }
            if (T == 0) s4 = *reinterpret_cast<const float4*>(sshift + 4 * j4);
            const float* sl = stage + (size_t)slot * SS_T * DP;
            const int32_t* sbs = ssub + slot * SS_T;
            const int nj = min(SS_TPS, ntt - T * SS_TPS);
            for (int j = 0; j < nj; ++j) {
                const int idx = T * SS_TPS + j, b = idx & 1, u = idx >> 1;
                if (u >= 1 && !warp_wait_bounded(&bars[SB_STFREE + b], (uint32_t)((u - 1) & 1), gerr)) {
                    if (lane == 0) atomicCAS(err, 0, ERR_TIMEOUT_EMPTY);
                    ok = false;
                    break;
                }
                uint8_t* ob = sop + (size_t)b * L::OP_BYTES;
#pragma unroll
                for (int it = 0; it < ITEMS; ++it) {
                    const int pl = (gt + 128 * it) / C4;   // point of the tile; 8 lanes share a row
                    const int pp = SS_KT * j + pl;
                    const int sv = sbs[pp];
                    const bool live = sv == 1 || sv == 2;
                    const float4 v4 = *reinterpret_cast<const float4*>(sl + (size_t)pp * DP + 4 * j4);
                    const float cv[4] = {v4.x - s4.x, v4.y - s4.y, v4.z - s4.z, v4.w - s4.w};
                    float hi[4], lo[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        hi[e] = tf32_rna(cv[e]);
                        lo[e] = tf32_rna(cv[e] - hi[e]);
                        if (!live) hi[e] = lo[e] = 0.f;
                    }
                    const uint32_t a0 = a_off0 + A_STEP * it, b_o = b_off0 + B_STEP * it;
                    const uint32_t a_c = sv == 2 ? a0 + 1024 : a0, a_z = sv == 2 ? a0 : a0 + 1024;
                    const uint4 h4 = make_uint4(__float_as_uint(hi[0]), __float_as_uint(hi[1]), __float_as_uint(hi[2]),
                                                __float_as_uint(hi[3]));
                    const uint4 l4 = make_uint4(__float_as_uint(lo[0]), __float_as_uint(lo[1]), __float_as_uint(lo[2]),
                                                __float_as_uint(lo[3]));
                    const uint4 z4 = make_uint4(0u, 0u, 0u, 0u);
                    *reinterpret_cast<uint4*>(ob + L::OP_AH + a_c) = h4;
                    *reinterpret_cast<uint4*>(ob + L::OP_AL + a_c) = l4;
                    *reinterpret_cast<uint4*>(ob + L::OP_AH + a_z) = z4;
                    *reinterpret_cast<uint4*>(ob + L::OP_AL + a_z) = z4;
                    *reinterpret_cast<uint4*>(ob + L::OP_BH + b_o) = h4;
                    *reinterpret_cast<uint4*>(ob + L::OP_BL + b_o) = l4;
                }
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                warp_arrive(&bars[SB_STFULL + b]);
            }
            if (!ok) break;
            warp_arrive(&bars[SB_EMPTY + slot]);   // the rows and sub-labels of this slot are consumed
            // the accumulation group that ended with the previous super-tile, while this one's products run
            if ((T & 1) == 0 && T >= 2) {
                if (!drain_group(T / 2 - 1)) { ok = false; break; }
                drained = T / 2;
            }
        }
        if (ok)
            for (int g = drained; g < ngr && ok; ++g) ok = drain_group(g);
        if (!ok) *abort_flag = 1;
    }
    tc_fence_before();
    __syncthreads();   // every role is done: copies landed, products complete, accumulators drained
    const bool good = *abort_flag == 0;
    double* xs = reinterpret_cast<double*>(smem + L::stage);   // [2][DP] sums S1
    double* xd = xs + 2 * DP;                                  // [DP] d = a - mu_k
    double* xn = xd + DP;                                      // [2] counts
    if (good) {
        if (warp >= 2 && do_sum) xs[dslot * DP + fi] = sacc;
        if (tid < DP) xd[tid] = (double)sshift[tid] - (double)muv[(size_t)3 * k * DP + tid];
        if (tid == 0) {
            xn[0] = (double)scnt[0];
            xn[1] = (double)scnt[1];
        }
    }
    __syncthreads();
    if (good) {
        double* out = part + (size_t)ch * 2 * SL;
        if (tid < 2) out[(size_t)tid * SL] = xn[tid];
        if (warp >= 2) {
            const double n = xn[dslot];
            if (do_s) {
                double* po = out + (size_t)dslot * SL + 1 + DP;
                const double di = xd[fi], si = xs[dslot * DP + fi];
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    const int j = 32 * hc + i;
                    if (fi <= j && j < DP) {
                        const double dj = xd[j], sj = xs[dslot * DP + j];
                        po[tri_index(DP, fi, j)] = acc[i] + di * sj + si * dj + n * di * dj;
                    }
                }
            }
            if (do_sum) out[(size_t)dslot * SL + 1 + fi] = sacc + n * xd[fi];
        }
    }
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(SS_TMEM_COLS));
    }
}

}  // namespace tc

constexpr size_t kTcSmemCap = 227 * 1024;

// B stages: the deepest ring that fits
static bool tc_config(int& bstages)
{
    for (int bs = tc::MAX_BSTAGES; bs >= 2; --bs)
        if (tc::smem_layout(bs).total <= kTcSmemCap) {
            bstages = bs;
            return true;
        }
    return false;
}

bool tc_supported(const dpmm_ctx* c, int K)
{
    int bs = 0;
    return c->prior == DPMM_PRIOR_GAUSSIAN && c->d_Btc != nullptr && c->d_Atc != nullptr && c->d_rbuf != nullptr &&
           (c->Dp == 32 || c->Dp == 64) && K >= 1 && K <= c->k_max && tc_config(bs);
}

// bias records follow the B tiles in the same allocation
static uint8_t* tc_bias_base(const dpmm_ctx* c)
{
    return c->d_Btc + (size_t)((c->k_max + tc::CPT - 1) / tc::CPT) * tc::STAGE_BYTES;
}

size_t tc_param_bytes(int k_max)
{
    return (size_t)((k_max + tc::CPT - 1) / tc::CPT) * (tc::STAGE_BYTES + tc::BIAS_REC);
}

dpmm_status pack_tc_params(dpmm_ctx* c, int K)
{
    if (!c->d_Btc || !(c->Dp == 32 || c->Dp == 64)) return DPMM_OK;
    const int NT = (K + tc::CPT - 1) / tc::CPT;
    const int total = NT * tc::BN * 8;
    tc::k_pack_b<<<(total + 255) / 256, 256, 0, c->stream>>>(c->d_Wt, K, c->Dp, NT, 0, c->d_Btc);
    DPMM_LAUNCHED();
    if (c->d_Bsub) {
        const int ts = K * tc::BN * 8;
        tc::k_pack_b<<<(ts + 255) / 256, 256, 0, c->stream>>>(c->d_Wt, K, c->Dp, K, 1, c->d_Bsub);
        DPMM_LAUNCHED();
    }
    const int nb = NT * (tc::BIAS_REC / 4);
    tc::k_pack_bias<<<(nb + 255) / 256, 256, 0, c->stream>>>(c->d_b, c->d_c, K, c->Dp, NT, tc_bias_base(c));
    DPMM_LAUNCHED();
    return DPMM_OK;
}

dpmm_status pack_tc_points(dpmm_ctx* c)
{
    if (!c->d_Atc) return DPMM_OK;
    const int64_t ntiles = (c->N + tc::BM - 1) / tc::BM;
    const int64_t total = ntiles * tc::BM * 8;
    tc::k_pack_a<<<(unsigned)((total + 255) / 256), 256, 0, c->stream>>>(c->d_x, c->N, c->Dp, ntiles, c->d_Atc);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

dpmm_status launch_cluster_labels_tc(dpmm_ctx* c, int K, int final_, const float* d_u, float* d_rout)
{
    int bstages = 0;
    if (!tc_supported(c, K) || !tc_config(bstages))
        return fail(DPMM_ERR_INVALID_ARG, "tensor-core label kernel: unsupported shape");
    const tc::SmemLayout L = tc::smem_layout(bstages);
    DPMM_CUDA_TRY(cudaFuncSetAttribute(tc::k_gauss_labels_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
    int32_t* err = c->d_aux + 4;
    DPMM_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int32_t), c->stream));
    const int64_t ntiles = (c->N + tc::BM - 1) / tc::BM;
    const int64_t nst = (ntiles + tc::HALVES - 1) / tc::HALVES;
    const unsigned grid = (unsigned)std::min<int64_t>(nst, c->num_sms);
    {
        KernelTimer kt(c, PH_LABEL_KERNEL);
        tc::k_gauss_labels_tc<<<grid, tc::THREADS, L.total, c->stream>>>(c->d_Atc, c->N, (int)ntiles, c->d_Btc,
                                                                         tc_bias_base(c), c->Dp, K, bstages, final_,
                                                                         c->d_rbuf, c->d_rpart, d_rout, err,
                                                                         c->stall_tc_mma);
        DPMM_LAUNCHED();
    }
    RngArgs r = rng_args(c, d_u);
    tc::k_draw_labels<<<(unsigned)((c->N + 255) / 256), 256, 0, c->stream>>>(c->d_rbuf, c->d_rpart, c->N, K, final_,
                                                                            r, c->d_labels);
    DPMM_LAUNCHED();
    int32_t h_err = 0;
    DPMM_CUDA_TRY(cudaMemcpyAsync(&h_err, err, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (h_err) return fail(DPMM_ERR_TIMEOUT, "tensor-core label kernel: bounded wait expired (code " +
                                                 std::to_string(h_err) + ")");
    return DPMM_OK;
}

bool tc_sub_supported(const dpmm_ctx* c)
{
    return c->prior == DPMM_PRIOR_GAUSSIAN && c->d_Bsub != nullptr && (c->Dp == 32 || c->Dp == 64) &&
           c->ll_mode != DPMM_LL_FP32;
}

template <int DP>
static dpmm_status launch_sub_labels_tc_t(dpmm_ctx* c, RngArgs r, float* d_rout, int32_t* err)
{
    auto kern = tc::k_sub_labels_tc<DP>;
    DPMM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::SubSmem::total));
    kern<<<c->max_chunks, 256, tc::SubSmem::total, c->stream>>>(c->d_x, c->d_perm, c->d_chunk, c->d_nchunks, c->d_Bsub,
                                                              c->d_b, c->d_c, c->d_lrw, r, c->d_sub, d_rout, err,
                                                              c->stall_tc_mma);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

dpmm_status launch_sub_labels_tc(dpmm_ctx* c, RngArgs r, float* d_rout, bool defer_check)
{
    int32_t* err = c->d_aux + 5;
    DPMM_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int32_t), c->stream));
    if (c->Dp == 64) DPMM_TRY(launch_sub_labels_tc_t<64>(c, r, d_rout, err));
    else DPMM_TRY(launch_sub_labels_tc_t<32>(c, r, d_rout, err));
    if (defer_check) {
        c->sub_err_pending = true;
        return DPMM_OK;
    }
    int32_t h_err = 0;
    DPMM_CUDA_TRY(cudaMemcpyAsync(&h_err, err, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (h_err) return fail(DPMM_ERR_TIMEOUT, "tensor-core sub-label kernel: bounded wait expired (code " +
                                                 std::to_string(h_err) + ")");
    return DPMM_OK;
}

bool tc_scan_supported(const dpmm_ctx* c, int K)
{
    return c->ll_mode != DPMM_LL_FP32 && tc_supported(c, K) && K <= tc::kScanMaxK;
}

template <int DP>
static dpmm_status launch_prune_scan_tc_t(dpmm_ctx* c, int K, int32_t* err)
{
    // single pass while [W_h | every other cluster's v] fits two B tiles, else the two-pass form
    auto kern = K - 1 <= tc::kScan1MaxCand ? tc::k_prune_scan1_tc<DP> : tc::k_prune_scan_tc<DP>;
    DPMM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::ScanSmem::total));
    kern<<<c->max_chunks, 256, tc::ScanSmem::total, c->stream>>>(
        c->d_x, c->d_perm, c->d_chunk, c->d_nchunks, c->d_Btc, c->d_b, c->d_c, c->d_mu, c->d_prune_lam, c->d_prune_M,
        c->d_prune_V, c->d_prune_beta, K, c->prune_margin, c->d_prune_rh, c->d_prune_cand, c->d_prune_cnt, err,
        c->stall_tc_mma);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

// the caller clears *d_err before and reads it after (with the pass's counters)
dpmm_status launch_prune_scan_tc(dpmm_ctx* c, int K, int32_t* d_err)
{
    if (!tc_scan_supported(c, K)) return fail(DPMM_ERR_INVALID_ARG, "tensor-core scan: unsupported shape");
    if (c->Dp == 64) return launch_prune_scan_tc_t<64>(c, K, d_err);
    return launch_prune_scan_tc_t<32>(c, K, d_err);
}

bool tc_stats_supported(const dpmm_ctx* c)
{
    return c->prior == DPMM_PRIOR_GAUSSIAN && (c->Dp == 32 || c->Dp == 64) && c->ll_mode != DPMM_LL_FP32;
}

template <int DP>
static dpmm_status launch_slot_stats_tc_t(dpmm_ctx* c, const uint8_t* d_mask, int32_t* err)
{
    auto kern = tc::k_slot_stats_tc<DP>;
    constexpr size_t sm = tc::StatSmem<DP>::total;
    DPMM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    kern<<<c->max_chunks, 256, sm, c->stream>>>(c->d_x, c->d_perm, c->d_chunk, c->d_nchunks, c->d_mu, c->d_sub,
                                                c->d_part, d_mask, err, c->stall_tc_mma);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

dpmm_status launch_slot_stats_tc(dpmm_ctx* c, const uint8_t* d_mask)
{
    if (!tc_stats_supported(c)) return fail(DPMM_ERR_INVALID_ARG, "tensor-core statistics: unsupported shape");
    int32_t* err = c->d_aux + 3;
    DPMM_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int32_t), c->stream));
    {
        KernelTimer kt(d_mask ? nullptr : c, PH_SLOT_STATS);   // full launches only (masked: a few clusters)
        if (c->Dp == 64) DPMM_TRY(launch_slot_stats_tc_t<64>(c, d_mask, err));
        else DPMM_TRY(launch_slot_stats_tc_t<32>(c, d_mask, err));
    }
    int32_t* h_err = reinterpret_cast<int32_t*>(c->h_pinned);
    h_err[1] = 0;
    DPMM_CUDA_TRY(cudaMemcpyAsync(h_err, err, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    if (c->sub_err_pending)
        DPMM_CUDA_TRY(cudaMemcpyAsync(h_err + 1, c->d_aux + 5, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->sub_err_pending = false;
    if (h_err[1]) return fail(DPMM_ERR_TIMEOUT, "tensor-core sub-label kernel: bounded wait expired (code " +
                                                    std::to_string(h_err[1]) + ")");
    if (*h_err) return fail(DPMM_ERR_TIMEOUT, "tensor-core statistics: bounded wait expired (code " +
                                                  std::to_string(*h_err) + ")");
    return DPMM_OK;
}

template <int DP>
static dpmm_status launch_sub_stats_tc_t(dpmm_ctx* c, RngArgs r, float* d_rout, int32_t* err)
{
    auto kern = tc::k_sub_stats_tc<DP>;
    constexpr size_t sm = tc::SubStatSmem<DP>::total;
    DPMM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    kern<<<c->max_chunks, tc::SS_THREADS, sm, c->stream>>>(c->d_x, c->d_perm, c->d_chunk, c->d_nchunks, c->d_Bsub,
                                                            c->d_b, c->d_c, c->d_lrw, c->d_mu, r, c->d_sub, d_rout,
                                                            c->d_part, err, c->stall_tc_mma);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

bool tc_sub_stats_supported(const dpmm_ctx* c)
{
    return c->fuse_sub_stats && tc_sub_supported(c) && tc_stats_supported(c);
}

dpmm_status launch_sub_stats_tc(dpmm_ctx* c, RngArgs r, float* d_rout)
{
    if (!tc_sub_stats_supported(c)) return fail(DPMM_ERR_INVALID_ARG, "fused sub-label statistics: unsupported shape");
    int32_t* err = c->d_aux + 3;
    DPMM_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int32_t), c->stream));
    {
        KernelTimer kt(c, PH_SLOT_STATS);
        if (c->Dp == 64) DPMM_TRY(launch_sub_stats_tc_t<64>(c, r, d_rout, err));
        else DPMM_TRY(launch_sub_stats_tc_t<32>(c, r, d_rout, err));
    }
    int32_t* h_err = reinterpret_cast<int32_t*>(c->h_pinned);
    DPMM_CUDA_TRY(cudaMemcpyAsync(h_err, err, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (*h_err) return fail(DPMM_ERR_TIMEOUT, "fused sub-label statistics kernel: bounded wait expired (code " +
                                                  std::to_string(*h_err) + ")");
    return DPMM_OK;
}

}  // namespace dpmm

namespace dpmm {
namespace tc {

// ============================================================================= multinomial label phase
// cudaKernel_multinomial::log_likelihood_labels (cudaKernel_multinomial.cu:22-35, 60-76: r_k(x) =
// sum_d x_d log theta_kd, no weight term) for every cluster as one contraction on the tensor cores:
// C[p, k] = sum_d X[p, d] T[k, d] with the counts X stored as BF16 (exact: the upload checks that
// every count is a BF16 value) and log theta split into three BF16 terms (hi + mid + lo = the FP32
// value exactly), so r is the FP32 dot product of the SIMT form up to the order of the additions.
// Operands are packed once in the exact shared-memory image (K-major, 128-byte swizzle): the counts
// per (128-point tile, 64-category block) at upload, log theta per 64-category block after every
// parameter update; each pipeline stage is then two cp.async.bulk copies.
//
// Persistent CTAs (one per SM) walk the 128-point tiles:
//   warp 0      producer: per (tile, block) the counts (16 KB) and the three log theta parts
//               (3 x Kp x 128 B) into a ring of stages
//   warp 1      allocates TMEM; lane 0 issues per block 4 k-steps x 3 parts of tcgen05.mma
//               (kind::f16, M = 128, N = Kp, K = 16) into one of two accumulators
//   warps 2-5   epilogue (TMEM lane quarter = warp % 4): per point the K values of r, written
//               cluster-major to rbuf[k][point] (32 points per store), and the point's max and sum of
//               exp (or its first maximum, final mode) as the partials k_draw_labels reads; then the
//               softmax + alias draw runs in k_draw_labels as for the Gaussian tensor-core phase.
// Every wait is bounded; on expiry the CTA records the error, stops issuing, waits (bounded) for the
// copies and products it issued and frees its TMEM.
constexpr int MT_KB = 64;                          // categories per block: one 128-byte BF16 row
constexpr int MT_A = BM * MT_KB * 2;               // 16 KB of counts per (tile, block)
constexpr int MT_PARTS = 3;                        // log theta = hi + mid + lo (BF16)
constexpr int MT_MAX_KP = 224;                     // clusters per contraction (N of the MMA)
constexpr int MT_THREADS = 192;
constexpr int MT_MAX_STAGES = 8;

__host__ __device__ constexpr uint32_t mt_stage_bytes(int Kp) { return (uint32_t)(MT_A + MT_PARTS * Kp * 128); }

__global__ void __launch_bounds__(MT_THREADS, 1) k_mult_labels_tc(
    const uint8_t* __restrict__ Acnt, int64_t N, int ntiles, int nkb, const uint8_t* __restrict__ Bth, int Kp, int K,
    int stages, int final_, float* __restrict__ rbuf, float* __restrict__ part, float* __restrict__ r_out,
    int32_t* __restrict__ err, int stall)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const uint32_t SB = mt_stage_bytes(Kp);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)stages * SB);
    uint64_t* empty = full + MT_MAX_STAGES;
    uint64_t* afull = empty + MT_MAX_STAGES;         // [2] accumulator a holds a finished tile
    uint64_t* aempty = afull + 2;                    // [2] the epilogue has read accumulator a
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(aempty + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const volatile int32_t* gerr = err;
    uint32_t ncols = 32;
    while (ncols < (uint32_t)(2 * Kp)) ncols <<= 1;

    if (tid == 0) {
        for (int s = 0; s < stages; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(afull + a, 1);
            mbar_init(aempty + a, 4);                // one arrival per epilogue warp
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        if (lane == 0) {
            int64_t g = 0;   // (tile, block) pairs issued
            bool ok = true;
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
                for (int kb = 0; kb < nkb; ++kb, ++g) {
                    const int s = (int)(g % stages);
                    if (g >= stages && !mbar_wait_bounded(empty + s, (uint32_t)(((g / stages) - 1) & 1), gerr)) {
                        atomicCAS(err, 0, ERR_TIMEOUT_EMPTY);
                        ok = false;
                        break;
                    }
                    uint8_t* dst = smem + (size_t)s * SB;
                    mbar_arrive_expect_tx(full + s, SB);
                    bulk_copy_g2s(dst, Acnt + ((size_t)tile * nkb + kb) * MT_A, MT_A, full + s);
                    bulk_copy_g2s(dst + MT_A, Bth + (size_t)kb * MT_PARTS * Kp * 128, MT_PARTS * Kp * 128, full + s);
                }
            }
            // nothing may land in shared memory after the CTA exits: wait for the last use of every stage
            for (int64_t q = g - 1; q >= 0 && q >= g - stages; --q)
                mbar_wait_bounded(full + (int)(q % stages), (uint32_t)((q / stages) & 1), nullptr);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer (stall, test seam:
        // nothing is issued, so the waits for the products run out and report ERR_TIMEOUT_*)
        if (lane == 0 && !stall) {
            const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(Kp >> 3) << 17) |
                                   ((uint32_t)(BM >> 4) << 24);
            int64_t g = 0;
            int it = 0;
            bool ok = true;
            uint64_t* last = nullptr;   // the barrier of the last commit and its phase
            uint32_t last_par = 0;
            for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++it) {
                const int a = it & 1;
                if (it >= 2 && !mbar_wait_bounded(aempty + a, (uint32_t)(((it >> 1) - 1) & 1), gerr)) {
                    atomicCAS(err, 0, ERR_TIMEOUT_TEMPTY);
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t td = tmem_base + (uint32_t)(a * Kp);
                for (int kb = 0; kb < nkb; ++kb, ++g) {
                    const int s = (int)(g % stages);
                    if (!mbar_wait_bounded(full + s, (uint32_t)((g / stages) & 1), gerr)) {
                        atomicCAS(err, 0, ERR_TIMEOUT_FULL);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = smem_u32(smem + (size_t)s * SB);
                    const uint64_t da = sw128_desc(sa);
#pragma unroll
                    for (int ks = 0; ks < MT_KB / 16; ++ks)
#pragma unroll
                        for (int p = 0; p < MT_PARTS; ++p) {
                            const uint64_t db = sw128_desc(sa + MT_A + (uint32_t)(p * Kp * 128));
                            const uint32_t acc = (kb | ks | p) != 0 ? 1u : 0u;
                            asm volatile(
                                "{\n\t.reg .pred q;\n\t"
                                "setp.ne.b32 q, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, q;\n\t}" ::"r"(td),
                                "l"(da + 2 * ks), "l"(db + 2 * ks), "r"(idesc), "r"(acc)
                                : "memory");
                        }
                    umma_commit(empty + s);
                    last = empty + s;
                    last_par = (uint32_t)((g / stages) & 1);
                }
                if (!ok) break;
                umma_commit(afull + a);
                last = afull + a;
                last_par = (uint32_t)((it >> 1) & 1);
            }
            if (!ok && last) mbar_wait_bounded(last, last_par, nullptr);   // no product in flight at dealloc
        }
    } else {
        // ------------------------------------------------------------ epilogue
        const int q = warp & 3;
        const int row = q * 32 + lane;
        int it = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
            const int a = it & 1;
            if (!warp_wait_bounded(afull + a, (uint32_t)((it >> 1) & 1), gerr)) {
                if (lane == 0) atomicCAS(err, 0, ERR_TIMEOUT_TFULL);
                break;
            }
            tc_fence_after();
            const int64_t pt = (int64_t)tile * BM + row;
            const bool live = pt < N;
            const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(a * Kp);
            float mx = -INFINITY;
            int arg = -1;
            for (int c0 = 0; c0 < Kp; c0 += 32) {
                uint32_t v[32];
                tmem_ld32(taddr + (uint32_t)c0, v);
#pragma unroll
                for (int m = 0; m < 32; ++m) {
                    const int k = c0 + m;
                    const float r = __uint_as_float(v[m]);
                    if (k < K) {
                        if (live) {
                            rbuf[(size_t)k * N + pt] = r;
                            if (r_out) r_out[(size_t)pt * K + k] = r;
                        }
                        if (r > mx) {   // first maximum wins (cudaKernel.cu:405-424)
                            mx = r;
                            arg = k;
                        }
                    }
                }
            }
            float sum = 0.f;
            if (!final_) {
                for (int c0 = 0; c0 < Kp; c0 += 32) {
                    uint32_t v[32];
                    tmem_ld32(taddr + (uint32_t)c0, v);
#pragma unroll
                    for (int m = 0; m < 32; ++m)
                        if (c0 + m < K) sum += __expf(__uint_as_float(v[m]) - mx);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(aempty + a);
            if (live) {
                // the partials of k_draw_labels: half 0 holds every cluster, half 1 none
                part[pt] = mx;
                part[N + pt] = final_ ? __int_as_float(arg) : sum;
                part[2 * N + pt] = -INFINITY;
                part[3 * N + pt] = final_ ? __int_as_float(-1) : 0.f;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(ncols));
    }
}

// counts (FP32 rows, stride Dp) -> BF16 tiles in the shared-memory image: Apack[(t * nkb + kb)] = 16 KB
// holding points 128 t .. +127, categories 64 kb .. +63 (zero past N / D).  inexact counts a count
// that BF16 does not hold exactly.
__global__ void k_pack_mult_a(const float* __restrict__ x, int64_t N, int D, int Dp, int64_t ntiles, int nkb,
                              uint8_t* __restrict__ Apack, int32_t* __restrict__ inexact)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;   // (tile, block, row, 8-chunk)
    if (e >= ntiles * nkb * BM * 8) return;
    const int ch = (int)(e % 8), row = (int)((e / 8) % BM);
    const int64_t tb = e / (8 * BM);
    const int kb = (int)(tb % nkb);
    const int64_t t = tb / nkb;
    const int64_t pt = t * BM + row;
    __align__(16) __nv_bfloat16 v[8];
    int bad = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int d = kb * MT_KB + ch * 8 + j;
        const float f = (pt < N && d < D) ? x[pt * Dp + d] : 0.f;
        v[j] = __float2bfloat16_rn(f);
        bad |= __bfloat162float(v[j]) != f;
    }
    if (bad) atomicAdd(inexact, 1);
    *reinterpret_cast<uint4*>(Apack + (size_t)tb * MT_A + sw128_offset(row, ch * 8)) = *reinterpret_cast<const uint4*>(v);
}

// log theta of the cluster slots (3k, FP32 rows of stride Dp) -> three BF16 parts in the shared-memory
// image: Bpack[kb][part] = Kp rows x 128 B (zero past K / D)
__global__ void k_pack_mult_b(const float* __restrict__ lt, int K, int D, int Dp, int Kp, int nkb,
                              uint8_t* __restrict__ Bpack)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;   // (block, row, 8-chunk)
    if (e >= nkb * Kp * 8) return;
    const int ch = e % 8, k = (e / 8) % Kp, kb = e / (8 * Kp);
    __align__(16) __nv_bfloat16 hi[8], mid[8], lo[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int d = kb * MT_KB + ch * 8 + j;
        const float f = (k < K && d < D) ? lt[(size_t)3 * k * Dp + d] : 0.f;
        hi[j] = __float2bfloat16_rn(f);
        const float r1 = f - __bfloat162float(hi[j]);
        mid[j] = __float2bfloat16_rn(r1);
        lo[j] = __float2bfloat16_rn(r1 - __bfloat162float(mid[j]));
    }
    uint8_t* base = Bpack + (size_t)kb * MT_PARTS * Kp * 128;
    const uint32_t off = sw128_offset(k, ch * 8);
    *reinterpret_cast<uint4*>(base + off) = *reinterpret_cast<const uint4*>(hi);
    *reinterpret_cast<uint4*>(base + (size_t)Kp * 128 + off) = *reinterpret_cast<const uint4*>(mid);
    *reinterpret_cast<uint4*>(base + (size_t)2 * Kp * 128 + off) = *reinterpret_cast<const uint4*>(lo);
}

}  // namespace tc

static int mt_kp(int K) { return std::max(32, (K + 31) / 32 * 32); }

static int mt_stages(int Kp)
{
    const size_t avail = kTcSmemCap - 1024 - 256;
    return (int)std::min<size_t>(tc::MT_MAX_STAGES, avail / tc::mt_stage_bytes(Kp));
}

bool tc_mult_supported(const dpmm_ctx* c, int K)
{
    return c->prior == DPMM_PRIOR_MULTINOMIAL && c->d_Amult != nullptr && c->mult_tc_ok && c->d_rbuf != nullptr &&
           c->ll_mode != DPMM_LL_FP32 && K >= 1 && K <= c->k_max && mt_kp(K) <= tc::MT_MAX_KP && mt_stages(mt_kp(K)) >= 2;
}

size_t mult_tc_a_bytes(int64_t N, int D)
{
    return (size_t)((N + tc::BM - 1) / tc::BM) * (size_t)((D + tc::MT_KB - 1) / tc::MT_KB) * tc::MT_A;
}

size_t mult_tc_b_bytes(int k_max, int D)
{
    const int kp = std::min(tc::MT_MAX_KP, mt_kp(k_max));
    return (size_t)((D + tc::MT_KB - 1) / tc::MT_KB) * tc::MT_PARTS * kp * 128;
}

dpmm_status pack_mult_tc_points(dpmm_ctx* c)
{
    if (!c->d_Amult) return DPMM_OK;
    const int64_t ntiles = (c->N + tc::BM - 1) / tc::BM;
    const int nkb = (c->D + tc::MT_KB - 1) / tc::MT_KB;
    int32_t* inexact = c->d_aux + 8;
    DPMM_CUDA_TRY(cudaMemsetAsync(inexact, 0, sizeof(int32_t), c->stream));
    const int64_t items = ntiles * nkb * tc::BM * 8;
    tc::k_pack_mult_a<<<(unsigned)((items + 255) / 256), 256, 0, c->stream>>>(c->d_x, c->N, c->D, c->Dp, ntiles, nkb,
                                                                             c->d_Amult, inexact);
    DPMM_LAUNCHED();
    int32_t h = 0;
    DPMM_CUDA_TRY(cudaMemcpyAsync(&h, inexact, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->mult_tc_ok = h == 0;   // counts that BF16 does not hold exactly: the FP32 SIMT form only
    return DPMM_OK;
}

dpmm_status pack_mult_tc_params(dpmm_ctx* c, int K)
{
    if (!c->d_Amult || !c->mult_tc_ok || mt_kp(K) > tc::MT_MAX_KP) return DPMM_OK;
    const int Kp = mt_kp(K), nkb = (c->D + tc::MT_KB - 1) / tc::MT_KB;
    const int items = nkb * Kp * 8;
    tc::k_pack_mult_b<<<(items + 255) / 256, 256, 0, c->stream>>>(c->d_mu, K, c->D, c->Dp, Kp, nkb, c->d_Bmult);
    DPMM_LAUNCHED();
    c->mult_tc_K = K;
    return DPMM_OK;
}

dpmm_status launch_mult_labels_tc(dpmm_ctx* c, int K, int final_, const float* d_u, float* d_rout)
{
    if (!tc_mult_supported(c, K)) return fail(DPMM_ERR_INVALID_ARG, "tensor-core multinomial labels: unsupported shape");
    if (c->mult_tc_K != K) DPMM_TRY(pack_mult_tc_params(c, K));
    const int Kp = mt_kp(K), stages = mt_stages(Kp);
    const size_t sm = 1024 + (size_t)stages * tc::mt_stage_bytes(Kp) + (2 * tc::MT_MAX_STAGES + 4) * 8 + 16;
    DPMM_CUDA_TRY(cudaFuncSetAttribute(tc::k_mult_labels_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int32_t* err = c->d_aux + 7;
    DPMM_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int32_t), c->stream));
    const int64_t ntiles = (c->N + tc::BM - 1) / tc::BM;
    const int nkb = (c->D + tc::MT_KB - 1) / tc::MT_KB;
    const unsigned grid = (unsigned)std::min<int64_t>(ntiles, c->num_sms);
    {
        KernelTimer kt(c, PH_LABEL_KERNEL);
        tc::k_mult_labels_tc<<<grid, tc::MT_THREADS, sm, c->stream>>>(c->d_Amult, c->N, (int)ntiles, nkb, c->d_Bmult,
                                                                      Kp, K, stages, final_, c->d_rbuf, c->d_rpart,
                                                                      d_rout, err, c->stall_tc_mma);
        DPMM_LAUNCHED();
    }
    RngArgs r = rng_args(c, d_u);
    tc::k_draw_labels<<<(unsigned)((c->N + 255) / 256), 256, 0, c->stream>>>(c->d_rbuf, c->d_rpart, c->N, K, final_,
                                                                            r, c->d_labels);
    DPMM_LAUNCHED();
    int32_t h_err = 0;
    DPMM_CUDA_TRY(cudaMemcpyAsync(&h_err, err, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (h_err) return fail(DPMM_ERR_TIMEOUT, "tensor-core multinomial label kernel: bounded wait expired (code " +
                                                 std::to_string(h_err) + ")");
    return DPMM_OK;
}

}  // namespace dpmm
