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
// of the reference (cudaKernel.cu:374-424, 27-124), one thread per point.
//
// CTA roles (320 threads): warp 0 streams B tiles (2 clusters = 128 columns, hi + lo, 32 KB,
// stored pre-swizzled in global memory) with cp.async.bulk into a 2-3 stage ring; warp 1
// allocates TMEM and issues tcgen05.mma (M=128, N=128, K=16; 12 per tile) into a
// double-buffered accumulator (2 x 128 columns); warps 2-9 are the epilogue.  Every mbarrier
// wait is bounded: on timeout the CTA records an error code, stops issuing work, drains what it
// issued (bounded) and frees its TMEM.
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
constexpr uint32_t TMEM_COLS = 512;        // accumulators in 0-255, the tile's r in 256 + k
constexpr uint32_t R_COL0 = 2 * BN;
constexpr int DRAIN_WARPS = 8;             // two per TMEM lane quarter, one cluster each
constexpr int DRAW_WARPS = 4;              // one per TMEM lane quarter
constexpr int WARP_DRAIN0 = 2, WARP_DRAW0 = WARP_DRAIN0 + DRAIN_WARPS;
constexpr int THREADS = 32 * (2 + DRAIN_WARPS + DRAW_WARPS);

enum : int {
    ERR_TIMEOUT_FULL = 1, ERR_TIMEOUT_EMPTY = 2, ERR_TIMEOUT_TFULL = 3, ERR_TIMEOUT_TEMPTY = 4,
    ERR_TIMEOUT_AFULL = 5, ERR_TIMEOUT_AEMPTY = 6, ERR_TIMEOUT_RFULL = 7, ERR_TIMEOUT_REMPTY = 8
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

// Single-thread bounded wait.  Gives up after WAIT_LIMIT_NS, or early when another CTA of the
// launch has already reported an error (gerr != nullptr).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, const volatile int32_t* gerr)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t i = 1;; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 255) == 0) {
            if (global_ns() - t0 > WAIT_LIMIT_NS) return false;
            if (gerr && *gerr) return false;
        }
    }
}

// Warp-uniform bounded wait: every lane observes the phase, and all lanes take the same
// decision (the epilogue's tcgen05.ld is warp-collective).
__device__ __forceinline__ bool warp_wait_bounded(uint64_t* bar, uint32_t parity, const volatile int32_t* gerr)
{
    const int lane = threadIdx.x & 31;
    uint64_t t0 = lane == 0 ? global_ns() : 0;
    for (uint32_t i = 1;; ++i) {
        const bool ok = mbar_try_wait(bar, parity);
        if (__all_sync(0xffffffffu, ok)) return true;
        if ((i & 255) == 0) {
            int stop = 0;
            if (lane == 0) stop = (global_ns() - t0 > WAIT_LIMIT_NS) || (gerr && *gerr);
            if (__shfl_sync(0xffffffffu, stop, 0)) return false;
        }
    }
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

// 64 consecutive accumulator columns of this thread's TMEM lane (warp-collective)
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, uint32_t (&r)[64])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, "
        "%32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, "
        "%48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
          "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
          "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
          "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
          "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void bf16_split(float v, __nv_bfloat16& hi, __nv_bfloat16& lo)
{
    hi = __float2bfloat16_rn(v);
    lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

// ------------------------------------------------------------------------- B packing
// Bpack[t] = 32 KB: hi (16 KB) then lo (16 KB) of the 128 x 64 K-major swizzled tile holding
// rows n = (c, j) -> W_{2t+c}(i, j) over i (zero outside the K clusters / the dimension).
__global__ void k_pack_b(const float* __restrict__ Wt, int K, int Dp, int NT, uint8_t* __restrict__ Bpack)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;   // (t, n, chunk)
    if (e >= NT * BN * 8) return;
    const int t = e / (BN * 8);
    const int n = (e / 8) % BN;
    const int ch = e % 8;
    const int k = CPT * t + n / KD;
    const int j = n % KD;
    __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int i = ch * 8 + q;
        float w = 0.f;
        if (k < K && j < Dp && i < Dp) w = Wt[((size_t)3 * k * Dp + j) * Dp + i];
        bf16_split(w, hi[q], lo[q]);
    }
    uint8_t* base = Bpack + (size_t)t * STAGE_BYTES;
    const uint32_t off = sw128_offset(n, ch * 8);
    *reinterpret_cast<uint4*>(base + off) = *reinterpret_cast<const uint4*>(hi);
    *reinterpret_cast<uint4*>(base + B_BYTES + off) = *reinterpret_cast<const uint4*>(lo);
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
// Persistent: one CTA per SM walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ...
//
//   warp 0      producer: A tile (32 KB) into an A ring, B tiles (32 KB) into a B ring
//   warp 1      MMA issuer: 12 tcgen05.mma per N tile into a double-buffered accumulator
//               (TMEM columns 0-255)
//   warps 2-9   drain: TMEM accumulator -> r = c - |z|^2 / 2 for one cluster of the N tile per
//               warp (two warps per TMEM lane quarter); r goes to TMEM columns 256 + k, and a
//               running max / sum of exp (or first maximum, final mode) per point and half
//   warps 10-13 draw: copy the tile's r from TMEM to a shared-memory row per point, release
//               the TMEM r buffer, then softmax + alias draw (or argmax) one thread per point,
//               while the next tile's MMAs and drain proceed
//
// r table in shared memory: one row of KS = K rounded up to odd floats per point, so the draw
// warps' stores (32 points x one cluster) hit 32 distinct banks.
__host__ __device__ constexpr int r_stride(int K) { return K | 1; }

struct SmemLayout {
    int astages, bstages;
    size_t a, b, r, part, bar, total;
};

__host__ __device__ inline SmemLayout smem_layout(int K, int astages, int bstages)
{
    SmemLayout L;
    L.astages = astages;
    L.bstages = bstages;
    L.a = 0;                                            // astages x 32 KB (1024-aligned)
    L.b = (size_t)astages * A_TILE;                     // bstages x 32 KB
    L.r = L.b + (size_t)bstages * STAGE_BYTES;          // BM x r_stride(K) floats
    L.part = (L.r + (size_t)BM * r_stride(K) * 4 + 15) / 16 * 16;   // 4 x BM partials
    L.bar = L.part + (size_t)4 * BM * 4;
    L.total = L.bar + 16 * 8 + 16 + 1024;               // barriers, tmem slot + flag, alignment slack
    return L;
}

__device__ __forceinline__ void tmem_st1(uint32_t taddr, float v)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};" ::"r"(taddr), "r"(__float_as_uint(v))
                 : "memory");
}

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

__global__ void __launch_bounds__(THREADS, 1) k_gauss_labels_tc(
    const uint8_t* __restrict__ Apack, int64_t N, int ntiles, const uint8_t* __restrict__ Bpack,
    const float* __restrict__ bvec, const float* __restrict__ cvec, int Dp, int K, int astages, int bstages,
    int final_, RngArgs rng, int32_t* __restrict__ labels, float* __restrict__ r_out, int32_t* __restrict__ err)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const SmemLayout L = smem_layout(K, astages, bstages);
    uint8_t* sA = smem + L.a;
    uint8_t* sB = smem + L.b;
    float* sr = reinterpret_cast<float*>(smem + L.r);
    float* spart = reinterpret_cast<float*>(smem + L.part);   // [half][2][BM]: max, sum (or best, arg)
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L.bar);
    uint64_t* full = bars;            // [bstages <= 3]
    uint64_t* empty = bars + 3;       // [3]
    uint64_t* afull = bars + 6;       // [astages <= 2]
    uint64_t* aempty = bars + 8;      // [2]
    uint64_t* tfull = bars + 10;      // [2]
    uint64_t* tempty = bars + 12;     // [2]
    uint64_t* rfull = bars + 14;      // r of a tile is in TMEM (drain -> draw)
    uint64_t* rempty = bars + 15;     // TMEM r buffer copied out (draw -> drain)
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 16);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int NT = (K + CPT - 1) / CPT;
    const int KS = r_stride(K);
    const volatile int32_t* gerr = err;

    if (tid == 0) {
        *abort_flag = *gerr ? 1 : 0;
        for (int s = 0; s < bstages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int s = 0; s < astages; ++s) {
            mbar_init(&afull[s], 1);
            mbar_init(&aempty[s], 1);
        }
        for (int t = 0; t < 2; ++t) {
            mbar_init(&tfull[t], 1);
            mbar_init(&tempty[t], DRAIN_WARPS * 32);
        }
        mbar_init(rfull, DRAIN_WARPS * 32);
        mbar_init(rempty, DRAW_WARPS * 32);
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
            for (int tile = blockIdx.x; tile < ntiles && !*abort_flag; tile += gridDim.x, ++la) {
                const int sa = la % astages;
                if (!mbar_wait_bounded(&aempty[sa], ((la / astages) & 1) ^ 1, gerr)) {
                    atomicCAS(err, 0, ERR_TIMEOUT_AEMPTY);
                    *abort_flag = 1;
                    break;
                }
                mbar_arrive_expect_tx(&afull[sa], A_TILE);
                bulk_copy_g2s(sA + (size_t)sa * A_TILE, Apack + (size_t)tile * A_TILE, A_TILE, &afull[sa]);
                bool ok = true;
                for (int nt = 0; nt < NT; ++nt, ++gb) {
                    const int s = gb % bstages;
                    if (!mbar_wait_bounded(&empty[s], ((gb / bstages) & 1) ^ 1, gerr)) {
                        atomicCAS(err, 0, ERR_TIMEOUT_EMPTY);
                        *abort_flag = 1;
                        ok = false;   // gb stays the count of B copies issued
                        break;
                    }
                    mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
                    bulk_copy_g2s(sB + (size_t)s * STAGE_BYTES, Bpack + (size_t)nt * STAGE_BYTES, STAGE_BYTES,
                                  &full[s]);
                }
                if (!ok) { ++la; break; }   // this tile's A copy was issued
            }
            // drain: every copy issued has landed before shared memory is released
            for (int q = la > astages ? la - astages : 0; q < la; ++q)
                mbar_wait_bounded(&afull[q % astages], (q / astages) & 1, nullptr);
            for (int q = gb > bstages ? gb - bstages : 0; q < gb; ++q)
                mbar_wait_bounded(&full[q % bstages], (q / bstages) & 1, nullptr);
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer
        if (lane == 0) {
            int g = 0, la = 0, issued = 0;
            for (int tile = blockIdx.x; tile < ntiles && !*abort_flag; tile += gridDim.x, ++la) {
                const int sa = la % astages;
                if (!mbar_wait_bounded(&afull[sa], (la / astages) & 1, gerr)) {
                    atomicCAS(err, 0, ERR_TIMEOUT_AFULL);
                    *abort_flag = 1;
                    break;
                }
                const uint32_t a_hi = smem_u32(sA + (size_t)sa * A_TILE), a_lo = a_hi + A_BYTES;
                bool ok = true;
                for (int nt = 0; nt < NT; ++nt, ++g) {
                    const int s = g % bstages, t = g & 1;
                    if (!mbar_wait_bounded(&full[s], (g / bstages) & 1, gerr)) {
                        atomicCAS(err, 0, ERR_TIMEOUT_FULL);
                        ok = false;
                        break;
                    }
                    if (!mbar_wait_bounded(&tempty[t], ((g >> 1) & 1) ^ 1, gerr)) {
                        atomicCAS(err, 0, ERR_TIMEOUT_TEMPTY);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d = tmem_base + (uint32_t)(t * BN);
                    const uint32_t b_hi = smem_u32(sB + (size_t)s * STAGE_BYTES), b_lo = b_hi + B_BYTES;
                    const uint32_t as[3] = {a_hi, a_lo, a_hi};
                    const uint32_t bs[3] = {b_hi, b_hi, b_lo};
#pragma unroll
                    for (int prod = 0; prod < 3; ++prod)
#pragma unroll
                        for (int ks = 0; ks < KD / 16; ++ks)
                            umma_bf16(d, sw128_desc(as[prod] + ks * 32), sw128_desc(bs[prod] + ks * 32),
                                      (prod | ks) != 0 ? 1u : 0u);
                    umma_commit(&empty[s]);
                    umma_commit(&tfull[t]);
                    issued = g + 1;
                }
                umma_commit(&aempty[sa]);   // the A slot is free once this tile's MMAs complete
                if (!ok) {
                    *abort_flag = 1;
                    break;
                }
            }
            // drain: the last MMAs issued have completed before TMEM is freed
            if (issued > 0) mbar_wait_bounded(&tfull[(issued - 1) & 1], ((issued - 1) >> 1) & 1, nullptr);
        }
    } else if (warp < WARP_DRAW0) {
        // ---------------- drain: TMEM accumulator -> r (quarter = warp % 4, cluster c of each N tile)
        const int quarter = warp & 3;
        const int c = (warp - WARP_DRAIN0) >> 2;
        const int p = quarter * 32 + lane;
        const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
        int g = 0, la = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++la) {
            if (__any_sync(0xffffffffu, *abort_flag != 0)) break;
            // the draw warps have taken the previous tile's r and partials
            if (la > 0 && !warp_wait_bounded(rempty, (la - 1) & 1, gerr)) {
                if (lane == 0) atomicCAS(err, 0, ERR_TIMEOUT_REMPTY);
                *abort_flag = 1;
                break;
            }
            const int64_t pt = (int64_t)tile * BM + p;
            float m = -INFINITY, sum = 0.f;   // running max and sum of exp(r - max); final: best, arg
            int arg = -1;
            bool ok = true;
            for (int nt = 0; nt < NT; ++nt, ++g) {
                const int t = g & 1;
                if (!warp_wait_bounded(&tfull[t], (g >> 1) & 1, gerr)) {
                    if (lane == 0) atomicCAS(err, 0, ERR_TIMEOUT_TFULL);
                    ok = false;
                    break;
                }
                tc_fence_after();
                const int k = nt * CPT + c;
                if (k < K) {
                    uint32_t v[64];
                    tmem_ld64(tmem_base + lane_addr + (uint32_t)(t * BN + c * KD), v);
                    const float4* bk = reinterpret_cast<const float4*>(bvec + (size_t)3 * k * Dp);
                    float q0 = 0.f, q1 = 0.f;
#pragma unroll
                    for (int j4 = 0; j4 < KD / 4; ++j4) {
                        const float4 b4 = j4 * 4 < Dp ? __ldg(bk + j4) : make_float4(0.f, 0.f, 0.f, 0.f);
                        const float z0 = __uint_as_float(v[4 * j4 + 0]) - b4.x;
                        const float z1 = __uint_as_float(v[4 * j4 + 1]) - b4.y;
                        const float z2 = __uint_as_float(v[4 * j4 + 2]) - b4.z;
                        const float z3 = __uint_as_float(v[4 * j4 + 3]) - b4.w;
                        q0 = fmaf(z0, z0, q0);
                        q1 = fmaf(z1, z1, q1);
                        q0 = fmaf(z2, z2, q0);
                        q1 = fmaf(z3, z3, q1);
                    }
                    const float r = __ldg(cvec + 3 * k) - 0.5f * (q0 + q1);
                    if (final_) {
                        if (arg < 0 || m < r) { m = r; arg = k; }   // first maximum in cluster order
                    } else {
                        if (r > m) {
                            sum = sum * __expf(m - r) + 1.f;
                            m = r;
                        } else {
                            sum += __expf(r - m);
                        }
                        tmem_st1(tmem_base + lane_addr + R_COL0 + (uint32_t)k, r);
                    }
                    if (r_out && pt < N) r_out[pt * K + k] = r;
                }
                tc_fence_before();
                mbar_arrive(&tempty[t]);
            }
            if (!ok) {
                *abort_flag = 1;
                break;
            }
            spart[(2 * c) * BM + p] = m;
            spart[(2 * c + 1) * BM + p] = final_ ? __int_as_float(arg) : sum;
            if (!final_) asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            tc_fence_before();
            mbar_arrive(rfull);
        }
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");   // nothing in flight at dealloc
    } else {
        // ---------------- draw: one thread per point of the lane quarter (warp % 4)
        const int quarter = warp & 3;
        const int p = quarter * 32 + lane;
        const uint32_t lane_addr = (uint32_t)(quarter * 32) << 16;
        float* row = sr + (size_t)p * KS;
        int la = 0;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++la) {
            if (__any_sync(0xffffffffu, *abort_flag != 0)) break;
            if (!warp_wait_bounded(rfull, la & 1, gerr)) {
                if (lane == 0) atomicCAS(err, 0, ERR_TIMEOUT_RFULL);
                *abort_flag = 1;
                break;
            }
            tc_fence_after();
            const float m0 = spart[0 * BM + p], x0 = spart[1 * BM + p];
            const float m1 = spart[2 * BM + p], x1 = spart[3 * BM + p];
            if (!final_) {
                for (int c0 = 0; c0 < K; c0 += 32) {
                    uint32_t v[32];
                    tmem_ld32(tmem_base + lane_addr + R_COL0 + (uint32_t)c0, v);
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        if (c0 + j < K) row[c0 + j] = __uint_as_float(v[j]);
                }
            }
            tc_fence_before();
            mbar_arrive(rempty);
            const int64_t pt = (int64_t)tile * BM + p;
            if (pt >= N) continue;
            if (final_) {
                // update_labels_by_max_index_kernel (cudaKernel.cu:405-424): first maximum wins
                const int a0 = __float_as_int(x0), a1 = __float_as_int(x1);
                int arg = a0;
                if (a1 >= 0 && (a0 < 0 || m0 < m1 || (m1 == m0 && a1 < a0))) arg = a1;
                labels[pt] = arg + 1;
            } else {
                // build_log_likelihood_array_kernel (cudaKernel.cu:374-403): max, exp, normalise
                const float mx = fmaxf(m0, m1);
                const float sum = x0 * __expf(m0 - mx) + x1 * __expf(m1 - mx);
                const float inv = 1.0f / sum, fk = (float)K;
                int ns = 0;
                for (int k = 0; k < K; ++k) {
                    const float y = (__expf(row[k] - mx) * inv) * fk;
                    row[k] = y;
                    ns += y < 1.f ? 1 : 0;
                }
                float u1, u2;
                draw_uniform2(rng, pt, u1, u2);
                labels[pt] = alias_draw_stream_ns(row, 1, K, ns, u1, u2);
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

}  // namespace tc

constexpr size_t kTcSmemCap = 227 * 1024;

// (A slots, B stages) for K clusters: the deepest rings that fit
static bool tc_config(int K, int& astages, int& bstages)
{
    const int cand[4][2] = {{2, 3}, {2, 2}, {1, 3}, {1, 2}};
    for (const auto& cb : cand)
        if (tc::smem_layout(K, cb[0], cb[1]).total <= kTcSmemCap) {
            astages = cb[0];
            bstages = cb[1];
            return true;
        }
    return false;
}

bool tc_supported(const dpmm_ctx* c, int K)
{
    int as = 0, bs = 0;
    return c->prior == DPMM_PRIOR_GAUSSIAN && c->d_Btc != nullptr && c->d_Atc != nullptr &&
           (c->Dp == 32 || c->Dp == 64) && K >= 1 && K <= (int)(tc::TMEM_COLS - tc::R_COL0) &&
           tc_config(K, as, bs);
}

dpmm_status pack_tc_params(dpmm_ctx* c, int K)
{
    if (!c->d_Btc || !(c->Dp == 32 || c->Dp == 64)) return DPMM_OK;
    const int NT = (K + tc::CPT - 1) / tc::CPT;
    const int total = NT * tc::BN * 8;
    tc::k_pack_b<<<(total + 255) / 256, 256, 0, c->stream>>>(c->d_Wt, K, c->Dp, NT, c->d_Btc);
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
    int astages = 0, bstages = 0;
    if (!tc_supported(c, K) || !tc_config(K, astages, bstages))
        return fail(DPMM_ERR_INVALID_ARG, "tensor-core label kernel: unsupported shape");
    const tc::SmemLayout L = tc::smem_layout(K, astages, bstages);
    RngArgs r = rng_args(c, d_u);
    DPMM_CUDA_TRY(cudaFuncSetAttribute(tc::k_gauss_labels_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
    int32_t* err = c->d_aux + 4;
    DPMM_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int32_t), c->stream));
    const int64_t ntiles = (c->N + tc::BM - 1) / tc::BM;
    const unsigned grid = (unsigned)std::min<int64_t>(ntiles, c->num_sms);
    tc::k_gauss_labels_tc<<<grid, tc::THREADS, L.total, c->stream>>>(c->d_Atc, c->N, (int)ntiles, c->d_Btc, c->d_b,
                                                                     c->d_c, c->Dp, K, astages, bstages, final_, r,
                                                                     c->d_labels, d_rout, err);
    DPMM_LAUNCHED();
    int32_t h_err = 0;
    DPMM_CUDA_TRY(cudaMemcpyAsync(&h_err, err, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (h_err) return fail(DPMM_ERR_TIMEOUT, "tensor-core label kernel: bounded wait expired (code " +
                                                 std::to_string(h_err) + ")");
    return DPMM_OK;
}

}  // namespace dpmm
