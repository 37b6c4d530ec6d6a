// dpmm_device.cuh -- device helpers shared by the kernels: uniforms (caller-supplied,
// Philox4x32-10, or the cuRAND XORWOW device API in compat mode) and the Walker alias
// draw with the reference's exact construction order.
#pragma once

#include <curand_kernel.h>
#include <stdint.h>

#include "dpmm_internal.h"

namespace dpmm {

// Upper-triangle pair count of the scatter matrix, and the index of (i, j), i <= j, in its
// row-major upper triangle (the layout of the statistics records)
__host__ __device__ constexpr int tri(int dp) { return dp * (dp + 1) / 2; }
__host__ __device__ constexpr int tri_index(int dp, int i, int j) { return i * dp - i * (i - 1) / 2 + (j - i); }

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy as 1, 2, 3",
// SC'11): ten rounds of the 4x32 bijection keyed by a 64-bit key, with the multipliers and
// Weyl key increments published in that paper.
struct Philox4 {
    uint32_t v[4];
};

__device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                 uint32_t k0, uint32_t k1)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(M0, c0), lo0 = M0 * c0;
        uint32_t hi1 = __umulhi(M1, c2), lo1 = M1 * c2;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += W0;
        k1 += W1;
    }
    Philox4 o;
    o.v[0] = c0; o.v[1] = c1; o.v[2] = c2; o.v[3] = c3;
    return o;
}

// 24 random bits -> float in (0, 1] (the range curand_uniform returns)
__device__ __forceinline__ float u01_from_bits(uint32_t x)
{
    return (float)((x >> 8) + 1u) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ Philox4 philox_point(const RngArgs& r, int64_t pt)
{
    pt += r.offset;   // keyed by the global point index
    return philox4x32_10((uint32_t)pt, (uint32_t)((uint64_t)pt >> 32), (uint32_t)r.ctr,
                         (uint32_t)(r.ctr >> 32), (uint32_t)r.seed, (uint32_t)(r.seed >> 32));
}

// Two uniforms for point pt (the two curand_uniform() calls of cudaKernel.cu:115-116).
__device__ __forceinline__ void draw_uniform2(const RngArgs& r, int64_t pt, float& u1, float& u2)
{
    if (r.ucaller) {
        u1 = r.ucaller[2 * pt];
        u2 = r.ucaller[2 * pt + 1];
    } else if (r.kind == DPMM_RNG_CURAND_XORWOW) {
        curandStateXORWOW st = r.states[pt];
        u1 = curand_uniform(&st);
        u2 = curand_uniform(&st);
        r.states[pt] = st;
    } else {
        Philox4 o = philox_point(r, pt);
        u1 = u01_from_bits(o.v[0]);
        u2 = u01_from_bits(o.v[1]);
    }
}

// A label phase that settles a point without drawing still consumes its two uniforms from a
// stateful per-point stream (cuRAND XORWOW), so later draws stay those of the dense phase; the
// caller-supplied and counter-based sources need nothing.
__device__ __forceinline__ void skip_uniform2(const RngArgs& r, int64_t pt)
{
    if (!r.ucaller && r.kind == DPMM_RNG_CURAND_XORWOW) {
        float u1, u2;
        draw_uniform2(r, pt, u1, u2);
    }
}

// One uniform for point pt (initial label draws, cudaKernel.cu:144-170).
__device__ __forceinline__ float draw_uniform1(const RngArgs& r, int64_t pt)
{
    if (r.ucaller) return r.ucaller[pt];
    if (r.kind == DPMM_RNG_CURAND_XORWOW) {
        curandStateXORWOW st = r.states[pt];
        float u = curand_uniform(&st);
        r.states[pt] = st;
        return u;
    }
    return u01_from_bits(philox_point(r, pt).v[0]);
}

// 32 random bits for point pt (the curand() of cudaKernel.cu:210, :252).
__device__ __forceinline__ uint32_t draw_bits(const RngArgs& r, const uint32_t* bits, int64_t pt)
{
    if (bits) return bits[pt];
    if (r.kind == DPMM_RNG_CURAND_XORWOW) {
        curandStateXORWOW st = r.states[pt];
        uint32_t v = curand(&st);
        r.states[pt] = st;
        return v;
    }
    return philox_point(r, pt).v[2];
}

// Column chosen by the first uniform: (int)(u1 * (n - 1 + 0.999999) + 1) evaluated in double
// exactly as cudaKernel.cu:115 does (float uniform promoted to double).  For u1 in (0, 1] the
// column is already in [1, n]; the clamp only keeps a caller's out-of-range uniform inside the table.
__device__ __forceinline__ int alias_column(int n, float u1)
{
    int col = (int)((double)u1 * ((double)(n - 1) + 0.999999) + 1.0);
    return col < 1 ? 1 : (col > n ? n : col);
}

// Walker alias construction + draw in the order of cudaKernel.cu:27-124.  The arrays are
// accessed through an accessor so the same code serves shared-memory tables interleaved
// across the points of a tile (index * stride + lane) and small per-thread arrays.
// Preconditions: y(1..n) = p_i * n.  Indices 0..n+1 are used.  Returns the 1-based label.
template <typename T, typename IdxT, typename Acc>
__device__ __forceinline__ int alias_draw(int n, Acc acc, float u1, float u2)
{
    T* __restrict__ y = acc.y;
    IdxT* __restrict__ a = acc.a;
    IdxT* __restrict__ b = acc.b;
    const int s = acc.stride;
    for (int i = 0; i <= n + 1; ++i) {
        a[i * s] = (IdxT)i;
        b[i * s] = (IdxT)i;
    }
    y[0] = (T)0;
    y[(n + 1) * s] = (T)2;
    int i = 0, j = n + 1, t;
    for (;;) {
        do { i++; } while (y[(int)b[i * s] * s] < (T)1);
        do { j--; } while ((T)1 <= y[(int)b[j * s] * s]);
        if (j <= i) break;
        t = b[i * s]; b[i * s] = b[j * s]; b[j * s] = (IdxT)t;
    }
    i = j;
    j++;
    while (0 < i) {
        while (y[(int)b[j * s] * s] <= (T)1) j++;
        if (n < j) break;
        const int bj = b[j * s], bi = b[i * s];
        y[bj * s] = y[bj * s] - ((T)1 - y[bi * s]);
        a[bi * s] = (IdxT)bj;
        if (y[bj * s] < (T)1) {
            b[i * s] = (IdxT)bj;
            b[j * s] = (IdxT)bi;
            j++;
        } else {
            i--;
        }
    }
    const int col = alias_column(n, u1);
    int label = col;
    if (y[col * s] < (T)u2) label = a[col * s];
    return label;
}

template <typename T, typename IdxT>
struct AliasAcc {
    T* y;
    IdxT* a;
    IdxT* b;
    int stride;
};

// Two-category draw used by the sub-cluster phase: the general construction with n = 2 on
// a 4-entry table, with the reference's float->double promotions replaced by float maths.
__device__ __forceinline__ int alias_draw2(float p1, float p2, float u1, float u2)
{
    float y[4];
    uint8_t a[4], b[4];
    y[1] = p1 * 2.0f;
    y[2] = p2 * 2.0f;
    AliasAcc<float, uint8_t> acc{y, a, b, 1};
    return alias_draw<float, uint8_t>(2, acc, u1, u2);
}

// ---------------------------------------------------------------------------------------------
// Streamed form of the same alias draw (one thread, no index tables).  y[(k - 1) * stride] =
// p_k * K for the 1-based categories k = 1..K; returns the label drawn with (u1, u2).
//
// Only the drawn column's final (y, alias) matter, and the reference's two loops
// (cudaKernel.cu:56-111) determine them as a merge of two streams:
//  * the partition leaves the smalls (y < 1) at positions 1..ns: a small at q <= ns stays, and
//    the larges of [1, ns] trade places with the smalls of (ns, K], the i-th large from the
//    left with the i-th small from the right;
//  * the pairing consumes smalls from position ns downwards (a displaced large's slot yields
//    the next small of (ns, K] walking upwards) and larges from position ns + 1 upwards (a
//    displaced small's slot yields the next large of [1, ns] walking downwards);
//  * with D the deficit (1 - y) consumed so far and C the excess (y - 1) of the larges taken so
//    far, a small is aliased to the current large, which is replaced by the next one with
//    positive excess while C <= D; a large whose C is reached by D ends at y = 1 + C - D and,
//    when D > C, is aliased to the next large with positive excess.
// The merge stops as soon as the drawn column is settled.  D and C are FP64 running sums in the
// reference's consumption order.
// Small/large flags of up to 256 categories as a bitmask in registers: bit (q - 1) % 32 of word
// (q - 1) / 32 is set when category q is small.  The walks of the merge become bit scans.
struct SmallMask {
    uint32_t w[8];
    int K;

    __device__ __forceinline__ uint32_t word(int i) const
    {
        uint32_t v = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (j == i) v = w[j];
        return v;
    }
    __device__ __forceinline__ bool small(int q) const { return (word((q - 1) >> 5) >> ((q - 1) & 31)) & 1u; }
    // smallest small q > x (K + 1 if none)
    __device__ __forceinline__ int next_small_after(int x) const
    {
        int res = K + 1;
#pragma unroll
        for (int j = 7; j >= 0; --j) {
            uint32_t m = w[j];
            const int lo = x - 32 * j;   // clear bits b with 32j + b + 1 <= x
            m = lo <= 0 ? m : (lo >= 32 ? 0u : m & (~0u << lo));
            if (m) res = 32 * j + __ffs(m);
        }
        return res;
    }
    // largest large q < x (0 if none)
    __device__ __forceinline__ int prev_large_before(int x) const
    {
        int res = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int nv = K - 32 * j;   // valid bits in word j
            uint32_t m = ~w[j] & (nv >= 32 ? ~0u : (nv <= 0 ? 0u : (1u << nv) - 1u));
            const int hi = x - 1 - 32 * j;   // keep bits b with 32j + b + 1 < x
            m = hi >= 32 ? m : (hi <= 0 ? 0u : m & ((1u << hi) - 1u));
            if (m) res = 32 * j + 32 - __clz(m);
        }
        return res;
    }
};

// The same flags read from y itself (any K): linear walks.  YF: y(i) for 0-based i.
template <typename YF>
struct ReadFlags {
    YF y;
    int K;
    __device__ __forceinline__ bool small(int q) const { return y(q - 1) < 1.f; }
    __device__ __forceinline__ int next_small_after(int x) const
    {
        int q = x + 1;
        while (q <= K && !small(q)) ++q;
        return q;
    }
    __device__ __forceinline__ int prev_large_before(int x) const
    {
        int q = x - 1;
        while (q >= 1 && small(q)) --q;
        return q;
    }
};

// The merge of the two consumption streams (see above).  y(i) returns y of category i + 1 and
// must return the same value on every call.
template <typename YF, typename Flags>
__device__ __forceinline__ int alias_merge(const YF& y, int K, int ns, const Flags& fl, float u1, float u2)
{
    const int col = alias_column(K, u1);
    const float yc = y(col - 1);
    if (yc == 1.f) return col;           // a large without excess is never consumed

    int P = ns + 1;     // small-stream position (descending)
    int sr = ns;        // last small of (ns, K] taken (ascending)
    int Q = ns;         // large-stream position (ascending)
    int ll = ns + 1;    // last large of [1, ns] taken (descending)
    double D = 0.0, C = 0.0, Ccol = 0.0;
    bool col_taken = false;

    // next large with positive excess in consumption order (0 if none); adds its excess to C
    auto next_large = [&]() -> int {
        while (++Q <= K) {
            int e = Q;
            if (fl.small(Q)) {
                ll = fl.prev_large_before(ll);
                if (ll < 1) return 0;     // unreachable: (ns, K] holds as many smalls as [1, ns] larges
                e = ll;
            }
            const double ex = (double)y(e - 1) - 1.0;
            if (ex > 0.0) {
                C += ex;
                return e;
            }
        }
        return 0;
    };
    // the large that col passes its deficit to, once D has reached col's C
    auto settle_col = [&]() -> int {
        if (!(1.0 + Ccol - D < (double)u2)) return col;
        const int a = next_large();
        return a != 0 ? a : col;
    };

    int cur = 0;
    for (;;) {
        // Fast path: the next 8 positions of the small stream hold their own smalls (no displaced
        // large among them), col is not one of them, and the current large still has capacity
        // after all 8: none of these steps can change the outcome, so take them at once (same
        // summation order as single steps).
        if (cur != 0 && P > 8 && (col >= P || col < P - 8)) {
            float v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = y(P - 2 - i);
            bool all_small = true;
#pragma unroll
            for (int i = 0; i < 8; ++i) all_small = all_small && v[i] < 1.f;
            if (all_small) {
                double Dn = D;
#pragma unroll
                for (int i = 0; i < 8; ++i) Dn += 1.0 - (double)v[i];
                if (Dn < C) {
                    D = Dn;
                    P -= 8;
                    continue;
                }
            }
        }
        if (--P < 1) return col;          // every small paired: col keeps itself
        int s = P;
        if (!fl.small(P)) {
            sr = fl.next_small_after(sr);
            if (sr > K) return col;       // unreachable, as above
            s = sr;
        }
        while (C <= D) {                  // the current large is used up: take the next
            cur = next_large();
            if (cur == 0) return col;     // no large left: this and later smalls keep themselves
            if (cur == col) {
                col_taken = true;
                Ccol = C;
                if (Ccol <= D) return settle_col();   // used up at once by the carried deficit
            }
        }
        if (s == col) return yc < u2 ? cur : col;
        D += 1.0 - (double)y(s - 1);
        if (col_taken && D >= Ccol) return settle_col();
    }
}

// Alias draw over K categories given y(i) = p_{i+1} * K (FP32): register bitmask walks for
// K <= 256, reads otherwise.  SF: is_small(i), the small/large split the merge follows (y(i) < 1,
// or an equivalent cheaper test; at an exact tie either answer keeps the walk consistent: a
// small with y >= 1 adds no deficit and a large with y <= 1 has no excess to give).
template <typename YF, typename SF>
__device__ __forceinline__ int alias_draw_y(const YF& y, const SF& is_small, int K, float u1, float u2)
{
    if (K <= 256) {
        SmallMask sm;
        sm.K = K;
        int ns = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            uint32_t m = 0;
            const int kend = min(K, 32 * j + 32);
            for (int k = 32 * j; k < kend; ++k) m |= (is_small(k) ? 1u : 0u) << (k - 32 * j);
            sm.w[j] = m;
            ns += __popc(m);
        }
        if (ns == K - 1) {
            // One large L: it absorbs every small's deficit (its excess equals their total up to
            // rounding, well below 1e-3), so a drawn small with y < 0.999 is aliased to L wherever it
            // sits in the consumption order.  Otherwise (col = L, or y near 1) walk the merge.
            const int col = alias_column(K, u1);
            if (sm.small(col)) {
                const float yc = y(col - 1);
                if (yc < 0.999f) return yc < u2 ? sm.prev_large_before(K + 1) : col;
            }
        }
        return alias_merge(y, K, ns, sm, u1, u2);
    }
    int ns = 0;
    for (int k = 0; k < K; ++k) ns += y(k) < 1.f ? 1 : 0;
    return alias_merge(y, K, ns, ReadFlags<YF>{y, K}, u1, u2);
}

// y stored in memory: ys[(k - 1) * stride] for category k.
__device__ __forceinline__ int alias_draw_stream(const float* __restrict__ ys, int64_t stride, int K, float u1,
                                                 float u2)
{
    auto y = [=](int i) -> float { return ys[(size_t)i * stride]; };
    auto is_small = [=](int i) -> bool { return ys[(size_t)i * stride] < 1.f; };
    return alias_draw_y(y, is_small, K, u1, u2);
}

}  // namespace dpmm
