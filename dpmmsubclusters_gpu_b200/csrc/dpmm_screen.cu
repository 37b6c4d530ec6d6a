// dpmm_screen.cu -- learned split/merge screen.  No counterpart in the reference, which evaluates the
// exact Hastings ratio of every split candidate (local_clusters_actions.cpp:244-285) and every
// cluster pair (local_clusters_actions.cpp:287-321) each iteration.  Here:
//
//   k_screen_slots_niw / _dir   per statistics slot: posterior quantities; for cluster slots the
//                               exact log marginal likelihood, log det psi' and (NIW) the inverse
//                               Cholesky factor of psi'.  No Cholesky of the sub-cluster slots.
//   k_screen_merge_feat         32 features of every pair i < j (one warp per pair): the exact count
//                               term of the merge ratio plus a proxy of the marginal-likelihood
//                               term that needs no Cholesky of the merged scatter (Minkowski's
//                               determinant inequality for log|B_i + B_j|, a rank-one correction
//                               for the mean shift, diagonal and Mahalanobis separations)
//   k_screen_split_feat         the same for every cluster's split into its two sub-clusters
//   k_screen_mlp                32 -> 64 -> 64 -> 1 ReLU MLP, BF16-rounded weights, FP32 accumulate
//   k_screen_topk               the `top` best-scored eligible candidates, ascending candidate order
//   k_*_list                    exact FP64 ratios (the arithmetic of dpmm_hastings.cu) for a list
//   k_mlp_grad_tile, k_mlp_adam training: forward + backward over 64-row tiles (per-tile partial
//                               gradients, deterministic), fixed-order reduction and Adam update
//
// The feature definitions are restated in FP64 numpy by the screen oracle (test infrastructure).
#include <cuda_bf16.h>
#include <math.h>

#include <algorithm>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "dpmm_internal.h"
#include "dpmm_niw.cuh"

namespace dpmm {

// per-slot record (FP64), kScrRec values
enum { R_N = 0, R_KP = 1, R_VP = 2, R_LD = 3, R_HD = 4, R_TR = 5, R_L = 6, R_LST = 7, R_TAU = 8 };
// (Dirichlet: R_KP holds A = sum a', R_VP holds A0 = sum alpha0, R_TR the mean count per point;
//  NIW cluster slots: R_TAU = tr(B^-1 P0), B = nu' psi', P0 = nu0 psi0 + kappa0 m0 m0^T)

__device__ __forceinline__ double slog(double x) { return copysign(log1p(fabs(x)), x); }

__device__ __forceinline__ double logaddexp2v(double a, double b)
{
    const double m = fmax(a, b);
    return m + log1p(exp(-fabs(a - b)));
}

// (x - 1/2) ln x - x + ln(2 pi) / 2 for x > 0, else 0
__device__ __forceinline__ double stirling(double x)
{
    return x > 0 ? (x - 0.5) * log(x) - x + 0.91893853320467274178 : 0.0;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// pair row (row-major over the strict upper triangle of K x K) -> (i, j)
__device__ __forceinline__ void unrank_pair(long long row, int K, int& i, int& j)
{
    // largest i with start(i) = i (2K - i - 1) / 2 <= row
    int lo = 0, hi = K - 2;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const long long st = (long long)mid * (2LL * K - mid - 1) / 2;
        if (st <= row) lo = mid;
        else hi = mid - 1;
    }
    i = lo;
    j = (int)(row - (long long)lo * (2LL * K - lo - 1) / 2) + lo + 1;
}

__device__ double count_term_merge(double ni, double nj, double alpha)
{
    const double n = ni + nj;
    return -log(alpha) + lgamma(alpha) - 2 * lgamma(0.5 * alpha) + lgamma(n) - lgamma(n + alpha) +
           lgamma(ni + 0.5 * alpha) - lgamma(ni) - lgamma(nj) + lgamma(nj + 0.5 * alpha);
}

// NIW log marginal likelihood (niw.cpp:122-138) given the posterior log|psi'| and the lgamma sum g
__device__ double niw_lml_hat(double n, int D, double k0, double v0, double ld0, double kp, double vp, double ldp,
                              double g)
{
    return -n * D * 0.5 * log(M_PI) + g + (v0 / 2.0) * (D * log(v0) + ld0) - (vp / 2.0) * (D * log(vp) + ldp) +
           (D / 2.0) * log(k0 / kp);
}

// sum over d = 1..D of log(max(m - d + 1, 1)) over this lane's d (lanes stride 32); a warp sum gives
// the log-determinant scale of a Wishart scatter of m points
__device__ __forceinline__ double lw_part(double m, int D, int lane)
{
    double s = 0;
    for (int d = 1 + lane; d <= D; d += 32) s += log(fmax(m - d + 1.0, 1.0));
    return s;
}

// the 32 features of one candidate (roles a, b and their union u); rows are written by lane 0
__device__ void screen_assemble(float* __restrict__ f, bool merge, bool gauss, int D, double alpha, double P, double T,
                                double na, double nb, double nu, double La, double Lb, double Lu, double qa, double qb,
                                double r1, double gsc, double gapa, double gapb, double gapu, double ldd, double md,
                                double pf, double tra, double trb, const double* ex)
{
    const double Dd = (double)D;
    double v[kScrF];
    const double e27 = ex[0], e28 = ex[1], e29 = ex[2], e30 = ex[3];
    v[0] = merge ? 1.0 : -1.0;
    v[1] = gauss ? 1.0 : -1.0;
    v[2] = slog(P) / 8;
    v[3] = slog(T) / 8;
    v[4] = slog(P - T) / 8;
    v[5] = log1p(na) / 16;
    v[6] = log1p(nb) / 16;
    v[7] = log1p(nu) / 16;
    v[8] = na / (na + nb);
    v[9] = log(Dd) / 8;
    v[10] = log(alpha) / 4;
    v[11] = fmin(fmax(La / (na * Dd), -8.0), 8.0) / 8;
    v[12] = fmin(fmax(Lb / (nb * Dd), -8.0), 8.0) / 8;
    v[13] = fmin(fmax(Lu / (nu * Dd), -8.0), 8.0) / 8;
    v[14] = log1p(qa) / 8;
    v[15] = log1p(qb) / 8;
    v[16] = log1p(r1) / 8;
    v[17] = slog(gsc) / 8;
    v[18] = gapa;
    v[19] = gapb;
    v[20] = gapu;
    v[21] = ldd;
    v[22] = log1p(md) / 8;
    v[23] = pf;
    v[24] = log(fmax(tra, 1e-30)) / 8;
    v[25] = log(fmax(trb, 1e-30)) / 8;
    v[26] = slog(P / (na + nb)) / 8;
    v[27] = slog(e27) / 8;
    v[28] = slog(e28) / 8;
    v[29] = slog(e29) / 8;
    v[30] = e30;
    v[31] = 0.0;
#pragma unroll
    for (int q = 0; q < kScrF; ++q) f[q] = (float)v[q];
}

// ------------------------------------------------------------------------------ per-slot quantities
// NIW: one block per slot (3K).  vec[s] = posterior mean m'[D] then diag(psi')[D].  Cluster slots also
// get the exact log marginal likelihood, log det psi', tau and the inverse Cholesky factor of psi'.
// psi0_identity: the prior scale is the identity and its mean zero (tau needs no prior matrix then).
// Dynamic shared memory: D*D doubles (the Cholesky factor, then its inverse).
template <int DP>
__global__ void __launch_bounds__(RegChol<DP>::T) k_screen_slots_niw(const double* __restrict__ stats, int stat_len,
                                                                      int D, double k0, double v0, double ld0,
                                                                      const double* __restrict__ prior,
                                                                      int psi0_identity, double* __restrict__ rec,
                                                                      double* __restrict__ vec, float* __restrict__ linv)
{
    __shared__ double sh[RegChol<DP>::SMEM];
    extern __shared__ double Lm[];
    double* red = sh + 3 * DP;
    const int s = blockIdx.x;
    const double* st = stats + (size_t)s * stat_len;
    const double n = st[0];
    const double* m0 = prior;
    const double* psi0 = prior + D;
    double* r = rec + (size_t)s * kScrRec;
    double* vmean = vec + (size_t)s * 2 * D;
    double* vdiag = vmean + D;
    const double kp = k0 + n, vp = v0 + n;
    double h = 0, t = 0;
    for (int d = threadIdx.x; d < D; d += blockDim.x) {
        // the expressions of niw_lml_reg for m'[d] and psi'(d, d)
        const double m = (m0[d] * k0 + st[1 + d]) / kp;
        const size_t dd = (size_t)d * D + d;
        const double tm = v0 * psi0[dd] + k0 * m0[d] * m0[d];
        const double pdd = (tm - kp * m * m + st[1 + D + dd]) / vp;
        vmean[d] = m;
        vdiag[d] = pdd;
        h += log(pdd);
        t += pdd;
    }
    double ld = 0, L = 0, tau = 0;
    if (s % 3 == 0 && n > 0) {
        NiwExtras ex;
        L = niw_lml_reg<DP>(D, n, st + 1, st + 1 + D, nullptr, nullptr, k0, v0, m0, psi0, ld0, sh, &ex, Lm);
        ld = ex.ld;
        h = ex.hd;
        t = ex.tr;
        for (int e = threadIdx.x; e < D * D; e += blockDim.x) {   // zero the upper triangle of the factor
            const int i = e % D, j = e / D;
            if (i < j) Lm[e] = 0.0;
        }
        __syncthreads();
        block_tri_inverse(Lm, D);          // Lm now holds Y = L^-1 (lower)
        // tau = tr(psi'^-1 P0) / nu' = sum over rows r of y_r^T P0 y_r / nu', P0 = nu0 psi0 + kappa0 m0 m0^T
        for (int rr = threadIdx.x; rr < D; rr += blockDim.x) {
            double acc = 0;
            if (psi0_identity) {
                for (int a = 0; a <= rr; ++a) {
                    const double y = Lm[(size_t)a * D + rr];
                    acc += y * y;
                }
                acc *= v0;
            } else {
                double ym = 0;
                for (int a = 0; a <= rr; ++a) {
                    const double ya = Lm[(size_t)a * D + rr];
                    ym += ya * m0[a];
                    double q = 0;
                    for (int b = 0; b <= rr; ++b) q += psi0[(size_t)b * D + a] * Lm[(size_t)b * D + rr];
                    acc += ya * q;
                }
                acc = v0 * acc + k0 * ym * ym;
            }
            tau += acc;
        }
        tau = block_sum(tau, red) / vp;
        float* Li = linv + (size_t)(s / 3) * D * D;
        for (int e = threadIdx.x; e < D * D; e += blockDim.x) Li[e] = (float)Lm[e];
    } else {
        h = block_sum(h, red);
        t = block_sum(t, red);
    }
    if (threadIdx.x == 0) {
        r[R_N] = n;
        r[R_KP] = kp;
        r[R_VP] = vp;
        r[R_LD] = ld;
        r[R_HD] = h;
        r[R_TR] = t;
        r[R_L] = L;
        r[R_LST] = 0.0;
        r[R_TAU] = tau;
    }
}

// Dirichlet: one block per slot.  vec[s] = p = a' / sum a' [D] then a' [D].
__global__ void __launch_bounds__(kHThreads) k_screen_slots_dir(const double* __restrict__ stats, int stat_len, int D,
                                                                const double* __restrict__ alpha0,
                                                                double* __restrict__ rec, double* __restrict__ vec)
{
    __shared__ double red[33];
    const int s = blockIdx.x;
    const double* st = stats + (size_t)s * stat_len;
    const double n = st[0];
    double* vp_ = vec + (size_t)s * 2 * D;
    double* va = vp_ + D;
    double A0 = 0, A = 0, sst = 0;
    for (int d = threadIdx.x; d < D; d += blockDim.x) {
        const double a0 = alpha0[d], a = a0 + st[1 + d];
        va[d] = a;
        A0 += a0;
        A += a;
        sst += stirling(a) - stirling(a0);
    }
    A0 = block_sum(A0, red);
    A = block_sum(A, red);
    sst = block_sum(sst, red);
    for (int d = threadIdx.x; d < D; d += blockDim.x) vp_[d] = A > 0 ? (alpha0[d] + st[1 + d]) / A : 0.0;
    double L = 0.0;
    if (s % 3 == 0) L = mult_lml_block(D, n, st + 1, nullptr, alpha0, red);
    if (threadIdx.x == 0) {
        double* r = rec + (size_t)s * kScrRec;
        r[R_N] = n;
        r[R_KP] = A;
        r[R_VP] = A0;
        r[R_LD] = 0.0;
        r[R_HD] = 0.0;
        r[R_TR] = n > 0 ? (A - A0) / n : 0.0;
        r[R_L] = L;
        r[R_LST] = stirling(A0) - stirling(A) + sst;
        r[R_TAU] = 0.0;
    }
}

// ------------------------------------------------------------------------------ features
constexpr int kFeatWarps = 8;

template <bool GAUSS>
__global__ void __launch_bounds__(32 * kFeatWarps) k_screen_merge_feat(const double* __restrict__ rec,
                                                                        const double* __restrict__ vec,
                                                                        const float* __restrict__ linv, int D, int K,
                                                                        long long pairs, double k0, double v0, double ld0,
                                                                        double alpha, const double* __restrict__ alpha0,
                                                                        float* __restrict__ feat, double* __restrict__ prox)
{
    __shared__ double sdelta[kFeatWarps][GAUSS ? kMaxGaussDim : 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long row = (long long)blockIdx.x * kFeatWarps + warp;
    if (row >= pairs) return;   // warp-uniform; the kernel has no block-wide barrier
    int i, j;
    unrank_pair(row, K, i, j);
    const double* ri = rec + (size_t)(3 * i) * kScrRec;
    const double* rj = rec + (size_t)(3 * j) * kScrRec;
    float* out = feat + (size_t)row * kScrF;
    const double ni = ri[R_N], nj = rj[R_N];
    if (ni == 0 || nj == 0) {
        out[lane] = 0.f;
        if (lane == 0) prox[row] = 0.0;
        return;
    }
    const double n = ni + nj;
    const double* vi = vec + (size_t)(3 * i) * 2 * D;
    const double* vj = vec + (size_t)(3 * j) * 2 * D;
    if (GAUSS) {
        const double* di = vi + D;
        const double* dj = vj + D;
        double s_lsum = 0, s_li = 0, s_lj = 0, s_md = 0;
        for (int d = lane; d < D; d += 32) {
            const double dl = vi[d] - vj[d];
            sdelta[warp][d] = dl;
            const double bi = ri[R_VP] * di[d], bj = rj[R_VP] * dj[d];
            s_lsum += log(bi + bj);
            s_li += log(bi);
            s_lj += log(bj);
            s_md += dl * dl / (di[d] + dj[d]);
        }
        __syncwarp();
        // delta^T psi'^-1 delta = |L^-1 delta|^2 for both clusters; lane r owns rows r, r + 32, ...
        const float* Li = linv + (size_t)i * D * D;
        const float* Lj = linv + (size_t)j * D * D;
        double qi = 0, qj = 0;
        for (int r = lane; r < D; r += 32) {
            double zi = 0, zj = 0;
            for (int c = 0; c <= r; ++c) {
                const double dc = sdelta[warp][c];
                zi += (double)Li[(size_t)c * D + r] * dc;
                zj += (double)Lj[(size_t)c * D + r] * dc;
            }
            qi += zi * zi;
            qj += zj * zj;
        }
        const double vu = v0 + n, ku = k0 + n;
        double g = 0;
        for (int d = 1 + lane; d <= D; d += 32) g += lgamma(vu / 2.0 + (1 - d) / 2.0) - lgamma(v0 / 2.0 + (1 - d) / 2.0);
        double wu = lw_part(n, D, lane), wi = lw_part(ni, D, lane), wj = lw_part(nj, D, lane);
        wu = warp_sum(wu);
        wi = warp_sum(wi);
        wj = warp_sum(wj);
        s_lsum = warp_sum(s_lsum);
        s_li = warp_sum(s_li);
        s_lj = warp_sum(s_lj);
        s_md = warp_sum(s_md);
        qi = warp_sum(qi);
        qj = warp_sum(qj);
        g = warp_sum(g);
        if (lane != 0) return;
        const double T = count_term_merge(ni, nj, alpha);
        const double lbi = D * log(ri[R_VP]) + ri[R_LD], lbj = D * log(rj[R_VP]) + rj[R_LD];
        const double lbm = D * logaddexp2v(lbi / D, lbj / D);
        const double ai = qi / ri[R_VP], aj = qj / rj[R_VP];
        const double h = ai + aj > 0 ? ai * aj / (ai + aj) : 0.0;
        const double c = ri[R_KP] * rj[R_KP] / (ri[R_KP] + rj[R_KP]);
        const double ti = ri[R_TAU], tj = rj[R_TAU];
        const double ht = ti + tj > 0 ? ti * tj / (ti + tj) : 0.0;
        const double g0 = wu - D * logaddexp2v(wi / D, wj / D);   // expected Wishart gap
        // log|B_u|, B_u = B_i + B_j - P0 + c delta delta^T: Minkowski's bound plus the expected Wishart
        // gap, the prior scatter counted once (first order), the mean-shift term
        const double lbu = lbm + g0 - ht + log1p(c * h);
        const double ldu = lbu - D * log(vu);
        const double Lu = niw_lml_hat(n, D, k0, v0, ld0, ku, vu, ldu, g);
        const double P = T + Lu - ri[R_L] - rj[R_L];
        const double gdiag = s_lsum - D * logaddexp2v(s_li / D, s_lj / D);
        const double hdu = s_lsum - D * log(vu);
        const double ex[4] = {vu * ht / 2, vu * g0 / 2, 0.0, 0.0};
        screen_assemble(out, true, true, D, alpha, P, T, ni, nj, n, ri[R_L], rj[R_L], Lu, qi, qj, c * h,
                        vu * gdiag / 2, (ri[R_HD] - ri[R_LD]) / D, (rj[R_HD] - rj[R_LD]) / D, (hdu - ldu) / D,
                        (ri[R_LD] - rj[R_LD]) / D, s_md / D, v0 / vu, ri[R_TR] / D, rj[R_TR] / D, ex);
        prox[row] = P;
    } else {
        const double* ai_ = vi + D;
        const double* aj_ = vj + D;
        double Au = 0, sst = 0, chi = 0;
        for (int d = lane; d < D; d += 32) {
            const double a0 = alpha0[d];
            const double au = ai_[d] + aj_[d] - a0;
            Au += au;
            sst += stirling(au) - stirling(a0);
            const double ps = vi[d] + vj[d];
            if (ps > 0) chi += (vi[d] - vj[d]) * (vi[d] - vj[d]) / ps;
        }
        Au = warp_sum(Au);
        sst = warp_sum(sst);
        chi = warp_sum(chi);
        if (lane != 0) return;
        const double A0 = ri[R_VP];
        const double T = count_term_merge(ni, nj, alpha);
        const double Lstu = stirling(A0) - stirling(Au) + sst;
        const double P = T + Lstu - ri[R_LST] - rj[R_LST];
        const double c = ni * nj / n;
        const double ex[4] = {0.0, 0.0, 0.0, 0.0};
        screen_assemble(out, true, false, D, alpha, P, T, ni, nj, n, ri[R_LST], rj[R_LST], Lstu, ni * chi, nj * chi,
                        c * chi, 0.0, 0.0, 0.0, 0.0, 0.0, chi, A0 / Au, ri[R_TR], rj[R_TR], ex);
        prox[row] = P;
    }
}

template <bool GAUSS>
__global__ void __launch_bounds__(32 * kFeatWarps) k_screen_split_feat(const double* __restrict__ rec,
                                                                        const double* __restrict__ vec,
                                                                        const float* __restrict__ linv, int D, int K,
                                                                        double k0, double v0, double ld0, double alpha,
                                                                        float* __restrict__ feat, double* __restrict__ prox)
{
    __shared__ double sdelta[kFeatWarps][GAUSS ? kMaxGaussDim : 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int k = blockIdx.x * kFeatWarps + warp;
    if (k >= K) return;
    const double* rc = rec + (size_t)(3 * k) * kScrRec;
    const double* rl = rc + kScrRec;
    const double* rr = rl + kScrRec;
    float* out = feat + (size_t)k * kScrF;
    const double nl = rl[R_N], nr = rr[R_N], n = rc[R_N];
    if (nl == 0 || nr == 0 || n == 0) {
        out[lane] = 0.f;
        if (lane == 0) prox[k] = 0.0;
        return;
    }
    const double* vc = vec + (size_t)(3 * k) * 2 * D;
    const double* vl = vc + 2 * D;
    const double* vr = vl + 2 * D;
    const double T = log(alpha) + lgamma(nl) + lgamma(nr) - lgamma(nl + nr);
    if (GAUSS) {
        const double* dc = vc + D;
        const double* dl = vl + D;
        const double* dr = vr + D;
        double s_lsum = 0, s_ll = 0, s_lr = 0, s_md = 0, s_qd = 0;
        for (int d = lane; d < D; d += 32) {
            const double de = vl[d] - vr[d];
            sdelta[warp][d] = de;
            const double bl = rl[R_VP] * dl[d], br = rr[R_VP] * dr[d];
            s_lsum += log(bl + br);
            s_ll += log(bl);
            s_lr += log(br);
            s_md += de * de / (dl[d] + dr[d]);
            s_qd += de * de / dc[d];
        }
        __syncwarp();
        const float* Lc = linv + (size_t)k * D * D;
        double q = 0;
        for (int r = lane; r < D; r += 32) {
            double z = 0;
            for (int c = 0; c <= r; ++c) z += (double)Lc[(size_t)c * D + r] * sdelta[warp][c];
            q += z * z;
        }
        double gl = 0, gr = 0;
        for (int d = 1 + lane; d <= D; d += 32) {
            const double p0 = lgamma(v0 / 2.0 + (1 - d) / 2.0);
            gl += lgamma(rl[R_VP] / 2.0 + (1 - d) / 2.0) - p0;
            gr += lgamma(rr[R_VP] / 2.0 + (1 - d) / 2.0) - p0;
        }
        double wu = lw_part(nl + nr, D, lane), wl = lw_part(nl, D, lane), wr = lw_part(nr, D, lane);
        wu = warp_sum(wu);
        wl = warp_sum(wl);
        wr = warp_sum(wr);
        s_lsum = warp_sum(s_lsum);
        s_ll = warp_sum(s_ll);
        s_lr = warp_sum(s_lr);
        s_md = warp_sum(s_md);
        s_qd = warp_sum(s_qd);
        q = warp_sum(q);
        gl = warp_sum(gl);
        gr = warp_sum(gr);
        if (lane != 0) return;
        const double clr = rl[R_KP] * rr[R_KP] / (rl[R_KP] + rr[R_KP]);
        // children's log|B| from the parent's exact one: log|B_l + B_r - P0| = log|B_c| + log(1 - c y)
        // (Sherman-Morrison, y = delta^T B_c^-1 delta); the prior scatter (first order) and the expected
        // Wishart gap give D log(|B_l|^(1/D) + |B_r|^(1/D)); the children keep the ratio of their
        // diagonal (Hadamard) log-determinants
        const double om = fmax(1.0 - clr * q / rc[R_VP], 1e-12);
        const double g0 = wu - D * logaddexp2v(wl / D, wr / D);
        const double lbc = D * log(rc[R_VP]) + rc[R_LD];
        const double hbl = D * log(rl[R_VP]) + rl[R_HD], hbr = D * log(rr[R_VP]) + rr[R_HD];
        const double d0 = lbc + log(om) + rc[R_TAU] - g0 - D * logaddexp2v(hbl / D, hbr / D);
        const double ldl = hbl + d0 - D * log(rl[R_VP]), ldr = hbr + d0 - D * log(rr[R_VP]);
        const double Ll = niw_lml_hat(nl, D, k0, v0, ld0, rl[R_KP], rl[R_VP], ldl, gl);
        const double Lr = niw_lml_hat(nr, D, k0, v0, ld0, rr[R_KP], rr[R_VP], ldr, gr);
        const double P = T + Ll + Lr - rc[R_L];
        // second estimate: the parent's Hadamard gap stands in for the children's
        const double gapc = rc[R_HD] - rc[R_LD];
        const double Ll2 = niw_lml_hat(nl, D, k0, v0, ld0, rl[R_KP], rl[R_VP], rl[R_HD] - gapc, gl);
        const double Lr2 = niw_lml_hat(nr, D, k0, v0, ld0, rr[R_KP], rr[R_VP], rr[R_HD] - gapc, gr);
        const double P2 = T + Ll2 + Lr2 - rc[R_L];
        const double gdiag = s_lsum - D * logaddexp2v(s_ll / D, s_lr / D);
        const double ex[4] = {rc[R_VP] * rc[R_TAU] / 2, rc[R_VP] * g0 / 2, P2, -log(om) / 8};
        screen_assemble(out, false, true, D, alpha, P, T, nl, nr, n, Ll, Lr, rc[R_L], q, s_qd, clr * q / rc[R_VP],
                        rc[R_VP] * gdiag / 2, gapc / D, gapc / D, gapc / D, (ldl - ldr) / D, s_md / D, v0 / rc[R_VP],
                        rl[R_TR] / D, rr[R_TR] / D, ex);
        prox[k] = P;
    } else {
        double chi = 0;
        for (int d = lane; d < D; d += 32) {
            const double ps = vl[d] + vr[d];
            if (ps > 0) chi += (vl[d] - vr[d]) * (vl[d] - vr[d]) / ps;
        }
        chi = warp_sum(chi);
        if (lane != 0) return;
        const double P = T + rl[R_LST] + rr[R_LST] - rc[R_LST];
        const double cc = nl * nr / (nl + nr);
        const double ex[4] = {0.0, 0.0, 0.0, 0.0};
        screen_assemble(out, false, false, D, alpha, P, T, nl, nr, n, rl[R_LST], rr[R_LST], rc[R_LST], nl * chi,
                        nr * chi, cc * chi, 0.0, 0.0, 0.0, 0.0, 0.0, chi, rc[R_VP] / rc[R_KP], rl[R_TR], rr[R_TR], ex);
        prox[k] = P;
    }
}

// ------------------------------------------------------------------------------ MLP inference
// w: deployed parameters (weights already rounded to BF16, biases FP32), kScrParams floats
constexpr int kMlpThreads = 64;

__global__ void __launch_bounds__(kMlpThreads) k_screen_mlp(const float* __restrict__ feat, long long rows,
                                                            const float* __restrict__ w, float* __restrict__ score)
{
    __shared__ float sw[kScrParams];
    for (int e = threadIdx.x; e < kScrParams; e += blockDim.x) sw[e] = w[e];
    __syncthreads();
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    float x[kScrF];
    const float4* xr = reinterpret_cast<const float4*>(feat + (size_t)r * kScrF);
#pragma unroll
    for (int q = 0; q < kScrF / 4; ++q) {
        const float4 v = xr[q];
        x[4 * q] = v.x;
        x[4 * q + 1] = v.y;
        x[4 * q + 2] = v.z;
        x[4 * q + 3] = v.w;
    }
    const float* W1 = sw + kScrOffW1;
    const float* b1 = sw + kScrOffB1;
    const float* W2 = sw + kScrOffW2;
    const float* b2 = sw + kScrOffB2;
    const float* w3 = sw + kScrOffW3;
    float h1[kScrH];
#pragma unroll
    for (int h = 0; h < kScrH; ++h) {
        float acc = b1[h];
#pragma unroll
        for (int f = 0; f < kScrF; ++f) acc = fmaf(W1[h * kScrF + f], x[f], acc);
        h1[h] = fmaxf(acc, 0.f);
    }
    float z = sw[kScrOffB3];
#pragma unroll 4
    for (int h = 0; h < kScrH; ++h) {
        float acc = b2[h];
#pragma unroll
        for (int k = 0; k < kScrH; ++k) acc = fmaf(W2[h * kScrH + k], h1[k], acc);
        z = fmaf(w3[h], fmaxf(acc, 0.f), z);
    }
    score[r] = z;
}

// FP32 parameters -> deployed form (weights rounded to nearest-even BF16, biases kept)
__global__ void k_screen_deploy(const float* __restrict__ p, float* __restrict__ w)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= kScrParams) return;
    const bool weight = (e < kScrOffB1) || (e >= kScrOffW2 && e < kScrOffB2) || (e >= kScrOffW3 && e < kScrOffB3);
    w[e] = weight ? __bfloat162float(__float2bfloat16_rn(p[e])) : p[e];
}

// ------------------------------------------------------------------------------ selection
constexpr int kTopThreads = 1024;
constexpr int kTopCache = 8;       // candidates a thread keeps in registers (rows <= kTopThreads * kTopCache)

// rank order: higher score first, then lower candidate index; NaN scores rank as -inf
__device__ __forceinline__ bool ranks_before(float sa, long long ia, float sb, long long ib)
{
    return sa > sb || (sa == sb && ia < ib);
}

__device__ __forceinline__ bool row_eligible(long long r, int merge, int K, const uint8_t* __restrict__ elig)
{
    if (!merge) return elig[r] != 0;
    int i, j;
    unrank_pair(r, K, i, j);
    return elig[i] && elig[j];
}

// (score, index) of the best candidate ranked after (ps, pi), over a warp; index -1 when none
__device__ __forceinline__ void warp_best(float& bs, long long& bi)
{
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const float os = __shfl_xor_sync(0xffffffffu, bs, o);
        const long long oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (oi >= 0 && (bi < 0 || ranks_before(os, oi, bs, bi))) {
            bs = os;
            bi = oi;
        }
    }
}

// `top` rounds; round t picks the best eligible candidate ranked after round t-1's pick
__global__ void __launch_bounds__(kTopThreads) k_screen_topk(const float* __restrict__ score, long long rows, int merge,
                                                             int K, const uint8_t* __restrict__ elig, int top,
                                                             int32_t* __restrict__ sel, int32_t* __restrict__ nsel)
{
    __shared__ float ws[kTopThreads / 32];
    __shared__ long long wi[kTopThreads / 32];
    __shared__ int32_t picked[kScrMaxTop];
    __shared__ float prev_s;
    __shared__ long long prev_i;
    __shared__ int npicked;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool cached = rows <= (long long)kTopThreads * kTopCache;
    float cs[kTopCache];
    long long ci[kTopCache];
#pragma unroll
    for (int q = 0; q < kTopCache; ++q) {
        const long long r = threadIdx.x + (long long)q * kTopThreads;
        ci[q] = -1;
        cs[q] = -INFINITY;
        if (cached && r < rows && row_eligible(r, merge, K, elig)) {
            const float v = score[r];
            cs[q] = v != v ? -INFINITY : v;
            ci[q] = r;
        }
    }
    if (threadIdx.x == 0) {
        prev_s = INFINITY;
        prev_i = -1;
        npicked = 0;
    }
    __syncthreads();
    for (int t = 0; t < top; ++t) {
        const float ps = prev_s;
        const long long pi = prev_i;
        float bs = -INFINITY;
        long long bi = -1;
        if (cached) {
#pragma unroll
            for (int q = 0; q < kTopCache; ++q)
                if (ci[q] >= 0 && ranks_before(ps, pi, cs[q], ci[q]) && (bi < 0 || ranks_before(cs[q], ci[q], bs, bi))) {
                    bs = cs[q];
                    bi = ci[q];
                }
        } else {
            for (long long r = threadIdx.x; r < rows; r += blockDim.x) {
                if (!row_eligible(r, merge, K, elig)) continue;
                float v = score[r];
                if (v != v) v = -INFINITY;
                if (!ranks_before(ps, pi, v, r)) continue;        // already picked
                if (bi < 0 || ranks_before(v, r, bs, bi)) {
                    bs = v;
                    bi = r;
                }
            }
        }
        warp_best(bs, bi);
        if (lane == 0) {
            ws[warp] = bs;
            wi[warp] = bi;
        }
        __syncthreads();
        if (warp == 0) {
            bs = lane < (int)(blockDim.x >> 5) ? ws[lane] : -INFINITY;
            bi = lane < (int)(blockDim.x >> 5) ? wi[lane] : -1;
            warp_best(bs, bi);
            if (lane == 0) {
                if (bi >= 0) {
                    picked[npicked++] = (int32_t)bi;
                    prev_s = bs;
                    prev_i = bi;
                } else {
                    prev_i = -2;   // nothing left
                }
            }
        }
        __syncthreads();
        if (prev_i == -2) break;
    }
    if (threadIdx.x == 0) {
        const int m = npicked;
        for (int a = 1; a < m; ++a) {   // ascending candidate order
            const int32_t v = picked[a];
            int b = a - 1;
            while (b >= 0 && picked[b] > v) {
                picked[b + 1] = picked[b];
                --b;
            }
            picked[b + 1] = v;
        }
        for (int a = 0; a < m; ++a) sel[a] = picked[a];
        *nsel = m;
    }
}

// ------------------------------------------------------------------------------ exact ratios of a list
// log marginal likelihood of the listed slots (the arithmetic of k_slot_lml), one block per slot
// (sel, nullable: clusters whose slots use the second prior k1, v1, ld1, prior1 -- the outlier layout)
template <int DP>
__global__ void __launch_bounds__(RegChol<DP>::T) k_slot_lml_list(const double* __restrict__ stats, int stat_len, int D,
                                                                   int gauss, double k0, double v0, double ld0,
                                                                   const double* __restrict__ prior, double k1,
                                                                   double v1, double ld1,
                                                                   const double* __restrict__ prior1,
                                                                   const uint8_t* __restrict__ sel,
                                                                   const int32_t* __restrict__ slots,
                                                                   double* __restrict__ lml)
{
    __shared__ double sh[RegChol<DP>::SMEM];
    const int s = slots[blockIdx.x];
    if (sel && sel[s / 3]) {
        k0 = k1;
        v0 = v1;
        ld0 = ld1;
        prior = prior1;
    }
    const double* st = stats + (size_t)s * stat_len;
    double v;
    if (gauss)
        v = niw_lml_reg<DP>(D, st[0], st + 1, st + 1 + D, nullptr, nullptr, k0, v0, prior, prior + D, ld0, sh);
    else
        v = mult_lml_block(D, st[0], st + 1, nullptr, prior, sh + 3 * DP);
    if (threadIdx.x == 0) lml[s] = v;
}

// exact merge ratios of the listed pairs (the arithmetic of k_merge_hr), one block per pair; the merged
// cluster takes cluster i's prior (shared_actions.cpp:88-95)
template <int DP>
__global__ void __launch_bounds__(RegChol<DP>::T) k_merge_hr_list(const double* __restrict__ stats, int stat_len, int D,
                                                                   int gauss, double k0, double v0, double ld0,
                                                                   const double* __restrict__ prior, double k1,
                                                                   double v1, double ld1,
                                                                   const double* __restrict__ prior1,
                                                                   const uint8_t* __restrict__ sel,
                                                                   const double* __restrict__ lml,
                                                                   const int32_t* __restrict__ pairs, double alpha,
                                                                   double* __restrict__ out)
{
    __shared__ double sh[RegChol<DP>::SMEM];
    const int i = pairs[2 * blockIdx.x], j = pairs[2 * blockIdx.x + 1];
    if (sel && sel[i]) {
        k0 = k1;
        v0 = v1;
        ld0 = ld1;
        prior = prior1;
    }
    const double v = merge_log_hr_reg<DP>(stats, stat_len, D, gauss, k0, v0, ld0, prior, lml, i, j, alpha, sh);
    if (threadIdx.x == 0) out[blockIdx.x] = v;
}

__global__ void k_split_hr_list(const double* __restrict__ stats, int stat_len, const double* __restrict__ lml,
                                const int32_t* __restrict__ idx, int n, double alpha, double* __restrict__ out)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) out[t] = split_log_hr_slot(stats, stat_len, lml, idx[t], alpha);
}

// ------------------------------------------------------------------------------ training
constexpr int kTile = 64;          // rows per training block
constexpr int kTrainThreads = 256;
constexpr int kXS = kScrF + 1;     // padded row strides in shared memory
constexpr int kHS = kScrH + 1;
constexpr size_t kTrainSmemFloats = (size_t)kScrH * kXS /*W1*/ + kScrH /*b1*/ + (size_t)kScrH * kHS /*W2*/ +
                                    kScrH /*b2*/ + kScrH /*w3*/ + 1 /*b3*/ + (size_t)kTile * kXS /*X*/ +
                                    4 * (size_t)kTile * kHS /*H1 H2 dH2 dH1*/ + 2 * kTile /*dz, t*/;

// One 64-row tile of a minibatch: forward, mean-squared-error backward, partial gradient of the tile.
// rows of the batch: idx[b0 + r] (or b0 + r when idx is null), r < min(64, batch - b0).
// part[blockIdx.x][kScrParams] = gradient sum over the tile, part[...][kScrParams] = loss sum.
// Every sum runs over the tile's rows in order: the result does not depend on scheduling.
__global__ void __launch_bounds__(kTrainThreads) k_mlp_grad_tile(const float* __restrict__ X, const float* __restrict__ tgt,
                                                                 const int64_t* __restrict__ idx, int64_t batch0,
                                                                 int batch, const float* __restrict__ p,
                                                                 float* __restrict__ part)
{
    extern __shared__ float sm[];
    float* W1 = sm;
    float* b1 = W1 + kScrH * kXS;
    float* W2 = b1 + kScrH;
    float* b2 = W2 + kScrH * kHS;
    float* w3 = b2 + kScrH;
    float* b3 = w3 + kScrH;
    float* Xs = b3 + 1;
    float* H1 = Xs + kTile * kXS;
    float* H2 = H1 + kTile * kHS;
    float* dH2 = H2 + kTile * kHS;
    float* dH1 = dH2 + kTile * kHS;
    float* dz = dH1 + kTile * kHS;
    float* ts = dz + kTile;
    const int tid = threadIdx.x;
    const int r0 = blockIdx.x * kTile;
    const int nr = min(kTile, batch - r0);
    const float invB = 1.0f / (float)batch;
    for (int e = tid; e < kScrH * kScrF; e += blockDim.x) W1[(e / kScrF) * kXS + e % kScrF] = p[kScrOffW1 + e];
    for (int e = tid; e < kScrH * kScrH; e += blockDim.x) W2[(e / kScrH) * kHS + e % kScrH] = p[kScrOffW2 + e];
    for (int e = tid; e < kScrH; e += blockDim.x) {
        b1[e] = p[kScrOffB1 + e];
        b2[e] = p[kScrOffB2 + e];
        w3[e] = p[kScrOffW3 + e];
    }
    if (tid == 0) b3[0] = p[kScrOffB3];
    for (int e = tid; e < kTile * kScrF; e += blockDim.x) {
        const int r = e / kScrF, f = e % kScrF;
        float v = 0.f;
        if (r < nr) {
            const int64_t row = idx ? idx[batch0 + r0 + r] : batch0 + r0 + r;
            v = X[(size_t)row * kScrF + f];
        }
        Xs[r * kXS + f] = v;
    }
    for (int r = tid; r < kTile; r += blockDim.x) {
        float v = 0.f;
        if (r < nr) {
            const int64_t row = idx ? idx[batch0 + r0 + r] : batch0 + r0 + r;
            v = tgt[row];
        }
        ts[r] = v;
    }
    __syncthreads();
    // forward
    for (int e = tid; e < kTile * kScrH; e += blockDim.x) {
        const int r = e / kScrH, h = e % kScrH;
        float acc = b1[h];
        for (int f = 0; f < kScrF; ++f) acc = fmaf(W1[h * kXS + f], Xs[r * kXS + f], acc);
        H1[r * kHS + h] = fmaxf(acc, 0.f);
    }
    __syncthreads();
    for (int e = tid; e < kTile * kScrH; e += blockDim.x) {
        const int r = e / kScrH, h = e % kScrH;
        float acc = b2[h];
        for (int k = 0; k < kScrH; ++k) acc = fmaf(W2[h * kHS + k], H1[r * kHS + k], acc);
        H2[r * kHS + h] = fmaxf(acc, 0.f);
    }
    __syncthreads();
    if (tid < kTile) {
        const int r = tid;
        float z = b3[0];
        for (int h = 0; h < kScrH; ++h) z = fmaf(w3[h], H2[r * kHS + h], z);
        const float e = z - ts[r];
        dz[r] = r < nr ? 2.f * e * invB : 0.f;
        ts[r] = r < nr ? e * e * invB : 0.f;    // per-row loss term
    }
    __syncthreads();
    // backward
    for (int e = tid; e < kTile * kScrH; e += blockDim.x) {
        const int r = e / kScrH, h = e % kScrH;
        dH2[r * kHS + h] = H2[r * kHS + h] > 0.f ? dz[r] * w3[h] : 0.f;
    }
    __syncthreads();
    for (int e = tid; e < kTile * kScrH; e += blockDim.x) {
        const int r = e / kScrH, k = e % kScrH;
        float acc = 0.f;
        for (int h = 0; h < kScrH; ++h) acc = fmaf(dH2[r * kHS + h], W2[h * kHS + k], acc);
        dH1[r * kHS + k] = H1[r * kHS + k] > 0.f ? acc : 0.f;
    }
    __syncthreads();
    float* out = part + (size_t)blockIdx.x * (kScrParams + 1);
    for (int e = tid; e < kScrH * kScrH; e += blockDim.x) {       // dW2[h][k] = sum_r dH2[r][h] H1[r][k]
        const int h = e / kScrH, k = e % kScrH;
        float acc = 0.f;
        for (int r = 0; r < kTile; ++r) acc = fmaf(dH2[r * kHS + h], H1[r * kHS + k], acc);
        out[kScrOffW2 + e] = acc;
    }
    for (int e = tid; e < kScrH * kScrF; e += blockDim.x) {       // dW1[h][f] = sum_r dH1[r][h] X[r][f]
        const int h = e / kScrF, f = e % kScrF;
        float acc = 0.f;
        for (int r = 0; r < kTile; ++r) acc = fmaf(dH1[r * kHS + h], Xs[r * kXS + f], acc);
        out[kScrOffW1 + e] = acc;
    }
    for (int h = tid; h < kScrH; h += blockDim.x) {
        float g1 = 0.f, g2 = 0.f, g3 = 0.f;
        for (int r = 0; r < kTile; ++r) {
            g1 += dH1[r * kHS + h];
            g2 += dH2[r * kHS + h];
            g3 = fmaf(dz[r], H2[r * kHS + h], g3);
        }
        out[kScrOffB1 + h] = g1;
        out[kScrOffB2 + h] = g2;
        out[kScrOffW3 + h] = g3;
    }
    if (tid == 0) {
        float gb = 0.f, ls = 0.f;
        for (int r = 0; r < kTile; ++r) {
            gb += dz[r];
            ls += ts[r];
        }
        out[kScrOffB3] = gb;
        out[kScrParams] = ls;
    }
}

// Sum of the tiles' partial gradients (fixed order), optional copy out, optional Adam step
// (Kingma & Ba 2015, bias-corrected).  loss_out[0] = loss of the batch.
__global__ void k_mlp_adam(const float* __restrict__ part, int ntiles, float* __restrict__ p, float* __restrict__ m,
                           float* __restrict__ v, int step, float lr, float beta1, float beta2, float eps,
                           float* __restrict__ grad_out, float* __restrict__ loss_out)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e > kScrParams) return;
    float g = 0.f;
    for (int b = 0; b < ntiles; ++b) g += part[(size_t)b * (kScrParams + 1) + e];
    if (e == kScrParams) {
        if (loss_out) loss_out[0] = g;
        return;
    }
    if (grad_out) grad_out[e] = g;
    if (lr > 0.f) {
        const float mm = beta1 * m[e] + (1.f - beta1) * g;
        const float vv = beta2 * v[e] + (1.f - beta2) * g * g;
        m[e] = mm;
        v[e] = vv;
        const float mh = mm / (1.f - powf(beta1, (float)step));
        const float vh = vv / (1.f - powf(beta2, (float)step));
        p[e] -= lr * mh / (sqrtf(vh) + eps);
    }
}

// ------------------------------------------------------------------------------ launchers (context)
template <int DP>
static dpmm_status launch_slots_niw(dpmm_ctx* c, int K)
{
    const size_t sm = sizeof(double) * (size_t)c->D * c->D;
    DPMM_TRY(allow_smem(k_screen_slots_niw<DP>, sm));
    k_screen_slots_niw<DP><<<3 * K, RegChol<DP>::T, sm, c->stream>>>(
        c->d_stats, c->stat_len, c->D, c->prior_k, c->prior_v, c->prior_logdet, c->d_prior, c->prior_identity ? 1 : 0,
        c->d_scr_rec, c->d_scr_vec, c->d_scr_linv);
    return DPMM_OK;
}

dpmm_status launch_screen_features(dpmm_ctx* c, int K, int kind, double alpha)
{
    if (!c->prior_set) return fail(DPMM_ERR_STATE, "prior hyper-parameters not set");
    DPMM_TRY(ensure_stats(c, K));
    const bool gauss = c->prior == DPMM_PRIOR_GAUSSIAN;
    const int D = c->D;
    if (gauss) {
        dpmm_status st = DPMM_OK;
        DPMM_WITH_DP(c->Dp, (st = launch_slots_niw<DP>(c, K)));
        DPMM_TRY(st);
    } else {
        k_screen_slots_dir<<<3 * K, kHThreads, 0, c->stream>>>(c->d_stats, c->stat_len, D, c->d_prior, c->d_scr_rec,
                                                               c->d_scr_vec);
    }
    DPMM_LAUNCHED();
    if (kind == DPMM_SCREEN_MERGE) {
        const long long pairs = (long long)K * (K - 1) / 2;
        if (pairs == 0) return DPMM_OK;
        const unsigned grid = (unsigned)((pairs + kFeatWarps - 1) / kFeatWarps);
        if (gauss)
            k_screen_merge_feat<true><<<grid, 32 * kFeatWarps, 0, c->stream>>>(
                c->d_scr_rec, c->d_scr_vec, c->d_scr_linv, D, K, pairs, c->prior_k, c->prior_v, c->prior_logdet, alpha,
                c->d_prior, c->d_scr_feat, c->d_scr_prox);
        else
            k_screen_merge_feat<false><<<grid, 32 * kFeatWarps, 0, c->stream>>>(
                c->d_scr_rec, c->d_scr_vec, c->d_scr_linv, D, K, pairs, 0.0, 0.0, 0.0, alpha, c->d_prior, c->d_scr_feat,
                c->d_scr_prox);
    } else {
        const unsigned grid = (unsigned)((K + kFeatWarps - 1) / kFeatWarps);
        if (gauss)
            k_screen_split_feat<true><<<grid, 32 * kFeatWarps, 0, c->stream>>>(
                c->d_scr_rec, c->d_scr_vec, c->d_scr_linv, D, K, c->prior_k, c->prior_v, c->prior_logdet, alpha,
                c->d_scr_feat, c->d_scr_prox);
        else
            k_screen_split_feat<false><<<grid, 32 * kFeatWarps, 0, c->stream>>>(
                c->d_scr_rec, c->d_scr_vec, c->d_scr_linv, D, K, 0.0, 0.0, 0.0, alpha, c->d_scr_feat, c->d_scr_prox);
    }
    DPMM_LAUNCHED();
    return DPMM_OK;
}

static long long screen_rows(int K, int kind) { return kind == DPMM_SCREEN_MERGE ? (long long)K * (K - 1) / 2 : K; }

dpmm_status launch_screen_select(dpmm_ctx* c, int K, int kind, double alpha, int top)
{
    if (!c->scr_params_set) return fail(DPMM_ERR_STATE, "screen parameters not set (dpmm_screen_set_params)");
    DPMM_TRY(launch_screen_features(c, K, kind, alpha));
    const long long rows = screen_rows(K, kind);
    if (rows > 0) {
        k_screen_mlp<<<(unsigned)((rows + kMlpThreads - 1) / kMlpThreads), kMlpThreads, 0, c->stream>>>(
            c->d_scr_feat, rows, c->d_scr_wdep, c->d_scr_score);
        DPMM_LAUNCHED();
    }
    k_screen_topk<<<1, kTopThreads, 0, c->stream>>>(c->d_scr_score, rows, kind == DPMM_SCREEN_MERGE, K, c->d_scr_elig,
                                                    top, c->d_scr_sel, c->d_scr_sel + kScrMaxTop);
    DPMM_LAUNCHED();
    return DPMM_OK;
}

dpmm_status launch_hastings_list(dpmm_ctx* c, int K, int kind, double alpha, int n, int nslots)
{
    if (!c->prior_set) return fail(DPMM_ERR_STATE, "prior hyper-parameters not set");
    DPMM_TRY(ensure_stats(c, K));
    const int gauss = c->prior == DPMM_PRIOR_GAUSSIAN;
    if (n == 0) return DPMM_OK;
    const int dp = gauss ? c->Dp : 4;
    const bool out2 = c->outlier_layout != 0;
    const double* p2 = out2 ? c->d_prior2 : c->d_prior;
    const uint8_t* sel = out2 ? c->d_prior_sel : nullptr;
    DPMM_WITH_DP(dp, (k_slot_lml_list<DP><<<nslots, RegChol<DP>::T, 0, c->stream>>>(
                         c->d_stats, c->stat_len, c->D, gauss, c->prior_k, c->prior_v, c->prior_logdet, c->d_prior,
                         c->prior2_k, c->prior2_v, c->prior2_logdet, p2, sel, c->d_scr_slots, c->d_lml)));
    DPMM_LAUNCHED();
    if (kind == DPMM_SCREEN_MERGE) {
        DPMM_WITH_DP(dp, (k_merge_hr_list<DP><<<n, RegChol<DP>::T, 0, c->stream>>>(
                             c->d_stats, c->stat_len, c->D, gauss, c->prior_k, c->prior_v, c->prior_logdet, c->d_prior,
                             c->prior2_k, c->prior2_v, c->prior2_logdet, p2, sel, c->d_lml, c->d_scr_list, alpha,
                             c->d_scr_hr)));
    } else {
        k_split_hr_list<<<(n + 127) / 128, 128, 0, c->stream>>>(c->d_stats, c->stat_len, c->d_lml, c->d_scr_list, n,
                                                                alpha, c->d_scr_hr);
    }
    DPMM_LAUNCHED();
    return DPMM_OK;
}

}  // namespace dpmm

using namespace dpmm;

// ============================================================================== C ABI (context)
extern "C" dpmm_status dpmm_screen_set_params(dpmm_ctx* c, const float* params)
{
    if (!c || !params) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    for (int e = 0; e < kScrParams; ++e)
        if (!std::isfinite(params[e])) return fail(DPMM_ERR_NUMERIC, "screen parameters hold NaN or Inf");
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_scr_w, params, sizeof(float) * kScrParams, cudaMemcpyHostToDevice, c->stream));
    k_screen_deploy<<<(kScrParams + 255) / 256, 256, 0, c->stream>>>(c->d_scr_w, c->d_scr_wdep);
    DPMM_LAUNCHED();
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    g_h2d_bytes.fetch_add(sizeof(float) * kScrParams, std::memory_order_relaxed);
    c->scr_params_set = true;
    return DPMM_OK;
}

static dpmm_status check_kind(const dpmm_ctx* c, int K, int kind)
{
    if (!c || K < 1 || K > c->k_max) return fail(DPMM_ERR_INVALID_ARG, "invalid context or K");
    if (kind != DPMM_SCREEN_SPLIT && kind != DPMM_SCREEN_MERGE) return fail(DPMM_ERR_INVALID_ARG, "unknown screen kind");
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_screen_features(dpmm_ctx* c, int K, int kind, double alpha, float* features, double* proxy)
{
    DPMM_TRY(check_kind(c, K, kind));
    if (!(alpha > 0)) return fail(DPMM_ERR_INVALID_ARG, "alpha must be positive");
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    {
        PhaseTimer pt(c, kind == DPMM_SCREEN_MERGE ? PH_MERGE_HR : PH_SPLIT_HR);
        DPMM_TRY(launch_screen_features(c, K, kind, alpha));
    }
    const long long rows = screen_rows(K, kind);
    if (features && rows > 0) {
        DPMM_CUDA_TRY(cudaMemcpyAsync(features, c->d_scr_feat, sizeof(float) * kScrF * (size_t)rows,
                                      cudaMemcpyDeviceToHost, c->stream));
        g_d2h_bytes.fetch_add(sizeof(float) * kScrF * (size_t)rows, std::memory_order_relaxed);
    }
    if (proxy && rows > 0) {
        DPMM_CUDA_TRY(cudaMemcpyAsync(proxy, c->d_scr_prox, sizeof(double) * (size_t)rows, cudaMemcpyDeviceToHost,
                                      c->stream));
        g_d2h_bytes.fetch_add(sizeof(double) * (size_t)rows, std::memory_order_relaxed);
    }
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_screen_select(dpmm_ctx* c, int K, int kind, double alpha, const uint8_t* eligible, int top,
                                          int32_t* selected, int32_t* n_selected, float* scores)
{
    DPMM_TRY(check_kind(c, K, kind));
    if (!eligible || !selected || !n_selected) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    if (top < 1 || top > kScrMaxTop)
        return fail(DPMM_ERR_INVALID_ARG, "top must be in [1, " + std::to_string(kScrMaxTop) + "]");
    if (!(alpha > 0)) return fail(DPMM_ERR_INVALID_ARG, "alpha must be positive");
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    {
        PhaseTimer pt(c, kind == DPMM_SCREEN_MERGE ? PH_MERGE_HR : PH_SPLIT_HR);
        DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_scr_elig, eligible, (size_t)K, cudaMemcpyHostToDevice, c->stream));
        g_h2d_bytes.fetch_add((uint64_t)K, std::memory_order_relaxed);
        DPMM_TRY(launch_screen_select(c, K, kind, alpha, top));
    }
    int32_t* h = reinterpret_cast<int32_t*>(c->h_pinned);
    DPMM_CUDA_TRY(cudaMemcpyAsync(h, c->d_scr_sel, sizeof(int32_t) * (kScrMaxTop + 1), cudaMemcpyDeviceToHost, c->stream));
    g_d2h_bytes.fetch_add(sizeof(int32_t) * (kScrMaxTop + 1), std::memory_order_relaxed);
    const long long rows = screen_rows(K, kind);
    if (scores && rows > 0) {
        DPMM_CUDA_TRY(cudaMemcpyAsync(scores, c->d_scr_score, sizeof(float) * (size_t)rows, cudaMemcpyDeviceToHost,
                                      c->stream));
        g_d2h_bytes.fetch_add(sizeof(float) * (size_t)rows, std::memory_order_relaxed);
    }
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    const int m = h[kScrMaxTop];
    if (m < 0 || m > top) return fail(DPMM_ERR_CUDA, "screen selection returned an invalid count");
    std::memcpy(selected, h, sizeof(int32_t) * m);
    *n_selected = m;
    return DPMM_OK;
}

static dpmm_status hastings_list(dpmm_ctx* c, int K, int kind, double alpha, int n, const int32_t* items, double* out)
{
    DPMM_TRY(check_kind(c, K, kind));
    if (n < 0 || n > kScrMaxTop) return fail(DPMM_ERR_INVALID_ARG, "list length must be in [0, 256]");
    if (n > 0 && (!items || !out)) return fail(DPMM_ERR_INVALID_ARG, "null argument");
    if (!(alpha > 0)) return fail(DPMM_ERR_INVALID_ARG, "alpha must be positive");
    // slots whose log marginal likelihood the ratios read (each once)
    std::vector<int32_t> list, slots;
    std::vector<uint8_t> seen(3 * (size_t)K, 0);
    auto add_slot = [&](int s) {
        if (!seen[s]) {
            seen[s] = 1;
            slots.push_back(s);
        }
    };
    for (int t = 0; t < n; ++t) {
        if (kind == DPMM_SCREEN_MERGE) {
            const int i = items[2 * t], j = items[2 * t + 1];
            if (i < 0 || j < 0 || i >= K || j >= K || i == j) return fail(DPMM_ERR_INVALID_ARG, "pair index out of range");
            list.push_back(i);
            list.push_back(j);
            add_slot(3 * i);
            add_slot(3 * j);
        } else {
            const int k = items[t];
            if (k < 0 || k >= K) return fail(DPMM_ERR_INVALID_ARG, "cluster index out of range");
            list.push_back(k);
            for (int s = 0; s < 3; ++s) add_slot(3 * k + s);
        }
    }
    DPMM_CUDA_TRY(cudaSetDevice(c->device));
    {
        PhaseTimer pt(c, kind == DPMM_SCREEN_MERGE ? PH_MERGE_HR : PH_SPLIT_HR);
        if (n > 0) {
            DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_scr_list, list.data(), sizeof(int32_t) * list.size(),
                                          cudaMemcpyHostToDevice, c->stream));
            DPMM_CUDA_TRY(cudaMemcpyAsync(c->d_scr_slots, slots.data(), sizeof(int32_t) * slots.size(),
                                          cudaMemcpyHostToDevice, c->stream));
            g_h2d_bytes.fetch_add(sizeof(int32_t) * (list.size() + slots.size()), std::memory_order_relaxed);
        }
        DPMM_TRY(launch_hastings_list(c, K, kind, alpha, n, (int)slots.size()));
    }
    if (n > 0) {
        DPMM_CUDA_TRY(cudaMemcpyAsync(out, c->d_scr_hr, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
        g_d2h_bytes.fetch_add(sizeof(double) * n, std::memory_order_relaxed);
    }
    DPMM_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_split_hastings_list(dpmm_ctx* c, int K, double alpha, int n, const int32_t* clusters,
                                                double* split_log_hr)
{
    return hastings_list(c, K, DPMM_SCREEN_SPLIT, alpha, n, clusters, split_log_hr);
}

extern "C" dpmm_status dpmm_merge_hastings_list(dpmm_ctx* c, int K, double alpha, int n, const int32_t* pairs,
                                                double* merge_log_hr)
{
    return hastings_list(c, K, DPMM_SCREEN_MERGE, alpha, n, pairs, merge_log_hr);
}

// ============================================================================== C ABI (standalone MLP)
namespace {

// device buffers of one standalone call, freed on every exit path
struct DevBufs {
    std::vector<void*> ptrs;
    cudaStream_t stream = nullptr;
    ~DevBufs()
    {
        if (stream) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    dpmm_status alloc(T** p, size_t count)
    {
        *p = nullptr;
        cudaError_t e = cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(count, 1));
        if (e != cudaSuccess) {
            *p = nullptr;
            return cuda_status(e, "cudaMalloc");
        }
        ptrs.push_back(*p);
        return DPMM_OK;
    }
};

dpmm_status begin(int device, DevBufs& b)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(DPMM_ERR_NO_DEVICE, "no CUDA device available");
    if (device < 0 || device >= ndev) return fail(DPMM_ERR_INVALID_ARG, "device ordinal out of range");
    DPMM_CUDA_TRY(cudaSetDevice(device));
    DPMM_CUDA_TRY(cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking));
    return DPMM_OK;
}

size_t train_smem() { return sizeof(float) * kTrainSmemFloats; }

dpmm_status enable_train_smem()
{
    DPMM_CUDA_TRY(cudaFuncSetAttribute(k_mlp_grad_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem()));
    return DPMM_OK;
}

}  // namespace

extern "C" dpmm_status dpmm_screen_forward(const float* features, int64_t rows, const float* params, float* scores,
                                           int32_t device)
{
    if (!features || !params || !scores || rows < 0) return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    if (rows == 0) return DPMM_OK;
    DevBufs b;
    DPMM_TRY(begin(device, b));
    float *dX, *dp, *dw, *ds;
    DPMM_TRY(b.alloc(&dX, (size_t)rows * kScrF));
    DPMM_TRY(b.alloc(&dp, kScrParams));
    DPMM_TRY(b.alloc(&dw, kScrParams));
    DPMM_TRY(b.alloc(&ds, (size_t)rows));
    DPMM_CUDA_TRY(cudaMemcpyAsync(dX, features, sizeof(float) * kScrF * (size_t)rows, cudaMemcpyHostToDevice, b.stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(dp, params, sizeof(float) * kScrParams, cudaMemcpyHostToDevice, b.stream));
    k_screen_deploy<<<(kScrParams + 255) / 256, 256, 0, b.stream>>>(dp, dw);
    DPMM_LAUNCHED();
    k_screen_mlp<<<(unsigned)((rows + kMlpThreads - 1) / kMlpThreads), kMlpThreads, 0, b.stream>>>(dX, rows, dw, ds);
    DPMM_LAUNCHED();
    DPMM_CUDA_TRY(cudaMemcpyAsync(scores, ds, sizeof(float) * (size_t)rows, cudaMemcpyDeviceToHost, b.stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(b.stream));
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_screen_loss_grad(const float* features, const float* targets, int32_t rows,
                                             const float* params, float* loss, float* grad, int32_t device)
{
    if (!features || !targets || !params || !loss || !grad || rows < 1) return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    DevBufs b;
    DPMM_TRY(begin(device, b));
    DPMM_TRY(enable_train_smem());
    const int ntiles = (rows + kTile - 1) / kTile;
    float *dX, *dt, *dp, *dpart, *dg, *dl;
    DPMM_TRY(b.alloc(&dX, (size_t)rows * kScrF));
    DPMM_TRY(b.alloc(&dt, (size_t)rows));
    DPMM_TRY(b.alloc(&dp, kScrParams));
    DPMM_TRY(b.alloc(&dpart, (size_t)ntiles * (kScrParams + 1)));
    DPMM_TRY(b.alloc(&dg, kScrParams));
    DPMM_TRY(b.alloc(&dl, 1));
    DPMM_CUDA_TRY(cudaMemcpyAsync(dX, features, sizeof(float) * kScrF * (size_t)rows, cudaMemcpyHostToDevice, b.stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(dt, targets, sizeof(float) * (size_t)rows, cudaMemcpyHostToDevice, b.stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(dp, params, sizeof(float) * kScrParams, cudaMemcpyHostToDevice, b.stream));
    k_mlp_grad_tile<<<ntiles, kTrainThreads, train_smem(), b.stream>>>(dX, dt, nullptr, 0, rows, dp, dpart);
    DPMM_LAUNCHED();
    k_mlp_adam<<<(kScrParams + 1 + 255) / 256, 256, 0, b.stream>>>(dpart, ntiles, dp, nullptr, nullptr, 0, 0.f, 0.f, 0.f,
                                                                   0.f, dg, dl);
    DPMM_LAUNCHED();
    DPMM_CUDA_TRY(cudaMemcpyAsync(grad, dg, sizeof(float) * kScrParams, cudaMemcpyDeviceToHost, b.stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(loss, dl, sizeof(float), cudaMemcpyDeviceToHost, b.stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(b.stream));
    return DPMM_OK;
}

extern "C" dpmm_status dpmm_screen_train(const float* features, const float* targets, int64_t rows, int32_t epochs,
                                         int32_t batch, float lr, uint64_t seed, float* params, float* epoch_loss,
                                         int32_t device)
{
    if (!features || !targets || !params || rows < 1 || epochs < 1 || batch < 1 || !(lr > 0))
        return fail(DPMM_ERR_INVALID_ARG, "invalid argument");
    if (batch > rows) batch = (int32_t)rows;
    DevBufs b;
    DPMM_TRY(begin(device, b));
    DPMM_TRY(enable_train_smem());
    const int ntiles = (batch + kTile - 1) / kTile;
    const int64_t steps_per_epoch = rows / batch;    // the last partial batch of an epoch is dropped
    float *dX, *dt, *dp, *dm, *dv, *dpart, *dl;
    int64_t* didx;
    DPMM_TRY(b.alloc(&dX, (size_t)rows * kScrF));
    DPMM_TRY(b.alloc(&dt, (size_t)rows));
    DPMM_TRY(b.alloc(&dp, kScrParams));
    DPMM_TRY(b.alloc(&dm, kScrParams));
    DPMM_TRY(b.alloc(&dv, kScrParams));
    DPMM_TRY(b.alloc(&dpart, (size_t)ntiles * (kScrParams + 1)));
    DPMM_TRY(b.alloc(&dl, (size_t)steps_per_epoch));
    DPMM_TRY(b.alloc(&didx, (size_t)rows));
    DPMM_CUDA_TRY(cudaMemcpyAsync(dX, features, sizeof(float) * kScrF * (size_t)rows, cudaMemcpyHostToDevice, b.stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(dt, targets, sizeof(float) * (size_t)rows, cudaMemcpyHostToDevice, b.stream));
    DPMM_CUDA_TRY(cudaMemcpyAsync(dp, params, sizeof(float) * kScrParams, cudaMemcpyHostToDevice, b.stream));
    DPMM_CUDA_TRY(cudaMemsetAsync(dm, 0, sizeof(float) * kScrParams, b.stream));
    DPMM_CUDA_TRY(cudaMemsetAsync(dv, 0, sizeof(float) * kScrParams, b.stream));
    std::vector<int64_t> perm(rows);
    std::vector<float> losses((size_t)steps_per_epoch);
    std::mt19937_64 gen(seed);
    int step = 0;
    for (int ep = 0; ep < epochs; ++ep) {
        // Fisher-Yates shuffle of the row order, one per epoch
        for (int64_t q = 0; q < rows; ++q) perm[q] = q;
        for (int64_t q = rows - 1; q > 0; --q) {
            const int64_t r = (int64_t)(gen() % (uint64_t)(q + 1));
            std::swap(perm[q], perm[r]);
        }
        DPMM_CUDA_TRY(cudaMemcpyAsync(didx, perm.data(), sizeof(int64_t) * rows, cudaMemcpyHostToDevice, b.stream));
        for (int64_t s = 0; s < steps_per_epoch; ++s) {
            ++step;
            k_mlp_grad_tile<<<ntiles, kTrainThreads, train_smem(), b.stream>>>(dX, dt, didx, s * batch, batch, dp, dpart);
            DPMM_LAUNCHED();
            k_mlp_adam<<<(kScrParams + 1 + 255) / 256, 256, 0, b.stream>>>(dpart, ntiles, dp, dm, dv, step, lr, 0.9f,
                                                                           0.999f, 1e-8f, nullptr, dl + s);
            DPMM_LAUNCHED();
        }
        DPMM_CUDA_TRY(cudaMemcpyAsync(losses.data(), dl, sizeof(float) * steps_per_epoch, cudaMemcpyDeviceToHost,
                                      b.stream));
        DPMM_CUDA_TRY(cudaStreamSynchronize(b.stream));
        double acc = 0;
        for (float v : losses) acc += v;
        if (epoch_loss) epoch_loss[ep] = steps_per_epoch ? (float)(acc / steps_per_epoch) : 0.f;
    }
    DPMM_CUDA_TRY(cudaMemcpyAsync(params, dp, sizeof(float) * kScrParams, cudaMemcpyDeviceToHost, b.stream));
    DPMM_CUDA_TRY(cudaStreamSynchronize(b.stream));
    return DPMM_OK;
}
