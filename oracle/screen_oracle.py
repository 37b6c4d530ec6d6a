"""CPU oracle of the learned split/merge screen -- TEST INFRASTRUCTURE ONLY.

Only tests/ (and the screen training script's held-out report) use this module, as the checker of
the device kernels in dpmmsubclusters_gpu_b200/csrc/dpmm_screen.cu.  Nothing on the product path
imports it.

The screen has no counterpart in the reference: it ranks split and merge candidates so that the
exact FP64 Hastings ratio (the reference's should_split_local, local_clusters_actions.cpp:215-242,
and should_merge, shared_actions.cpp:88-111) is computed for the best-ranked ones only.  This file
restates, in FP64 numpy:
  * the per-slot posterior quantities (niw.cpp:23-49 posterior; niw.cpp:122-138 and
    multinomial_prior.cpp:56-67 log marginal likelihoods),
  * the 32 candidate features (definitions below, mirrored by the device kernels),
  * the 32 -> 64 -> 64 -> 1 ReLU MLP, its mean-squared-error loss and gradient.

Statistics layout: 3K slots (slot 3k cluster k, 3k+1 its l, 3k+2 its r sub-cluster) of
(count, sum[D], S[D*D] column-major) (NIW) or (count, sum[D]) (Dirichlet), FP64, the layout
dpmm_create_sufficient_statistics returns.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import gammaln

F = 32          # features per candidate
H = 64          # hidden width
# parameter vector layout (FP32 on the device): W1[H][F], b1[H], W2[H][H], b2[H], w3[H], b3
OFF_W1, OFF_B1 = 0, H * F
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
NPARAM = OFF_B3 + 1

LOG_PI = math.log(math.pi)
HALF_LOG_2PI = 0.5 * math.log(2 * math.pi)


def slog(x):
    """sign(x) * log(1 + |x|)"""
    return np.sign(x) * np.log1p(np.abs(x))


def stirling(x):
    """(x - 1/2) ln x - x + ln(2 pi)/2 (Stirling's series truncated after its leading terms) for
    x > 0, and 0 for x <= 0."""
    x = np.asarray(x, dtype=np.float64)
    safe = np.where(x > 0, x, 1.0)
    return np.where(x > 0, (safe - 0.5) * np.log(safe) - safe + HALF_LOG_2PI, 0.0)


def chi_distance(pa, pb):
    """sum over d with pa + pb > 0 of (pa - pb)^2 / (pa + pb)"""
    s = pa + pb
    ok = s > 0
    return float(np.sum((pa[ok] - pb[ok]) ** 2 / s[ok]))


def lmvgamma_diff(vp, v0, D):
    d = np.arange(1, D + 1)
    return float(np.sum(gammaln(vp / 2.0 + (1 - d) / 2.0) - gammaln(v0 / 2.0 + (1 - d) / 2.0)))


def niw_lml_hat(n, D, k0, v0, ld0, kp, vp, ldp):
    """log marginal likelihood of niw.cpp:122-138 for given posterior log|psi'| (exact when ldp is)."""
    return (-n * D * 0.5 * LOG_PI + lmvgamma_diff(vp, v0, D) + (v0 / 2.0) * (D * math.log(v0) + ld0)
            - (vp / 2.0) * (D * math.log(vp) + ldp) + (D / 2.0) * math.log(k0 / kp))


class Prior:
    def __init__(self, gauss, D, k0=1.0, m0=None, v0=None, psi0=None, alpha0=None):
        self.gauss, self.D = gauss, D
        if gauss:
            self.k0, self.v0 = float(k0), float(v0)
            self.m0 = np.asarray(m0, dtype=np.float64)
            self.psi0 = np.asarray(psi0, dtype=np.float64).reshape(D, D)
            self.ld0 = float(np.linalg.slogdet(self.psi0)[1])
        else:
            self.alpha0 = np.asarray(alpha0, dtype=np.float64)


def _split_stat(row, D, gauss):
    n = row[0]
    s = row[1:1 + D]
    S = row[1 + D:1 + D + D * D].reshape(D, D).T if gauss else None   # column-major
    return n, s, S


def slot_quantities(stats, K, prior):
    """Per slot: dict of posterior quantities the feature kernels use."""
    D, g = prior.D, prior.gauss
    out = []
    for q in range(3 * K):
        n, s, S = _split_stat(stats[q], D, g)
        r = {"n": float(n)}
        if g:
            kp, vp = prior.k0 + n, prior.v0 + n
            mp = (prior.m0 * prior.k0 + s) / kp
            U = np.triu(prior.v0 * prior.psi0 + prior.k0 * np.outer(prior.m0, prior.m0) - kp * np.outer(mp, mp) + S)
            psi = (U + np.triu(U, 1).T) / vp   # upper triangle mirrored (selfadjointView<Upper>)
            r.update(kp=kp, vp=vp, mean=mp, diag=np.diag(psi).copy(), psi=psi,
                     hd=float(np.sum(np.log(np.diag(psi)))), tr=float(np.trace(psi)))
            if q % 3 == 0:
                ld = float(np.linalg.slogdet(psi)[1]) if n > 0 else prior.ld0
                r["ld"] = ld
                r["L"] = 0.0 if n == 0 else niw_lml_hat(n, D, prior.k0, prior.v0, prior.ld0, kp, vp, ld)
                # tau = tr(B^-1 P0), B = nu' psi', P0 = nu0 psi0 + kappa0 m0 m0^T (the prior's scatter)
                P0 = prior.v0 * prior.psi0 + prior.k0 * np.outer(prior.m0, prior.m0)
                r["tau"] = float(np.trace(np.linalg.solve(psi, P0))) / vp if n > 0 else 0.0
        else:
            a = prior.alpha0 + s
            A0, A = float(prior.alpha0.sum()), float(a.sum())
            r.update(a=a, A=A, A0=A0, p=a / A if A > 0 else np.zeros(D),
                     Lst=float(stirling(A0) - stirling(A) + np.sum(stirling(a) - stirling(prior.alpha0))),
                     tr=float((A - A0) / n) if n > 0 else 0.0)
            if q % 3 == 0:
                r["L"] = 0.0 if n == 0 else float(gammaln(A0) - gammaln(A) + np.sum(gammaln(a) - gammaln(prior.alpha0)))
        out.append(r)
    return out


def _count_term_merge(ni, nj, alpha):
    n = ni + nj
    return (-math.log(alpha) + math.lgamma(alpha) - 2 * math.lgamma(0.5 * alpha) + math.lgamma(n) - math.lgamma(n + alpha)
            + math.lgamma(ni + 0.5 * alpha) - math.lgamma(ni) - math.lgamma(nj) + math.lgamma(nj + 0.5 * alpha))


def _count_term_split(nl, nr, alpha):
    return math.log(alpha) + math.lgamma(nl) + math.lgamma(nr) - math.lgamma(nl + nr)


def lw(m, D):
    """sum over d = 1..D of log(max(m - d + 1, 1)): log det of a Wishart scatter's expected scale"""
    d = np.arange(1, D + 1)
    return float(np.sum(np.log(np.maximum(m - d + 1.0, 1.0))))


def wishart_gap(na, nb, D):
    """Expected Minkowski gap log|W_a + W_b| - D log(|W_a|^(1/D) + |W_b|^(1/D)) of two scatters of the
    same covariance from na and nb points, through the Wishart log-determinant means."""
    return lw(na + nb, D) - D * logaddexp(lw(na, D) / D, lw(nb, D) / D)


def _assemble(kind, gauss, D, alpha, P, T, na, nb, nu, La, Lb, Lu, qa, qb, r1, gsc, gapa, gapb, gapu, ldd, md, prior_frac,
              tra, trb, e27=0.0, e28=0.0, e29=0.0, e30=0.0):
    f = np.zeros(F)
    f[0] = 1.0 if kind == "merge" else -1.0
    f[1] = 1.0 if gauss else -1.0
    f[2] = slog(P) / 8
    f[3] = slog(T) / 8
    f[4] = slog(P - T) / 8
    f[5] = math.log1p(na) / 16
    f[6] = math.log1p(nb) / 16
    f[7] = math.log1p(nu) / 16
    f[8] = na / (na + nb)
    f[9] = math.log(D) / 8
    f[10] = math.log(alpha) / 4
    f[11] = min(max(La / (na * D), -8.0), 8.0) / 8
    f[12] = min(max(Lb / (nb * D), -8.0), 8.0) / 8
    f[13] = min(max(Lu / (nu * D), -8.0), 8.0) / 8
    f[14] = math.log1p(qa) / 8
    f[15] = math.log1p(qb) / 8
    f[16] = math.log1p(r1) / 8
    f[17] = slog(gsc) / 8
    f[18] = gapa
    f[19] = gapb
    f[20] = gapu
    f[21] = ldd
    f[22] = math.log1p(md) / 8
    f[23] = prior_frac
    f[24] = math.log(max(tra, 1e-30)) / 8
    f[25] = math.log(max(trb, 1e-30)) / 8
    f[26] = slog(P / (na + nb)) / 8
    f[27] = slog(e27) / 8
    f[28] = slog(e28) / 8
    f[29] = slog(e29) / 8
    f[30] = e30
    return f


def logaddexp(a, b):
    return float(np.logaddexp(a, b))


def merge_features(stats, K, prior, alpha):
    """Features of every pair i < j (row-major over the strict upper triangle); rows of pairs with
    an empty cluster are zero.  Returns (features [K(K-1)/2, F], proxy P [K(K-1)/2])."""
    D, g = prior.D, prior.gauss
    sq = slot_quantities(stats, K, prior)
    rows, prox = [], []
    for i in range(K):
        for j in range(i + 1, K):
            a, b = sq[3 * i], sq[3 * j]
            ni, nj = a["n"], b["n"]
            if ni == 0 or nj == 0:
                rows.append(np.zeros(F))
                prox.append(0.0)
                continue
            n = ni + nj
            T = _count_term_merge(ni, nj, alpha)
            if g:
                ku, vu = prior.k0 + n, prior.v0 + n
                lbi, lbj = D * math.log(a["vp"]) + a["ld"], D * math.log(b["vp"]) + b["ld"]
                lbm = D * logaddexp(lbi / D, lbj / D)                 # Minkowski bound of log|B_i + B_j|
                delta = a["mean"] - b["mean"]
                qi = float(delta @ np.linalg.solve(a["psi"], delta))
                qj = float(delta @ np.linalg.solve(b["psi"], delta))
                ai, aj = qi / a["vp"], qj / b["vp"]
                h = ai * aj / (ai + aj) if ai + aj > 0 else 0.0
                c = a["kp"] * b["kp"] / (a["kp"] + b["kp"])
                ht = a["tau"] * b["tau"] / (a["tau"] + b["tau"]) if a["tau"] + b["tau"] > 0 else 0.0
                g0 = wishart_gap(ni, nj, D)
                # log|B_u|, B_u = B_i + B_j - P0 + c delta delta^T: Minkowski's bound plus the expected
                # Wishart gap, the prior scatter counted once (first order), the mean-shift term
                lbu = lbm + g0 - ht + math.log1p(c * h)
                ldu = lbu - D * math.log(vu)
                Lu = niw_lml_hat(n, D, prior.k0, prior.v0, prior.ld0, ku, vu, ldu)
                P = T + Lu - a["L"] - b["L"]
                bdi, bdj = a["vp"] * a["diag"], b["vp"] * b["diag"]
                gdiag = float(np.sum(np.log(bdi + bdj)) - D * logaddexp(np.sum(np.log(bdi)) / D, np.sum(np.log(bdj)) / D))
                md = float(np.sum(delta ** 2 / (a["diag"] + b["diag"]))) / D
                hdu = float(np.sum(np.log((bdi + bdj) / vu)))   # diagonal of B_i + B_j over nu_u
                f = _assemble("merge", True, D, alpha, P, T, ni, nj, n, a["L"], b["L"], Lu, qi, qj, c * h,
                              vu * gdiag / 2, (a["hd"] - a["ld"]) / D, (b["hd"] - b["ld"]) / D, (hdu - ldu) / D,
                              (a["ld"] - b["ld"]) / D, md, prior.v0 / vu, a["tr"] / D, b["tr"] / D,
                              vu * ht / 2, vu * g0 / 2)
            else:
                au = prior.alpha0 + (a["a"] - prior.alpha0) + (b["a"] - prior.alpha0)
                A0 = a["A0"]
                Lstu = float(stirling(A0) - stirling(au.sum()) + np.sum(stirling(au) - stirling(prior.alpha0)))
                P = T + Lstu - a["Lst"] - b["Lst"]
                pa, pb = a["p"], b["p"]
                chi = chi_distance(pa, pb)
                c = ni * nj / n
                f = _assemble("merge", False, D, alpha, P, T, ni, nj, n, a["Lst"], b["Lst"], Lstu, ni * chi, nj * chi,
                              c * chi, 0.0, 0.0, 0.0, 0.0, 0.0, chi, A0 / au.sum(), a["tr"], b["tr"])
            rows.append(f)
            prox.append(P)
    return np.array(rows).reshape(-1, F), np.array(prox)


def split_features(stats, K, prior, alpha):
    """Features of every cluster's split (row k); rows with N_l == 0 or N_r == 0 are zero."""
    D, g = prior.D, prior.gauss
    sq = slot_quantities(stats, K, prior)
    rows, prox = [], []
    for k in range(K):
        c, l, r = sq[3 * k], sq[3 * k + 1], sq[3 * k + 2]
        nl, nr, n = l["n"], r["n"], c["n"]
        if nl == 0 or nr == 0:
            rows.append(np.zeros(F))
            prox.append(0.0)
            continue
        T = _count_term_split(nl, nr, alpha)
        if g:
            delta = l["mean"] - r["mean"]
            q = float(delta @ np.linalg.solve(c["psi"], delta))
            qd = float(np.sum(delta ** 2 / c["diag"]))
            clr = l["kp"] * r["kp"] / (l["kp"] + r["kp"])
            # children's log|B| from the parent's exact one: log|B_l + B_r - P0| = log|B_c| + log(1 - c y)
            # (Sherman-Morrison, y = delta^T B_c^-1 delta), the prior scatter (first order) and the
            # expected Wishart gap give D log(|B_l|^(1/D) + |B_r|^(1/D)); the children keep the ratio of
            # their diagonal (Hadamard) log-determinants
            y = q / c["vp"]
            om = max(1.0 - clr * y, 1e-12)
            g0 = wishart_gap(nl, nr, D)
            lbc = D * math.log(c["vp"]) + c["ld"]
            hbl, hbr = D * math.log(l["vp"]) + l["hd"], D * math.log(r["vp"]) + r["hd"]
            d0 = lbc + math.log(om) + c["tau"] - g0 - D * logaddexp(hbl / D, hbr / D)
            ldl, ldr = hbl + d0 - D * math.log(l["vp"]), hbr + d0 - D * math.log(r["vp"])
            Ll = niw_lml_hat(nl, D, prior.k0, prior.v0, prior.ld0, l["kp"], l["vp"], ldl)
            Lr = niw_lml_hat(nr, D, prior.k0, prior.v0, prior.ld0, r["kp"], r["vp"], ldr)
            P = T + Ll + Lr - c["L"]
            # second estimate: the parent's Hadamard gap stands in for the children's
            gapc = c["hd"] - c["ld"]
            Ll2 = niw_lml_hat(nl, D, prior.k0, prior.v0, prior.ld0, l["kp"], l["vp"], l["hd"] - gapc)
            Lr2 = niw_lml_hat(nr, D, prior.k0, prior.v0, prior.ld0, r["kp"], r["vp"], r["hd"] - gapc)
            P2 = T + Ll2 + Lr2 - c["L"]
            bdl, bdr = l["vp"] * l["diag"], r["vp"] * r["diag"]
            gdiag = float(np.sum(np.log(bdl + bdr)) - D * logaddexp(np.sum(np.log(bdl)) / D, np.sum(np.log(bdr)) / D))
            md = float(np.sum(delta ** 2 / (l["diag"] + r["diag"]))) / D
            f = _assemble("split", True, D, alpha, P, T, nl, nr, n, Ll, Lr, c["L"], q, qd, clr * q / c["vp"],
                          c["vp"] * gdiag / 2, gapc / D, gapc / D, gapc / D, (ldl - ldr) / D, md, prior.v0 / c["vp"],
                          l["tr"] / D, r["tr"] / D, c["vp"] * c["tau"] / 2, c["vp"] * g0 / 2, P2, -math.log(om) / 8)
        else:
            P = T + l["Lst"] + r["Lst"] - c["Lst"]
            pl, pr = l["p"], r["p"]
            chi = chi_distance(pl, pr)
            cc = nl * nr / (nl + nr)
            f = _assemble("split", False, D, alpha, P, T, nl, nr, n, l["Lst"], r["Lst"], c["Lst"], nl * chi, nr * chi,
                          cc * chi, 0.0, 0.0, 0.0, 0.0, 0.0, chi, c["A0"] / c["A"], l["tr"], r["tr"])
        rows.append(f)
        prox.append(P)
    return np.array(rows).reshape(-1, F), np.array(prox)


# ----------------------------------------------------------------------------------- MLP
def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(H, F), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H), p[OFF_B2:OFF_W3],
            p[OFF_W3:OFF_B3], p[OFF_B3])


def bf16_round(w):
    """Round FP32 values to BF16 (round to nearest even), returned as float64."""
    a = np.asarray(w, dtype=np.float32).copy()
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def deployed(p):
    """Parameters as the inference kernel uses them: weights rounded to BF16, biases FP32."""
    q = np.asarray(p, dtype=np.float32).astype(np.float64)
    for lo, hi in ((OFF_W1, OFF_B1), (OFF_W2, OFF_B2), (OFF_W3, OFF_B3)):
        q[lo:hi] = bf16_round(q[lo:hi])
    return q


def forward(p, X):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    h1 = np.maximum(X @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    return h2 @ w3 + b3, h1, h2


def loss_grad(p, X, t):
    """Mean squared error (1/B) sum (z - t)^2 and its gradient with respect to p."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    B = X.shape[0]
    z, h1, h2 = forward(p, X)
    loss = float(np.sum((z - t) ** 2) / B)
    dz = 2.0 * (z - t) / B
    g = np.zeros(NPARAM)
    g[OFF_W3:OFF_B3] = h2.T @ dz
    g[OFF_B3] = dz.sum()
    dh2 = np.outer(dz, w3) * (h2 > 0)
    g[OFF_W2:OFF_B2] = (dh2.T @ h1).reshape(-1)
    g[OFF_B2:OFF_W3] = dh2.sum(0)
    dh1 = (dh2 @ W2) * (h1 > 0)
    g[OFF_W1:OFF_B1] = (dh1.T @ X).reshape(-1)
    g[OFF_B1:OFF_W2] = dh1.sum(0)
    return loss, g


def init_params(seed):
    """He-uniform initial weights, zero biases."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM)
    p[OFF_W1:OFF_B1] = rng.uniform(-1, 1, H * F) * math.sqrt(6.0 / F)
    p[OFF_W2:OFF_B2] = rng.uniform(-1, 1, H * H) * math.sqrt(6.0 / H)
    p[OFF_W3:OFF_B3] = rng.uniform(-1, 1, H) * math.sqrt(6.0 / H)
    return p.astype(np.float32)


def adam_step(p, m, v, g, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (Kingma & Ba 2015) with bias correction; returns new (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v


def target(log_hr, lo=-30.0, hi=10.0):
    """Regression target of a candidate: its exact log Hastings ratio clamped to [lo, hi], / 10."""
    return np.clip(np.asarray(log_hr, dtype=np.float64), lo, hi) / 10.0


def select_top(scores, eligible_rows, top):
    """Rows of the `top` best scores among eligible rows (higher score first, then lower row; NaN
    ranks as -inf), returned in ascending row order -- the rule of the device selection."""
    s = np.asarray(scores, dtype=np.float64).copy()
    s[np.isnan(s)] = -np.inf
    rows = np.flatnonzero(np.asarray(eligible_rows, dtype=bool))
    order = sorted(rows.tolist(), key=lambda r: (-s[r], r))
    return np.array(sorted(order[:top]), dtype=np.int64)


def merge_row_eligibility(elig, K):
    """eligible pair rows (row-major over i < j) from per-cluster eligibility"""
    e = np.asarray(elig, dtype=bool)
    return np.array([e[i] and e[j] for i in range(K) for j in range(i + 1, K)], dtype=bool)


def exact_merge_log_hr(stats, i, j, prior, alpha):
    """The exact FP64 merge ratio of clusters i, j (shared_actions.cpp:88-99; niw.cpp:122-138) from
    slot statistics, for checking the proxy."""
    D = prior.D
    u = stats[3 * i] + stats[3 * j]
    one = np.stack([u, stats[3 * i + 1], stats[3 * i + 2]])
    L_u = slot_quantities(one, 1, prior)[0]["L"]
    sq = slot_quantities(stats, stats.shape[0] // 3, prior)
    ni, nj = sq[3 * i]["n"], sq[3 * j]["n"]
    return _count_term_merge(ni, nj, alpha) + L_u - sq[3 * i]["L"] - sq[3 * j]["L"]
