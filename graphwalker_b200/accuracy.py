"""How close a Monte Carlo visit estimate should be to its exact expectation.

A query of B walks from one source estimates each vertex's expected visits
per walk, mu_v, by c_v / B, where c_v counts the walks' visits to v.  The
exact mu comes from the FP64 power series (gw_expected_visits).  Monte Carlo
noise alone makes c / B differ from mu, and makes the top-k of c differ from
the top-k of mu wherever mu has near-ties at the cut.  This module states
what that noise predicts, so a measured error can be judged against it
instead of merely reported.

The noise model: c_v ~ Poisson(B * mu_v), independently per vertex.  It is
the standard approximation for counts summed over many independent walks.
It understates the variance where one walk revisits a vertex (a walk makes
at most L visits, so Var c_v <= L * B * mu_v, the bound that `l1_bound`
uses).

* `expected_l1`: E sum_v |c_v / B - mu_v|, in closed form from the Poisson
  mean absolute deviation, 2 e^-lam lam^(m+1) / m!  with m = floor(lam);
  `l1_sigma` is its standard deviation, sqrt(sum_v (lam_v - MAD_v^2)) / B.
* `expected_overlap`: the mean, over seeded resamples of c, of the overlap
  between the top-k of c (count desc, id asc, nonzero counts only; the
  engine's top-k order) and the top-k of mu (mu desc, id asc);
  `overlap_sigma` is its standard deviation over the resamples.
* `l1_bound`: sum_v sqrt(L * mu_v / B) >= E||c / B - mu||_1 (Cauchy-Schwarz
  with Var c_v <= L * B * mu_v), a bound that holds without the model.
"""
from __future__ import annotations

import numpy as np


def _gammaln(x: np.ndarray) -> np.ndarray:
    from scipy.special import gammaln
    return gammaln(x)


def poisson_mad(lam: np.ndarray) -> np.ndarray:
    """E|X - lam| for X ~ Poisson(lam), elementwise (0 where lam == 0)."""
    lam = np.asarray(lam, dtype=np.float64)
    out = np.zeros_like(lam)
    pos = lam > 0
    lp = lam[pos]
    m = np.floor(lp)
    out[pos] = 2.0 * np.exp(-lp + (m + 1.0) * np.log(lp) - _gammaln(m + 1.0))
    return out


def exact_topk(mu: np.ndarray, k: int) -> np.ndarray:
    """The k vertices of largest mu, ties broken by the smaller id (only mu > 0)."""
    mu = np.asarray(mu, dtype=np.float64)
    cand = np.flatnonzero(mu > 0)
    if len(cand) > 4 * k:
        vals = mu[cand]
        kth = np.partition(vals, len(vals) - k)[len(vals) - k]
        cand = cand[vals >= kth]
    order = cand[np.lexsort((cand, -mu[cand]))]
    return order[:k]


def count_topk(ids: np.ndarray, counts: np.ndarray, k: int) -> np.ndarray:
    """Top-k of integer counts over the given ids: count desc, id asc, counts > 0."""
    ids = np.asarray(ids)
    counts = np.asarray(counts).astype(np.int64)
    keep = counts > 0
    ids, counts = ids[keep], counts[keep]
    if len(counts) > 4 * k:
        # only counts >= the k-th largest can be listed; sort just those
        kth = np.partition(counts, len(counts) - k)[len(counts) - k]
        sel = counts >= kth
        ids, counts = ids[sel], counts[sel]
    return ids[np.lexsort((ids, -counts))][:k]


def expected_accuracy(mu: np.ndarray, budget: int, L: int, k: int = 100, resamples: int = 100,
                      seed: int = 0, max_candidates: int = 1_000_000) -> dict:
    """The Poisson model's expected L1 error and top-k overlap of a B-walk
    estimate of mu (see the module docstring), with their spreads."""
    mu = np.asarray(mu, dtype=np.float64)
    B = float(budget)
    lam = B * mu
    mad = poisson_mad(lam)
    out = {"model": "c_v ~ Poisson(B mu_v), independent", "budget": int(budget), "k": int(k),
           "expected_l1": float(mad.sum() / B),
           "l1_sigma": float(np.sqrt(max(0.0, float((lam - mad * mad).sum()))) / B),
           "l1_bound": float(np.sqrt(L * mu / B).sum())}
    top = exact_topk(mu, k)
    if len(top) == 0:
        out.update(expected_overlap=0.0, overlap_sigma=0.0, candidates=0, resamples=0)
        return out
    # Vertices far below the k-th rate cannot reach the sampled top-k: keep
    # those whose count could plausibly pass the k-th one (7 sigma each side;
    # a Poisson count beyond 7 sigma has probability below 1e-10).  The
    # candidates are the highest rates, at most max_candidates of them.
    lam_k = lam[top[-1]]
    cut = lam_k - 7.0 * np.sqrt(lam_k) - 7.0
    cand = np.flatnonzero(lam > 0) if cut <= 0 else np.flatnonzero(lam >= _lam_floor(cut))
    if len(cand) > max_candidates:
        cand = cand[np.argpartition(-lam[cand], max_candidates - 1)[:max_candidates]]
    rng = np.random.default_rng(seed)
    exact = set(top.tolist())
    ov = []
    for _ in range(resamples):
        c = rng.poisson(lam[cand])
        got = count_topk(cand, c, k)
        ov.append(len(exact.intersection(got.tolist())))
    out.update(expected_overlap=float(np.mean(ov)), overlap_sigma=float(np.std(ov)),
               candidates=int(len(cand)), resamples=int(resamples))
    return out


def _lam_floor(cut: float) -> float:
    """Smallest rate lam whose count reaches `cut` within 7 sigma:
    lam + 7 sqrt(lam) + 7 >= cut."""
    s = max(0.0, -3.5 + np.sqrt(12.25 + max(0.0, cut - 7.0)))
    return s * s


def measured_accuracy(mu: np.ndarray, budget: int, L: int, top_ids: np.ndarray, counts: np.ndarray | None = None,
                      k: int = 100, resamples: int = 100, seed: int = 0) -> dict:
    """The measured top-k overlap (and L1 error, when the full per-vertex
    counts are given) beside the model's expectation for the same budget;
    `within_3_sigma` says whether the measurement is no worse than the
    expectation minus three standard deviations."""
    exp = expected_accuracy(mu, budget, L, k=k, resamples=resamples, seed=seed)
    exact = set(exact_topk(mu, k).tolist())
    got = [int(x) for x in np.asarray(top_ids).ravel() if int(x) != 0xFFFFFFFF]
    res = dict(exp)
    res["top_overlap"] = len(exact.intersection(got))
    ok = res["top_overlap"] >= exp["expected_overlap"] - 3.0 * exp["overlap_sigma"]
    if counts is not None:
        c = np.asarray(counts, dtype=np.float64)
        res["l1_error"] = float(np.abs(c / float(budget) - np.asarray(mu, np.float64)).sum())
        ok = ok and res["l1_error"] <= exp["expected_l1"] + 3.0 * exp["l1_sigma"]
    res["within_3_sigma"] = bool(ok)
    return res
