"""Seeded synthetic spectra for the benchmark workloads and parity tests.

No public dataset is involved: every spectrum is drawn from numpy's
``default_rng(seed)``.  The Marchenko-Pastur draws use the inverse-CDF
method on a 2**20-point grid, as the workloads specify.
"""
from __future__ import annotations

import numpy as np


def mp_edges(c: float, sigma2: float = 1.0) -> tuple[float, float]:
    s = np.sqrt(c)
    return sigma2 * (1.0 - s) ** 2, sigma2 * (1.0 + s) ** 2


def mp_inverse_cdf(u: np.ndarray, c: float, sigma2: float = 1.0, grid: int = 1 << 20) -> np.ndarray:
    """Map uniforms u in [0,1) to MP(c, sigma2) quantiles (0 < c <= 1)."""
    a, b = mp_edges(c, sigma2)
    x = np.linspace(a, b, grid)
    with np.errstate(invalid="ignore", divide="ignore"):
        f = np.sqrt(np.clip((b - x) * (x - a), 0.0, None)) / (2.0 * np.pi * c * sigma2 * x)
    f = np.nan_to_num(f, nan=0.0, posinf=0.0)
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (f[1:] + f[:-1]) * np.diff(x))])
    cdf /= cdf[-1]
    return np.interp(u, cdf, x)


def mp_spectrum(p: int, c: float, sigma2: float = 1.0, seed: int = 0, rng=None) -> np.ndarray:
    """p i.i.d. MP draws by inverse CDF, sorted ascending."""
    rng = np.random.default_rng(seed) if rng is None else rng
    return np.sort(mp_inverse_cdf(rng.random(p), c, sigma2))


def wishart_spiked(n: int = 4000, p: int = 1000, spikes=(12.0, 7.0, 4.0), seed: int = 0) -> np.ndarray:
    """Eigenvalues of X^T X / n, X n x p i.i.d. N(0,1) with columns scaled by
    sqrt of diag(spikes..., 1, ..., 1).  Sorted ascending."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, p))
    scale = np.ones(p)
    scale[: len(spikes)] = np.sqrt(np.asarray(spikes, dtype=np.float64))
    x *= scale[None, :]
    s = x.T @ x / n
    return np.ascontiguousarray(np.sort(np.linalg.eigvalsh(s)))


def mp_with_spikes(p: int, c: float, n_spikes: int, lo: float, hi: float, seed: int,
                   log_uniform: bool = True, sigma2: float = 1.0) -> np.ndarray:
    """MP bulk with the first n_spikes draws replaced by spikes in [lo, hi]."""
    rng = np.random.default_rng(seed)
    ev = mp_inverse_cdf(rng.random(p), c, sigma2)
    if n_spikes:
        if log_uniform:
            sp = np.exp(rng.uniform(np.log(lo), np.log(hi), n_spikes))
        else:
            sp = rng.uniform(lo, hi, n_spikes)
        ev[:n_spikes] = sp
    return np.ascontiguousarray(np.sort(ev))


# ---------------------------------------------------------------- workloads --
def config1(seed: int = 0) -> np.ndarray:
    """Wishart n=4000, p=1000 (c=0.25), population diag(12,7,4,1,...,1)."""
    return wishart_spiked(4000, 1000, (12.0, 7.0, 4.0), seed)


def config2(p: int, seed: int = 2) -> np.ndarray:
    """MP(c=0.5, sigma2=1) by inverse CDF, sorted; used with eta = 1/sqrt(p)."""
    return mp_spectrum(p, 0.5, 1.0, seed)


def config3(p: int = 1_000_000, seed: int = 3) -> np.ndarray:
    """MP bulk (c=0.1) + 20 spikes log-uniform in [3, 50]."""
    return mp_with_spikes(p, 0.1, 20, 3.0, 50.0, seed, log_uniform=True)


def config4(n_spectra: int = 4096, seed: int = 4, p_lo: int = 256, p_hi: int = 16384,
            grid: int = 1 << 14):
    """Uneven batch: p log-uniform in [p_lo, p_hi], MP bulk with c ~ U[0.05, 0.9],
    sigma2 log-uniform in [0.5, 2], 0-5 spikes in [(1+sqrt c)^2 sigma2 1.5, 30]
    placed at the top.  Returns (values, offsets, etas).  Each spectrum has
    its own (c, sigma2), so the inverse CDF uses a 2**14-point grid by default
    (ample for p <= 16384; the 2**20 grid of the single-spectrum workloads
    would cost minutes for 4096 spectra)."""
    rng = np.random.default_rng(seed)
    ps = np.round(np.exp(rng.uniform(np.log(p_lo), np.log(p_hi), n_spectra))).astype(np.int64)
    out = []
    for p in ps:
        c = rng.uniform(0.05, 0.9)
        s2 = np.exp(rng.uniform(np.log(0.5), np.log(2.0)))
        k = int(rng.integers(0, 6))
        ev = np.sort(mp_inverse_cdf(rng.random(int(p)), c, s2, grid))
        if k:
            lo = (1.0 + np.sqrt(c)) ** 2 * s2 * 1.5
            ev[-k:] = np.sort(rng.uniform(lo, 30.0, k))
        out.append(np.sort(ev))
    offs = np.zeros(n_spectra + 1, np.int64)
    offs[1:] = np.cumsum(ps)
    vals = np.ascontiguousarray(np.concatenate(out))
    etas = 1.0 / np.sqrt(ps.astype(np.float64))
    return vals, offs, etas


def config5(p: int, seed: int = 5) -> np.ndarray:
    """MP bulk (c=0.3) + 5 spikes uniform in [4, 20]."""
    return mp_with_spikes(p, 0.3, 5, 4.0, 20.0, seed, log_uniform=False)


def log_spectrum(p: int) -> np.ndarray:
    """ln(1..p), the reference's canonical test spectrum (testutil.rs:10-12)."""
    return np.log(np.arange(1, p + 1, dtype=np.float64))


def harness_spectrum(p: int) -> np.ndarray:
    """The reference benchmarks' deterministic MP-like spectrum
    (benches/support/mod.rs:17-35 ``Lcg``, 65-80 ``harness_spectrum``): a
    c = 0.5 Marchenko-Pastur support filled uniformly by a 64-bit LCG seeded
    with 42, plus two outliers hi*2.3 and lo*0.35, sorted ascending (p < 3:
    the first p LCG draws, unsorted)."""
    c = 0.5
    lo = (1.0 - float(np.sqrt(c))) ** 2
    hi = (1.0 + float(np.sqrt(c))) ** 2
    mask = (1 << 64) - 1
    state = 42
    n = p if p < 3 else p - 2
    out = np.empty(n)
    for k in range(n):
        state = (state * 6364136223846793005 + 1442695040888963407) & mask
        out[k] = lo + ((state >> 11) / float(1 << 53)) * (hi - lo)
    if p < 3:
        return out
    return np.sort(np.concatenate([out, [hi * 2.3, lo * 0.35]]))
