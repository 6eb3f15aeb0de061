"""Seeded synthetic time series for benchmarks and tests.

White N(0, 1) noise (variance series of ones) plus pulse trains with a von
Mises pulse shape, exp(kappa (cos 2 pi phi - 1)) with
kappa = ln 2 / (1 - cos(pi duty)) (duty = full width at half maximum as a
fraction of the period), and a Taylor phase model about the middle of the
observation: phi(t) = f0 (t - d(t)), d(t) = a t^2 / (2c) + j t^3 / (6c)
(+ x sin(2 pi t / Pb + phi0) for a circular binary).
Amplitudes are set so that the noiseless pulse folded at its true parameters
and scored by the boxcar scorer reaches the requested S/N.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

C_LIGHT = 299792458.0


@dataclass
class Pulsar:
    f0: float
    accel: float = 0.0
    jerk: float = 0.0
    duty: float = 0.05
    snr: float = 10.0
    # circular orbit: Roemer delay x sin(2 pi t / porb + phi0), x in light-seconds
    porb: float = 0.0
    x: float = 0.0
    phi0: float = 0.0


def von_mises_profile(nbins: int, duty: float, oversample: int = 32) -> np.ndarray:
    kappa = np.log(2.0) / (1.0 - np.cos(np.pi * duty))
    phi = (np.arange(nbins * oversample) + 0.5) / (nbins * oversample)
    p = np.exp(kappa * (np.cos(2 * np.pi * phi) - 1.0))
    return p.reshape(nbins, oversample).mean(axis=1)


def _boxcar_snr(x: np.ndarray, widths) -> float:
    # Boxcar S/N of a unit-variance profile (same template as the scorer).
    n = x.size
    best = -np.inf
    for w in widths:
        h = np.sqrt((n - w) / (n * w))
        b = w * h / (n - w)
        ext = np.concatenate([x, x[:w]])
        win = np.convolve(ext, np.ones(w), mode="valid")[:n]
        best = max(best, (h + b) * win.max() - b * x.sum())
    return float(best)


def amplitude_for_snr(snr: float, nsamps: int, nbins: int, duty: float, widths) -> float:
    """Per-sample peak amplitude giving the target folded boxcar S/N."""
    prof = von_mises_profile(nbins, duty)
    # Folded signal in bin b: A * (nsamps / nbins) * prof_b; noise sd per bin
    # sqrt(nsamps / nbins): the normalised profile is A * sqrt(nsamps/nbins) * prof.
    unit = _boxcar_snr(np.sqrt(nsamps / nbins) * prof, widths)
    return snr / unit


def inject(ts: np.ndarray, tsamp: float, psr: Pulsar, nbins: int, widths, chunk: int = 1 << 20) -> None:
    n = ts.size
    t_ref = n * tsamp / 2.0
    kappa = np.log(2.0) / (1.0 - np.cos(np.pi * psr.duty))
    amp = amplitude_for_snr(psr.snr, n, nbins, psr.duty, widths)
    for i0 in range(0, n, chunk):
        t = (np.arange(i0, min(n, i0 + chunk)) * tsamp) - t_ref
        delay = psr.accel * t * t / (2 * C_LIGHT) + psr.jerk * t**3 / (6 * C_LIGHT)
        if psr.porb > 0:
            delay = delay + psr.x * np.sin(2 * np.pi * t / psr.porb + psr.phi0)
        phase = psr.f0 * (t - delay)
        ts[i0 : i0 + t.size] += (amp * np.exp(kappa * (np.cos(2 * np.pi * phase) - 1.0))).astype(np.float32)


def make_series(nsamps: int, tsamp: float, seed: int, pulsars=(), nbins: int = 64, widths=(1, 2, 4, 8)):
    rng = np.random.default_rng(seed)
    ts_e = rng.standard_normal(nsamps, dtype=np.float32)
    for p in pulsars:
        inject(ts_e, tsamp, p, nbins, widths)
    ts_v = np.ones(nsamps, dtype=np.float32)
    return ts_e, ts_v


def taylor_accel_workload(seed: int = 7, n_signals: int = 4):
    """Taylor FFA (f, fdot) workload: 2^22 samples at 64 us, seed 7, four
    signals with f ~ U(5, 50) Hz, accel ~ U(-150, 150) m/s^2 and fold
    S/N ~ U(8, 20); searched over f in [5, 50] Hz, |accel| <= 200 m/s^2 at
    nbins = 64 with boxcar widths {1, 2, 3, 4, 6, 8, 12, 16}."""
    nsamps, tsamp, nbins = 1 << 22, 64e-6, 64
    widths = [1, 2, 3, 4, 6, 8, 12, 16]
    rng = np.random.default_rng(seed + 1000)
    pulsars = [
        Pulsar(f0=float(rng.uniform(5, 50)), accel=float(rng.uniform(-150, 150)),
               duty=0.05, snr=float(rng.uniform(8, 20)))
        for _ in range(n_signals)
    ]
    ts_e, ts_v = make_series(nsamps, tsamp, seed, pulsars, nbins, widths)
    params = dict(nsamps=nsamps, tsamp=tsamp, nbins=nbins, eta=2.0,
                  param_limits=[[-200.0, 200.0], [5.0, 50.0]], score_widths=widths)
    return ts_e, ts_v, params, pulsars


def mc_cascade_workload(ntrials: int = 1 << 20, nbins: int = 64, nstages: int = 8, seed: int = 99,
                        n_grid: int = 64):
    """Monte-Carlo cascade inputs: ntrials folded profiles of nbins float32 bins,
    N(0, 1) per bin plus a von Mises pulse (duty ~ U(2 %, 20 %), random phase)
    scaled to an injected S/N ~ U(0, 20) against unit-variance noise. Stage s
    (0-based) adds fresh noise of the input's variance (so the variance
    doubles) and the signal again times 2**s (a coherent signal doubles too);
    its pruning threshold rises linearly from 2 to 6 and every stage is counted
    against the same 64-threshold grid (0 .. 16). Trials with injected
    S/N >= 8 are flagged for the detection counts. All arrays come from one
    numpy generator (seed), so the CPU and GPU paths see the same numbers."""
    rng = np.random.default_rng(seed)
    duty = rng.uniform(0.02, 0.20, ntrials)
    snr = rng.uniform(0.0, 20.0, ntrials).astype(np.float32)
    phase = rng.random(ntrials)
    x = (np.arange(nbins) + 0.5) / nbins
    kappa = np.log(2.0) / (1.0 - np.cos(np.pi * duty))
    shape = np.exp(kappa[:, None] * (np.cos(2 * np.pi * (x[None, :] - phase[:, None])) - 1.0))
    shape /= np.sqrt((shape ** 2).sum(axis=1, keepdims=True))
    signal = (shape * snr[:, None]).astype(np.float32)
    folds0 = (rng.standard_normal((ntrials, nbins), dtype=np.float32) + signal).astype(np.float32)
    cls = (snr >= 8.0).astype(np.uint8)
    noises = []
    var = 1.0
    for _ in range(nstages):
        nz = rng.standard_normal((ntrials, nbins), dtype=np.float32)
        nz *= np.float32(np.sqrt(var))
        noises.append(nz)
        var *= 2.0
    thresholds = np.linspace(2.0, 6.0, nstages).astype(np.float32)
    grids = [np.linspace(0.0, 16.0, n_grid).astype(np.float32) for _ in range(nstages)]
    return folds0, signal, cls, noises, thresholds, grids


def jerk_prune_workload(seed: int = 11, n_signals: int = 2):
    """Jerk search through the pruning tree: 2^23 samples at 64 us (537 s),
    seed 11, two circular binaries (Pb ~ U(2, 6) h, x ~ U(0.5, 2) lt-s,
    f ~ U(20, 200) Hz, fold S/N ~ U(10, 14)); FFA to 32 segments
    (bseg_ffa = 2^18), jerk in [-0.4, 0.4] m/s^3, accel in [-457, 457] m/s^2,
    f in [20, 200] Hz, nbins 32; per-level thresholds rising linearly from 3
    to 8 over the 31 pruning levels."""
    nsamps, tsamp, nbins = 1 << 23, 64e-6, 32
    rng = np.random.default_rng(seed + 1000)
    pulsars = [
        Pulsar(f0=float(rng.uniform(20, 200)), duty=0.05, snr=float(rng.uniform(10, 14)),
               porb=float(rng.uniform(2, 6)) * 3600.0, x=float(rng.uniform(0.5, 2.0)),
               phi0=float(rng.uniform(0, 2 * np.pi)))
        for _ in range(n_signals)
    ]
    ts_e, ts_v = make_series(nsamps, tsamp, seed, pulsars, nbins, (1, 2, 4, 8))
    params = dict(nsamps=nsamps, tsamp=tsamp, nbins=nbins, eta=1.0, bseg_ffa=1 << 18,
                  param_limits=[[-0.4, 0.4], [-457.0, 457.0], [20.0, 200.0]])
    thresholds = np.linspace(3.0, 8.0, 31).astype(np.float32)
    return ts_e, ts_v, params, thresholds, pulsars


def multi_series_workload(nseries: int = 512, seed: int = 3, tsamp: float = 64e-6):
    """Many beams / DM trials: nseries float32 series with lengths
    log-uniform in [2^18, 2^22] samples at 64 us, N(0, 1) noise (variance
    series of ones); one in eight carries a pulsar with period ~ U(20, 500) ms
    and fold S/N ~ U(6, 20). Searched over periods 20-500 ms (f 2-50 Hz) at
    nbins 128 with widths {1,2,3,4,6,8,12,16}."""
    rng = np.random.default_rng(seed)
    lengths = np.exp(rng.uniform(np.log(2.0 ** 18), np.log(2.0 ** 22), nseries)).astype(np.int64)
    widths = [1, 2, 3, 4, 6, 8, 12, 16]
    data = []
    for k, n in enumerate(lengths):
        ts_e = rng.standard_normal(int(n), dtype=np.float32)
        if k % 8 == 0:
            psr = Pulsar(f0=1.0 / float(rng.uniform(0.020, 0.500)), duty=0.05, snr=float(rng.uniform(6, 20)))
            inject(ts_e, tsamp, psr, 128, widths)
        data.append((ts_e, np.ones(int(n), dtype=np.float32)))
    params = dict(tsamp=tsamp, nbins=128, f_range=(2.0, 50.0), widths=widths, eta=1.0)
    return data, params
