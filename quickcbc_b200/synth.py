"""Seeded synthetic events for the likelihood hot path.

No public data set is used: every event is coloured Gaussian noise plus one
injected IMRPhenomD signal, in the normalisation of the QuickCBC reference:

* data ``D`` is the half-complex FFT scaled by sqrt(Tobs)/N
  (QuickCBC.c:254-313), so the noise in bin i has Re, Im ~ N(0, S_i/4) and
  <n|n> = 2 per bin under the inner product of Utilities.c:716-736;
* ``SN`` is the analytic one-sided PSD
  S(f) = 1e-49 [ x^-4.14 - 5 x^-2 + 111 (1 - x^2 + x^4/2) / (1 + x^2/2) ],
  x = f / 215 Hz, stored per bin with row length N/2 + 1 (the reference's
  ``double_matrix(Nifo, N/2)`` allocates N/2 + 1 entries, Utilities.c:2981);
* ``freq`` is the reference's frequency vector: freq[0] = 1/Tobs and
  freq[i] = i/Tobs (QuickCBC.c:419-420);
* parameters use the reference's 11-entry layout (QuickCBC.c:1867):
  [0] ln(Mc kg) [1] ln(Mt kg) [2] chi1 [3] chi2 [4] phi0 [5] t_c
  [6] ln(D_L m) [7] alpha [8] sin(delta) [9] psi [10] cos(iota).

The injected waveform comes from a caller-supplied template function
(``template(params) -> h[Nifo, N]``), so a test can inject with the oracle and
the benchmark can inject with the product; the distance is scaled so that the
network optimal SNR over the analysis band equals the requested value.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
import numpy as np

MSUN_SI = 1.988546954961461467461011951140572744e30
PC_SI = 3.085677581491367278913937957796471611e16
FMAX = 1024.0           # reference analysis band upper edge (ConstCBC.h:33)
NP = 11


def psd(f):
    """Analytic PSD of the synthetic configs (one-sided, strain^2/Hz)."""
    x = np.asarray(f, dtype=np.float64) / 215.0
    x2 = x * x
    return 1e-49 * (x ** -4.14 - 5.0 / x2 + 111.0 * (1.0 - x2 + 0.5 * x2 * x2) / (1.0 + 0.5 * x2))


def masses_to_params(m1, m2):
    """(m1, m2) in Msun -> (ln Mc_kg, ln Mt_kg)."""
    mt = m1 + m2
    eta = m1 * m2 / (mt * mt)
    mc = mt * eta ** 0.6
    return np.log(mc * MSUN_SI), np.log(mt * MSUN_SI)


@dataclass
class Event:
    """One analysis: detector network, data, PSD, frequency grid, injection."""
    labels: np.ndarray           # int32 [Nifo], 0=H1 1=L1 2=V1
    Tobs: float
    fs: float
    N: int
    fmin: float
    GMST: float
    D: np.ndarray                # [Nifo, N] half-complex
    SN: np.ndarray               # [Nifo, N/2+1]
    freq: np.ndarray             # [N/2]
    inj: np.ndarray              # [11]
    snr: float
    seed: int
    meta: dict = field(default_factory=dict)

    @property
    def nifo(self):
        return len(self.labels)

    @property
    def imin(self):
        return int(self.Tobs * self.fmin)

    @property
    def imax(self):
        return min(int(self.Tobs * FMAX), self.N // 2)


def make_grid(Tobs, fs):
    N = int(round(Tobs * fs))
    freq = np.arange(N // 2, dtype=np.float64) / Tobs
    freq[0] = 1.0 / Tobs
    return N, freq


def make_psd_rows(nifo, N, Tobs):
    f = np.arange(N // 2 + 1, dtype=np.float64) / Tobs
    f[0] = 1.0 / Tobs
    S = psd(f)
    return np.ascontiguousarray(np.broadcast_to(S, (nifo, N // 2 + 1)))


def inner(a, b, S, imin, imax, N):
    """4 sum_{i in [imin,imax)} (Re a Re b + Im a Im b)/S_i  (Utilities.c:716-736)."""
    i = np.arange(imin, imax)
    k = N - i
    return 4.0 * np.sum((a[i] * b[i] + a[k] * b[k]) / S[i])


def random_extrinsic(rng, p):
    p[4] = rng.uniform(0.0, 2.0 * np.pi)
    p[7] = rng.uniform(0.0, 2.0 * np.pi)
    p[8] = rng.uniform(-1.0, 1.0)
    p[9] = rng.uniform(0.0, np.pi)
    p[10] = rng.uniform(-1.0, 1.0)
    return p


def make_event(template, *, labels, Tobs, fs, fmin, m1, m2, chi1, chi2, snr, seed, tc=None):
    """Coloured Gaussian noise + one injection scaled to network SNR ``snr``.

    ``template(net_info, params) -> h[Nifo, N]`` where ``net_info`` is a dict
    with labels/Tobs/GMST/N/freq.
    """
    rng = np.random.default_rng(seed)
    labels = np.asarray(labels, dtype=np.int32)
    nifo = len(labels)
    N, freq = make_grid(Tobs, fs)
    SN = make_psd_rows(nifo, N, Tobs)
    GMST = rng.uniform(0.0, 2.0 * np.pi)
    p = np.zeros(NP)
    p[0], p[1] = masses_to_params(m1, m2)
    p[2], p[3] = chi1, chi2
    p[5] = Tobs - 2.0 if tc is None else tc
    p[6] = np.log(400e6 * PC_SI)
    random_extrinsic(rng, p)
    info = dict(labels=labels, Tobs=Tobs, GMST=GMST, N=N, freq=freq, fmin=fmin)
    imin, imax = int(Tobs * fmin), min(int(Tobs * FMAX), N // 2)
    h = template(info, p)
    s2 = sum(inner(h[i], h[i], SN[i], imin, imax, N) for i in range(nifo))
    if s2 > 0:
        p[6] += np.log(np.sqrt(s2) / snr)
        h = template(info, p)
    D = np.zeros((nifo, N))
    half = N // 2
    for i in range(nifo):
        sig = np.sqrt(SN[i, 1:half] / 4.0)
        D[i, 1:half] = rng.normal(size=half - 1) * sig
        D[i, N - 1:half:-1] = rng.normal(size=half - 1) * sig
    D += h
    D[:, 0] = 0.0
    D[:, half] = 0.0
    return Event(labels=labels, Tobs=float(Tobs), fs=float(fs), N=N, fmin=float(fmin), GMST=GMST,
                 D=np.ascontiguousarray(D), SN=SN, freq=freq, inj=p, snr=float(snr), seed=seed)


def draw_params(rng, B, inj, *, mc=(10.0, 30.0), q=(0.25, 1.0), chi=(-0.9, 0.9), dtc=0.05,
                dl_factor=(0.5, 2.0)):
    """Parameter sets drawn around an injection (chirp mass, mass ratio and
    spins uniform, t_c jitter, uniform phase/polarisation, isotropic sky)."""
    P = np.zeros((B, NP))
    Mc = rng.uniform(*mc, size=B)
    qq = rng.uniform(*q, size=B)
    m1 = Mc * (1.0 + qq) ** 0.2 / qq ** 0.6
    m2 = m1 * qq
    P[:, 0], P[:, 1] = masses_to_params(m1, m2)
    P[:, 2] = rng.uniform(*chi, size=B)
    P[:, 3] = rng.uniform(*chi, size=B)
    P[:, 4] = rng.uniform(0.0, 2.0 * np.pi, size=B)
    P[:, 5] = inj[5] + rng.uniform(-dtc, dtc, size=B)
    P[:, 6] = inj[6] + np.log(rng.uniform(*dl_factor, size=B))
    P[:, 7] = rng.uniform(0.0, 2.0 * np.pi, size=B)
    P[:, 8] = rng.uniform(-1.0, 1.0, size=B)
    P[:, 9] = rng.uniform(0.0, np.pi, size=B)
    P[:, 10] = rng.uniform(-1.0, 1.0, size=B)
    return P


def jitter_params(rng, B, center, scale=1e-3):
    """Parameter sets in a small neighbourhood of ``center`` (chains near the
    posterior peak); angular entries stay in range."""
    P = np.tile(np.asarray(center, dtype=np.float64), (B, 1))
    P[:, 0] += scale * 0.1 * rng.normal(size=B)
    P[:, 1] += scale * rng.normal(size=B)
    P[:, 2] = np.clip(P[:, 2] + 10 * scale * rng.normal(size=B), -0.95, 0.95)
    P[:, 3] = np.clip(P[:, 3] + 10 * scale * rng.normal(size=B), -0.95, 0.95)
    P[:, 4] = np.mod(P[:, 4] + 50 * scale * rng.normal(size=B), 2 * np.pi)
    P[:, 5] += scale * 1e-2 * rng.normal(size=B)
    P[:, 6] += 10 * scale * rng.normal(size=B)
    P[:, 7] = np.mod(P[:, 7] + 10 * scale * rng.normal(size=B), 2 * np.pi)
    P[:, 8] = np.clip(P[:, 8] + 10 * scale * rng.normal(size=B), -1, 1)
    P[:, 9] = np.mod(P[:, 9] + 10 * scale * rng.normal(size=B), np.pi)
    P[:, 10] = np.clip(P[:, 10] + 10 * scale * rng.normal(size=B), -1, 1)
    # keep eta <= 0.25: Mc <= Mt * 0.25^(3/5)
    lim = P[:, 1] + 0.6 * np.log(0.25)
    P[:, 0] = np.minimum(P[:, 0], lim - 1e-9)
    return P


def wrap_params(P):
    """Parameter sets brought back into the reference's ranges: phase, alpha and psi wrapped,
    sin(delta) and cos(iota) reflected into [-1, 1], spins clipped to the prior's +-0.85, and
    eta = (Mc/Mt)^(5/3) above 0.25 reflected about 0.25 at fixed (well-measured) chirp mass."""
    P = np.array(P, dtype=np.float64)
    for k, period in ((4, 2 * np.pi), (7, 2 * np.pi), (9, np.pi)):
        P[:, k] = np.mod(P[:, k], period)
    for k in (8, 10):
        x = np.mod(P[:, k] + 1.0, 4.0)
        P[:, k] = np.where(x > 2.0, 4.0 - x, x) - 1.0
    P[:, 2:4] = np.clip(P[:, 2:4], -0.85, 0.85)
    eta = np.exp((P[:, 0] - P[:, 1]) / 0.6)
    over = eta > 0.25
    P[over, 1] = P[over, 0] - 0.6 * np.log(np.clip(0.5 - eta[over], 0.05, 0.25 - 1e-12))
    return P


def fisher_steps(rng, B, fisher):
    """B Gaussian steps with covariance F^-1 for the 11 x 11 Fisher matrix F (e.g. Fisher_Het,
    QuickCBC.c:5446), drawn along F's eigenvectors as the reference sampler's eigen-jumps are
    (update, QuickCBC.c:2268-2282); eigenvalues below 10 are raised to 10, as the reference's
    FisherEvec does (QuickCBC.c:2510-2516)."""
    F = np.asarray(fisher, dtype=np.float64)
    lam, V = np.linalg.eigh(0.5 * (F + F.T))
    return (rng.normal(size=(B, NP)) / np.sqrt(np.maximum(lam, 10.0))) @ V.T


def cloud_at_drops(rng, center, fisher, drops, lnl, iters=40):
    """Parameter sets about ``center`` whose lnL lies the given amounts below lnL(center): set b
    is center + t_b s_b (wrapped), s_b a Fisher step (fisher_steps) and t_b > 0 found by bisection
    on lnL(center) - lnL(center + t s_b) = drops[b].  ``lnl(P) -> [B]`` evaluates a batch (sets
    it rejects at -1e20 count as infinitely far).  Chains at the posterior's width sit 0.5-10
    below the peak, wider ones tens below, and burn-in points hundreds below.  A high-SNR
    likelihood is far from quadratic beyond a fraction of a Fisher step, which is why the
    distance along each step is searched rather than scaled."""
    drops = np.asarray(drops, dtype=np.float64)
    B = len(drops)
    c = np.asarray(center, dtype=np.float64)
    S = fisher_steps(rng, B, fisher)
    L0 = float(lnl(c[None, :])[0])

    def drop(t):
        return L0 - np.asarray(lnl(wrap_params(c[None, :] + t[:, None] * S)), dtype=np.float64)

    lo, hi = np.zeros(B), np.full(B, 1.0)
    for _ in range(20):                       # grow hi until it passes the target
        short = drop(hi) < drops
        if not short.any():
            break
        hi[short] *= 2.0
    for _ in range(iters):
        mid = 0.5 * (lo + hi)
        below = drop(mid) < drops
        lo = np.where(below, mid, lo)
        hi = np.where(below, hi, mid)
    return wrap_params(c[None, :] + (0.5 * (lo + hi))[:, None] * S)


# --- the synthetic workloads (sizes from the reference's usage) -------------
CONFIGS = {
    1: dict(labels=[0, 1], Tobs=4.0, fs=2048.0, fmin=16.0, m1=36.0, m2=29.0, chi1=0.3, chi2=-0.1,
            snr=24.0, seed=1000, batch=16),
    2: dict(labels=[0, 1, 2], Tobs=16.0, fs=4096.0, fmin=20.0, m1=30.0, m2=25.0, chi1=0.2, chi2=0.1,
            snr=20.0, seed=2000, batch=2048),
    3: dict(labels=[0, 1, 2], Tobs=128.0, fs=4096.0, fmin=20.0, m1=1.45, m2=1.30, chi1=0.03, chi2=-0.02,
            snr=30.0, seed=3000, batch=4096),
}


def config_event(c, template, **over):
    kw = dict(CONFIGS[c])
    kw.update(over)
    kw.pop("batch", None)
    return make_event(template, **kw)


# --- config 4: many uneven events in one launch -----------------------------
TOBS_CHOICES = (4.0, 8.0, 16.0, 32.0, 64.0)


def chirp_time(mc_msun, f):
    """Newtonian time to merger from frequency f (s)."""
    return 2.18 * (1.21 / mc_msun) ** (5.0 / 3.0) * (100.0 / f) ** (8.0 / 3.0)


def uneven_event_specs(n_events=256, seed=4000, fmin=20.0):
    """Per-event settings of the uneven batch: total mass log-uniform 2.5-150 Msun,
    mass ratio U[0.25, 1], aligned spins U[-0.5, 0.5], the shortest Tobs in
    {4, 8, 16, 32, 64} s holding the chirp from fmin plus 2 s, fs 4096 Hz below
    20 Msun total mass else 2048 Hz, 1-3 detectors in random order, SNR U[10, 40].
    Event e uses seed `seed + e`."""
    specs = []
    for e in range(n_events):
        rng = np.random.default_rng(seed + e)
        mt = float(np.exp(rng.uniform(np.log(2.5), np.log(150.0))))
        q = float(rng.uniform(0.25, 1.0))
        m1, m2 = mt / (1.0 + q), mt * q / (1.0 + q)
        mc = mt * (m1 * m2 / mt ** 2) ** 0.6
        need = chirp_time(mc, fmin) + 2.5
        Tobs = next((t for t in TOBS_CHOICES if t >= need), TOBS_CHOICES[-1])
        fs = 4096.0 if mt < 20.0 else 2048.0
        nifo = int(rng.integers(1, 4))
        labels = [int(x) for x in rng.permutation(3)[:nifo]]
        specs.append(dict(labels=labels, Tobs=Tobs, fs=fs, fmin=fmin, m1=m1, m2=m2,
                          chi1=float(rng.uniform(-0.5, 0.5)), chi2=float(rng.uniform(-0.5, 0.5)),
                          snr=float(rng.uniform(10.0, 40.0)), seed=seed + e))
    return specs


def uneven_params(events, chains=32, proposals=8, seed=4000 + 500000, scale=1e-3):
    """chains x proposals parameter sets around each event's injection; returns
    (event_of [B] int32, params [B, 11]) with sets grouped by event."""
    rng = np.random.default_rng(seed)
    n = chains * proposals
    P = np.vstack([jitter_params(rng, n, ev.inj, scale=scale) for ev in events])
    eo = np.repeat(np.arange(len(events), dtype=np.int32), n)
    return eo, P


# --- analysis input files ------------------------------------------------------
def time_series(ev):
    """Strain time series whose scaled FFT is the event's data: x = irfft of D (half-complex,
    scaled by sqrt(Tobs)/N) times N/sqrt(Tobs).  [Nifo, N]."""
    N = ev.N
    M = N // 2
    out = np.zeros((len(ev.labels), N))
    for i in range(len(ev.labels)):
        d = ev.D[i]
        X = np.zeros(M + 1, dtype=complex)
        X[0] = d[0]
        X[M] = d[M]
        X[1:M] = d[1:M] + 1j * d[N - 1:M:-1]
        out[i] = np.fft.irfft(X, n=N) * N / np.sqrt(ev.Tobs)
    return out


def psd_model_arrays(rng, nifo, Tobs, N, nsample=3, nknots=(24, 20, 16), nlines=(6, 4, 5)):
    """A spline-plus-lines PSD model of `nsample` samples per detector: knots from 1/Tobs to
    (N/2)/Tobs, log PSD of the analytic curve with 5 % scatter per sample, lines near 60 Hz
    multiples and calibration-like frequencies with heights 10-1000 and Q 500-5000.
    Returns (nspline, nlines, ffit [nifo, nsp], xspline [nifo, nsample, nsp],
    lines [nifo, nsample, nlm, 5])."""
    ns = np.array(nknots[:nifo], dtype=np.int32)
    nl = np.array(nlines[:nifo], dtype=np.int32)
    nsp, nlm = int(ns.max()), int(nl.max())
    ffit = np.zeros((nifo, nsp))
    xs = np.zeros((nifo, nsample, nsp))
    L = np.zeros((nifo, nsample, nlm, 5))
    fhi = (N // 2) / Tobs
    base = np.array([60.0, 120.0, 35.9, 331.3, 502.5, 999.7])
    for i in range(nifo):
        n = ns[i]
        ffit[i, :n] = np.concatenate([[1.0 / Tobs], np.geomspace(6.0, 0.8 * fhi, n - 2), [fhi]])
        for s in range(nsample):
            xs[i, s, :n] = np.log(psd(ffit[i, :n])) + 0.05 * rng.normal(size=n)
            for j in range(nl[i]):
                lf = base[j] * (1.0 + 1e-3 * rng.normal())
                L[i, s, j] = [lf, 10.0 ** rng.uniform(1, 3), rng.uniform(500, 5000), rng.uniform(0.5, 4.0),
                              rng.uniform(0.05, 0.5)]
    return ns, nl, ffit, xs, L


def write_analysis_files(directory, labels, Tobs, ttrig, x, SN, SM=None):
    """framed_ and spec_ files as SpecFit writes them (SpecFit.c:207-213, 888-897): rows
    "t x" with %.16e, rows "f SN SM PS" with %.15e (PS written as 0)."""
    N = x.shape[1]
    dt = Tobs / N
    for i, lab in enumerate(labels):
        fr = os.path.join(directory, "framed_%d_%d_%d.dat" % (int(Tobs), int(ttrig), lab))
        with open(fr, "w") as f:
            f.writelines("%.16e %.16e\n" % (k * dt, v) for k, v in enumerate(x[i]))
        sp = os.path.join(directory, "spec_%d_%d_%d.dat" % (int(Tobs), int(ttrig), lab))
        sm = SN[i] if SM is None else SM[i]
        with open(sp, "w") as f:
            f.writelines("%.15e %.15e %.15e %.15e\n" % (k / Tobs, SN[i][k], sm[k], 0.0) for k in range(N // 2))


def write_psd_model_files(directory, labels, nspline, nlines, ffit, xspline, lines):
    """summary_, ffile_, sfile_ and lfile_ files in the layout QuickCBC.c:322-378 reads."""
    nsample = xspline.shape[1]
    for i, lab in enumerate(labels):
        n, m = int(nspline[i]), int(nlines[i])
        with open(os.path.join(directory, "summary_%d.dat" % lab), "w") as f:
            f.write("%d %d %d\n" % (n, m, nsample))
        with open(os.path.join(directory, "ffile_%d.dat" % lab), "w") as f:
            f.writelines("%.16e\n" % v for v in ffit[i, :n])
        with open(os.path.join(directory, "sfile_%d.dat" % lab), "w") as f:
            f.writelines(" ".join("%.16e" % v for v in xspline[i, s, :n]) + "\n" for s in range(nsample))
        with open(os.path.join(directory, "lfile_%d.dat" % lab), "w") as f:
            for s in range(nsample):
                f.writelines(" ".join("%.16e" % v for v in lines[i, s, j]) + "\n" for j in range(m))
