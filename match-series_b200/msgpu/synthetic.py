"""Seeded synthetic image series standing in for electron-microscopy frame series.

Every frame is a lattice of Gaussian atom columns, sampled through a smooth
random displacement plus per-row horizontal scan jitter, with Poisson counting
noise.  No public dataset is involved; the shapes, sizes and value
distributions follow the workloads the benchmark names:

* ``square``  : square lattice, spacing 12 px, sigma 2 px, amplitudes U(0.6, 1.0),
  Poisson peak 50, displacement <= 2 px, row jitter sigma 0.5 px  (257^2 series)
* ``hex``     : hexagonal lattice, spacing 10 px, sigma 1.8 px, Poisson peak 30,
  displacement <= 3 px, row jitter sigma 0.7 px  (513^2 series)

Frames are returned in raw counts (float64); the registration pipeline
normalises them exactly like the reference preprocessing does.
"""
from __future__ import annotations

import dataclasses
import numpy as np


@dataclasses.dataclass(frozen=True)
class LatticeSpec:
    kind: str = "hex"          # "hex" or "square"
    spacing: float = 10.0      # px
    sigma: float = 1.8         # px, Gaussian column width
    amp_lo: float = 0.6
    amp_hi: float = 1.0
    peak: float = 30.0         # Poisson counts at amplitude 1
    max_disp: float = 3.0      # px, bound of the smooth displacement
    jitter: float = 0.7        # px, std of the per-row x jitter
    n_waves: int = 4
    wl_lo: float = 64.0        # px, sinusoid wavelengths
    wl_hi: float = 256.0


SQUARE_257 = LatticeSpec("square", 12.0, 2.0, 0.6, 1.0, 50.0, 2.0, 0.5)
HEX_513 = LatticeSpec("hex", 10.0, 1.8, 0.6, 1.0, 30.0, 3.0, 0.7)


def _lattice_basis(spec: LatticeSpec):
    a = spec.spacing
    if spec.kind == "hex":
        return np.array([a, 0.0]), np.array([0.5 * a, np.sqrt(3.0) / 2.0 * a])
    return np.array([a, 0.0]), np.array([0.0, a])


def clean_image(n: int, spec: LatticeSpec, px: np.ndarray, py: np.ndarray,
                amp_seed: int, origin=(3.3, 4.1)) -> np.ndarray:
    """Gaussian-column lattice evaluated at sample positions (px, py) in pixels."""
    a1, a2 = _lattice_basis(spec)
    B = np.stack([a1, a2], axis=1)  # columns are basis vectors
    Binv = np.linalg.inv(B)
    ox, oy = origin
    rx, ry = px - ox, py - oy
    f1 = Binv[0, 0] * rx + Binv[0, 1] * ry
    f2 = Binv[1, 0] * rx + Binv[1, 1] * ry
    i0 = np.floor(f1).astype(np.int64)
    j0 = np.floor(f2).astype(np.int64)
    rng = np.random.default_rng(amp_seed)
    span = int(np.ceil(2.0 * n / spec.spacing)) + 16
    amps = rng.uniform(spec.amp_lo, spec.amp_hi, size=(2 * span + 1, 2 * span + 1))
    reach = int(np.ceil(4.0 * spec.sigma / (spec.spacing * 0.5))) + 1
    out = np.zeros_like(px, dtype=np.float64)
    inv2s2 = 1.0 / (2.0 * spec.sigma * spec.sigma)
    for di in range(-reach, reach + 1):
        for dj in range(-reach, reach + 1):
            ii = i0 + di
            jj = j0 + dj
            cx = ox + ii * a1[0] + jj * a2[0]
            cy = oy + ii * a1[1] + jj * a2[1]
            d2 = (px - cx) ** 2 + (py - cy) ** 2
            amp = amps[np.clip(ii + span, 0, 2 * span), np.clip(jj + span, 0, 2 * span)]
            out += amp * np.exp(-d2 * inv2s2)
    return out


def smooth_displacement(n: int, spec: LatticeSpec, rng: np.random.Generator):
    """Sum of random sinusoids scaled to max |u| <= spec.max_disp (pixels)."""
    y, x = np.mgrid[0:n, 0:n].astype(np.float64)
    u = np.zeros((n, n))
    v = np.zeros((n, n))
    for _ in range(spec.n_waves):
        wl = rng.uniform(spec.wl_lo, spec.wl_hi)
        th = rng.uniform(0, 2 * np.pi)
        ph = rng.uniform(0, 2 * np.pi)
        k = 2 * np.pi / wl
        arg = k * (np.cos(th) * x + np.sin(th) * y) + ph
        au, av = rng.normal(size=2)
        u += au * np.sin(arg)
        v += av * np.sin(arg)
    m = np.sqrt(u * u + v * v).max()
    if m > 0:
        s = spec.max_disp * rng.uniform(0.5, 1.0) / m
        u *= s
        v *= s
    return u, v


def make_series(n: int, num_frames: int, spec: LatticeSpec = HEX_513, seed: int = 2000,
                noise: bool = True, first: int = 0):
    """Returns (frames[F, n, n] float64 counts, clean[F, n, n], disp[F, 2, n, n]).

    Frame f uses the generator seeded with ``seed + f``; the lattice amplitudes
    are shared by the series (seeded with ``seed``).  ``first`` > 0 returns
    frames first .. first + num_frames - 1 of the same series (a shard)."""
    y, x = np.mgrid[0:n, 0:n].astype(np.float64)
    frames = np.empty((num_frames, n, n))
    clean = np.empty((num_frames, n, n))
    disp = np.empty((num_frames, 2, n, n))
    for i in range(num_frames):
        f = first + i
        rng = np.random.default_rng(seed + f)
        u, v = smooth_displacement(n, spec, rng)
        u = u + rng.normal(0.0, spec.jitter, size=(n, 1))
        img = clean_image(n, spec, x + u, y + v, amp_seed=seed)
        clean[i] = spec.peak * img
        disp[i, 0] = u
        disp[i, 1] = v
        frames[i] = rng.poisson(spec.peak * img).astype(np.float64) if noise else spec.peak * img
    return frames, clean, disp


def smooth_field(n: int, rng: np.random.Generator, amp_px: float, shift_px=(0.0, 0.0)) -> np.ndarray:
    """A smooth displacement [x | y] in domain units (2 x n*n): a constant
    shift plus two plane sinusoids per component, amplitudes in pixels."""
    y, x = np.mgrid[0:n, 0:n] / (n - 1)
    out = np.zeros((2, n * n))
    for c in range(2):
        f = shift_px[c] + sum(amp_px * rng.uniform(0.3, 1.0) *
                              np.sin(2 * np.pi * (rng.uniform(0.5, 2) * x + rng.uniform(0.5, 2) * y) + rng.uniform(0, 6))
                              for _ in range(2))
        out[c] = (f / (n - 1)).ravel()
    return out


def ragged_workload(num_series: int = 16, frames_per_series: int = 8, sizes=(129, 257, 513, 1025),
                    seed: int = 3000):
    """Uneven series: each of a size drawn from `sizes`, a square or hexagonal
    lattice with spacing U(8, 16) px, Poisson peak U(20, 100), displacements
    up to 3 px; returns a list of (reference[n*n], templates[F, n*n])."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(num_series):
        n = int(rng.choice(sizes))
        spec = LatticeSpec("hex" if rng.random() < 0.5 else "square", float(rng.uniform(8, 16)), 1.8, 0.6, 1.0,
                           float(rng.uniform(20, 100)), 3.0, 0.5)
        fr, _, _ = make_series(n, frames_per_series + 1, spec, seed=seed + 100 * s)
        out.append((fr[0].reshape(-1).copy(), fr[1:].reshape(frames_per_series, -1).copy()))
    return out


def seismic_gathers(num_gathers: int = 32, nt: int = 2049, ntr: int = 257, seed: int = 4000, dt: float = 0.25e-3,
                    f0: float = 50.0, snr_db: float = 10.0):
    """Synthetic seismic gathers (num_gathers, ntr, nt): per trace, sparse
    reflectivity (Bernoulli 0.02 x N(0, 1)) at hyperbolic moveout times
    t(x) = sqrt(t0^2 + (x/v)^2) (offsets 0-200 m, v 1500-1800 m/s), plus a
    static shift per trace (uniform +-2 ms), convolved with a Ricker wavelet
    of f0 Hz at dt sampling, and Gaussian noise at snr_db.  Time runs along
    x (the line of a trace), traces along y."""
    rng = np.random.default_rng(seed)
    t = np.arange(nt) * dt
    tw = np.arange(-64, 65) * dt
    a = (np.pi * f0 * tw) ** 2
    ricker = (1 - 2 * a) * np.exp(-a)
    out = np.zeros((num_gathers, ntr, nt))
    for g in range(num_gathers):
        refl_t0 = t[rng.random(nt) < 0.02]
        amps = rng.normal(size=refl_t0.size)
        v = rng.uniform(1500, 1800)
        offsets = np.linspace(0, 200, ntr)
        statics = rng.uniform(-2e-3, 2e-3, ntr)
        for k in range(ntr):
            tt = np.sqrt(refl_t0 ** 2 + (offsets[k] / v) ** 2) + statics[k]
            spikes = np.zeros(nt)
            idx = np.round(tt / dt).astype(np.int64)
            ok = (idx >= 0) & (idx < nt)
            np.add.at(spikes, idx[ok], amps[ok])
            out[g, k] = np.convolve(spikes, ricker, mode="same")
        p_sig = np.mean(out[g] ** 2)
        out[g] += rng.normal(0, np.sqrt(p_sig / 10 ** (snr_db / 10)), out[g].shape)
    return out


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    """Peak signal-to-noise ratio of a against b, peak = range of b."""
    mse = float(np.mean((a - b) ** 2))
    rng = float(b.max() - b.min())
    return float("inf") if mse == 0 else 10.0 * np.log10(rng * rng / mse)


# --- the same lattice series generated on the GPU (torch) ----------------------
# For the learned warm start's training and evaluation sets, which need many
# large frames: the lattice, displacement and noise model of make_series,
# evaluated on a CUDA device.  The random numbers differ from make_series'
# (scalar draws from numpy, per-pixel draws from a torch generator), so the
# frames follow the same distribution but are not the same frames.

def random_spec(rng: np.random.Generator) -> LatticeSpec:
    """A lattice of the uneven-series distribution: square or hexagonal,
    spacing U(8, 16) px, column sigma 0.18 spacing, Poisson peak U(20, 100),
    displacements up to U(1, 3) px, row jitter U(0.3, 0.7) px."""
    a = float(rng.uniform(8, 16))
    return LatticeSpec("hex" if rng.random() < 0.5 else "square", a, 0.18 * a, 0.6, 1.0,
                       float(rng.uniform(20, 100)), float(rng.uniform(1, 3)), float(rng.uniform(0.3, 0.7)))


def make_series_torch(n: int, num_frames: int, spec: LatticeSpec, seed: int, device, noise: bool = True):
    """make_series on a CUDA device: frames [F, n, n] float64 counts (torch)."""
    import torch
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    kw = dict(dtype=torch.float64, device=device)
    y, x = torch.meshgrid(torch.arange(n, **kw), torch.arange(n, **kw), indexing="ij")
    a1, a2 = _lattice_basis(spec)
    Binv = np.linalg.inv(np.stack([a1, a2], axis=1))
    span = int(np.ceil(2.0 * n / spec.spacing)) + 16
    amps = torch.from_numpy(rng.uniform(spec.amp_lo, spec.amp_hi, size=(2 * span + 1, 2 * span + 1))).to(device)
    reach = int(np.ceil(4.0 * spec.sigma / (spec.spacing * 0.5))) + 1
    inv2s2 = 1.0 / (2.0 * spec.sigma * spec.sigma)
    ox, oy = 3.3, 4.1
    frames = torch.empty((num_frames, n, n), **kw)
    for f in range(num_frames):
        u = torch.zeros((n, n), **kw)
        v = torch.zeros((n, n), **kw)
        for _ in range(spec.n_waves):
            wl, th, ph = rng.uniform(spec.wl_lo, spec.wl_hi), rng.uniform(0, 2 * np.pi), rng.uniform(0, 2 * np.pi)
            k = 2 * np.pi / wl
            arg = k * (np.cos(th) * x + np.sin(th) * y) + ph
            au, av = rng.normal(size=2)
            s = torch.sin(arg)
            u += au * s
            v += av * s
        m = float(torch.sqrt(u * u + v * v).max())
        if m > 0:
            sc = spec.max_disp * rng.uniform(0.5, 1.0) / m
            u *= sc
            v *= sc
        u += torch.randn((n, 1), generator=g, **kw) * spec.jitter
        px, py = x + u - ox, y + v - oy
        f1 = Binv[0, 0] * px + Binv[0, 1] * py
        f2 = Binv[1, 0] * px + Binv[1, 1] * py
        i0, j0 = torch.floor(f1).long(), torch.floor(f2).long()
        img = torch.zeros((n, n), **kw)
        for di in range(-reach, reach + 1):
            for dj in range(-reach, reach + 1):
                ii, jj = i0 + di, j0 + dj
                cx = ii * a1[0] + jj * a2[0]
                cy = ii * a1[1] + jj * a2[1]
                d2 = (px - cx) ** 2 + (py - cy) ** 2
                amp = amps[(ii + span).clamp(0, 2 * span), (jj + span).clamp(0, 2 * span)]
                img += amp * torch.exp(-d2 * inv2s2)
        frames[f] = torch.poisson(spec.peak * img, generator=g) if noise else spec.peak * img
    return frames
