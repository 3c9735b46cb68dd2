"""Generates the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's own templates through oracle/_ref/ms_ref (built from the
quocmesh sources by oracle/Makefile.ref) on seeded synthetic lattice images
and stores inputs and outputs as compressed .npz files.  The reference's own
tests hold no golden vectors for this path, so these fixtures pin both the
CPU oracle and the CUDA path.  Run from the repository root:

    make -f oracle/Makefile.ref && python tests/golden/make_golden.py

(--ncc-only regenerates only the fixtures of the cross-correlation data term,
--series-only those of the series pipeline: composition, median, stages;
--io-only the array files written by the reference's savers, --l9-only the
full-size registration of the benchmark configuration.)
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "match-series_b200"))
import msor  # noqa: E402
from msgpu import synthetic as syn  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def n_of(level):
    return (1 << level) + 1


def ops(ref: msor.RefRunner, level: int, seed: int):
    n = n_of(level)
    rng = np.random.default_rng(seed)
    fr, _, _ = syn.make_series(n, 2, syn.HEX_513, seed=seed)
    raw_t = fr[1].ravel()
    R = ref.normalize(level, fr[0].ravel())
    T = ref.normalize(level, raw_t)
    px = rng.normal(0, 0.5 / (n - 1), n * n)     # about half a pixel
    py = rng.normal(0, 0.5 / (n - 1), n * n)
    bx = px.copy()
    bx[: n] += 2.0 / (n - 1)                       # push the first row past the boundary (clipping)
    d = {"level": level, "R": R, "T": T, "px": px, "py": py, "lam": 0.1, "raw_t": raw_t}
    for tag, qx in (("", px), ("_clip", bx)):
        r = ref.energy(level, R, T, qx, py, 0.1)
        d["E" + tag] = np.array([r["essd"], r["ereg"], r["e"]])
        d["DE" + tag] = np.stack([r["dex"], r["dey"]])
        d["F" + tag] = np.stack([r["fx"], r["fy"]])
    d["px_clip"] = bx
    x = rng.normal(size=n * n)
    d["smooth_in"] = x
    d["smooth_sigmas"] = np.array([1.0, 0.25, 0.01])
    d["smooth_out"] = np.stack([ref.smooth(level, s, x) for s in d["smooth_sigmas"]])
    d["restrict_out"] = ref.restrict(level, x)
    xc = rng.normal(size=n_of(level - 1) ** 2)
    d["prolong_in"] = xc
    d["prolong_out"] = ref.prolong(level - 1, xc)
    d["resample_out"] = ref.resample(level - 1, xc, level)
    big = 3.0 / (n - 1)
    qx, qy = rng.normal(0, big, n * n), rng.normal(0, big, n * n)
    d["deform_px"], d["deform_py"] = qx, qy
    d["deform_out"] = ref.deform(level, raw_t, qx, qy)
    d["normalize_out"] = T
    d["normalize_nosat_out"] = ref.normalize(level, raw_t, sat=-1, min_to_zero=1)
    np.savez_compressed(os.path.join(OUT, f"ops_L{level}.npz"), **d)


def gd(ref: msor.RefRunner, level: int, seed: int, lam: float, max_iter: int):
    n = n_of(level)
    fr, _, _ = syn.make_series(n, 2, syn.SQUARE_257, seed=seed)
    R = ref.normalize(level, fr[0].ravel())
    T = ref.normalize(level, fr[1].ravel())
    z = np.zeros(n * n)
    px, py, e, steps, trace = ref.gd_level(level, R, T, z, z, lam, max_iter)
    np.savez_compressed(os.path.join(OUT, f"gd_L{level}.npz"), level=level, R=R, T=T, lam=lam, max_iter=max_iter,
                        px=px, py=py, energy=e, steps=steps, trace=np.array(trace, dtype=np.float64))


def register(ref: msor.RefRunner, level: int, seed: int):
    n = n_of(level)
    fr, _, _ = syn.make_series(n, 2, syn.HEX_513, seed=seed)
    R = ref.normalize(level, fr[0].ravel())
    T = ref.normalize(level, fr[1].ravel())
    cases = [
        dict(start=4, stop=level, lam=0.1, lam_factor=1.0, max_iter=20, stop_eps=0.0, resample=0),
        dict(start=3, stop=level - 1, lam=0.2, lam_factor=0.5, max_iter=15, stop_eps=1e-7, resample=0),
        dict(start=4, stop=level, lam=0.1, lam_factor=1.0, max_iter=10, stop_eps=0.0, resample=1),
    ]
    out = {"level": level, "R": R, "T": T}
    for i, c in enumerate(cases):
        px, py, e = ref.register(level, c["start"], c["stop"], R, T, lam=c["lam"], lam_factor=c["lam_factor"],
                                 max_iter=c["max_iter"], stop_eps=c["stop_eps"], resample_phi=bool(c["resample"]))
        out[f"case{i}"] = np.array([c["start"], c["stop"], c["lam"], c["lam_factor"], c["max_iter"], c["stop_eps"],
                                    c["resample"]], dtype=np.float64)
        out[f"phi{i}"] = np.stack([px, py])
        out[f"E{i}"] = np.array([e])
    np.savez_compressed(os.path.join(OUT, f"register_L{level}.npz"), **out)


def series(ref: msor.RefRunner, level: int, F: int, seed: int):
    n = n_of(level)
    fr, clean, _ = syn.make_series(n, F, syn.SQUARE_257, seed=seed)
    frames = fr.reshape(F, -1)
    phis, mean, info = ref.series(level, 3, level, frames, 0.1, 1.0, 15)
    np.savez_compressed(os.path.join(OUT, f"series_L{level}.npz"), level=level, frames=frames, phis=phis,
                        mean=mean, energies=np.array(info["energies"]), start=3, lam=0.1, max_iter=15)


def ncc(ref: msor.RefRunner, level: int, seed: int, max_iter: int):
    """Normalized cross-correlation data term: energy and variation at a small
    displacement and at one that pushes points out of the domain, and a traced
    level solve from zero."""
    n = n_of(level)
    rng = np.random.default_rng(seed)
    fr, _, _ = syn.make_series(n, 2, syn.HEX_513, seed=seed)
    R = ref.normalize(level, fr[0].ravel())
    T = ref.normalize(level, fr[1].ravel())
    px = rng.normal(0, 0.5 / (n - 1), n * n)
    py = rng.normal(0, 0.5 / (n - 1), n * n)
    bx = px.copy()
    bx[: n] += 2.0 / (n - 1)
    d = {"level": level, "R": R, "T": T, "px": px, "py": py, "px_out": bx, "lam": 0.1, "max_iter": max_iter}
    for tag, qx in (("", px), ("_out", bx)):
        r = ref.energy(level, R, T, qx, py, 0.1, ncc=True)
        d["E" + tag] = np.array([r["essd"], r["ereg"], r["e"]])
        d["DE" + tag] = np.stack([r["dex"], r["dey"]])
        d["F" + tag] = np.stack([r["fx"], r["fy"]])
    z = np.zeros(n * n)
    gx, gy, e, steps, trace = ref.gd_level(level, R, T, z, z, 0.1, max_iter, ncc=True)
    d.update(gd_px=gx, gd_py=gy, gd_energy=e, gd_steps=steps, gd_trace=np.array(trace, dtype=np.float64))
    np.savez_compressed(os.path.join(OUT, f"ncc_L{level}.npz"), **d)


def ncc_register(ref: msor.RefRunner, level: int, seed: int):
    n = n_of(level)
    fr, _, _ = syn.make_series(n, 2, syn.HEX_513, seed=seed)
    R = ref.normalize(level, fr[0].ravel())
    T = ref.normalize(level, fr[1].ravel())
    px, py, e = ref.register(level, 4, level, R, T, lam=0.1, max_iter=15, ncc=True)
    np.savez_compressed(os.path.join(OUT, f"ncc_register_L{level}.npz"), level=level, R=R, T=T, start=4,
                        lam=0.1, max_iter=15, phi=np.stack([px, py]), E=np.array([e]))


def compose(ref: msor.RefRunner, level: int, seed: int):
    """ConcatAndSmoothlyExtendDeformations with a shifted d2 (a band of
    nodes leaves the domain and is extended) and with a small d2 (no node
    leaves), the initial guess being d2 as in series matching; and the
    median of warped frames for an odd and an even frame count."""
    n = n_of(level)
    rng = np.random.default_rng(seed)
    d1 = syn.smooth_field(n, rng, 1.5)
    d2 = syn.smooth_field(n, rng, 1.0, shift_px=(2.5, -1.5))
    d2s = syn.smooth_field(n, rng, 0.3)
    out = ref.compose(level, d1, d2)
    out_in = ref.compose(level, d1, d2s)
    F = 5
    fr, _, _ = syn.make_series(n, F, syn.HEX_513, seed=seed)
    frames = fr.reshape(F, -1)
    phis = np.stack([syn.smooth_field(n, rng, 2.0, shift_px=(rng.uniform(-3, 3), rng.uniform(-3, 3))) for _ in range(F)])
    med5 = ref.median(level, frames, phis, 0.5)
    med4 = ref.median(level, frames[:4], phis[:4], 0.25)
    np.savez_compressed(os.path.join(OUT, f"compose_L{level}.npz"), level=level, d1=d1, d2=d2, out=out, d2_in=d2s,
                        out_in=out_in, frames=frames, phis=phis, med5=med5, med4=med4)


def match_series(ref: msor.RefRunner, level: int, F: int, seed: int):
    """matchSeries<>() with accumulated deformations: stage 1 plus one extra
    stage against the median, refinement from level 5."""
    n = n_of(level)
    fr, _, _ = syn.make_series(n, F, syn.HEX_513, seed=seed)
    frames = fr.reshape(F, -1)
    kw = dict(start=3, stop=level, max_iter=12, refine_start=5, extra_stages=1, extra_lam_factor=0.3,
              use_median=True)
    phis, avg, med, cnt, energies, _ = ref.match_series(level, frames=frames, **kw)
    np.savez_compressed(os.path.join(OUT, f"match_series_L{level}.npz"), level=level, frames=frames, phis=phis,
                        avg=avg, median=med, count=cnt, energies1=energies[0], energies2=energies[1],
                        **{k: np.array(v) for k, v in kw.items()})


def match_series_conditioned(ref: msor.RefRunner, level: int, F: int, seed: int):
    """A configuration of the same loop on which the reference is well
    conditioned: when every input pixel moves by one ulp, the displacements
    move by spread_px at most (stored), so that an implementation whose sums
    are reordered can be held to a tight tolerance."""
    n = n_of(level)
    fr, _, _ = syn.make_series(n, F, syn.SQUARE_257, seed=seed)
    frames = fr.reshape(F, -1)
    kw = dict(start=5, stop=level, max_iter=6, refine_start=6, extra_stages=1, extra_lam_factor=1.0, use_median=True)
    phis, avg, med, cnt, energies, _ = ref.match_series(level, frames=frames, **kw)
    spread = 0.0
    for k in range(2):
        sign = np.random.default_rng(k).choice([-1.0, 1.0], size=frames.shape)
        q = ref.match_series(level, frames=np.nextafter(frames, frames + sign * np.inf), **kw)[0]
        spread = max(spread, float(np.abs(q - phis).max() * (n - 1)))
    np.savez_compressed(os.path.join(OUT, f"match_series_wc_L{level}.npz"), level=level, frames=frames, phis=phis,
                        avg=avg, median=med, count=cnt, energies1=energies[0], energies2=energies[1],
                        spread_px=spread, **{k: np.array(v) for k, v in kw.items()})


IO_FILES = (("ref_p9.q2bz", 9), ("ref_p8.dat.bz2", 8), ("ref_p5.pgm", 5), ("ref_pa.pgm", 10), ("ref_p2.pgm", 2),
            ("ref_p7.txt", 7), ("ref_p9.pgm", 9))


def io_files(ref: msor.RefRunner, seed: int):
    """Array files written by the reference's own savers (one per format and
    compression) and what the reference's loader reads back from each; and a
    displacement saved as the reference's per-component files."""
    d = os.path.join(OUT, "io")
    os.makedirs(d, exist_ok=True)
    rng = np.random.default_rng(seed)
    a = rng.normal(0, 50, (17, 33)) + 100
    expected = {"source": a}
    for name, t in IO_FILES:
        path = os.path.join(d, name)
        ref.save_array(a, path, t)
        expected[name] = ref.load_array(path)
    # DigitalMicrograph files (this repository's writer, the reference's reader)
    from msgpu.dmfile import dm_bytes
    for v, t in ((3, 6), (4, 4), (3, 2), (4, 10)):
        img = rng.normal(0, 100, (13, 21)) + (200 if t in (4, 10) else 0)
        if t in (4, 10):
            img = np.clip(img, 0, 255)
        name = f"dm_t{t}.dm{v}"
        with open(os.path.join(d, name), "wb") as f:
            f.write(dm_bytes([(rng.normal(size=(5, 7)), 6), (img, t)], v))
        expected[name] = ref.load_array(os.path.join(d, name))
    n = n_of(4)
    phi = rng.normal(0, 0.01, (2, n * n))
    ref.save_displacement(4, phi, os.path.join(d, "ref_deformation_04_%d.dat.bz2"))
    expected["deformation"] = phi
    np.savez_compressed(os.path.join(OUT, "io_expected.npz"), **expected)


def seismic(ref: msor.RefRunner, seed: int):
    """The seismic model's energy pieces (matchSeismicSeries): the line-shift
    NCC data term with its derivative on a non-square grid (one NaN line that
    is skipped, displacements that push points off their line), and the
    anisotropic regulariser of findXShift."""
    rng = np.random.default_rng(seed)
    d = {}
    for tag, (nx, ny) in (("a", (65, 9)), ("b", (40, 6))):
        x = np.arange(nx)
        R = np.stack([np.sin(x / 3.0 + k) + 0.1 * rng.normal(size=nx) for k in range(ny)])
        T = np.stack([np.sin((x - 1.3) / 3.0 + k) + 0.1 * rng.normal(size=nx) for k in range(ny)])
        phi = rng.normal(0, 1.5 / (nx - 1), (ny, nx))
        phi[0, :3] = -5.0 / (nx - 1)
        if tag == "a":
            R[4, :] = np.nan
        e, de = ref.lineshift(R, T, phi)
        ereg, kphi = ref.xshift_reg(phi, 0.3 if tag == "a" else 2.0)
        d.update({f"R_{tag}": R, f"T_{tag}": T, f"phi_{tag}": phi, f"E_{tag}": e, f"DE_{tag}": de,
                  f"yreg_{tag}": 0.3 if tag == "a" else 2.0, f"Ereg_{tag}": ereg, f"Kphi_{tag}": kphi})
    # the H1 metric's system matrix M + 0.5 sigma^2 L (its Cholesky inverse needs
    # SuiteSparse, which the reference does not vendor: only the matrix is pinned)
    for tag, (nx, ny, sg) in (("a", (33, 17, 1.0)), ("b", (40, 23, 0.03))):
        x = rng.normal(size=(ny, nx))
        d[f"h1x_{tag}"] = x
        d[f"h1sigma_{tag}"] = sg
        d[f"h1y_{tag}"] = ref.h1sys(x, sg)
    # the regulariser with laplaceWeight > 0 (w L M^-1 L + stiffX + yRegFactor stiffY)
    for tag, yreg, w in (("a", 0.3, 0.5), ("b", 2.0, 3.0)):
        elap, klap = ref.xshift_reg_laplace(d[f"phi_{tag}"], yreg, w)
        d.update({f"lapw_{tag}": w, f"Elap_{tag}": elap, f"Kphilap_{tag}": klap})
    phi5 = rng.normal(0, 0.2, (5, 7))
    elap, klap = ref.xshift_reg_laplace(phi5, 1.0, 1.5)
    d.update({"phi_c": phi5, "yreg_c": 1.0, "lapw_c": 1.5, "Elap_c": elap, "Kphilap_c": klap})
    # findXShiftYConst (forceNonDyadicXShiftYConst): one shift per line, the reference's own run
    for tag, (nx, ny, shift, nan_line) in (("a", (33, 9, 1.3, -1)), ("b", (65, 17, -2.0, 3))):
        x = np.arange(nx)
        R = np.stack([np.sin(x / 4.0 + 0.3 * k) + 0.05 * rng.normal(size=nx) for k in range(ny)])
        T = np.stack([np.sin((x - shift - 0.2 * k / ny) / 4.0 + 0.3 * k) + 0.05 * rng.normal(size=nx)
                      for k in range(ny)])
        if nan_line >= 0:
            R[nan_line, :] = np.nan
        ph0 = rng.normal(0, 0.3, (ny, nx)) / (nx - 1)
        ph, e = ref.xshift_yconst(R, T, 60, ph0)
        d.update({f"ycR_{tag}": R, f"ycT_{tag}": T, f"ycphi0_{tag}": ph0, f"ycphi_{tag}": ph, f"ycE_{tag}": e})
    # replaceEmptyLinesWithNaN: zero lines (also -0.0 and squares that underflow to 0) become NaN; a line with
    # a NaN, a subnormal square or one non-zero sample stays
    img = rng.normal(size=(12, 21))
    img[[0, 5, 11], :] = 0.0
    img[2, :] = -0.0
    img[3, :] = 1e-170
    img[4, :] = 0.0
    img[4, 7] = np.nan
    img[6, :] = 0.0
    img[6, 20] = 1e-160
    img[7, :] = 0.0
    img[7, 0] = -3.0
    d.update({"enR": img, "enOut": ref.empty_lines_to_nan(img)})
    # removeEmptyLinesFromImage: every third line recorded (the others empty, one all NaN), an empty block at
    # the top and at the bottom, without and with keepEmptyTopBottomBlocks
    rm = np.zeros((31, 17))
    rm[4:26:3] = rng.normal(size=(8, 17))
    rm[7, :] = np.nan
    rm[5, :] = np.nan
    rm[5, 3] = 0.5
    d.update({"rmR": rm, "rmOut0": ref.remove_empty_lines(rm, False), "rmOut1": ref.remove_empty_lines(rm, True)})
    np.savez_compressed(os.path.join(OUT, "seismic.npz"), **d)


def phi_digest(px, py) -> str:
    """SHA-256 of a displacement's bytes ([phi_x, phi_y], little-endian float64)."""
    import hashlib
    return hashlib.sha256(np.concatenate([px, py]).astype("<f8").tobytes()).hexdigest()


def exact_l9(seed: int, frames_n: int = 4):
    """The benchmark configuration at full size: templates 1..3 of a 513^2
    hexagonal-lattice series registered to frame 0 on levels 5..9 with 30
    gradient-flow steps per level, by the reference itself.  The raw frames
    are Poisson counts (integers), stored as uint8; the displacements (2 x
    263169 doubles per template) are too large to commit, so the fixture keeps
    their SHA-256 (a bit-for-bit comparison), every 16th node for
    diagnostics, and the exact final energies."""
    from concurrent.futures import ThreadPoolExecutor
    level, n = 9, n_of(9)
    fr, _, _ = syn.make_series(n, frames_n, syn.HEX_513, seed=seed)
    raw = fr.reshape(frames_n, -1)
    assert np.all(raw == np.round(raw)) and raw.min() >= 0 and raw.max() < 256
    raw8 = raw.astype(np.uint8)
    R = msor.RefRunner().normalize(level, raw8[0].astype(np.float64))

    def one(i):
        ref = msor.RefRunner()
        T = ref.normalize(level, raw8[i].astype(np.float64))
        return ref.register(level, 5, 9, R, T, lam=0.1, lam_factor=1.0, max_iter=30)

    with ThreadPoolExecutor(frames_n - 1) as ex:
        res = list(ex.map(one, range(1, frames_n)))
    sub = np.s_[::16, ::16]
    np.savez_compressed(os.path.join(OUT, "exact_L9.npz"), level=level, start=5, stop=9, lam=0.1, max_iter=30,
                        raw=raw8, energies=np.array([e for _, _, e in res]),
                        digests=np.array([phi_digest(px, py) for px, py, _ in res]),
                        phi_sub=np.stack([np.stack([px.reshape(n, n)[sub], py.reshape(n, n)[sub]])
                                          for px, py, _ in res]))


def main():
    if not msor.have_ref():
        raise SystemExit("oracle/_ref/ms_ref is missing: make -f oracle/Makefile.ref")
    ref = msor.RefRunner()
    if "--l9-only" in sys.argv:
        exact_l9(9001)
        return
    if "--seismic-only" in sys.argv:
        seismic(ref, 801)
        return
    if "--io-only" in sys.argv:
        io_files(ref, 701)
        return
    if "--series-only" in sys.argv:
        compose(ref, 6, 601)
        match_series(ref, 6, 4, 602)
        match_series_conditioned(ref, 6, 4, 623)
        return
    if "--ncc-only" in sys.argv:
        ncc(ref, 5, 501, 20)
        ncc(ref, 6, 502, 15)
        ncc_register(ref, 7, 503)
        return
    ops(ref, 5, 101)
    ops(ref, 6, 102)
    gd(ref, 5, 201, 0.1, 20)
    gd(ref, 6, 202, 0.05, 30)
    register(ref, 7, 301)
    series(ref, 6, 4, 401)
    ncc(ref, 5, 501, 20)
    ncc(ref, 6, 502, 15)
    ncc_register(ref, 7, 503)
    compose(ref, 6, 601)
    match_series(ref, 6, 4, 602)
    match_series_conditioned(ref, 6, 4, 623)
    io_files(ref, 701)
    seismic(ref, 801)
    exact_l9(9001)
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))


if __name__ == "__main__":
    main()
