"""ctypes binding of the FP64 CPU restatement (oracle/libmsoracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline leg of bench.py, as the checker.  The product never imports it.
Also wraps the reference driver oracle/_ref/ms_ref when it has been built.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmsoracle.so")
REF_BIN = os.path.join(HERE, "_ref", "ms_ref")

_dp = ctypes.POINTER(ctypes.c_double)


class Step(ctypes.Structure):
    _fields_ = [("iter", ctypes.c_int), ("energy", ctypes.c_double), ("tau", ctypes.c_double),
                ("sigma", ctypes.c_double), ("evals", ctypes.c_int)]


def build() -> None:
    subprocess.run(["make", "-s", "-f", os.path.join(HERE, "Makefile")], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.msor_ssd_energy.restype = ctypes.c_double
        L.msor_energy.restype = ctypes.c_double
        L.msor_register.restype = ctypes.c_double
        L.msor_gd_level.restype = ctypes.c_int
        L.msor_ncc_energy.restype = ctypes.c_double
        L.msor_lineshift.restype = ctypes.c_double
        L.msor_xshift_reg.restype = ctypes.c_double
        L.msor_xshift_reg_laplace.restype = ctypes.c_double
        L.msor_energy_dt.restype = ctypes.c_double
        L.msor_register_dt.restype = ctypes.c_double
        L.msor_gd_level_dt.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def n_of(level: int) -> int:
    return (1 << level) + 1


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def ssd_energy(level, R, T, px, py):
    return lib().msor_ssd_energy(level, _p(_c(R)), _p(_c(T)), _p(_c(px)), _p(_c(py)))


def energy(level, R, T, px, py, lam, ncc=False):
    ereg = ctypes.c_double()
    e = lib().msor_energy_dt(int(bool(ncc)), level, _p(_c(R)), _p(_c(T)), _p(_c(px)), _p(_c(py)),
                             ctypes.c_double(lam), ctypes.byref(ereg))
    return e, ereg.value


def denergy(level, R, T, px, py, lam, ncc=False):
    n = n_of(level)
    gx = np.zeros(n * n)
    gy = np.zeros(n * n)
    lib().msor_denergy_dt(int(bool(ncc)), level, _p(_c(R)), _p(_c(T)), _p(_c(px)), _p(_c(py)),
                          ctypes.c_double(lam), _p(gx), _p(gy))
    return gx, gy


def ncc_energy(level, R, T, px, py):
    return lib().msor_ncc_energy(level, _p(_c(R)), _p(_c(T)), _p(_c(px)), _p(_c(py)))


def mass_apply(level, u):
    out = np.zeros(n_of(level) ** 2)
    lib().msor_mass_apply(level, _p(_c(u)), _p(out))
    return out


def ssd_force(level, R, T, px, py):
    n = n_of(level)
    gx = np.zeros(n * n)
    gy = np.zeros(n * n)
    lib().msor_ssd_force(level, _p(_c(R)), _p(_c(T)), _p(_c(px)), _p(_c(py)), _p(gx), _p(gy))
    return gx, gy


def stiff_apply(level, u):
    out = np.zeros(n_of(level) ** 2)
    lib().msor_stiff_apply(level, _p(_c(u)), _p(out))
    return out


def smooth(level, sigma, x):
    out = np.zeros(n_of(level) ** 2)
    lib().msor_smooth(level, ctypes.c_double(sigma), _p(_c(x)), _p(out))
    return out


def restrict(fine_level, x):
    out = np.zeros(n_of(fine_level - 1) ** 2)
    lib().msor_restrict(fine_level, _p(_c(x)), _p(out))
    return out


def prolong(coarse_level, x):
    out = np.zeros(n_of(coarse_level + 1) ** 2)
    lib().msor_prolong(coarse_level, _p(_c(x)), _p(out))
    return out


def resample(src_level, x, dst_level):
    out = np.zeros(n_of(dst_level) ** 2)
    lib().msor_resample(src_level, _p(_c(x)), dst_level, _p(out))
    return out


def deform_image(level, img, px, py, ext=np.inf):
    out = np.zeros(n_of(level) ** 2)
    lib().msor_deform_image(level, _p(_c(img)), _p(_c(px)), _p(_c(py)), ctypes.c_double(ext), _p(out))
    return out


def normalize(img, sat=0.15, min_to_zero=1):
    a = _c(img).copy()
    lib().msor_normalize(_p(a), a.size, ctypes.c_double(sat), min_to_zero)
    return a


def gd_level(level, R, T, px, py, lam, max_iter, stop_eps=0.0, trace_cap=4096, ncc=False):
    px = _c(px).copy()
    py = _c(py).copy()
    tr = (Step * trace_cap)()
    e = ctypes.c_double()
    steps = lib().msor_gd_level_dt(int(bool(ncc)), level, _p(_c(R)), _p(_c(T)), _p(px), _p(py),
                                   ctypes.c_double(lam), max_iter, ctypes.c_double(stop_eps), ctypes.byref(e),
                                   tr, trace_cap)
    trace = [(tr[i].iter, tr[i].energy, tr[i].tau, tr[i].sigma, tr[i].evals) for i in range(min(steps, trace_cap))]
    return px, py, e.value, steps, trace


def register(max_level, start, stop, R, T, px=None, py=None, lam=0.1, lam_factor=1.0,
             max_iter=20, stop_eps=0.0, resample_phi=False, ncc=False):
    N = n_of(max_level) ** 2
    px = np.zeros(N) if px is None else _c(px).copy()
    py = np.zeros(N) if py is None else _c(py).copy()
    steps = (ctypes.c_int * max(1, stop - start + 1))()
    e = lib().msor_register_dt(int(bool(ncc)), max_level, start, stop, _p(_c(R)), _p(_c(T)), _p(px), _p(py),
                               ctypes.c_double(lam), ctypes.c_double(lam_factor), max_iter,
                               ctypes.c_double(stop_eps), int(bool(resample_phi)), steps)
    return px, py, e, list(steps)


def compose(level, d1, d2, init=None, with_iterations=False):
    """ConcatAndSmoothlyExtendDeformations of displacements d1, d2 (2 x N each);
    init: the solver's initial guess (default d2, as in series matching).
    with_iterations: also return the PCG steps of both components together."""
    N = n_of(level) ** 2
    out = (_c(d2) if init is None else _c(init)).reshape(2, N).copy()
    d1 = _c(d1).reshape(2, N)
    d2 = _c(d2).reshape(2, N)
    ox, oy = out[0].copy(), out[1].copy()
    its = lib().msor_compose(level, _p(d1[0].copy()), _p(d1[1].copy()), _p(d2[0].copy()), _p(d2[1].copy()),
                             _p(ox), _p(oy))
    res = np.stack([ox, oy])
    return (res, int(its)) if with_iterations else res


def lineshift(R, T, phix):
    """The seismic line-shift data term and its derivative; R, T, phix (ny, nx)."""
    R = _c(R)
    ny, nx = R.shape
    de = np.zeros((ny, nx))
    e = lib().msor_lineshift(nx, ny, _p(R.reshape(-1)), _p(_c(T).reshape(-1)), _p(_c(phix).reshape(-1)), _p(de))
    return float(e), de


def xshift_reg(phix, yreg):
    """findXShift's regulariser: (1/2 phi.K phi, K phi) for phix (ny, nx)."""
    ny, nx = phix.shape
    k = np.zeros((ny, nx))
    e = lib().msor_xshift_reg(nx, ny, ctypes.c_double(yreg), _p(_c(phix).reshape(-1)), _p(k))
    return float(e), k


def xshift_reg_laplace(phix, yreg, w):
    """findXShift's regulariser with laplaceWeight w > 0: (1/2 phi.K phi, K phi)."""
    ny, nx = phix.shape
    k = np.zeros((ny, nx))
    e = lib().msor_xshift_reg_laplace(nx, ny, ctypes.c_double(yreg), ctypes.c_double(w), _p(_c(phix).reshape(-1)),
                                      _p(k))
    return float(e), k


def h1sys_apply(x, sigma):
    """(M + 0.5 sigma^2 L) x on the grid of x (ny, nx)."""
    ny, nx = x.shape
    y = np.zeros((ny, nx))
    lib().msor_h1sys_apply(nx, ny, ctypes.c_double(sigma), _p(_c(x).reshape(-1)), _p(y))
    return y


def h1_metric(x, sigma):
    """(M + 0.5 sigma^2 L)^{-1} x, exact (band Cholesky)."""
    y = _c(x).copy()
    ny, nx = y.shape
    lib().msor_h1_metric(nx, ny, ctypes.c_double(sigma), _p(y.reshape(-1)))
    return y


def xshift(R, T, lam, yreg, max_iter, phix=None, trace_cap=4096, laplace_weight=0.0):
    """findXShift: returns (phix, energy, steps, trace rows (iter, energy, tau, sigma, evals))."""
    R = _c(R)
    ny, nx = R.shape
    ph = np.zeros((ny, nx)) if phix is None else _c(phix).copy()
    e = ctypes.c_double()
    tr = (Step * trace_cap)()
    steps = lib().msor_xshift(nx, ny, _p(R.reshape(-1)), _p(_c(T).reshape(-1)), ctypes.c_double(lam),
                              ctypes.c_double(yreg), ctypes.c_double(laplace_weight), max_iter, _p(ph.reshape(-1)),
                              ctypes.byref(e), tr, trace_cap)
    rows = [(tr[i].iter, tr[i].energy, tr[i].tau, tr[i].sigma, tr[i].evals) for i in range(min(steps, trace_cap))]
    return ph, e.value, steps, rows


def xshift_yconst(R, T, max_iter, phix=None):
    """findXShiftYConst: returns (phix (one value per line), energy, steps of the last descent)."""
    R = _c(R)
    ny, nx = R.shape
    ph = np.zeros((ny, nx)) if phix is None else _c(phix).copy()
    e = ctypes.c_double()
    steps = lib().msor_xshift_yconst(nx, ny, _p(R.reshape(-1)), _p(_c(T).reshape(-1)), max_iter,
                                     _p(ph.reshape(-1)), ctypes.byref(e))
    return ph, e.value, steps


def box_x(T, i):
    T = _c(T)
    ny, nx = T.shape
    out = np.zeros((ny, nx))
    lib().msor_box_x(_p(T.reshape(-1)), nx, ny, i, _p(out))
    return out


def remove_empty_lines(img, keep_top_bottom=False):
    """removeEmptyLinesFromImage of img (ny, nx); returns the cleaned image, or the code -1 / -2."""
    img = _c(img)
    ny, nx = img.shape
    out = np.zeros((ny, nx))
    n = lib().msor_remove_empty_lines(_p(img.reshape(-1)), nx, ny, int(keep_top_bottom), _p(out))
    return out[:n] if n >= 0 else n


def empty_lines_to_nan(img):
    """replaceEmptyLinesWithNaN on a copy of img (..., ny, nx); returns (copy, lines replaced)."""
    out = _c(img).copy()
    nx = out.shape[-1]
    n = lib().msor_empty_lines_to_nan(_p(out.reshape(-1)), nx, out.size // nx)
    return out, n


def warp_median(level, frames, phis, fill):
    N = n_of(level) ** 2
    out = np.zeros(N)
    lib().msor_warp_median(level, frames.shape[0], _p(_c(frames).reshape(-1)), _p(_c(phis).reshape(-1)),
                           ctypes.c_double(fill), _p(out))
    return out


def match_series(level, start, stop, frames, lam=0.1, lam_factor=1.0, max_iter=15, stop_eps=0.0, sat=0.15,
                 min_to_zero=1, refine_start=None, refine_stop=None, extra_stages=0, extra_lam_factor=1.0,
                 use_median=False, ncc=False):
    """matchSeries<>() with accumulated deformations, refinement and extra
    stages; returns the last stage's (phis m x 2 x N, avg, median, count) and
    the energies of every stage (one array per stage)."""
    F = frames.shape[0]
    N = n_of(level) ** 2
    rs = start if refine_start is None else refine_start
    rp = level if refine_stop is None else refine_stop
    m = F - 1 if extra_stages == 0 else F
    phis = np.zeros((m, 2, N))
    avg, med, cnt = np.zeros(N), np.zeros(N), np.zeros(N)
    ne = (F - 1) + extra_stages * F
    en = np.zeros(ne)
    lib().msor_match_series(1 if ncc else 0, level, start, stop, ctypes.c_double(lam), ctypes.c_double(lam_factor),
                            max_iter, ctypes.c_double(stop_eps), ctypes.c_double(sat), min_to_zero, rs, rp,
                            extra_stages, ctypes.c_double(extra_lam_factor), 1 if use_median else 0, F,
                            _p(_c(frames).reshape(-1)), _p(phis), _p(avg), _p(med), _p(cnt), _p(en))
    stages = [en[: F - 1]] + [en[F - 1 + k * F: F - 1 + (k + 1) * F] for k in range(extra_stages)]
    return phis, avg, med, cnt, stages


def warp_mean(level, frames, phis):
    n = n_of(level)
    F = frames.shape[0]
    mean = np.zeros(n * n)
    count = np.zeros(n * n)
    lib().msor_warp_mean(level, F, _p(_c(frames).reshape(-1)), _p(_c(phis).reshape(-1)), _p(mean), _p(count))
    return mean, count


# --- reference driver (oracle/_ref/ms_ref) ---------------------------------

def have_ref() -> bool:
    return os.path.exists(REF_BIN)


class RefRunner:
    """Runs the reference's own templates through oracle/_ref/ms_ref."""

    def __init__(self):
        self.dir = tempfile.mkdtemp(prefix="msref_")

    def _w(self, name, a):
        p = os.path.join(self.dir, name)
        _c(a).tofile(p)
        return p

    def _r(self, name, count=None):
        a = np.fromfile(os.path.join(self.dir, name), dtype=np.float64)
        return a if count is None else a[:count]

    def run(self, *args):
        subprocess.run([REF_BIN, *map(str, args)], check=True, stdout=subprocess.DEVNULL,
                       stderr=subprocess.DEVNULL)

    def energy(self, level, R, T, px, py, lam, ncc=False):
        N = n_of(level) ** 2
        self.run("energy_ncc" if ncc else "energy", level, self._w("R", R), self._w("T", T), self._w("px", px), self._w("py", py),
                 repr(float(lam)), os.path.join(self.dir, "e"))
        essd, ereg, etot = map(float, open(os.path.join(self.dir, "e.txt")).read().split())
        de = self._r("e_de.bin")
        return dict(essd=essd, ereg=ereg, e=etot, dex=de[:N], dey=de[N:2 * N], fx=de[2 * N:3 * N], fy=de[3 * N:])

    def smooth(self, level, sigma, x):
        self.run("smooth", level, repr(float(sigma)), self._w("in", x), os.path.join(self.dir, "out"))
        return self._r("out")

    def restrict(self, fine_level, x):
        self.run("restrict", fine_level, self._w("in", x), os.path.join(self.dir, "out"))
        return self._r("out")

    def prolong(self, coarse_level, x):
        self.run("prolong", coarse_level, self._w("in", x), os.path.join(self.dir, "out"))
        return self._r("out")

    def resample(self, src_level, x, dst_level):
        self.run("resample", src_level, self._w("in", x), dst_level, os.path.join(self.dir, "out"))
        return self._r("out")

    def deform(self, level, img, px, py):
        self.run("deform", level, self._w("img", img), self._w("px", px), self._w("py", py),
                 os.path.join(self.dir, "out"))
        return self._r("out")

    def compose(self, level, d1, d2, init=None):
        N = n_of(level) ** 2
        init = d2 if init is None else init
        self.run("compose", level, self._w("d1", _c(d1).reshape(-1)), self._w("d2", _c(d2).reshape(-1)),
                 self._w("io", _c(init).reshape(-1)), os.path.join(self.dir, "out"))
        return self._r("out").reshape(2, N)

    def median(self, level, frames, phis, fill):
        self.run("median", level, frames.shape[0], self._w("fr", frames), self._w("ph", phis), repr(float(fill)),
                 os.path.join(self.dir, "out"))
        return self._r("out")

    def lineshift(self, R, T, phix):
        ny, nx = R.shape
        self.run("lineshift", nx, ny, self._w("R", R), self._w("T", T), self._w("px", phix),
                 os.path.join(self.dir, "e"), os.path.join(self.dir, "de"))
        return float(self._r("e")[0]), self._r("de").reshape(ny, nx)

    def xshift_reg(self, phix, yreg):
        ny, nx = phix.shape
        self.run("xshiftreg", nx, ny, repr(float(yreg)), self._w("px", phix), os.path.join(self.dir, "e"),
                 os.path.join(self.dir, "k"))
        return float(self._r("e")[0]), self._r("k").reshape(ny, nx)

    def xshift_reg_laplace(self, phix, yreg, w):
        ny, nx = phix.shape
        self.run("xshiftlap", nx, ny, repr(float(yreg)), repr(float(w)), self._w("px", phix),
                 os.path.join(self.dir, "e"), os.path.join(self.dir, "k"))
        return float(self._r("e")[0]), self._r("k").reshape(ny, nx)

    def xshift_yconst(self, R, T, max_iter, phix):
        ny, nx = R.shape
        self.run("xshiftyconst", nx, ny, int(max_iter), self._w("R", R), self._w("T", T), self._w("px", phix),
                 os.path.join(self.dir, "po"), os.path.join(self.dir, "e"))
        return self._r("po").reshape(ny, nx), float(self._r("e")[0])

    def empty_lines_to_nan(self, img):
        img = _c(img)
        ny, nx = img.shape
        self.run("emptynan", nx, ny, self._w("img", img), os.path.join(self.dir, "out"))
        return self._r("out").reshape(ny, nx)

    def remove_empty_lines(self, img, keep_top_bottom=False):
        img = _c(img)
        ny, nx = img.shape
        self.run("rmempty", nx, ny, int(keep_top_bottom), self._w("img", img), os.path.join(self.dir, "out"))
        out = self._r("out")
        return out.reshape(-1, nx)

    def h1sys(self, x, sigma):
        ny, nx = x.shape
        self.run("h1sys", nx, ny, repr(float(sigma)), self._w("x", x), os.path.join(self.dir, "y"))
        return self._r("y").reshape(ny, nx)

    def save_array(self, a, path, type_):
        """qc::ScalarArray<QC_2D>::save of a (numY, numX) array to path."""
        ny, nx = a.shape
        self.run("save", nx, ny, self._w("arr", a), path, type_)

    def load_array(self, path):
        self.run("load", path, os.path.join(self.dir, "arr_out"), os.path.join(self.dir, "dims"))
        nx, ny = map(int, open(os.path.join(self.dir, "dims")).read().split())
        return self._r("arr_out").reshape(ny, nx)

    def save_displacement(self, level, phi, mask):
        self.run("savedef", level, self._w("def", phi), mask)

    def load_displacement(self, level, mask):
        self.run("loaddef", level, mask, os.path.join(self.dir, "def_out"))
        return self._r("def_out").reshape(2, -1)

    def normalize(self, level, img, sat=0.15, min_to_zero=1):
        self.run("normalize", level, self._w("img", img), repr(float(sat)), min_to_zero,
                 os.path.join(self.dir, "out"))
        return self._r("out")

    def gd_level(self, level, R, T, px, py, lam, max_iter, stop_eps=0.0, ncc=False):
        N = n_of(level) ** 2
        self.run("gdlevel_ncc" if ncc else "gdlevel", level, self._w("R", R), self._w("T", T), self._w("px", px), self._w("py", py),
                 repr(float(lam)), max_iter, repr(float(stop_eps)), os.path.join(self.dir, "phi"),
                 os.path.join(self.dir, "trace.txt"))
        phi = self._r("phi")
        lines = open(os.path.join(self.dir, "trace.txt")).read().splitlines()
        head = lines[0].split()
        final_e = float(head[head.index("final") + 1])
        steps = int(head[head.index("steps") + 1])
        rows = [l.split() for l in lines[1:]]
        trace = [(int(r[0]), float(r[1]), float(r[2]), float(r[3]), int(r[4])) for r in rows]
        return phi[:N], phi[N:], final_e, steps, trace

    def register(self, max_level, start, stop, R, T, px=None, py=None, lam=0.1, lam_factor=1.0,
                 max_iter=20, stop_eps=0.0, resample_phi=False, ncc=False):
        N = n_of(max_level) ** 2
        px = np.zeros(N) if px is None else px
        py = np.zeros(N) if py is None else py
        self.run("register_ncc" if ncc else "register", max_level, start, stop, self._w("R", R), self._w("T", T), self._w("px", px),
                 self._w("py", py), repr(float(lam)), repr(float(lam_factor)), max_iter, repr(float(stop_eps)),
                 int(bool(resample_phi)), os.path.join(self.dir, "phi"), os.path.join(self.dir, "e.txt"))
        phi = self._r("phi")
        return phi[:N], phi[N:], float(open(os.path.join(self.dir, "e.txt")).read())

    def match_series(self, level, start, stop, frames, lam=0.1, lam_factor=1.0, max_iter=15, stop_eps=0.0,
                     sat=0.15, min_to_zero=1, refine_start=None, refine_stop=None, extra_stages=0,
                     extra_lam_factor=1.0, use_median=False, ncc=False):
        """The reference's stage loop (see match_series); returns the same
        tuple plus per-stage timings."""
        F = frames.shape[0]
        N = n_of(level) ** 2
        rs = start if refine_start is None else refine_start
        rp = level if refine_stop is None else refine_stop
        out = os.path.join(self.dir, "ms")
        self.run("matchseries_ncc" if ncc else "matchseries", level, start, stop, repr(float(lam)),
                 repr(float(lam_factor)), max_iter, repr(float(stop_eps)), repr(float(sat)), min_to_zero, rs, rp,
                 extra_stages, repr(float(extra_lam_factor)), 1 if use_median else 0, F,
                 self._w("frames", frames), out)
        last = extra_stages + 1
        m = F - 1 if extra_stages == 0 else F
        phis = self._r(f"ms_phis{last}.bin").reshape(m, 2, N)
        avg, med, cnt = (self._r(f"ms_{k}{last}.bin") for k in ("avg", "median", "count"))
        stages = [dict() for _ in range(last)]
        timing = {}
        for line in open(out + ".txt"):
            t = line.split()
            if t[0] == "energy":
                stages[int(t[1]) - 1][int(t[2])] = float(t[3])
            elif t[0] == "stage":
                timing[int(t[1])] = dict(lam=float(t[3]), registration_seconds=float(t[5]),
                                         average_seconds=float(t[7]))
        energies = [np.array([d[i] for i in sorted(d)]) for d in stages]
        return phis, avg, med, cnt, energies, timing

    def series(self, max_level, start, stop, frames, lam, lam_factor, max_iter, stop_eps=0.0, sat=0.15,
               min_to_zero=1):
        F = frames.shape[0]
        N = n_of(max_level) ** 2
        self.run("series", max_level, start, stop, repr(float(lam)), repr(float(lam_factor)), max_iter,
                 repr(float(stop_eps)), repr(float(sat)), min_to_zero, F, self._w("frames", frames),
                 os.path.join(self.dir, "phis"), os.path.join(self.dir, "mean"), os.path.join(self.dir, "s.txt"))
        phis = self._r("phis").reshape(F, 2, N)
        mean = self._r("mean")
        info = {}
        energies = {}
        for line in open(os.path.join(self.dir, "s.txt")):
            t = line.split()
            if t[0] == "energy":
                energies[int(t[1])] = float(t[2])
            else:
                info[t[0]] = float(t[1])
        info["energies"] = [energies[i] for i in range(F)]
        return phis, mean, info
