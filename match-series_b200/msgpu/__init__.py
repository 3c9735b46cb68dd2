"""Python binding of the msgpu C ABI (include/msgpu.h).

The CUDA library libmsgpu.so is built in-tree by ``msgpu.build.build()``.  There
is no CPU fallback: every call goes to the CUDA kernels, and a missing library
or a missing GPU raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmsgpu.so")

MSGPU_OK = 0
MSGPU_ERR_INVALID_ARG = 1
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "SIZE", 3: "CUDA", 4: "UNSUPPORTED"}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class Params(ctypes.Structure):
    """msgpu_params: the parameter-file keys of the registration path."""
    _fields_ = [
        ("precision_level", ctypes.c_int),
        ("input_level", ctypes.c_int),
        ("start_level", ctypes.c_int),
        ("stop_level", ctypes.c_int),
        ("lambda_", ctypes.c_double),
        ("lambda_factor", ctypes.c_double),
        ("max_gd_iterations", ctypes.c_int),
        ("stop_epsilon", ctypes.c_double),
        ("saturation_percent", ctypes.c_double),
        ("normalize_min_to_zero", ctypes.c_int),
        ("dont_normalize_input", ctypes.c_int),
        ("resample_deformation", ctypes.c_int),
        ("use_fp64", ctypes.c_int),
        ("data_term", ctypes.c_int),
        ("sum_order", ctypes.c_int),
    ]


class SeriesParams(ctypes.Structure):
    """msgpu_series_params: the keys of matchSeries<>() beyond the registration."""
    _fields_ = [
        ("refine_start_level", ctypes.c_int),
        ("refine_stop_level", ctypes.c_int),
        ("num_extra_stages", ctypes.c_int),
        ("extra_stages_lambda_factor", ctypes.c_double),
        ("use_median_as_new_target", ctypes.c_int),
        ("dont_accumulate_deformation", ctypes.c_int),
    ]


class SeriesDesc(ctypes.Structure):
    """msgpu_series_desc: one series of a ragged batch."""
    _fields_ = [
        ("level", ctypes.c_int),
        ("num_templates", ctypes.c_int),
        ("reference", ctypes.c_void_p),
        ("templates", ctypes.c_void_p),
        ("phis_out", ctypes.c_void_p),
        ("energies_out", ctypes.c_void_p),
    ]


class LevelTuning(ctypes.Structure):
    """msgpu_level_tuning: scheduling of the level kernel on one level."""
    _fields_ = [("chunk_div", ctypes.c_int), ("chunk_max", ctypes.c_int), ("ctas_per_sm", ctypes.c_int),
                ("ms", ctypes.c_float)]


class Stats(ctypes.Structure):
    _fields_ = [("kernel_launches", ctypes.c_int), ("num_levels", ctypes.c_int), ("first_level", ctypes.c_int),
                ("level_ms", ctypes.c_float * 16), ("level_steps", ctypes.c_longlong * 16),
                ("level_evals", ctypes.c_longlong * 16), ("level_cluster", ctypes.c_int * 16),
                ("level_pass_cycles", (ctypes.c_longlong * 8) * 16), ("graph_replayed", ctypes.c_int),
                ("level_xs", (ctypes.c_longlong * 8) * 16)]

PASS_KINDS = ["energy0", "gradient", "vdown", "vcoarse", "vup", "ncg", "energy", "sync"]


class MsgpuError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"msgpu {STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None

EXPORTS = [
    "msgpu_params_default", "msgpu_abi_version", "msgpu_create", "msgpu_destroy", "msgpu_last_error",
    "msgpu_register_batch", "msgpu_register_batch_device", "msgpu_warp_mean", "msgpu_warp_mean_device",
    "msgpu_energy", "msgpu_smooth", "msgpu_restrict", "msgpu_prolong", "msgpu_normalize", "msgpu_gd_level",
    "msgpu_match_series_stage", "msgpu_match_series_stage_device", "msgpu_set_profiling", "msgpu_get_stats",
    "msgpu_set_trace", "msgpu_get_trace",
    "msgpu_set_data_term", "msgpu_series_params_default", "msgpu_match_series", "msgpu_match_series_device",
    "msgpu_compose", "msgpu_compose_device", "msgpu_warp_median", "msgpu_warp_median_device",
    "msgpu_io_last_error", "msgpu_read_array", "msgpu_write_array", "msgpu_read_arrays", "msgpu_read_displacement",
    "msgpu_write_displacement", "msgpu_read_arrays_start", "msgpu_io_wait", "msgpu_register_ragged",
    "msgpu_register_ragged_device", "msgpu_lineshift_energy", "msgpu_lineshift_energy_device", "msgpu_xshift_reg",
    "msgpu_xshift_reg_device", "msgpu_find_xshift", "msgpu_find_xshift_device", "msgpu_find_xshift_batch",
    "msgpu_net_num_params", "msgpu_net_create", "msgpu_net_destroy", "msgpu_net_input_level", "msgpu_net_set_tensor_cores", "msgpu_net_get_params",
    "msgpu_net_set_params", "msgpu_net_save", "msgpu_net_load", "msgpu_net_predict_device",
    "msgpu_net_train_step_device", "msgpu_net_loss_grad", "msgpu_prepare_images_device", "msgpu_register_batch_warm",
    "msgpu_register_batch_warm_device", "msgpu_find_xshift_yconst", "msgpu_find_xshift_yconst_device",
    "msgpu_empty_lines_to_nan", "msgpu_empty_lines_to_nan_device", "msgpu_remove_empty_lines",
    "msgpu_remove_empty_lines_device", "msgpu_set_wait_limits", "msgpu_set_sum_order", "msgpu_set_certified_steps", "msgpu_set_seismic_device_control", "msgpu_set_warm_schedule", "msgpu_warp_sum_device",
    "msgpu_mean_from_sums_device", "msgpu_set_graphs", "msgpu_get_tuning", "msgpu_set_tuning",
    "msgpu_autotune_device", "msgpu_gd_level_log", "msgpu_exact_sum_device",
]


def lib():
    """Loads libmsgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with msgpu.build.build() (no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        L.msgpu_last_error.restype = ctypes.c_char_p
        L.msgpu_last_error.argtypes = [ctypes.c_void_p]
        L.msgpu_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.msgpu_destroy.argtypes = [ctypes.c_void_p]
        L.msgpu_params_default.argtypes = [ctypes.POINTER(Params)]
        L.msgpu_params_default.restype = None
        L.msgpu_register_batch.argtypes = [ctypes.c_void_p, ctypes.POINTER(Params), _dp, _dp, ctypes.c_int, _dp,
                                           _dp, _dp, _ip]
        L.msgpu_register_batch_device.argtypes = [ctypes.c_void_p, ctypes.POINTER(Params), ctypes.c_void_p,
                                                  ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.msgpu_warp_mean.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, _dp]
        L.msgpu_warp_mean_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.msgpu_energy.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double,
                                   ctypes.c_int, _dp, _dp]
        L.msgpu_smooth.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp, _dp]
        L.msgpu_restrict.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.msgpu_prolong.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.msgpu_normalize.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp]
        L.msgpu_gd_level.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double,
                                     ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp, _ip, _dp, ctypes.c_int]
        L.msgpu_gd_level_log.argtypes = L.msgpu_gd_level.argtypes
        L.msgpu_exact_sum_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p]
        L.msgpu_match_series_stage.argtypes = [ctypes.c_void_p, ctypes.POINTER(Params), _dp, _dp, ctypes.c_int,
                                               _dp, _dp, _ip, _dp, _dp]
        L.msgpu_match_series_stage_device.argtypes = [ctypes.c_void_p, ctypes.POINTER(Params), ctypes.c_void_p,
                                                      ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                      ctypes.c_void_p, ctypes.c_void_p]
        L.msgpu_set_profiling.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.msgpu_set_trace.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint]
        L.msgpu_get_trace.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong]
        L.msgpu_get_trace.restype = ctypes.c_longlong
        L.msgpu_set_graphs.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.msgpu_get_tuning.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(LevelTuning)]
        L.msgpu_set_tuning.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(LevelTuning)]
        L.msgpu_autotune_device.argtypes = [ctypes.c_void_p, ctypes.POINTER(Params), ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.msgpu_set_data_term.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.msgpu_set_sum_order.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.msgpu_set_certified_steps.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.msgpu_set_seismic_device_control.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.msgpu_set_warm_schedule.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.msgpu_get_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(Stats)]
        L.msgpu_series_params_default.argtypes = [ctypes.POINTER(Params), ctypes.POINTER(SeriesParams)]
        L.msgpu_series_params_default.restype = None
        L.msgpu_match_series.argtypes = [ctypes.c_void_p, ctypes.POINTER(Params), ctypes.POINTER(SeriesParams), _dp,
                                         ctypes.c_int, _dp, _dp, _dp, _dp, _dp]
        L.msgpu_match_series_device.argtypes = [ctypes.c_void_p, ctypes.POINTER(Params),
                                                ctypes.POINTER(SeriesParams), ctypes.c_void_p, ctypes.c_int,
                                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_void_p]
        L.msgpu_compose.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp, _ip]
        L.msgpu_compose_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p]
        L.msgpu_warp_median.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp]
        L.msgpu_warp_median_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.msgpu_io_last_error.restype = ctypes.c_char_p
        L.msgpu_io_last_error.argtypes = []
        L.msgpu_read_array.argtypes = [ctypes.c_char_p, _dp, ctypes.c_longlong, _ip, _ip]
        L.msgpu_write_array.argtypes = [ctypes.c_char_p, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.msgpu_read_arrays.argtypes = [ctypes.POINTER(ctypes.c_char_p), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        _dp, ctypes.c_int]
        L.msgpu_read_displacement.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _dp]
        L.msgpu_write_displacement.argtypes = [ctypes.c_char_p, _dp, ctypes.c_int, ctypes.c_int]
        L.msgpu_read_arrays_start.argtypes = [ctypes.POINTER(ctypes.c_char_p), ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, _dp, ctypes.c_int]
        L.msgpu_read_arrays_start.restype = ctypes.c_void_p
        L.msgpu_io_wait.argtypes = [ctypes.c_void_p]
        _fp = ctypes.POINTER(ctypes.c_float)
        _v = ctypes.c_void_p
        L.msgpu_net_num_params.restype = ctypes.c_longlong
        L.msgpu_net_create.argtypes = [_v, ctypes.c_int, ctypes.c_ulonglong, ctypes.POINTER(_v)]
        L.msgpu_net_destroy.argtypes = [_v]
        L.msgpu_net_input_level.argtypes = [_v]
        L.msgpu_net_set_tensor_cores.argtypes = [_v, ctypes.c_int]
        L.msgpu_net_get_params.argtypes = [_v, _fp]
        L.msgpu_net_set_params.argtypes = [_v, _fp]
        L.msgpu_net_save.argtypes = [_v, ctypes.c_char_p]
        L.msgpu_net_load.argtypes = [_v, ctypes.c_char_p]
        L.msgpu_net_predict_device.argtypes = [_v, _v, ctypes.c_longlong, _v, ctypes.c_int, _v, _v]
        L.msgpu_net_train_step_device.argtypes = [_v, _v, ctypes.c_longlong, _v, _v, ctypes.c_int, ctypes.c_float,
                                                  _fp, _v]
        L.msgpu_net_loss_grad.argtypes = [_v, _dp, _dp, _dp, ctypes.c_int, _fp, _dp, _fp]
        L.msgpu_prepare_images_device.argtypes = [_v, ctypes.POINTER(Params), _v, ctypes.c_int, ctypes.c_int, _v, _v]
        L.msgpu_register_batch_warm.argtypes = [_v, ctypes.POINTER(Params), _v, _dp, _dp, ctypes.c_int, _dp,
                                                ctypes.c_double, _dp, _dp, _ip, _ip]
        L.msgpu_register_batch_warm_device.argtypes = [_v, ctypes.POINTER(Params), _v, _v, _v, ctypes.c_int, _v,
                                                       ctypes.c_double, _v, _v, _v, _ip, _v]
        L.msgpu_lineshift_energy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _dp]
        L.msgpu_lineshift_energy_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        _d = ctypes.c_double
        L.msgpu_xshift_reg.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _d, _d, _dp, _dp, _dp]
        L.msgpu_xshift_reg_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _d, _d,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.msgpu_find_xshift.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp, _d, _d, _d,
                                        ctypes.c_int, _dp, _dp, _ip]
        L.msgpu_find_xshift_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                               ctypes.c_void_p, _d, _d, _d, ctypes.c_int, ctypes.c_void_p, _dp, _ip,
                                               ctypes.c_void_p]
        L.msgpu_find_xshift_yconst.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_int,
                                               _dp, _dp, _ip]
        L.msgpu_find_xshift_yconst_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                      ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, _dp, _ip,
                                                      ctypes.c_void_p]
        L.msgpu_empty_lines_to_nan.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _ip]
        L.msgpu_empty_lines_to_nan_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                      ctypes.c_void_p, _ip, ctypes.c_void_p]
        L.msgpu_remove_empty_lines.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp,
                                               _ip]
        L.msgpu_remove_empty_lines_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                      ctypes.c_int, ctypes.c_void_p, _ip, ctypes.c_void_p]
        L.msgpu_find_xshift_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp,
                                              ctypes.c_int, _dp, _d, _d, _d, ctypes.c_int, _dp, _dp, _ip, ctypes.c_int]
        L.msgpu_register_ragged.argtypes = [ctypes.c_void_p, ctypes.POINTER(Params), ctypes.POINTER(SeriesDesc),
                                            ctypes.c_int]
        L.msgpu_register_ragged_device.argtypes = [ctypes.c_void_p, ctypes.POINTER(Params),
                                                   ctypes.POINTER(SeriesDesc), ctypes.c_int, ctypes.c_void_p]
        L.msgpu_set_wait_limits.argtypes = [ctypes.c_double, ctypes.c_double]
        L.msgpu_warp_sum_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p]
        L.msgpu_mean_from_sums_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        _lib = L
    return _lib


def set_wait_limits(level_wait_s: float = 0.0, barrier_wait_s: float = 0.0) -> None:
    """Bounds of the device-side waits for the whole process (<= 0: defaults
    of 4 s and 2 s); shorter bounds make the waits run out on purpose."""
    st = lib().msgpu_set_wait_limits(level_wait_s, barrier_wait_s)
    if st:
        raise MsgpuError(st, "invalid wait limits")


def default_params(**kw) -> Params:
    p = Params()
    lib().msgpu_params_default(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, "lambda_" if k == "lambda" else k, v)
    return p


# --- on-disk arrays (host only) ------------------------------------------------
def _io_check(st: int):
    if st != MSGPU_OK:
        raise MsgpuError(st, lib().msgpu_io_last_error().decode())


def read_array(path: str) -> np.ndarray:
    """A 2-D array file of the reference's formats as a (numY, numX) float64 array."""
    nx, ny = ctypes.c_int(), ctypes.c_int()
    _io_check(lib().msgpu_read_array(path.encode(), None, 0, ctypes.byref(nx), ctypes.byref(ny)))
    out = np.zeros(nx.value * ny.value)
    _io_check(lib().msgpu_read_array(path.encode(), _p(out), out.size, ctypes.byref(nx), ctypes.byref(ny)))
    return out.reshape(ny.value, nx.value)


def write_array(path: str, a, type_: int = 9):
    a = _f64(a)
    ny, nx = a.shape
    _io_check(lib().msgpu_write_array(path.encode(), _p(a), nx, ny, type_))


def read_arrays(paths, nx: int, ny: int, threads: int = 0) -> np.ndarray:
    """Frames of one size from many files, decoded by host threads; (count, ny, nx)."""
    out = np.zeros((len(paths), ny, nx))
    arr = (ctypes.c_char_p * len(paths))(*[p.encode() for p in paths])
    _io_check(lib().msgpu_read_arrays(arr, len(paths), nx, ny, _p(out), threads))
    return out


class ReadTask:
    """Background decoding of frames into `out` (see msgpu_read_arrays_start)."""

    def __init__(self, paths, nx: int, ny: int, out: np.ndarray, threads: int = 0):
        assert out.dtype == np.float64 and out.flags.c_contiguous and out.size >= len(paths) * nx * ny
        self._out = out
        arr = (ctypes.c_char_p * len(paths))(*[p.encode() for p in paths])
        self._h = lib().msgpu_read_arrays_start(arr, len(paths), nx, ny, _p(out), threads)
        if not self._h:
            _io_check(MSGPU_ERR_INVALID_ARG)

    def wait(self) -> np.ndarray:
        h, self._h = self._h, None
        if h:
            _io_check(lib().msgpu_io_wait(h))
        return self._out


def read_displacement(mask: str, n: int) -> np.ndarray:
    out = np.zeros((2, n * n))
    _io_check(lib().msgpu_read_displacement(mask.encode(), n, n, _p(out)))
    return out


def write_displacement(mask: str, phi, n: int):
    _io_check(lib().msgpu_write_displacement(mask.encode(), _p(_f64(phi).reshape(2, n * n)), n, n))


def default_series_params(params: Params, **kw) -> SeriesParams:
    s = SeriesParams()
    lib().msgpu_series_params_default(ctypes.byref(params), ctypes.byref(s))
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def n_of(level: int) -> int:
    return (1 << level) + 1


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class Context:
    """A msgpu_context bound to one CUDA device."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        st = lib().msgpu_create(device, ctypes.byref(self._h))
        if st != MSGPU_OK:
            raise MsgpuError(st, f"msgpu_create(device={device}) failed (no CUDA device?)")

    def close(self):
        if self._h:
            lib().msgpu_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != MSGPU_OK:
            msg = lib().msgpu_last_error(self._h)
            raise MsgpuError(st, msg.decode() if msg else "")

    # --- batch path -----------------------------------------------------
    def register_batch(self, params: Params, reference, templates, initial_phis=None):
        """Registers every template to the reference; returns (phis[F,2,N], energies[F], steps[F,levels])."""
        ref = _f64(reference).reshape(-1)
        tm = _f64(templates)
        F = tm.shape[0]
        tm = tm.reshape(F, -1)
        N = n_of(params.precision_level) ** 2
        nlev = params.stop_level - params.start_level + 1
        phis = np.zeros((F, 2, N))
        energies = np.zeros(F)
        steps = np.zeros((F, nlev), dtype=np.int32)
        ip = None
        if initial_phis is not None:
            ip = _f64(initial_phis).reshape(F, 2, N)
        self._check(lib().msgpu_register_batch(self._h, ctypes.byref(params), _p(ref), _p(tm), F,
                                               _p(ip) if ip is not None else None, _p(phis), _p(energies),
                                               steps.ctypes.data_as(_ip)))
        return phis, energies, steps

    def register_batch_device(self, params: Params, d_ref: int, d_templates: int, num_templates: int,
                              d_phis_out: int, d_energies: int = 0, d_steps: int = 0, d_init: int = 0,
                              stream: int = 0):
        self._check(lib().msgpu_register_batch_device(self._h, ctypes.byref(params), d_ref, d_templates,
                                                      num_templates, d_init or None, d_phis_out, d_energies or None,
                                                      d_steps or None, stream or None))

    def register_batch_warm(self, params: Params, net: "Net", reference, templates, plain_energies=None,
                            rel_tol: float = 1e-6):
        """register_batch started from the network's prediction at its output
        level (params.start_level stays the plain start, for the fallback);
        returns (phis[F,2,N], energies[F], steps[F,levels], warm_used[F])."""
        ref = _f64(reference).reshape(-1)
        tm = _f64(templates)
        F = tm.shape[0]
        tm = tm.reshape(F, -1)
        N = n_of(params.precision_level) ** 2
        nlev = params.stop_level - params.start_level + 1
        phis = np.zeros((F, 2, N))
        energies = np.zeros(F)
        steps = np.zeros((F, nlev), dtype=np.int32)
        used = np.zeros(F, dtype=np.int32)
        pe = None if plain_energies is None else _f64(plain_energies).reshape(F)
        self._check(lib().msgpu_register_batch_warm(self._h, ctypes.byref(params), net._h, _p(ref), _p(tm), F,
                                                    _p(pe) if pe is not None else None, float(rel_tol), _p(phis),
                                                    _p(energies), steps.ctypes.data_as(_ip),
                                                    used.ctypes.data_as(_ip)))
        return phis, energies, steps, used

    def register_batch_warm_device(self, params: Params, net: "Net", d_ref: int, d_templates: int,
                                   num_templates: int, d_phis_out: int, d_energies: int = 0, d_steps: int = 0,
                                   d_plain_energies: int = 0, rel_tol: float = 1e-6, stream: int = 0):
        """Returns warm_used[F] (host)."""
        used = np.zeros(num_templates, dtype=np.int32)
        self._check(lib().msgpu_register_batch_warm_device(
            self._h, ctypes.byref(params), net._h, d_ref, d_templates, num_templates, d_plain_energies or None,
            float(rel_tol), d_phis_out, d_energies or None, d_steps or None, used.ctypes.data_as(_ip),
            stream or None))
        return used

    def prepare_images_device(self, params: Params, d_images: int, count: int, level: int, d_out: int,
                              stream: int = 0):
        """The registration path's image preparation, restricted to `level`."""
        self._check(lib().msgpu_prepare_images_device(self._h, ctypes.byref(params), d_images, count, level, d_out,
                                                      stream or None))

    def warp_mean(self, level: int, frames, phis):
        fr = _f64(frames)
        F = fr.shape[0]
        N = n_of(level) ** 2
        ph = _f64(phis).reshape(F, 2, N)
        mean = np.zeros(N)
        count = np.zeros(N)
        self._check(lib().msgpu_warp_mean(self._h, level, _p(fr.reshape(F, N)), _p(ph), F, _p(mean), _p(count)))
        return mean, count

    def warp_mean_device(self, level: int, d_frames: int, d_phis: int, num_frames: int, d_mean: int, d_count: int,
                         stream: int = 0):
        self._check(lib().msgpu_warp_mean_device(self._h, level, d_frames, d_phis, num_frames, d_mean, d_count,
                                                 stream or None))

    def warp_sum_device(self, level: int, d_frames: int, d_phis: int, num_frames: int, d_sum: int, d_count: int,
                        d_last_mean: int = 0, stream: int = 0):
        """Per-pixel sums of the finite warped samples and their counts of
        this rank's frames (device pointers); see msgpu_warp_sum_device."""
        self._check(lib().msgpu_warp_sum_device(self._h, level, d_frames, d_phis, num_frames, d_sum, d_count,
                                                d_last_mean or None, stream or None))

    def mean_from_sums_device(self, level: int, d_sum: int, d_count: int, d_fill: int, d_mean: int,
                              stream: int = 0):
        self._check(lib().msgpu_mean_from_sums_device(self._h, level, d_sum, d_count, d_fill, d_mean,
                                                      stream or None))

    def match_series_stage(self, params: Params, reference, templates, out=None):
        """register_batch + warp_mean in one call; returns (phis, energies, steps, mean, count).
        ``out`` may hold preallocated (phis, energies, steps, mean, count) arrays."""
        ref = _f64(reference).reshape(-1)
        tm = _f64(templates)
        F = tm.shape[0]
        tm = tm.reshape(F, -1)
        N = n_of(params.precision_level) ** 2
        nlev = params.stop_level - params.start_level + 1
        if out is None:
            out = (np.zeros((F, 2, N)), np.zeros(F), np.zeros((F, nlev), dtype=np.int32), np.zeros(N), np.zeros(N))
        phis, energies, steps, mean, count = out
        self._check(lib().msgpu_match_series_stage(self._h, ctypes.byref(params), _p(ref), _p(tm), F, _p(phis),
                                                   _p(energies), steps.ctypes.data_as(_ip), _p(mean), _p(count)))
        return out

    def match_series_stage_device(self, params: Params, d_ref: int, d_templates: int, num_templates: int,
                                  d_phis: int, d_energies: int, d_steps: int, d_mean: int, d_count: int,
                                  stream: int = 0):
        self._check(lib().msgpu_match_series_stage_device(self._h, ctypes.byref(params), d_ref, d_templates,
                                                          num_templates, d_phis, d_energies or None, d_steps or None,
                                                          d_mean, d_count, stream or None))

    # --- seismic line-shift model ---------------------------------------------
    def lineshift_energy(self, R, T, phix, with_derivative=True):
        """FELineShiftRegisEnergy of (ny, nx) images; returns (E, DE or None)."""
        R = _f64(R)
        ny, nx = R.shape
        e = ctypes.c_double()
        de = np.zeros((ny, nx)) if with_derivative else None
        self._check(lib().msgpu_lineshift_energy(self._h, nx, ny, _p(R), _p(_f64(T)), _p(_f64(phix)),
                                                 ctypes.byref(e), _p(de) if de is not None else None))
        return e.value, de

    def lineshift_energy_device(self, nx, ny, num_images, d_R, d_T, d_phix, d_energy, d_de, stream):
        """msgpu_lineshift_energy_device on device pointers (d_de may be 0)."""
        self._check(lib().msgpu_lineshift_energy_device(self._h, nx, ny, num_images, d_R, d_T, d_phix, d_energy,
                                                        d_de or None, stream))

    def xshift_reg(self, phix, yreg, laplace_weight=0.0):
        """findXShift's regulariser: (1/2 phi.K phi, K phi)."""
        phix = _f64(phix)
        ny, nx = phix.shape
        e = ctypes.c_double()
        k = np.zeros((ny, nx))
        self._check(lib().msgpu_xshift_reg(self._h, nx, ny, float(yreg), float(laplace_weight), _p(phix),
                                           ctypes.byref(e), _p(k)))
        return e.value, k

    def find_xshift(self, R, T, lam, yreg, max_iter=500, phix=None, laplace_weight=0.0):
        """findXShift: returns (phix (ny, nx), energy, steps)."""
        R = _f64(R)
        ny, nx = R.shape
        ph = np.zeros((ny, nx)) if phix is None else _f64(phix).copy()
        e = ctypes.c_double()
        steps = ctypes.c_int()
        self._check(lib().msgpu_find_xshift(self._h, nx, ny, _p(R), _p(_f64(T)), float(lam), float(yreg),
                                            float(laplace_weight),
                                            int(max_iter), _p(ph), ctypes.byref(e), ctypes.byref(steps)))
        return ph, e.value, steps.value

    def find_xshift_yconst(self, R, T, max_iter=500, phix=None):
        """findXShiftYConst: returns (phix (ny, nx), one value per line; energy; steps of the last descent)."""
        R = _f64(R)
        ny, nx = R.shape
        ph = np.zeros((ny, nx)) if phix is None else _f64(phix).copy()
        e = ctypes.c_double()
        steps = ctypes.c_int()
        self._check(lib().msgpu_find_xshift_yconst(self._h, nx, ny, _p(R), _p(_f64(T)), int(max_iter), _p(ph),
                                                   ctypes.byref(e), ctypes.byref(steps)))
        return ph, e.value, steps.value

    def empty_lines_to_nan(self, img):
        """replaceEmptyLinesWithNaN on a copy of img (ny, nx) or (G, ny, nx); returns (copy, lines replaced)."""
        out = _f64(img).copy()
        nx, ny = out.shape[-1], out.shape[-2]
        n = ctypes.c_int()
        self._check(lib().msgpu_empty_lines_to_nan(self._h, nx, ny, out.size // (nx * ny), _p(out), ctypes.byref(n)))
        return out, n.value

    def remove_empty_lines(self, img, keep_top_bottom=False):
        """removeEmptyLinesFromImage of img (ny, nx); returns the cleaned image (lines, nx)."""
        img = _f64(img)
        ny, nx = img.shape
        out = np.zeros((ny, nx))
        n = ctypes.c_int()
        self._check(lib().msgpu_remove_empty_lines(self._h, nx, ny, _p(img), int(bool(keep_top_bottom)), _p(out),
                                                   ctypes.byref(n)))
        return out[:n.value].copy()

    def empty_lines_to_nan_device(self, d_img, nx, ny, num_images, stream):
        """In place on device memory; returns the number of lines replaced."""
        n = ctypes.c_int()
        self._check(lib().msgpu_empty_lines_to_nan_device(self._h, nx, ny, num_images, d_img, ctypes.byref(n),
                                                          stream))
        return n.value

    def update_non_dyadic_xshift(self, R, T, lam, yreg, phix, laplace_weight=0.0, max_iter=500,
                                 force_yconst=False, prev_energy=float("nan")):
        """The non-dyadic step of XShiftNonDyadicRegistrationMultilevelDescent:
        the empty lines of R and T become NaN (replaceEmptyLinesWithNaN,
        matchSeismicSeries.h:141-157, 179-185), and unless every sample of
        R + T is NaN (matchSeries.h:1217-1221) phix (ny, nx) is refined by
        findXShift, or by findXShiftYConst under forceNonDyadicXShiftYConst
        (matchSeismicSeries.h:195-202).  Returns (phix, energy, steps).  With
        nothing to register the reference skips updateNonDyadicDeformation, so
        its energy of the last solution keeps its previous value: phix comes
        back unchanged with prev_energy (the caller's last energy) and 0 steps."""
        R, _ = self.empty_lines_to_nan(R)
        T, _ = self.empty_lines_to_nan(T)
        if np.isnan(R + T).all():
            return _f64(phix).copy(), float(prev_energy), 0
        if force_yconst:
            return self.find_xshift_yconst(R, T, max_iter, phix)
        return self.find_xshift(R, T, lam, yreg, max_iter, phix, laplace_weight=laplace_weight)

    def find_xshift_batch(self, R, T, lam, yreg, max_iter=500, phix=None, workers=4, laplace_weight=0.0):
        """findXShift for images T (G, ny, nx) against R (ny, nx) or (G, ny, nx);
        returns (phix (G, ny, nx), energies[G], steps[G])."""
        T = _f64(T)
        G, ny, nx = T.shape
        R = _f64(R)
        per = 1 if R.ndim == 3 else 0
        ph = np.zeros((G, ny, nx)) if phix is None else _f64(phix).copy()
        en = np.zeros(G)
        st = np.zeros(G, dtype=np.int32)
        self._check(lib().msgpu_find_xshift_batch(self._h, nx, ny, G, _p(R), per, _p(T), float(lam), float(yreg),
                                                  float(laplace_weight),
                                                  int(max_iter), _p(ph), _p(en), st.ctypes.data_as(_ip),
                                                  int(workers)))
        return ph, en, st

    # --- ragged batches -----------------------------------------------------
    def register_ragged(self, params: Params, series):
        """series: list of (reference, templates) of any sizes 2^l+1 (square);
        returns a list of (phis[F,2,N], energies[F]) in the same order."""
        keep, descs, outs = [], [], []
        for ref, tm in series:
            ref = _f64(ref).reshape(-1)
            tm = _f64(tm)
            F = tm.shape[0]
            tm = tm.reshape(F, -1)
            n = int(round(ref.size ** 0.5))
            level = (n - 1).bit_length() - 1
            if (1 << level) + 1 != n or n * n != ref.size:
                raise ValueError("images must be (2^l+1)^2")
            phis = np.zeros((F, 2, n * n))
            en = np.zeros(F)
            keep += [ref, tm]
            outs.append((phis, en))
            descs.append(SeriesDesc(level, F, ref.ctypes.data, tm.ctypes.data, phis.ctypes.data, en.ctypes.data))
        arr = (SeriesDesc * len(descs))(*descs)
        self._check(lib().msgpu_register_ragged(self._h, ctypes.byref(params), arr, len(descs)))
        return outs

    def register_ragged_device(self, params: Params, descs, stream: int = 0):
        """descs: SeriesDesc entries holding device pointers."""
        arr = (SeriesDesc * len(descs))(*descs)
        self._check(lib().msgpu_register_ragged_device(self._h, ctypes.byref(params), arr, len(descs),
                                                       stream or None))

    # --- series pipeline ----------------------------------------------------
    def match_series(self, params: Params, series: SeriesParams, frames):
        """matchSeries<>(): returns (phis[m,2,N], energies, average, median, count) of the last stage;
        energies holds every stage's per-template energies in order."""
        fr = _f64(frames)
        F = fr.shape[0]
        fr = fr.reshape(F, -1)
        N = n_of(params.precision_level) ** 2
        m = F if series.num_extra_stages > 0 else F - 1
        phis = np.zeros((m, 2, N))
        energies = np.zeros((F - 1) + series.num_extra_stages * F)
        avg, med, cnt = np.zeros(N), np.zeros(N), np.zeros(N)
        self._check(lib().msgpu_match_series(self._h, ctypes.byref(params), ctypes.byref(series), _p(fr), F,
                                             _p(phis), _p(energies), _p(avg), _p(med), _p(cnt)))
        return phis, energies, avg, med, cnt

    def match_series_device(self, params: Params, series: SeriesParams, d_frames: int, num_frames: int,
                            d_phis: int, d_energies: int = 0, d_avg: int = 0, d_median: int = 0, d_count: int = 0,
                            stream: int = 0):
        self._check(lib().msgpu_match_series_device(self._h, ctypes.byref(params), ctypes.byref(series), d_frames,
                                                    num_frames, d_phis, d_energies or None, d_avg or None,
                                                    d_median or None, d_count or None, stream or None))

    def compose(self, level: int, d1, d2, init=None):
        """ConcatAndSmoothlyExtendDeformations; init (default d2) is the solver's initial guess.
        Returns (composition[2,N], pcg_iterations[2])."""
        N = n_of(level) ** 2
        a = _f64(d1).reshape(2, N)
        b = _f64(d2).reshape(2, N)
        out = (b if init is None else _f64(init).reshape(2, N)).copy()
        it = np.zeros(2, dtype=np.int32)
        self._check(lib().msgpu_compose(self._h, level, _p(a), _p(b), _p(out), it.ctypes.data_as(_ip)))
        return out, it

    def compose_device(self, level: int, d_d1: int, d_d2: int, d_inout: int, stream: int = 0):
        self._check(lib().msgpu_compose_device(self._h, level, d_d1, d_d2, d_inout, stream or None))

    def warp_median(self, level: int, frames, phis):
        fr = _f64(frames)
        F = fr.shape[0]
        N = n_of(level) ** 2
        ph = _f64(phis).reshape(F, 2, N)
        med = np.zeros(N)
        self._check(lib().msgpu_warp_median(self._h, level, _p(fr.reshape(F, N)), _p(ph), F, _p(med)))
        return med

    def set_profiling(self, on: bool):
        self._check(lib().msgpu_set_profiling(self._h, int(bool(on))))

    def set_trace(self, level: int, capacity: int = 1 << 20):
        """Record the pass timeline of the level kernel at `level` in
        profiled calls (-1: off); read it with trace()."""
        self._check(lib().msgpu_set_trace(self._h, int(level), int(capacity)))

    def trace(self) -> dict:
        """The pass timeline of the last profiled call: arrays t (ns, from
        the first event), event, cta, value (event codes in msgpu.h)."""
        n = lib().msgpu_get_trace(self._h, None, 0)
        if n < 0:
            raise MsgpuError(MSGPU_ERR_INVALID_ARG, "msgpu_get_trace")
        w = np.zeros(2 * max(n, 1), dtype=np.uint64)
        lib().msgpu_get_trace(self._h, w.ctypes.data, n)
        w = w[:2 * n].reshape(n, 2)
        order = np.argsort(w[:, 0], kind="stable")
        w = w[order]
        t = w[:, 0].astype(np.int64)
        return {"t": t - (t[0] if n else 0), "event": (w[:, 1] >> np.uint64(56)).astype(np.int32),
                "cta": ((w[:, 1] >> np.uint64(32)) & np.uint64(0xFFFFFF)).astype(np.int32),
                "value": (w[:, 1] & np.uint64(0xFFFFFFFF)).astype(np.int64)}

    def tuning(self, fp64: bool, level: int) -> dict:
        t = LevelTuning()
        self._check(lib().msgpu_get_tuning(self._h, int(bool(fp64)), level, ctypes.byref(t)))
        return {"chunk_div": t.chunk_div, "chunk_max": t.chunk_max, "ctas_per_sm": t.ctas_per_sm, "ms": t.ms}

    def set_tuning(self, fp64: bool, level: int, chunk_div: int = 0, chunk_max: int = 0, ctas_per_sm: int = 0,
                   ms: float = 0.0):
        t = LevelTuning(int(chunk_div), int(chunk_max), int(ctas_per_sm), float(ms))
        self._check(lib().msgpu_set_tuning(self._h, int(bool(fp64)), level, ctypes.byref(t)))

    def load_tuning(self, path: str = None):
        """Loads a tuning table (JSON written from msgpu_autotune_device's
        results; default: the table measured on B200 that ships with the
        package) into the context."""
        import json
        path = path or os.path.join(HERE, "tuning_b200.json")
        d = json.load(open(path))
        for prec, levels in d["levels"].items():
            for lv, t in levels.items():
                self.set_tuning(prec == "fp64", int(lv), t["chunk_div"], t["chunk_max"], t["ctas_per_sm"],
                                t.get("ms", 0.0))

    def autotune_device(self, params: Params, d_ref: int, d_templates: int, num_templates: int,
                        d_phis_scratch: int, stream: int = 0) -> dict:
        """msgpu_autotune_device; returns the chosen setting per level."""
        self._check(lib().msgpu_autotune_device(self._h, ctypes.byref(params), d_ref, d_templates, num_templates,
                                                d_phis_scratch, stream or None))
        return {lv: self.tuning(bool(params.use_fp64), lv)
                for lv in range(params.start_level, params.stop_level + 1)}

    def exact_sum_device(self, level: int, d_terms: int, d_out: int, stream: int = 0):
        """The reference-order (sequentially rounded) sum of (2^level+1)^2 doubles."""
        self._check(lib().msgpu_exact_sum_device(self._h, level, d_terms, d_out, stream or None))

    def set_graphs(self, on: bool):
        """CUDA-graph capture and replay of the device batch calls (default on)."""
        self._check(lib().msgpu_set_graphs(self._h, int(bool(on))))

    def stats(self) -> dict:
        s = Stats()
        self._check(lib().msgpu_get_stats(self._h, ctypes.byref(s)))
        k = s.num_levels
        return {"kernel_launches": s.kernel_launches, "first_level": s.first_level,
                "level_ms": list(s.level_ms[:k]), "level_steps": list(s.level_steps[:k]),
                "level_evals": list(s.level_evals[:k]), "level_cluster": list(s.level_cluster[:k]),
                "level_pass_cycles": [dict(zip(PASS_KINDS, list(s.level_pass_cycles[i]))) for i in range(k)],
                "graph_replayed": bool(s.graph_replayed),
                "level_exact_sums": [dict(zip(["passes", "cycles_predict", "certified_steps", "cycles_walk",
                                               "chunks", "chunks_term_by_term", "cycles_term_by_term",
                                               "cycles_walk_warps"], list(s.level_xs[i])))
                                     for i in range(k)]}

    # --- single operators ------------------------------------------------
    def energy(self, level, R, T, phix, phiy, lam, fp64=False):
        N = n_of(level) ** 2
        e = ctypes.c_double()
        de = np.zeros(2 * N)
        self._check(lib().msgpu_energy(self._h, level, _p(_f64(R)), _p(_f64(T)), _p(_f64(phix)), _p(_f64(phiy)),
                                       float(lam), int(fp64), ctypes.byref(e), _p(de)))
        return e.value, de[:N], de[N:]

    def smooth(self, level, sigma, x, fp64=False):
        out = np.zeros(n_of(level) ** 2)
        self._check(lib().msgpu_smooth(self._h, level, float(sigma), int(fp64), _p(_f64(x)), _p(out)))
        return out

    def restrict(self, fine_level, x):
        out = np.zeros(n_of(fine_level - 1) ** 2)
        self._check(lib().msgpu_restrict(self._h, fine_level, _p(_f64(x)), _p(out)))
        return out

    def prolong(self, coarse_level, x):
        out = np.zeros(n_of(coarse_level + 1) ** 2)
        self._check(lib().msgpu_prolong(self._h, coarse_level, _p(_f64(x)), _p(out)))
        return out

    def normalize(self, x, sat=0.15, min_to_zero=1):
        a = _f64(x).reshape(-1)
        out = np.zeros_like(a)
        self._check(lib().msgpu_normalize(self._h, _p(a), a.size, float(sat), int(min_to_zero), _p(out)))
        return out

    def set_data_term(self, data_term: int):
        """0: SSD, 1: normalized cross-correlation, for energy() and gd_level()."""
        self._check(lib().msgpu_set_data_term(self._h, int(data_term)))

    def set_sum_order(self, sum_order: int):
        """0: the reference's sequential order (default), 1: a fixed parallel
        order, for the FP64 sums of energy() and gd_level()."""
        self._check(lib().msgpu_set_sum_order(self._h, int(sum_order)))

    def set_warm_schedule(self, coarse_iters: int):
        """Warm-started batches: step limit of the levels below the stop
        level (0: maxGDIterations)."""
        self._check(lib().msgpu_set_warm_schedule(self._h, int(coarse_iters)))

    def set_seismic_device_control(self, on: bool):
        """findXShift's descent control on the device as one graph, or on
        the host (default, measured faster); the results are the same."""
        self._check(lib().msgpu_set_seismic_device_control(self._h, int(bool(on))))

    def set_certified_steps(self, on: bool):
        """Control steps on bounded sums where the bounds settle them (default
        on); off: every pass's sums added in the reference's order first.
        The results are the same either way."""
        self._check(lib().msgpu_set_certified_steps(self._h, int(bool(on))))

    def gd_level(self, level, R, T, phix, phiy, lam, max_iter, stop_eps=0.0, fp64=False, max_trace=256):
        px = _f64(phix).copy()
        py = _f64(phiy).copy()
        e = ctypes.c_double()
        st = ctypes.c_int()
        tr = np.zeros((max_trace, 4))
        self._check(lib().msgpu_gd_level(self._h, level, _p(_f64(R)), _p(_f64(T)), _p(px), _p(py), float(lam),
                                         int(max_iter), float(stop_eps), int(fp64), ctypes.byref(e),
                                         ctypes.byref(st), _p(tr), max_trace))
        steps = st.value
        return px, py, e.value, steps, tr[:min(steps, max_trace)]

    def gd_level_log(self, level, R, T, phix, phiy, lam, max_iter, stop_eps=0.0, fp64=True):
        """gd_level with the reference's per-level energy log: rows of
        (iteration - 1, lambda * E_reg at the new position, energy)."""
        px = _f64(phix).copy()
        py = _f64(phiy).copy()
        e = ctypes.c_double()
        st = ctypes.c_int()
        lg = np.zeros((max_iter + 1, 3))
        self._check(lib().msgpu_gd_level_log(self._h, level, _p(_f64(R)), _p(_f64(T)), _p(px), _p(py), float(lam),
                                             int(max_iter), float(stop_eps), int(fp64), ctypes.byref(e),
                                             ctypes.byref(st), _p(lg), max_iter + 1))
        return px, py, e.value, st.value, lg[:st.value + 1]


class Net:
    """The learned warm start (msgpu_net): a U-Net from the prepared image
    pair at `input_level` to the displacement at input_level - 1."""

    def __init__(self, ctx: Context, input_level: int = 8, seed: int = 1):
        self.ctx = ctx
        self.level = int(input_level)
        self._h = ctypes.c_void_p()
        ctx._check(lib().msgpu_net_create(ctx._h, self.level, int(seed), ctypes.byref(self._h)))

    @staticmethod
    def num_params() -> int:
        return int(lib().msgpu_net_num_params())

    def close(self):
        if self._h:
            lib().msgpu_net_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_tensor_cores(self, on: bool):
        """Forward convolutions on tcgen05 (default) or on mma.sync."""
        self.ctx._check(lib().msgpu_net_set_tensor_cores(self._h, int(bool(on))))

    def get_params(self):
        out = np.zeros(self.num_params(), dtype=np.float32)
        self.ctx._check(lib().msgpu_net_get_params(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def set_params(self, theta):
        t = np.ascontiguousarray(theta, dtype=np.float32)
        self.ctx._check(lib().msgpu_net_set_params(self._h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def save(self, path: str):
        self.ctx._check(lib().msgpu_net_save(self._h, path.encode()))

    def load(self, path: str):
        self.ctx._check(lib().msgpu_net_load(self._h, path.encode()))

    def predict_device(self, d_R: int, r_stride: int, d_T: int, batch: int, d_phi_out: int, stream: int = 0):
        self.ctx._check(lib().msgpu_net_predict_device(self._h, d_R, int(r_stride), d_T, int(batch), d_phi_out,
                                                       stream or None))

    def train_step_device(self, d_R: int, r_stride: int, d_T: int, d_target: int, batch: int, lr: float,
                          stream: int = 0, want_loss: bool = True):
        loss = ctypes.c_float()
        self.ctx._check(lib().msgpu_net_train_step_device(self._h, d_R, int(r_stride), d_T, d_target, int(batch),
                                                          float(lr), ctypes.byref(loss) if want_loss else None,
                                                          stream or None))
        return loss.value if want_loss else None

    def loss_grad(self, R, T, target):
        """Host arrays R, T [B, n0, n0], target [B, 2, N1] (domain units):
        returns (loss, phi [B, 2, N1], flat gradient)."""
        R = _f64(R)
        B = R.shape[0]
        n1 = (1 << (self.level - 1)) + 1
        phi = np.zeros((B, 2, n1 * n1))
        grad = np.zeros(self.num_params(), dtype=np.float32)
        loss = ctypes.c_float()
        self.ctx._check(lib().msgpu_net_loss_grad(self._h, _p(R), _p(_f64(T)), _p(_f64(target)), B,
                                                  ctypes.byref(loss), _p(phi),
                                                  grad.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return loss.value, phi, grad
