"""goferro_b200 — Python host layer over the B200 engine's C ABI.

The engine itself is ``libgoferro_b200.so`` (built in-tree from ``csrc/`` by
``build.py``); this module binds the entry points declared in
``include/goferro_b200.h`` with ctypes and mirrors the reference's run flow:
a deck directory in, RK4 steps, averages / fields / probes out.

There is no CPU path: if the library is missing or no sm_100 device is
present, ``Engine`` raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import numpy as np

from . import decks  # noqa: F401  (re-exported)

_HERE = os.path.dirname(os.path.abspath(__file__))
# GOFERRO_B200_LIB selects another build of the engine library (a build
# with different tile or occupancy settings); default: the in-tree build
LIB_PATH = os.environ.get("GOFERRO_B200_LIB") or os.path.join(_HERE, "libgoferro_b200.so")

GF_OK = 0
ERRORS = {-1: "GF_EINVAL", -2: "GF_EIO", -3: "GF_ECUDA", -4: "GF_ENOMEM", -5: "GF_ENAN",
          -6: "GF_ENODEV", -7: "GF_EUNSUPPORTED"}

FIELD = {"m": 0, "m_afm1": 1, "m_afm2": 2, "p": 3, "q": 4, "u": 5, "v": 6,
         "Ex": 7, "Ey": 8, "Ez": 9, "Hx": 10, "Hy": 11, "Hz": 12,
         "Hstat": 13, "Estat": 14, "E_cell": 15, "H_cell": 16, "strain": 17}
OBS = {"m": 0, "m_afm1": 1, "m_afm2": 2, "p": 3, "u": 4}
PRECISION = {"fp64": 0, "mixed": 1}   # GF_PRECISION_FP64, GF_PRECISION_MIXED_FP32

# every symbol include/goferro_b200.h declares
EXPORTS = ["gf_create_from_deck", "gf_create_from_deck_ex", "gf_advance", "gf_advance_eager", "gf_average", "gf_probe_em",
           "gf_field_dims", "gf_download", "gf_upload", "gf_download_device", "gf_upload_device",
           "gf_get_info", "gf_profile_steps", "gf_synchronize", "gf_stream", "gf_check_finite", "gf_last_error",
           "gf_destroy", "gf_version", "gf_field_mean_noalloc", "gf_check_quotients",
           "gf_adjoint_create", "gf_adjoint_set_alpha", "gf_adjoint_set_waveform", "gf_adjoint_forward",
           "gf_adjoint_backward", "gf_adjoint_final_m", "gf_adjoint_destroy",
           "gf_batch_create", "gf_batch_advance", "gf_batch_synchronize", "gf_batch_stream", "gf_batch_tuned_chunk",
           "gf_batch_last_error", "gf_batch_destroy", "gf_set_electrostatics",
           "gf_save_state", "gf_load_state"]


class GFInfo(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
                ("dt", ctypes.c_double), ("time", ctypes.c_double),
                ("step", ctypes.c_uint64), ("deck_steps", ctypes.c_uint64),
                ("n_materials", ctypes.c_int32),
                ("fm", ctypes.c_int32), ("afm", ctypes.c_int32), ("fe", ctypes.c_int32),
                ("elastic", ctypes.c_int32), ("em", ctypes.c_int32), ("demag_per_stage", ctypes.c_int32),
                ("n_fm", ctypes.c_uint64), ("n_afm", ctypes.c_uint64), ("n_fe", ctypes.c_uint64),
                ("device_bytes", ctypes.c_uint64),
                ("launches_per_step", ctypes.c_int32), ("precision", ctypes.c_int32)]


class GFKernelTime(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 40), ("launches", ctypes.c_int32), ("total_ms", ctypes.c_double)]


class GFError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load_library(path: Optional[str] = None) -> ctypes.CDLL:
    """Load the engine library (once) and declare the C signatures."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"engine library not built: {p} (run __graft_entry__.build())")
    lib = ctypes.CDLL(p)
    vp, c_int, c_u64, c_dbl_p = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double)
    lib.gf_create_from_deck.argtypes = [ctypes.c_char_p, c_int, ctypes.POINTER(vp)]
    lib.gf_create_from_deck_ex.argtypes = [ctypes.c_char_p, c_int, c_int, ctypes.POINTER(vp)]
    lib.gf_advance.argtypes = [vp, c_u64]
    lib.gf_advance_eager.argtypes = [vp, c_u64]
    lib.gf_average.argtypes = [vp, c_int, c_dbl_p]
    lib.gf_probe_em.argtypes = [vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, c_dbl_p, c_dbl_p]
    lib.gf_field_dims.argtypes = [vp, c_int, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_size_t)]
    lib.gf_download.argtypes = [vp, c_int, c_dbl_p, ctypes.c_size_t]
    lib.gf_upload.argtypes = [vp, c_int, c_dbl_p, ctypes.c_size_t]
    lib.gf_download_device.argtypes = [vp, c_int, vp, ctypes.c_size_t]
    lib.gf_upload_device.argtypes = [vp, c_int, vp, ctypes.c_size_t]
    lib.gf_get_info.argtypes = [vp, ctypes.POINTER(GFInfo)]
    lib.gf_profile_steps.argtypes = [vp, c_u64, ctypes.POINTER(GFKernelTime), c_int, ctypes.POINTER(c_int)]
    lib.gf_synchronize.argtypes = [vp]
    lib.gf_stream.argtypes = [vp]
    lib.gf_stream.restype = vp
    lib.gf_check_finite.argtypes = [vp]
    lib.gf_last_error.argtypes = [vp]
    lib.gf_last_error.restype = ctypes.c_char_p
    lib.gf_destroy.argtypes = [vp]
    lib.gf_destroy.restype = None
    lib.gf_version.restype = ctypes.c_char_p
    lib.gf_field_mean_noalloc.argtypes = [vp, c_u64, ctypes.c_double, vp, vp]
    lib.gf_check_quotients.argtypes = [ctypes.c_double, c_u64, c_u64, ctypes.POINTER(c_u64)]
    lib.gf_adjoint_create.argtypes = [vp, c_int, c_int, ctypes.POINTER(vp)]
    lib.gf_adjoint_set_alpha.argtypes = [vp, c_dbl_p, ctypes.c_size_t]
    lib.gf_adjoint_set_waveform.argtypes = [vp, c_dbl_p, ctypes.c_size_t]
    lib.gf_adjoint_forward.argtypes = [vp, c_u64, c_dbl_p]
    lib.gf_adjoint_backward.argtypes = [vp, c_dbl_p, c_dbl_p, c_dbl_p]
    lib.gf_adjoint_final_m.argtypes = [vp, c_dbl_p, ctypes.c_size_t]
    lib.gf_adjoint_destroy.argtypes = [vp]
    lib.gf_adjoint_destroy.restype = None
    lib.gf_set_electrostatics.argtypes = [vp, c_int, ctypes.POINTER(c_int)]
    lib.gf_save_state.argtypes = [vp, ctypes.c_char_p]
    lib.gf_load_state.argtypes = [vp, ctypes.c_char_p]
    lib.gf_batch_create.argtypes = [ctypes.POINTER(vp), c_int, c_int, ctypes.POINTER(vp)]
    lib.gf_batch_advance.argtypes = [vp, c_u64]
    lib.gf_batch_synchronize.argtypes = [vp]
    lib.gf_batch_stream.argtypes = [vp]
    lib.gf_batch_stream.restype = vp
    lib.gf_batch_tuned_chunk.argtypes = [vp, c_int]
    lib.gf_batch_last_error.argtypes = [vp]
    lib.gf_batch_last_error.restype = ctypes.c_char_p
    lib.gf_batch_destroy.argtypes = [vp]
    lib.gf_batch_destroy.restype = None
    if path is None:
        _lib = lib
    return lib


class Engine:
    """One engine instance (device memory, stream, CUDA graphs) for a deck.

    precision: "fp64" (the parity form) or "mixed" (FP32 state and stencils
    with compensated RK4 accumulation; FP64 at the interface)."""

    def __init__(self, deck_dir: str, device: int = -1, lib: Optional[ctypes.CDLL] = None, precision: str = "fp64"):
        self.lib = lib or load_library()
        h = ctypes.c_void_p()
        rc = self.lib.gf_create_from_deck_ex(os.fsencode(deck_dir), device, PRECISION[precision], ctypes.byref(h))
        if rc != GF_OK:
            raise GFError(rc, self.lib.gf_last_error(None).decode())
        self.h = h
        self.info = self.get_info()

    # -- plumbing --------------------------------------------------------
    def _check(self, rc: int) -> None:
        if rc != GF_OK:
            raise GFError(rc, self.lib.gf_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.gf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- API -------------------------------------------------------------
    def get_info(self) -> GFInfo:
        info = GFInfo()
        self._check(self.lib.gf_get_info(self.h, ctypes.byref(info)))
        return info

    def advance(self, nsteps: int, graph: bool = True) -> None:
        fn = self.lib.gf_advance if graph else self.lib.gf_advance_eager
        self._check(fn(self.h, int(nsteps)))

    def synchronize(self) -> None:
        self._check(self.lib.gf_synchronize(self.h))

    def average(self, obs: str) -> np.ndarray:
        out = (ctypes.c_double * 3)()
        self._check(self.lib.gf_average(self.h, OBS[obs], out))
        return np.array(out[:], dtype=np.float64)

    def probe_em(self, i: int, j: int, k: int) -> Tuple[np.ndarray, np.ndarray]:
        e = (ctypes.c_double * 3)()
        h = (ctypes.c_double * 3)()
        self._check(self.lib.gf_probe_em(self.h, i, j, k, e, h))
        return np.array(e[:]), np.array(h[:])

    def field_dims(self, name: str):
        dims = (ctypes.c_int64 * 3)()
        cnt = ctypes.c_size_t()
        self._check(self.lib.gf_field_dims(self.h, FIELD[name], dims, ctypes.byref(cnt)))
        return tuple(dims[:]), cnt.value

    def download(self, name: str) -> np.ndarray:
        dims, cnt = self.field_dims(name)
        buf = np.empty(cnt, dtype=np.float64)
        self._check(self.lib.gf_download(self.h, FIELD[name], buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), cnt))
        ncomp = cnt // (dims[0] * dims[1] * dims[2])
        return buf.reshape((ncomp,) + dims) if ncomp > 1 else buf.reshape(dims)

    def upload(self, name: str, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        self._check(self.lib.gf_upload(self.h, FIELD[name], a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.size))

    def profile_steps(self, nsteps: int) -> dict:
        """Advance `nsteps` steps with per-launch events; returns
        {kernel family: (launches, total_ms)}."""
        recs = (GFKernelTime * 64)()
        n = ctypes.c_int()
        self._check(self.lib.gf_profile_steps(self.h, int(nsteps), recs, 64, ctypes.byref(n)))
        return {recs[i].name.decode(): (recs[i].launches, recs[i].total_ms) for i in range(n.value)}

    def save_state(self, path: str) -> None:
        self._check(self.lib.gf_save_state(self.h, os.fsencode(path)))

    def load_state(self, path: str) -> None:
        self._check(self.lib.gf_load_state(self.h, os.fsencode(path)))
        self.info = self.get_info()

    def set_electrostatics(self, enable: bool = True) -> int:
        """Enable the electrostatic (depolarisation) solve; returns the
        set-up iteration count."""
        used = ctypes.c_int()
        self._check(self.lib.gf_set_electrostatics(self.h, int(bool(enable)), ctypes.byref(used)))
        return used.value

    def check_finite(self) -> None:
        self._check(self.lib.gf_check_finite(self.h))

    def stream(self) -> int:
        return self.lib.gf_stream(self.h) or 0


def version() -> str:
    return load_library().gf_version().decode()


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Adjoint:
    """Discrete adjoint of an FP64 engine's ferromagnetic RK4 step
    (gf_adjoint_*): <m_x>(t) forward from the engine's current state, and the
    gradients of a loss of that trace with respect to an x-directed
    excitation waveform (n_wave piecewise-constant samples, A/m) and the
    per-cell damping alpha."""

    def __init__(self, engine: "Engine", n_wave: int, checkpoint_every: int = 200):
        self.engine = engine
        self.lib = engine.lib
        self.n_wave = int(n_wave)
        h = ctypes.c_void_p()
        engine._check(self.lib.gf_adjoint_create(engine.h, self.n_wave, int(checkpoint_every), ctypes.byref(h)))
        self.h = h
        self.n = engine.info.nx * engine.info.ny * engine.info.nz
        self.nsteps = None

    def set_alpha(self, alpha: np.ndarray) -> None:
        a = np.ascontiguousarray(alpha, dtype=np.float64).ravel()
        self.engine._check(self.lib.gf_adjoint_set_alpha(self.h, _dp(a), a.size))

    def set_waveform(self, w: np.ndarray) -> None:
        a = np.ascontiguousarray(w, dtype=np.float64).ravel()
        self.engine._check(self.lib.gf_adjoint_set_waveform(self.h, _dp(a), a.size))

    def forward(self, nsteps: int) -> np.ndarray:
        tr = np.empty(int(nsteps) + 1, dtype=np.float64)
        self.engine._check(self.lib.gf_adjoint_forward(self.h, int(nsteps), _dp(tr)))
        self.nsteps = int(nsteps)
        return tr

    def backward(self, dloss_dmx: np.ndarray):
        g = np.ascontiguousarray(dloss_dmx, dtype=np.float64).ravel()
        if self.nsteps is None or g.size != self.nsteps + 1:
            raise ValueError("dloss_dmx needs nsteps+1 values of the last forward run")
        gw = np.empty(self.n_wave, dtype=np.float64)
        ga = np.empty(self.n, dtype=np.float64)
        self.engine._check(self.lib.gf_adjoint_backward(self.h, _dp(g), _dp(gw), _dp(ga)))
        return gw, ga

    def final_m(self) -> np.ndarray:
        m = np.empty(3 * self.n, dtype=np.float64)
        self.engine._check(self.lib.gf_adjoint_final_m(self.h, _dp(m), m.size))
        i = self.engine.info
        return m.reshape(3, i.nx, i.ny, i.nz)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.gf_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Batch:
    """Several engines advanced together by one CUDA graph per step
    (gf_batch_*); with autotune the elastic tile's x-chunk is picked per
    engine by timing.  The engines remain owned by the caller and must not be
    advanced directly while the batch exists."""

    def __init__(self, engines, autotune: bool = True):
        self.engines = list(engines)
        self.lib = self.engines[0].lib
        arr = (ctypes.c_void_p * len(self.engines))(*[e.h.value for e in self.engines])
        h = ctypes.c_void_p()
        rc = self.lib.gf_batch_create(arr, len(self.engines), int(bool(autotune)), ctypes.byref(h))
        if rc != GF_OK:
            raise GFError(rc, self.lib.gf_batch_last_error(None).decode())
        self.h = h

    def _check(self, rc: int) -> None:
        if rc != GF_OK:
            raise GFError(rc, self.lib.gf_batch_last_error(self.h).decode())

    def advance(self, nsteps: int) -> None:
        self._check(self.lib.gf_batch_advance(self.h, int(nsteps)))

    def synchronize(self) -> None:
        self._check(self.lib.gf_batch_synchronize(self.h))

    def stream(self) -> int:
        return self.lib.gf_batch_stream(self.h) or 0

    def tuned_chunk(self, index: int) -> int:
        return int(self.lib.gf_batch_tuned_chunk(self.h, int(index)))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.gf_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
