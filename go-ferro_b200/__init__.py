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
         "Hstat": 13, "Estat": 14, "E_cell": 15, "H_cell": 16, "strain": 17,
         "strain_static": 18, "eigenstrain_static": 19, "force_store": 20, "Jp1": 21, "Jp2": 22, "Jp3": 23}
OBS = {"m": 0, "m_afm1": 1, "m_afm2": 2, "p": 3, "u": 4}
PRECISION = {"fp64": 0, "mixed": 1}   # GF_PRECISION_FP64, GF_PRECISION_MIXED_FP32

# every symbol include/goferro_b200.h declares
EXPORTS = ["gf_create_from_deck", "gf_create_from_deck_ex", "gf_advance", "gf_advance_eager", "gf_average", "gf_probe_em",
           "gf_field_dims", "gf_download", "gf_upload", "gf_download_device", "gf_upload_device",
           "gf_get_info", "gf_profile_steps", "gf_synchronize", "gf_stream", "gf_check_finite", "gf_last_error",
           "gf_destroy", "gf_version", "gf_field_mean_noalloc", "gf_check_quotients",
           "gf_adjoint_create", "gf_adjoint_set_alpha", "gf_adjoint_set_waveform", "gf_adjoint_forward",
           "gf_adjoint_backward", "gf_adjoint_final_m", "gf_adjoint_set_store_limit", "gf_adjoint_store_info",
           "gf_adjoint_destroy",
           "gf_write_outputs", "gf_run_deck", "gf_batch_create", "gf_batch_create_ex", "gf_batch_plan", "gf_batch_advance", "gf_batch_synchronize",
           "gf_batch_stream", "gf_batch_tuned_chunk",
           "gf_batch_last_error", "gf_batch_destroy", "gf_set_electrostatics", "gf_set_elastostatics",
           "gf_save_state", "gf_load_state", "gf_create", "gf_set_table", "gf_stage_begin", "gf_stage_commit",
           "gf_static_solve"]

TABLE = {"Hext": 0, "Eext": 1}      # GF_TABLE_HEXT, GF_TABLE_EEXT
STATIC = {"magnetic": 0, "electric": 1}   # GF_STATIC_MAGNETIC, GF_STATIC_ELECTRIC

_d, _i32, _i64, _u64, _ch = ctypes.c_double, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_char


class GFMaterialParams(ctypes.Structure):
    """gf_material_params: one material as read from materials.in."""
    _fields_ = [("c11", _d), ("c12", _d), ("c44", _d), ("density", _d), ("elast_mass_damping", _d),
                ("elast_stiff_damping", _d), ("if_FM", _i32), ("Ms", _d), ("gyro", _d), ("FM_damping", _d),
                ("anisotropy_type", _i32), ("K1", _d), ("K2", _d), ("Aex", _d), ("iDMI", _d), ("lamda100", _d),
                ("lamda111", _d), ("if_AFM", _i32), ("Ms_AFM", _d * 2), ("gyro_AFM", _d * 2), ("damping_AFM", _d * 2),
                ("K1_AFM", _d * 2), ("uniaxis_AFM", _d * 3), ("Aex_AFM", _d * 2), ("J_AFM", _d),
                ("lamda100_AFM", _d * 2), ("lamda111_AFM", _d * 2), ("if_spin_pump", _i32), ("spin_hall_angle", _d),
                ("spin_mix_cond", _d), ("spin_diffus_length", _d), ("if_FE", _i32), ("FE_mass", _d), ("FE_damping", _d),
                ("a1", _d), ("a11", _d), ("a12", _d), ("a111", _d), ("a112", _d), ("a123", _d), ("a1111", _d),
                ("a1112", _d), ("a1122", _d), ("a1123", _d), ("G11", _d), ("Q11", _d), ("Q12", _d), ("Q44", _d),
                ("f11", _d), ("f12", _d), ("f44", _d), ("if_PEC", _i32), ("r_permittivity", _d), ("conductivity", _d),
                ("comp_n", _d * 3), ("omega_plasma_n", _d * 3), ("tao_e_n", _d * 3)]


class GFRunParams(ctypes.Structure):
    """gf_run_params: the parsed system_setting.in values a run needs."""
    _fields_ = [("nx", _i64), ("ny", _i64), ("nz", _i64), ("dx", _d), ("dy", _d), ("dz", _d),
                ("periodicX", _i32), ("periodicY", _i32), ("periodicZ", _i32),
                ("step", _u64), ("dt", _d), ("if_OrientRotate", _i32), ("Tg2c", (_d * 3) * 3),
                ("theta_mag", _d), ("phi_mag", _d), ("px_init", _d), ("py_init", _d), ("pz_init", _d),
                ("Hext_stat", _d * 3), ("Hext_altr", _d * 3), ("H_altr_freq", _d * 3), ("if_prescribe_Hext", _i32),
                ("Eext_stat", _d * 3), ("Eext_altr", _d * 3), ("E_altr_freq", _d * 3), ("if_prescribe_Eext", _i32),
                ("if_magnetostatics", _i32), ("if_mag_1Dmodel", _i32), ("if_demag_factor", _i32), ("demag_fac", _d * 3),
                ("if_elec_1Dmodel", _i32), ("if_elec_1D_compensate", _i32), ("scale_elec", _d),
                ("elec_solver_limit", _i32), ("elec_solver_tol", _d),
                ("if_EMdynamic", _i32), ("if_input_planeEM_E", _i32), ("planeEM_E", _d * 3), ("planeEM_E_freq", _d * 3),
                ("if_EM_fromP", _i32), ("if_EM_fromM", _i32), ("if_EM_backaction_on_P", _i32),
                ("if_EM_backaction_on_M", _i32), ("if_1D_ABC", _i32), ("if_1D_ABC_ELAST_onlytop", _i32),
                ("if_1D_ABC_EM_onlytop", _i32), ("weighting_factor_fourth_Liao", _d), ("if_PEC_XY", _i32),
                ("if_PEC_Z", _i32), ("if_Jf_input", _i32), ("Jfin_lo", _i64 * 3), ("Jfin_hi", _i64 * 3),
                ("Jf_input_type", _i32), ("Jf_input_component", _ch), ("pad_", _ch * 3), ("Jf_input_amp", _d),
                ("Jf_input_freq", _d), ("Jf_input_sigma", _d), ("num_Jf_cycles", _u64),
                ("if_elastodynamics", _i32), ("if_elasto_backaction_from_pORm", _i32), ("if_elasto_on_pORm", _i32),
                ("if_gaussian_strain_pulse", _i32), ("input_strain_type", _i32), ("input_strain_sourcez", _i32),
                ("input_strain_component", _ch), ("pad2_", _ch * 7), ("sigma_gauss", _d), ("amplitude_gauss", _d),
                ("num_strain_cycles", _u64), ("if_elastostatic", _i32), ("if_flexo", _i32), ("if_prescribed_m", _i32),
                ("if_spin_pumping", _i32), ("scale_elasto", _d), ("elasto_solver_limit", _i32),
                ("elasto_solver_tol", _d)]


def material_params(m) -> GFMaterialParams:
    """gf_material_params of a decks.Material (the values materials.in holds)."""
    p = GFMaterialParams()
    p.c11, p.c12, p.c44, p.density = m.c11, m.c12, m.c44, m.density
    p.elast_mass_damping, p.elast_stiff_damping = m.mass_damping, m.stiff_damping
    p.if_FM, p.Ms, p.gyro, p.FM_damping = int(m.fm), m.Ms, m.gyro, m.alpha
    p.anisotropy_type, p.K1, p.K2, p.Aex, p.iDMI = int(m.aniso_type), m.K1, m.K2, m.Aex, m.iDMI
    p.lamda100, p.lamda111 = m.lam100, m.lam111
    p.if_AFM = int(m.afm)
    p.Ms_AFM[:] = list(m.afm_Ms); p.gyro_AFM[:] = list(m.afm_gyro); p.damping_AFM[:] = list(m.afm_alpha)
    p.K1_AFM[:] = list(m.afm_K1); p.uniaxis_AFM[:] = list(m.afm_axis); p.Aex_AFM[:] = list(m.afm_Aex)
    p.J_AFM = m.J_AFM
    p.lamda100_AFM[:] = list(m.afm_lam100); p.lamda111_AFM[:] = list(m.afm_lam111)
    p.if_spin_pump = int(m.spin_pump)
    p.spin_hall_angle, p.spin_mix_cond, p.spin_diffus_length = m.spin
    p.if_FE, p.FE_mass, p.FE_damping = int(m.fe), m.fe_mass, m.fe_damping
    p.a1, p.a11, p.a12, p.a111, p.a112, p.a123 = m.a1, m.a11, m.a12, m.a111, m.a112, m.a123
    p.a1111, p.a1112, p.a1122, p.a1123 = m.a1111, m.a1112, m.a1122, m.a1123
    p.G11, p.Q11, p.Q12, p.Q44, p.f11, p.f12, p.f44 = m.G11, m.Q11, m.Q12, m.Q44, m.f11, m.f12, m.f44
    p.if_PEC, p.r_permittivity, p.conductivity = int(m.pec), m.er, m.cond
    for k in range(3):
        p.comp_n[k], p.omega_plasma_n[k], p.tao_e_n[k] = m.drude[k]
    return p


def run_params(d) -> GFRunParams:
    """gf_run_params of a decks.Deck (the values system_setting.in holds)."""
    r = GFRunParams()
    r.nx, r.ny, r.nz, r.dx, r.dy, r.dz = d.nx, d.ny, d.nz, d.dx, d.dy, d.dz
    r.periodicX, r.periodicY, r.periodicZ = (int(x) for x in d.periodic)
    r.step, r.dt, r.if_OrientRotate = int(d.steps), d.dt, int(d.Tg2c is not None)
    T = np.eye(3) if d.Tg2c is None else np.asarray(d.Tg2c, dtype=np.float64)
    for i in range(3):
        for j in range(3):
            r.Tg2c[i][j] = float(T[i, j])
    r.theta_mag, r.phi_mag = d.theta_mag, d.phi_mag
    r.px_init, r.py_init, r.pz_init = d.p_init
    r.Hext_stat[:] = list(d.Hext_stat); r.Hext_altr[:] = list(d.Hext_altr); r.H_altr_freq[:] = list(d.H_altr_freq)
    r.if_prescribe_Hext = int(d.Hext_table is not None)
    r.Eext_stat[:] = list(d.Eext_stat); r.Eext_altr[:] = list(d.Eext_altr); r.E_altr_freq[:] = list(d.E_altr_freq)
    r.if_magnetostatics, r.if_mag_1Dmodel, r.if_demag_factor = int(d.magnetostatics), int(d.mag_1D), int(d.demag_factor)
    r.demag_fac[:] = list(d.demag_fac)
    r.scale_elec, r.elec_solver_limit, r.elec_solver_tol = d.scale_elec, int(d.elec_limit), d.elec_tol
    r.if_EMdynamic, r.if_input_planeEM_E = int(d.em), int(d.planeEM)
    r.planeEM_E[:] = list(d.planeEM_E); r.planeEM_E_freq[:] = list(d.planeEM_freq)
    r.if_EM_fromP, r.if_EM_fromM = int(d.em_fromP), int(d.em_fromM)
    r.if_EM_backaction_on_P, r.if_EM_backaction_on_M = int(d.em_back_P), int(d.em_back_M)
    r.if_1D_ABC, r.if_1D_ABC_ELAST_onlytop, r.if_1D_ABC_EM_onlytop = int(d.abc_1D), int(d.abc_elast_onlytop), int(d.abc_em_onlytop)
    r.weighting_factor_fourth_Liao = d.liao_w
    r.if_Jf_input = int(d.jf)
    r.Jfin_lo[:] = list(d.jf_lo); r.Jfin_hi[:] = list(d.jf_hi)
    r.Jf_input_type, r.Jf_input_component = int(d.jf_type), d.jf_comp.encode()
    r.Jf_input_amp, r.Jf_input_freq, r.Jf_input_sigma, r.num_Jf_cycles = d.jf_amp, d.jf_freq, d.jf_sigma, int(d.jf_cycles)
    r.if_elastodynamics, r.if_elasto_backaction_from_pORm, r.if_elasto_on_pORm = int(d.elastic), int(d.elasto_back), int(d.elasto_on)
    r.if_gaussian_strain_pulse, r.input_strain_type, r.input_strain_sourcez = int(d.strain_pulse), int(d.strain_type), int(d.strain_z)
    r.input_strain_component = d.strain_comp.encode()
    r.sigma_gauss, r.amplitude_gauss, r.num_strain_cycles = d.sigma_gauss, d.amp_gauss, int(d.strain_cycles)
    r.if_spin_pumping = int(d.spin_pumping)
    r.if_flexo = int(d.flexo)
    r.if_elastostatic = int(d.elastostatic)
    r.scale_elasto, r.elasto_solver_limit, r.elasto_solver_tol = d.scale_elasto, int(d.elasto_limit), d.elasto_tol
    r.if_elec_1Dmodel, r.if_elec_1D_compensate = int(d.elec_1D), int(d.elec_1D_comp)
    return r


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
    lib.gf_adjoint_set_store_limit.argtypes = [vp, ctypes.c_int64]
    lib.gf_adjoint_store_info.argtypes = [vp, ctypes.POINTER(c_int), ctypes.POINTER(ctypes.c_int64)]
    lib.gf_adjoint_destroy.argtypes = [vp]
    lib.gf_adjoint_destroy.restype = None
    lib.gf_set_electrostatics.argtypes = [vp, c_int, ctypes.POINTER(c_int)]
    lib.gf_set_elastostatics.argtypes = [vp, c_int, ctypes.POINTER(c_int)]
    lib.gf_save_state.argtypes = [vp, ctypes.c_char_p]
    lib.gf_load_state.argtypes = [vp, ctypes.c_char_p]
    lib.gf_write_outputs.argtypes = [vp, ctypes.c_char_p, c_int]
    lib.gf_run_deck.argtypes = [vp, ctypes.c_char_p]
    lib.gf_batch_create.argtypes = [ctypes.POINTER(vp), c_int, c_int, ctypes.POINTER(vp)]
    lib.gf_batch_create_ex.argtypes = [ctypes.POINTER(vp), c_int, c_int, c_int, ctypes.POINTER(vp)]
    lib.gf_batch_plan.argtypes = [vp]
    lib.gf_batch_plan.restype = ctypes.c_char_p
    lib.gf_batch_advance.argtypes = [vp, c_u64]
    lib.gf_batch_synchronize.argtypes = [vp]
    lib.gf_batch_stream.argtypes = [vp]
    lib.gf_batch_stream.restype = vp
    lib.gf_batch_tuned_chunk.argtypes = [vp, c_int]
    lib.gf_batch_last_error.argtypes = [vp]
    lib.gf_batch_last_error.restype = ctypes.c_char_p
    lib.gf_batch_destroy.argtypes = [vp]
    lib.gf_batch_destroy.restype = None
    lib.gf_create.argtypes = [ctypes.POINTER(GFRunParams), ctypes.POINTER(GFMaterialParams), c_int,
                              ctypes.POINTER(ctypes.c_uint32), c_int, c_int, ctypes.POINTER(vp)]
    lib.gf_set_table.argtypes = [vp, c_int, c_dbl_p, c_dbl_p, ctypes.c_int64]
    lib.gf_stage_begin.argtypes = [vp, c_int]
    lib.gf_stage_commit.argtypes = [vp, c_int]
    lib.gf_static_solve.argtypes = [vp, c_int]
    if path is None:
        _lib = lib
    return lib


class Engine:
    """One engine instance (device memory, stream, CUDA graphs) for a deck.

    precision: "fp64" (the parity form) or "mixed" (FP32 state and stencils
    with compensated RK4 accumulation; FP64 at the interface)."""

    def __init__(self, deck_dir: Optional[str], device: int = -1, lib: Optional[ctypes.CDLL] = None,
                 precision: str = "fp64", _handle=None):
        self.lib = lib or load_library()
        if _handle is not None:
            h = _handle
        else:
            h = ctypes.c_void_p()
            rc = self.lib.gf_create_from_deck_ex(os.fsencode(deck_dir), device, PRECISION[precision], ctypes.byref(h))
            if rc != GF_OK:
                raise GFError(rc, self.lib.gf_last_error(None).decode())
        self.h = h
        self.info = self.get_info()

    @classmethod
    def from_params(cls, deck, device: int = -1, precision: str = "fp64", lib: Optional[ctypes.CDLL] = None):
        """Engine from a decks.Deck's values through gf_create (no files):
        the run and material structs, the per-cell ids, then the deck's
        restart arrays through gf_upload and its H table through gf_set_table."""
        lib = lib or load_library()
        run = run_params(deck)
        mats = (GFMaterialParams * len(deck.materials))(*[material_params(m) for m in deck.materials])
        mc = np.ascontiguousarray(deck.material_cell().ravel(), dtype=np.uint32)
        h = ctypes.c_void_p()
        rc = lib.gf_create(ctypes.byref(run), mats, len(deck.materials), mc.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                           device, PRECISION[precision], ctypes.byref(h))
        if rc != GF_OK:
            raise GFError(rc, lib.gf_last_error(None).decode())
        eng = cls(None, lib=lib, _handle=h)
        if deck.Hext_table is not None:
            eng.set_table("Hext", deck.Hext_table[:, 0], deck.Hext_table[:, 1:4])
        for name, arr in (("m", deck.m0), ("m_afm1", None if deck.afm0 is None else deck.afm0[:3]),
                          ("m_afm2", None if deck.afm0 is None else deck.afm0[3:]), ("p", deck.p0), ("q", deck.q0),
                          ("u", deck.u0), ("v", deck.v0)):
            if arr is not None:
                eng.upload(name, arr)
        return eng

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

    def write_outputs(self, directory: str, initial: bool = False) -> None:
        """The reference's text outputs due at the current step (or its
        step-0 block) into directory (gf_write_outputs)."""
        self._check(self.lib.gf_write_outputs(self.h, directory.encode(), int(bool(initial))))

    def run_deck(self, directory: str) -> None:
        """The deck's whole run with the reference's output schedule
        (gf_run_deck)."""
        self._check(self.lib.gf_run_deck(self.h, directory.encode()))

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

    def set_elastostatics(self, enable: bool = True) -> int:
        """Enable the elastostatic (static strain) solve; returns the set-up
        iteration count."""
        used = ctypes.c_int()
        self._check(self.lib.gf_set_elastostatics(self.h, int(bool(enable)), ctypes.byref(used)))
        return used.value

    def check_finite(self) -> None:
        self._check(self.lib.gf_check_finite(self.h))

    def set_table(self, which: str, times: np.ndarray, xyz: np.ndarray) -> None:
        t = np.ascontiguousarray(times, dtype=np.float64)
        v = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        self._check(self.lib.gf_set_table(self.h, TABLE[which], _dp(t), _dp(v), t.size))

    def stage_begin(self, stage: int) -> None:
        self._check(self.lib.gf_stage_begin(self.h, int(stage)))

    def stage_commit(self, stage: int) -> None:
        self._check(self.lib.gf_stage_commit(self.h, int(stage)))

    def static_solve(self, which: str) -> None:
        self._check(self.lib.gf_static_solve(self.h, STATIC.get(which, -1)))

    def stream(self) -> int:
        return self.lib.gf_stream(self.h) or 0


def version() -> str:
    return load_library().gf_version().decode()


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Adjoint:
    """Discrete adjoint of an engine's ferromagnetic RK4 step, with its
    magnetoelastic coupling on elastodynamic decks (gf_adjoint_*): <m_x>(t)
    forward from the engine's current state, and the gradients of a loss of
    that trace with respect to an x-directed excitation waveform (n_wave
    piecewise-constant samples, A/m) and the per-cell damping alpha.  On a
    mixed-form engine the adjoint's fields are FP32 (the gradients FP64)."""

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

    def set_store_limit(self, nbytes: int) -> None:
        """Device memory the backward run may hold for a block's stage store:
        -1 automatic (the default), 0 never (recompute each step's stages),
        or a byte count; both layouts give identical gradients."""
        self.engine._check(self.lib.gf_adjoint_set_store_limit(self.h, int(nbytes)))

    def store_info(self):
        """(used, bytes): whether the last backward run kept the stage store,
        and the memory its layout held."""
        used, nbytes = ctypes.c_int(), ctypes.c_int64()
        self.engine._check(self.lib.gf_adjoint_store_info(self.h, ctypes.byref(used), ctypes.byref(nbytes)))
        return bool(used.value), int(nbytes.value)

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


BATCH_MODES = {"auto": 0, "branches": 1, "phases": 2, "persistent": 3}


class Batch:
    """Several engines advanced together by one CUDA graph per step
    (gf_batch_*).  mode "phases": mixed-form TDGL / elastodynamics / FDTD
    engines, each RK stage a few launches over the work items of every
    engine; "persistent": the same engines and work items, the whole step as
    one cooperative launch with grid barriers between the phases;
    "branches": one graph branch per engine; "auto": branches when some
    engine does not allow the phase mode, else (with autotune) the fastest
    of the three over timed steps.  With autotune the tile x-chunk (and, in
    the phase mode, the fusion of phase A) is picked by timing; plan()
    describes the choice.  The engines remain owned by the caller and must not be
    advanced directly while the batch exists."""

    def __init__(self, engines, autotune: bool = True, mode: str = "auto"):
        self.engines = list(engines)
        self.lib = self.engines[0].lib
        arr = (ctypes.c_void_p * len(self.engines))(*[e.h.value for e in self.engines])
        h = ctypes.c_void_p()
        rc = self.lib.gf_batch_create_ex(arr, len(self.engines), int(bool(autotune)), BATCH_MODES[mode], ctypes.byref(h))
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

    def plan(self) -> str:
        return self.lib.gf_batch_plan(self.h).decode()

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
