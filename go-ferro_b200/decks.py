"""GO-Ferro input decks: writer, seeded initial conditions and the run presets.

The decks are the reference's positional text files (read.cpp:4-237):
``system_setting.in`` (8-line geometry block, then one item group per line),
``materials.in`` (a title line and the fields of each material) and the
optional restart / table files (``m.in``, ``p.in``, ``q.in``, ``Hext.in``, ...).
The same deck directory drives the reference (its oracle build) and this
engine (``gf_create_from_deck``), so a run is defined once.

Seeded initial conditions use SplitMix64 (seed = 20241203 + preset number) in
cell storage order; a cell's draws are consumed in component order.
"""
from __future__ import annotations

import dataclasses
import math
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

MU0 = 1.256637061e-6          # magnetic_system.h:14
C0 = 2.99792458e8             # EMdynamic_system.h:14
ETA0 = 376.730313668          # vacuum impedance mu0*c


# --------------------------------------------------------------------------
# seeded random numbers
# --------------------------------------------------------------------------
def splitmix64(seed: int, count: int) -> np.ndarray:
    """`count` uniform doubles in [0,1) from SplitMix64 (53-bit mantissa)."""
    mask = (1 << 64) - 1
    out = np.empty(count, dtype=np.float64)
    # vectorised: state_i = seed + (i+1) * golden
    golden = np.uint64(0x9E3779B97F4A7C15)
    idx = np.arange(1, count + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed & mask) + idx * golden
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    out[:] = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return out


# --------------------------------------------------------------------------
# materials
# --------------------------------------------------------------------------
@dataclass
class Material:
    """Fields of one materials.in entry, in read order (read.cpp:121-205)."""
    title: str = "material"
    c11: float = 0.0
    c12: float = 0.0
    c44: float = 0.0
    density: float = 1.0
    mass_damping: float = 0.0
    stiff_damping: float = 0.0
    fm: bool = False
    Ms: float = 0.0
    gyro: float = 0.0
    alpha: float = 0.0
    aniso_type: int = 0
    K1: float = 0.0
    K2: float = 0.0
    Aex: float = 0.0
    iDMI: float = 0.0
    lam100: float = 0.0
    lam111: float = 0.0
    afm: bool = False
    afm_Ms: tuple = (0.0, 0.0)
    afm_gyro: tuple = (0.0, 0.0)
    afm_alpha: tuple = (0.0, 0.0)
    afm_K1: tuple = (0.0, 0.0)
    afm_axis: tuple = (0.0, 0.0, 1.0)
    afm_Aex: tuple = (0.0, 0.0)
    J_AFM: float = 0.0
    afm_lam100: tuple = (0.0, 0.0)
    afm_lam111: tuple = (0.0, 0.0)
    spin_pump: bool = False
    spin: tuple = (0.0, 0.0, 1.0)
    fe: bool = False
    fe_mass: float = 0.0
    fe_damping: float = 0.0
    a1: float = 0.0
    a11: float = 0.0
    a12: float = 0.0
    a111: float = 0.0
    a112: float = 0.0
    a123: float = 0.0
    a1111: float = 0.0
    a1112: float = 0.0
    a1122: float = 0.0
    a1123: float = 0.0
    G11: float = 0.0
    Q11: float = 0.0
    Q12: float = 0.0
    Q44: float = 0.0
    f11: float = 0.0
    f12: float = 0.0
    f44: float = 0.0
    pec: bool = False
    er: float = 1.0
    cond: float = 0.0
    # Drude poles: (weight, plasma frequency, relaxation time); weight 1 on
    # pole 1 with zero plasma frequency is "no dispersion" (the reference
    # normalises the weights, global.cpp:360-362)
    drude: tuple = ((1.0, 0.0, 1.0), (0.0, 0.0, 1.0), (0.0, 0.0, 1.0))


def _b(v: bool) -> str:
    return "true" if v else "false"


def _f(v: float) -> str:
    return repr(float(v))


def material_text(m: Material) -> str:
    L = [m.title,
         f"{_f(m.c11)} {_f(m.c12)} {_f(m.c44)}",
         _f(m.density),
         f"{_f(m.mass_damping)} {_f(m.stiff_damping)}",
         _b(m.fm),
         f"{_f(m.Ms)} {_f(m.gyro)} {_f(m.alpha)}",
         str(int(m.aniso_type)),
         f"{_f(m.K1)} {_f(m.K2)}",
         _f(m.Aex),
         _f(m.iDMI),
         f"{_f(m.lam100)} {_f(m.lam111)}",
         _b(m.afm),
         " ".join(_f(x) for x in m.afm_Ms),
         " ".join(_f(x) for x in m.afm_gyro),
         " ".join(_f(x) for x in m.afm_alpha),
         " ".join(_f(x) for x in m.afm_K1),
         " ".join(_f(x) for x in m.afm_axis),
         " ".join(_f(x) for x in m.afm_Aex),
         _f(m.J_AFM),
         " ".join(_f(x) for x in m.afm_lam100),
         " ".join(_f(x) for x in m.afm_lam111),
         _b(m.spin_pump),
         " ".join(_f(x) for x in m.spin),
         _b(m.fe),
         f"{_f(m.fe_mass)} {_f(m.fe_damping)}",
         _f(m.a1),
         f"{_f(m.a11)} {_f(m.a12)}",
         f"{_f(m.a111)} {_f(m.a112)} {_f(m.a123)}",
         f"{_f(m.a1111)} {_f(m.a1112)} {_f(m.a1122)} {_f(m.a1123)}",
         _f(m.G11),
         f"{_f(m.Q11)} {_f(m.Q12)} {_f(m.Q44)}",
         f"{_f(m.f11)} {_f(m.f12)} {_f(m.f44)}",
         _b(m.pec),
         _f(m.er),
         _f(m.cond)]
    for w, wp, tau in m.drude:
        L.append(f"{_f(w)} {_f(wp)} {_f(tau)}")
    return "\n".join(L) + "\n"


# --------------------------------------------------------------------------
# deck
# --------------------------------------------------------------------------
@dataclass
class Deck:
    """One run: geometry, switches, materials and initial-condition arrays.

    Field names follow global.h:30-176; the writer emits them in the order
    read.cpp expects.
    """
    nx: int = 8
    ny: int = 8
    nz: int = 8
    dx: float = 2e-9
    dy: float = 2e-9
    dz: float = 2e-9
    periodic: tuple = (True, True, False)
    nx_work: Optional[int] = None
    ny_work: Optional[int] = None
    layers: List[tuple] = field(default_factory=lambda: [(8, 1)])   # (nz, material id) bottom -> top
    steps: int = 10
    dt: float = 1e-15
    materials: List[Material] = field(default_factory=list)
    theta_mag: float = 0.0
    phi_mag: float = 0.0
    p_init: tuple = (0.0, 0.0, 0.0)
    Hext_stat: tuple = (0.0, 0.0, 0.0)
    Hext_altr: tuple = (0.0, 0.0, 0.0)
    H_altr_freq: tuple = (0.0, 0.0, 0.0)
    Eext_stat: tuple = (0.0, 0.0, 0.0)
    Eext_altr: tuple = (0.0, 0.0, 0.0)
    E_altr_freq: tuple = (0.0, 0.0, 0.0)
    magnetostatics: bool = False
    mag_1D: bool = False
    demag_factor: bool = False
    demag_fac: tuple = (0.0, 0.0, 1.0)
    em: bool = False
    planeEM: bool = False
    planeEM_E: tuple = (0.0, 0.0, 0.0)
    planeEM_freq: tuple = (0.0, 0.0, 0.0)
    em_fromP: bool = False
    em_fromM: bool = False
    em_back_P: bool = False
    em_back_M: bool = False
    elastic: bool = False
    # electrostatic solver settings (read.cpp:56): scale of the homogeneous
    # reference permittivity, iteration limit, tolerance
    spin_pumping: bool = False
    flexo: bool = False          # if_flexo (flexoelectric coupling)
    # text-output schedule of the time loop: output name -> step interval
    # (absent or 0 = off); names follow the deck's if_output_* switches:
    # ave, m, magcell, AFMm, p, em, em_onecell, strain, Hstat, Estat, eig0,
    # q, uv, force, emYee, Jp, Jishe; em_onecell_index is 1-based
    outputs: dict = field(default_factory=lambda: {"ave": 1})
    # prescribed-m test mode (if_prescribed_m): k = 0 ferromagnetic cells
    # precess on a cone of precess_angle degrees at precess_freq Hz
    prescribed_m: bool = False
    precess_angle: float = 0.0
    precess_freq: float = 0.0
    em_onecell_index: int = 0
    # electrostatics: 1-D model and its compensation (if_elec_1Dmodel,
    # if_elec_1D_compensate)
    elec_1D: bool = False
    elec_1D_comp: bool = False
    # static strain: if_elastostatic, the solver settings of read.cpp:64, and
    # the restart inputs strain_stat.in (global frame) / eigenstraint0_crt.in
    # (crystal frame), each (6, nx, ny, nz) in xx yy zz yz xz xy order
    elastostatic: bool = False
    scale_elasto: float = 1.0
    elasto_limit: int = 0
    elasto_tol: float = 1e-8
    strain_t0: Optional[np.ndarray] = None
    eig_t0: Optional[np.ndarray] = None
    scale_elec: float = 1.0
    elec_limit: int = 0
    elec_tol: float = 1e-8
    elasto_back: bool = False
    elasto_on: bool = False
    strain_pulse: bool = False
    strain_type: int = 2
    strain_z: int = 0
    strain_comp: str = "x"
    sigma_gauss: float = 0.0
    amp_gauss: float = 0.0
    strain_cycles: int = 0
    abc_1D: bool = False
    abc_elast_onlytop: bool = False
    abc_em_onlytop: bool = False
    liao_w: float = 0.5
    jf: bool = False
    jf_lo: tuple = (0, 0, 0)
    jf_hi: tuple = (0, 0, 0)
    jf_type: int = 0
    jf_comp: str = "x"
    jf_amp: float = 0.0
    jf_freq: float = 0.0
    jf_sigma: float = 0.0
    jf_cycles: int = 0
    # initial conditions / tables (None = deck's own uniform initialisation)
    m0: Optional[np.ndarray] = None        # (3, nx, ny, nz)
    afm0: Optional[np.ndarray] = None      # (6, nx, ny, nz): m1 then m2
    p0: Optional[np.ndarray] = None
    q0: Optional[np.ndarray] = None
    u0: Optional[np.ndarray] = None
    v0: Optional[np.ndarray] = None
    force0: Optional[np.ndarray] = None    # (3, nx, ny, nz): elastoforce.in (stiffness-damping force store)
    jp0: Optional[list] = None             # three (3, nx, ny, nz): Jp1.in..Jp3.in (Drude pole currents)
    Hext_table: Optional[np.ndarray] = None    # (K, 4): t Hx Hy Hz
    # crystal orientation: Tg2c, the global-to-crystal rotation (3x3); when
    # set, if_OrientRotate is true (read.cpp:30-37; Tc2g is its transpose)
    Tg2c: Optional[np.ndarray] = None
    # per-cell material ids (nx, ny, nz); when set, if_read_struct is true and
    # struct.in replaces the layer stack's cell assignment (read.cpp:280-294,
    # global.cpp:67-83)
    struct: Optional[np.ndarray] = None
    name: str = "deck"

    @property
    def n(self) -> int:
        return self.nx * self.ny * self.nz

    def material_cell(self) -> np.ndarray:
        """Per-cell material id as set_global builds it (global.cpp:65-83)."""
        if self.struct is not None:
            return np.asarray(self.struct, dtype=np.uint8).reshape(self.nx, self.ny, self.nz).copy()
        mc = np.zeros((self.nx, self.ny, self.nz), dtype=np.uint8)
        nxw = self.nx if self.nx_work is None else self.nx_work
        nyw = self.ny if self.ny_work is None else self.ny_work
        i0, j0 = (self.nx - nxw) // 2, (self.ny - nyw) // 2
        z = 0
        for nzl, mid in self.layers:
            mc[i0:i0 + nxw, j0:j0 + nyw, z:z + nzl] = mid
            z += nzl
        return mc

    def _out(self, name: str) -> str:
        step = int(self.outputs.get(name, 0))
        return f"{_b(step > 0)} {max(step, 1)}"

    def system_setting_text(self) -> str:
        nxw = self.nx if self.nx_work is None else self.nx_work
        nyw = self.ny if self.ny_work is None else self.ny_work
        nl = len(self.layers)
        L = [f"{self.nx} {self.ny} {self.nz}",
             f"{_f(self.dx)} {_f(self.dy)} {_f(self.dz)}",
             " ".join(_b(v) for v in self.periodic),
             _b(self.struct is not None),
             f"{nxw} {nyw}",
             str(nl),
             f"1 1 {nl}",
             " ".join(str(int(l[0])) for l in self.layers),
             str(int(self.steps)),
             _f(self.dt),
             str(len(self.materials)),
             " ".join(str(int(l[1])) for l in self.layers),
             _b(self.Tg2c is not None),
             *(" ".join(_f(x) for x in row) for row in (np.eye(3) if self.Tg2c is None else np.asarray(self.Tg2c))),
             f"{_f(self.theta_mag)} {_f(self.phi_mag)}",
             " ".join(_f(x) for x in self.p_init),
             "false",
             " ".join(_f(x) for x in self.Hext_stat),
             " ".join(_f(x) for x in self.Hext_altr),
             " ".join(_f(x) for x in self.H_altr_freq),
             f"{_b(self.Hext_table is not None)} {0 if self.Hext_table is None else len(self.Hext_table)}",
             " ".join(_f(x) for x in self.Eext_stat),
             " ".join(_f(x) for x in self.Eext_altr),
             " ".join(_f(x) for x in self.E_altr_freq),
             "false 0",
             f"{_b(self.magnetostatics)} {_b(self.mag_1D)}",
             f"{_b(self.demag_factor)} " + " ".join(_f(x) for x in self.demag_fac),
             f"{_b(self.elec_1D)} {_b(self.elec_1D_comp)}",
             f"{_b(self.em)} {_b(self.planeEM)}",
             " ".join(_f(x) for x in self.planeEM_E),
             " ".join(_f(x) for x in self.planeEM_freq),
             f"{_b(self.em_fromP)} {_b(self.em_fromM)}",
             f"{_b(self.em_back_P)} {_b(self.em_back_M)}",
             "0 0 0.0",
             f"{_f(self.scale_elec)} {int(self.elec_limit)} {_f(self.elec_tol)}",
             f"{_b(self.elastic)} {_b(self.elasto_back)} {_b(self.elasto_on)}",
             f"{_b(self.strain_pulse)} {int(self.strain_type)} {int(self.strain_z)}",
             f"{self.strain_comp} {_f(self.sigma_gauss)} {_f(self.amp_gauss)} {int(self.strain_cycles)}",
             f"{_b(self.elastostatic)} false",
             "false false",
             "0 0 0.0 0.0 0.0",
             f"{_f(self.scale_elasto)} {int(self.elasto_limit)} {_f(self.elasto_tol)}",
             f"{_b(self.abc_1D)} {_b(self.abc_elast_onlytop)} {_b(self.abc_em_onlytop)} {_f(self.liao_w)}",
             "false false",
             f"{_b(self.flexo)}",
             f"{_b(self.spin_pumping)}",
             f"{_b(self.m0 is not None)} {_b(self.afm0 is not None)} false",
             f"{_b(self.p0 is not None)} false",
             f"false {_b(self.jp0 is not None)}",
             f"{_b(self.u0 is not None)} {_b(self.strain_t0 is not None)} {_b(self.eig_t0 is not None)}",
             _b(self.force0 is not None),
             self._out("ave"),
             f"{self._out('m')} {self._out('magcell')}",
             self._out("AFMm"),
             self._out("p"),
             f"{self._out('em')} {self._out('em_onecell')} {int(self.em_onecell_index)}",
             self._out("strain"),
             self._out("Hstat"),
             self._out("Estat"),
             self._out("eig0"),
             self._out("q"),
             self._out("uv"),
             self._out("force"),
             self._out("emYee"),
             self._out("Jp"),
             self._out("Jishe"),
             _b(self.jf),
             " ".join(str(int(x)) for x in self.jf_lo),
             " ".join(str(int(x)) for x in self.jf_hi),
             f"{int(self.jf_type)} {self.jf_comp} {_f(self.jf_amp)} {_f(self.jf_freq)} {_f(self.jf_sigma)} {int(self.jf_cycles)}",
             f"{_b(self.prescribed_m)} {_f(self.precess_angle)} {_f(self.precess_freq)}"]
        return "\n".join(L) + "\n"


def _write_restart(path: str, arr: np.ndarray) -> None:
    """'i j k a b c' lines, 1-based, %.17e (inoutput.cpp:11-27 layout)."""
    ncomp, nx, ny, nz = arr.shape
    ii, jj, kk = np.meshgrid(np.arange(1, nx + 1), np.arange(1, ny + 1), np.arange(1, nz + 1), indexing="ij")
    cols = [ii.ravel(), jj.ravel(), kk.ravel()] + [arr[c].ravel() for c in range(ncomp)]
    fmt = "%d %d %d" + " %.17e" * ncomp
    data = np.column_stack(cols)
    np.savetxt(path, data, fmt=fmt)


def write_deck(deck: Deck, directory: str) -> str:
    """Write every file of `deck` into `directory` (created if needed)."""
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, "system_setting.in"), "w") as f:
        f.write(deck.system_setting_text())
    with open(os.path.join(directory, "materials.in"), "w") as f:
        for m in deck.materials:
            f.write(material_text(m))
    if deck.m0 is not None:
        _write_restart(os.path.join(directory, "m.in"), deck.m0)
    if deck.afm0 is not None:
        _write_restart(os.path.join(directory, "m_AFM.in"), deck.afm0)
    if deck.p0 is not None:
        _write_restart(os.path.join(directory, "p.in"), deck.p0)
        q = deck.q0 if deck.q0 is not None else np.zeros_like(deck.p0)
        _write_restart(os.path.join(directory, "q.in"), q)
    if deck.u0 is not None:
        _write_restart(os.path.join(directory, "u.in"), deck.u0)
        v = deck.v0 if deck.v0 is not None else np.zeros_like(deck.u0)
        _write_restart(os.path.join(directory, "v.in"), v)
    if deck.force0 is not None:
        _write_restart(os.path.join(directory, "elastoforce.in"), deck.force0)
    if deck.jp0 is not None:
        for pole, a in enumerate(deck.jp0):
            _write_restart(os.path.join(directory, f"Jp{pole + 1}.in"), a)
    if deck.strain_t0 is not None:
        _write_restart(os.path.join(directory, "strain_stat.in"), deck.strain_t0)
    if deck.eig_t0 is not None:
        _write_restart(os.path.join(directory, "eigenstraint0_crt.in"), deck.eig_t0)
    if deck.Hext_table is not None:
        np.savetxt(os.path.join(directory, "Hext.in"), deck.Hext_table, fmt="%.17e")
    if deck.struct is not None:
        # one line per cell: x y z id, 1-based coordinates
        mc = deck.material_cell()
        i, j, k = np.meshgrid(np.arange(deck.nx), np.arange(deck.ny), np.arange(deck.nz), indexing="ij")
        rows = np.stack([i.ravel() + 1, j.ravel() + 1, k.ravel() + 1, mc.ravel().astype(np.int64)], axis=1)
        np.savetxt(os.path.join(directory, "struct.in"), rows, fmt="%d")
    return directory


# --------------------------------------------------------------------------
# material sets used by the presets
# --------------------------------------------------------------------------
def yig(alpha: float = 0.01, magnetoelastic: bool = False) -> Material:
    """YIG-like ferrimagnet treated as a ferromagnet (FM and magnetoelastic presets)."""
    c11, c12, c44 = 2.69e11, 1.077e11, 0.764e11
    lam100 = lam111 = 0.0
    if magnetoelastic:
        B1, B2 = 3.48e5, 6.96e5
        lam100 = -2.0 * B1 / (3.0 * (c11 - c12))      # inverse of read.cpp:141
        lam111 = -B2 / (3.0 * c44)                     # inverse of read.cpp:142
    return Material(title="YIG", c11=c11, c12=c12, c44=c44, density=5170.0,
                    fm=True, Ms=1.4e5, gyro=1.76e11 * MU0, alpha=alpha, aniso_type=1,
                    K1=-610.0, K2=0.0, Aex=3.7e-12, lam100=lam100, lam111=lam111, er=15.0)


def ggg() -> Material:
    """GGG-like non-magnetic garnet substrate (constants chosen for the
    coupled magnetoelastic preset)."""
    return Material(title="GGG", c11=2.86e11, c12=1.16e11, c44=0.905e11, density=7080.0, er=12.0)


def afm_uniaxial(alpha: float = 0.01, magnetoelastic: bool = False) -> Material:
    """Two-sublattice uniaxial antiferromagnet (NiO-like magnitudes; easy
    axis z, inter-sublattice exchange field of order 10^7 A/m), on GGG-like
    elastic constants."""
    lam = (2e-5, 2e-5) if magnetoelastic else (0.0, 0.0)
    return Material(title="AFM", c11=2.86e11, c12=1.16e11, c44=0.905e11, density=6800.0,
                    afm=True, afm_Ms=(4.0e5, 4.0e5), afm_gyro=(1.76e11 * MU0, 1.76e11 * MU0),
                    afm_alpha=(alpha, alpha), afm_K1=(2.0e4, 2.0e4), afm_axis=(0.0, 0.0, 1.0),
                    afm_Aex=(2.0e-12, 2.0e-12), J_AFM=5.0e6, afm_lam100=lam, afm_lam111=lam, er=12.0)


def tilt_afm0(shape, seed: int, mc: np.ndarray, max_deg: float = 2.0) -> np.ndarray:
    """m1 along +z and m2 along -z in cells where mc is true, each tilted by
    an independent seeded angle of at most max_deg (splitmix64 draws)."""
    a = tilt_m0(shape, seed, mc, max_deg)
    b = -tilt_m0(shape, seed + 7, mc, max_deg)
    return np.concatenate([a, b], axis=0)


def pto() -> Material:
    """PbTiO3-like ferroelectric at 300 K (ferroelectric preset).  FE mass,
    damping, gradient coefficient and background permittivity are chosen
    here."""
    return Material(title="PTO", c11=2.3e11, c12=1.0e11, c44=1.2e11, density=7.9e3,
                    fe=True, fe_mass=1.7e-18, fe_damping=1.7e-6,
                    a1=3.8e5 * (300.0 - 479.0), a11=-7.3e7, a12=7.5e8,
                    a111=2.6e8, a112=6.1e8, a123=-3.7e9,
                    G11=5.1e-10, Q11=0.089, Q12=-0.026, Q44=0.0675, er=10.0)


def rotation(ax_deg: float, az_deg: float) -> np.ndarray:
    """An orthogonal global-to-crystal rotation: az_deg about z, then ax_deg
    about x."""
    a, b = math.radians(ax_deg), math.radians(az_deg)
    rz = np.array([[math.cos(b), -math.sin(b), 0.0], [math.sin(b), math.cos(b), 0.0], [0.0, 0.0, 1.0]])
    rx = np.array([[1.0, 0.0, 0.0], [0.0, math.cos(a), -math.sin(a)], [0.0, math.sin(a), math.cos(a)]])
    return rx @ rz


def tilt_m0(shape, seed: int, mc: np.ndarray, max_deg: float = 1.0) -> np.ndarray:
    """m along z with a uniform random tilt theta in [0, max_deg] degrees and
    azimuth in [0, 2 pi), one pair of draws per cell in storage order; zero in
    non-magnetic cells."""
    nx, ny, nz = shape
    r = splitmix64(seed, 2 * nx * ny * nz).reshape(nx * ny * nz, 2)
    th = np.deg2rad(max_deg) * r[:, 0]
    ph = 2.0 * np.pi * r[:, 1]
    m = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)]).reshape(3, nx, ny, nz)
    return m * (mc != 0)[None]


def gaussian_derivative_pulse(steps: int, dt: float, peak_T: float, sigma: float, bias_T: float) -> np.ndarray:
    """Prescribed H table (Hext.in): row i at t_i = i*dt holds
    Hx = (peak/mu0) sqrt(e) ((t-5s)/s) exp(-(t-5s)^2/(2 s^2)), Hz = bias/mu0."""
    t = np.arange(steps + 1, dtype=np.float64) * dt
    a = (t - 5.0 * sigma) / sigma
    hx = (peak_T / MU0) * math.sqrt(math.e) * a * np.exp(-0.5 * a * a)
    hz = np.full_like(t, bias_T / MU0)
    return np.column_stack([t, hx, np.zeros_like(t), hz])


# --------------------------------------------------------------------------
# presets (the three benchmark workloads, optionally scaled down for tests)
# --------------------------------------------------------------------------
def preset_fm_demag(nx=64, ny=64, nz=16, steps=4000, dt=5e-15) -> Deck:
    """FM LLG + FFT magnetostatics, YIG-like, 0.1 T bias along z,
    1 mT Gaussian-derivative x pulse of 1 ps width, seeded <=1 deg tilt."""
    d = Deck(nx=nx, ny=ny, nz=nz, dx=2e-9, dy=2e-9, dz=2e-9, periodic=(True, True, False),
             layers=[(nz, 1)], steps=steps, dt=dt, materials=[yig(0.01)],
             magnetostatics=True, name=f"fm_demag_{nx}x{ny}x{nz}")
    d.m0 = tilt_m0((nx, ny, nz), 20241203 + 1, d.material_cell())
    d.Hext_table = gaussian_derivative_pulse(steps, dt, 1e-3, 1e-12, 0.1)
    return d


def preset_magnetoelastic(nx=128, ny=128, nz=96, sub=56, film=32, steps=10000, dt=None) -> Deck:
    """Magnetoelastic YIG film on a GGG-like substrate with
    elastodynamics and Maxwell FDTD; bottom-plane 0.3 THz shear source of
    1 pm amplitude; vacuum above the film; Courant-limited dt."""
    dx = 2e-9
    vac = nz - sub - film
    assert vac >= 0
    if dt is None:
        dt = 0.9 * 2.0 * math.sqrt(2.0) * dx / (2.0 * math.sqrt(3.0) * C0)
    layers = [(sub, 1), (film, 2)] + ([(vac, 0)] if vac > 0 else [])
    d = Deck(nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, dz=dx, periodic=(True, True, False), layers=layers,
             steps=steps, dt=dt, materials=[ggg(), yig(1e-3, magnetoelastic=True)],
             magnetostatics=True, Hext_stat=(0.0, 0.0, 0.1 / MU0),
             em=True, em_fromM=True, em_back_M=True,
             elastic=True, elasto_back=True, elasto_on=True,
             strain_pulse=True, strain_type=2, strain_z=0, strain_comp="x",
             sigma_gauss=0.3e12, strain_cycles=0, abc_1D=False, liao_w=0.5,
             name=f"magnetoelastic_{nx}x{ny}x{nz}")
    vs = math.sqrt(ggg().c44 / ggg().density)
    # peak |u| of the (cos - 1) source is 2 A vs / (2 pi f) = 1 pm
    d.amp_gauss = 1e-12 * 2.0 * math.pi * d.sigma_gauss / (2.0 * vs)
    d.m0 = tilt_m0((nx, ny, nz), 20241203 + 2, (d.material_cell() == 2))
    return d


def preset_ferroelectric(nx=128, ny=128, nz=128, steps=40000, dt=None, pulse=True) -> Deck:
    """PbTiO3-like TDGL + electrostriction + elastodynamics + FDTD,
    seeded uniform random P within +-1e-3 C/m^2, z-polarised Gaussian sheet
    current (J_f type 4, width 1 ps) radiating ~100 kV/cm."""
    dx = 1e-9
    if dt is None:
        dt = 0.9 * 2.0 * math.sqrt(2.0) * dx / (2.0 * math.sqrt(3.0) * C0)
    d = Deck(nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, dz=dx, periodic=(True, True, False), layers=[(nz, 1)],
             steps=steps, dt=dt, materials=[pto()],
             em=True, em_fromP=True, em_back_P=True,
             elastic=True, elasto_back=True, elasto_on=True, abc_1D=True,
             name=f"ferroelectric_{nx}x{ny}x{nz}")
    r = splitmix64(20241203 + 3, 3 * d.n).reshape(d.n, 3)
    d.p0 = (2e-3 * r - 1e-3).T.reshape(3, nx, ny, nz).copy()
    d.q0 = np.zeros_like(d.p0)
    if pulse:
        kz = max(1, nz // 8)
        d.jf = True
        d.jf_lo = (0, 0, kz)
        d.jf_hi = (nx - 1, ny - 1, kz)
        d.jf_type = 4
        d.jf_comp = "z"
        d.jf_freq = 1e-12           # type 4 reads the Gaussian width from Jf_input_freq
        E0 = 1e7                    # 100 kV/cm
        d.jf_amp = 2.0 * E0 / (ETA0 * dx)
    return d


PRESETS = {
    "fm_demag": preset_fm_demag,
    "magnetoelastic": preset_magnetoelastic,
    "ferroelectric": preset_ferroelectric,
}
