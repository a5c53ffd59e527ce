"""The stencil kernels divide by run constants (cell sizes, dt, the RK4
weights 3 and 6) with a precomputed reciprocal and two residual corrections
instead of the general division.  The reference divides with IEEE division;
these tests check, through gf_check_quotients, that both give the same bits
on many numerators, half of them chosen next to rounding midpoints."""
import ctypes
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _divisors(gf):
    D = gf.decks
    ds = [2e-9, 1e-9, 3e-9, 2.5e-9, 3.0, 6.0]
    ds += [D.preset_magnetoelastic(nx=8, ny=8, nz=96).dt, D.preset_ferroelectric(nx=8, ny=8, nz=8).dt,
           D.preset_fm_demag(nx=8, ny=8, nz=8).dt]
    rng = np.random.default_rng(20241203)
    ds += list(10.0 ** rng.uniform(-18, 3, size=8))
    return ds


def test_quotients_match_ieee_division(gf):
    lib = gf.load_library()
    total = 0
    for i, d in enumerate(_divisors(gf)):
        bad = ctypes.c_uint64(99)
        rc = lib.gf_check_quotients(float(d), 1 << 24, 1000 + i, ctypes.byref(bad))
        assert rc == 0, lib.gf_last_error(None).decode()
        assert bad.value == 0, f"d={d!r}: {bad.value} quotients differ from IEEE division"
        total += 1 << 24
    assert total > 0


def test_quotient_check_rejects_bad_divisor(gf):
    lib = gf.load_library()
    bad = ctypes.c_uint64(0)
    assert lib.gf_check_quotients(0.0, 16, 1, ctypes.byref(bad)) == -1
    assert lib.gf_check_quotients(math.inf, 16, 1, ctypes.byref(bad)) == -1
