"""CPU-side tests: the C-ABI library loads and exports every declared entry
point; deck parsing and option validation (host logic, no GPU needed); the
oracle reproduces its golden fixtures; the oracle's host FFT matches numpy."""
import ctypes
import json
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "goferro_b200.h")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(gf_[a-z_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(gf):
    lib = gf.load_library()
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), f"missing export {s}"
    assert sorted(gf.EXPORTS) == syms
    assert b"sm_100a" in lib.gf_version()


def _create(gf, deck_dir):
    lib = gf.load_library()
    h = ctypes.c_void_p()
    rc = lib.gf_create_from_deck(os.fsencode(deck_dir), -1, ctypes.byref(h))
    msg = lib.gf_last_error(None).decode()
    if rc == 0:
        lib.gf_destroy(h)
    return rc, msg


def test_missing_deck_is_an_io_error(gf, tmp_path):
    rc, msg = _create(gf, str(tmp_path / "nope"))
    assert rc == -2 and "system_setting.in" in msg


def test_truncated_deck_reports_the_field(gf, tmp_path):
    d = gf.decks.preset_fm_demag(nx=8, ny=8, nz=4, steps=2)
    gf.decks.write_deck(d, str(tmp_path))
    txt = open(tmp_path / "system_setting.in").read().splitlines()
    open(tmp_path / "system_setting.in", "w").write("\n".join(txt[:30]) + "\n")
    rc, msg = _create(gf, str(tmp_path))
    assert rc == -2 and "cannot read" in msg


@pytest.mark.parametrize("tweak,needle", [
    (lambda d: setattr(d.materials[0], "afm", True), "nonzero Ms_AFM1/2"),
    (lambda d: (setattr(d.materials[1], "afm", True), setattr(d.materials[1], "afm_Ms", (1e5, 1e5)),
                setattr(d.materials[1], "afm_Aex", (1e-12, 1e-12))), "both ferromagnetic and antiferromagnetic"),
    (lambda d: setattr(d.materials[0], "drude", ((1.0, 1e15, 0.0), (0, 0, 1), (0, 0, 1))), "tao_e = 0"),
    (lambda d: setattr(d.materials[0], "drude", ((0.0, 0.0, 1.0), (0, 0, 1), (0, 0, 1))), "NaN"),
])
def test_unsupported_options_are_rejected_before_device_use(gf, tmp_path, tweak, needle):
    d = gf.decks.preset_magnetoelastic(nx=8, ny=8, nz=12, sub=5, film=4, steps=2)
    tweak(d)
    gf.decks.write_deck(d, str(tmp_path))
    rc, msg = _create(gf, str(tmp_path))
    assert rc == -7 and needle in msg


def test_valid_deck_reaches_the_device_check(gf, tmp_path):
    """A valid deck parses; without a GPU creation stops at the device check."""
    d = gf.decks.preset_ferroelectric(nx=8, ny=8, nz=10, steps=2)
    gf.decks.write_deck(d, str(tmp_path))
    rc, msg = _create(gf, str(tmp_path))
    import torch
    if torch.cuda.is_available():
        assert rc == 0
    else:
        assert rc in (-6, -3), msg


def test_splitmix_is_deterministic_and_uniform(gf):
    a = gf.decks.splitmix64(20241204, 100000)
    b = gf.decks.splitmix64(20241204, 100000)
    assert np.array_equal(a, b)
    assert 0.0 <= a.min() and a.max() < 1.0
    assert abs(a.mean() - 0.5) < 0.01


def test_tilt_is_within_one_degree(gf):
    d = gf.decks.preset_fm_demag(nx=8, ny=8, nz=4, steps=2)
    m = d.m0.reshape(3, -1)
    assert np.allclose(np.linalg.norm(m, axis=0), 1.0)
    assert np.degrees(np.arccos(m[2].min())) <= 1.0 + 1e-9


@pytest.mark.parametrize("name", json.load(open(os.path.join(GOLDEN, "cases.json"))).keys())
def test_oracle_reproduces_golden(gf, refrun, tmp_path, name):
    """The oracle is deterministic: re-running it on the regenerated deck
    gives the committed fixture bit for bit."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    d, steps, probe = mg.make_deck(name)
    gf.decks.write_deck(d, str(tmp_path / "deck"))
    r = refrun.run(str(tmp_path / "deck"), str(tmp_path / "out"), steps=steps, probe=probe, dump=True)
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    assert np.array_equal(r["trace"], g["trace"])
    for k in r["fields"]:
        assert np.array_equal(r["fields"][k], g[k]), k


def test_oracle_host_fft_matches_numpy(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text(r'''
#include "cufft.h"
#include <cstdio>
#include <vector>
int main(){int nx=6,ny=10,nz=12;long n=nx*ny*nz,h=nx*ny*(nz/2+1);
std::vector<double>a(n),b(n);std::vector<cufftDoubleComplex>k(h);
for(long i=0;i<n;i++)a[i]=((i*7919)%1013)/1013.0-0.5;
cufftHandle p,q;cufftPlan3d(&p,nx,ny,nz,CUFFT_D2Z);cufftPlan3d(&q,nx,ny,nz,CUFFT_Z2D);
cufftExecD2Z(p,a.data(),k.data());cufftExecZ2D(q,k.data(),b.data());
fwrite(a.data(),8,n,stdout);fwrite(k.data(),16,h,stdout);fwrite(b.data(),8,n,stdout);}
''')
    exe = tmp_path / "t"
    subprocess.run(["g++", "-O2", "-I", os.path.join(ROOT, "oracle", "shim"), str(src),
                    os.path.join(ROOT, "oracle", "shim", "host_fft.cpp"), "-o", str(exe)], check=True)
    raw = subprocess.run([str(exe)], check=True, capture_output=True).stdout
    n, h = 6 * 10 * 12, 6 * 10 * 7
    a = np.frombuffer(raw[:8 * n]).reshape(6, 10, 12)
    k = np.frombuffer(raw[8 * n:8 * n + 16 * h], dtype=np.complex128).reshape(6, 10, 7)
    b = np.frombuffer(raw[8 * n + 16 * h:]).reshape(6, 10, 12)
    ref = np.fft.rfftn(a)
    assert np.max(np.abs(k - ref)) < 1e-12 * np.max(np.abs(ref))
    assert np.max(np.abs(b / n - a)) < 1e-14
