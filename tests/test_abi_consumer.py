"""The C ABI from C and C++ consumers, not only from ctypes.

CPU (no GPU needed):
* tests/abi/abi_consumer.cpp — a C++ program that includes
  include/goferro_b200.h and links libgoferro_b200.so — compiles and links;
* tests/abi/refclass_binding.cpp — the method-level binding of the reference's
  four system classes over the ABI — compiles against the reference's own
  headers (skipped where the reference sources are absent);
* the layouts of gf_run_params and gf_material_params seen by a C compiler
  equal the ctypes mirrors the Python host uses.

GPU: the consumer's traces, driven by gf_advance and by main.cpp's
per-system stage calls (gf_stage_begin / gf_stage_commit), equal each other
bit for bit and GO-Ferro's own solver to 1e-10; an engine created from parsed
values (gf_create) equals the deck-created one bit for bit; gf_set_table
stands in for Hext.in.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ABI = os.path.join(ROOT, "tests", "abi")
LIBDIR = os.path.join(ROOT, "go-ferro_b200")
REF_DIR = os.environ.get("GOFERRO_REF_DIR", "/root/reference")


def build_consumer(out_dir):
    exe = os.path.join(out_dir, "abi_consumer")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ABI, "abi_consumer.cpp"), "-L" + LIBDIR, "-lgoferro_b200",
                    "-Wl,-rpath," + LIBDIR, "-o", exe], check=True)
    return exe


def test_consumer_compiles_and_links(gf, tmp_path):
    gf.load_library()
    exe = build_consumer(str(tmp_path))
    # without arguments it prints its usage and touches no device
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.skipif(not os.path.isdir(REF_DIR), reason="reference sources absent")
def test_class_binding_compiles_against_reference_headers():
    subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-w", "-I" + os.path.join(ROOT, "oracle", "shim"),
                    "-I" + REF_DIR, "-I" + os.path.join(ROOT, "include"), os.path.join(ABI, "refclass_binding.cpp")],
                   check=True)


def _c_layout(tmp_path, struct, ctype):
    fields = [f[0] for f in ctype._fields_]
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "goferro_b200.h"', "int main(void) {",
           f'  printf("%zu\\n", sizeof({struct}));']
    src += [f'  printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    src += ["  return 0;", "}"]
    c = tmp_path / f"{struct}.c"
    c.write_text("\n".join(src))
    exe = str(tmp_path / struct)
    subprocess.run(["gcc", "-std=c99", "-I" + os.path.join(ROOT, "include"), str(c), "-o", exe], check=True)
    out = [int(x) for x in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    return out[0], dict(zip(fields, out[1:]))


@pytest.mark.parametrize("struct,attr", [("gf_run_params", "GFRunParams"), ("gf_material_params", "GFMaterialParams")])
def test_param_struct_layouts_match_c(gf, tmp_path, struct, attr):
    ctype = getattr(gf, attr)
    size, offs = _c_layout(tmp_path, struct, ctype)
    assert size == ctypes.sizeof(ctype)
    for name, off in offs.items():
        assert getattr(ctype, name).offset == off, name


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def _consumer_trace(exe, deck_dir, mode, steps, probe):
    args = [exe, deck_dir, mode, str(steps)] + ([str(x) for x in probe] if probe else [])
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return np.loadtxt(r.stdout.splitlines(), ndmin=2)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["magnetoelastic", "ferroelectric", "fm_demag"])
def test_consumer_traces_match_reference(gf, refrun, tmp_path, case):
    if case == "magnetoelastic":
        d = gf.decks.preset_magnetoelastic(nx=8, ny=16, nz=12, sub=5, film=4, steps=12)
        d.amp_gauss *= 1e6
        probe = (4, 8, 7)
    elif case == "ferroelectric":
        d = gf.decks.preset_ferroelectric(nx=8, ny=8, nz=10, steps=12)
        probe = (4, 4, 5)
    else:
        d = gf.decks.preset_fm_demag(nx=16, ny=16, nz=8, steps=12)
        probe = None
    ddir = str(tmp_path / "deck")
    gf.decks.write_deck(d, ddir)
    exe = build_consumer(str(tmp_path))
    adv = _consumer_trace(exe, ddir, "advance", 12, probe)
    stg = _consumer_trace(exe, ddir, "stages", 12, probe)
    assert np.array_equal(adv, stg)
    ref = refrun.run(ddir, str(tmp_path / "ref"), steps=12, probe=probe)["trace"]
    assert adv.shape == ref.shape
    for c in range(1, 22):
        scale = float(np.max(np.abs(ref[:, c])))
        err = float(np.max(np.abs(adv[:, c] - ref[:, c])))
        assert err <= 1e-10 * scale or (scale == 0 and err == 0), f"column {c}: {err / max(scale, 1e-300):.3e}"


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["magnetoelastic", "ferroelectric", "fm_demag"])
def test_params_create_equals_deck_create(gf, tmp_path, case):
    if case == "magnetoelastic":
        d = gf.decks.preset_magnetoelastic(nx=8, ny=16, nz=12, sub=5, film=4, steps=9)
        d.amp_gauss *= 1e6
    elif case == "ferroelectric":
        d = gf.decks.preset_ferroelectric(nx=8, ny=8, nz=10, steps=9)
    else:
        d = gf.decks.preset_fm_demag(nx=16, ny=16, nz=8, steps=9)   # prescribed H table, m.in
    gf.decks.write_deck(d, str(tmp_path))
    fields = [f for f in ("m", "p", "q", "u", "v", "Ex", "Hz", "Hstat") ]
    out = []
    for make in (lambda: gf.Engine(str(tmp_path), device=0), lambda: gf.Engine.from_params(d, device=0)):
        with make() as eng:
            eng.advance(9)
            got = {}
            for f in fields:
                try:
                    got[f] = eng.download(f)
                except gf.GFError:
                    pass
            out.append(got)
    assert sorted(out[0]) == sorted(out[1])
    for f in out[0]:
        assert np.array_equal(out[0][f], out[1][f]), f


@pytest.mark.gpu
def test_stage_calls_out_of_order_are_rejected(gf, tmp_path):
    d = gf.decks.preset_ferroelectric(nx=8, ny=8, nz=10, steps=4)
    gf.decks.write_deck(d, str(tmp_path))
    with gf.Engine(str(tmp_path), device=0) as eng:
        with pytest.raises(gf.GFError):
            eng.stage_commit(1)              # no step open
        with pytest.raises(gf.GFError):
            eng.stage_begin(2)               # a step starts with stage 1
        eng.stage_begin(1)
        eng.stage_commit(1)
        with pytest.raises(gf.GFError):
            eng.stage_commit(3)              # stage 2 not done
        with pytest.raises(gf.GFError):
            eng.advance(1)                   # step still open
        for s in (2, 3, 4):
            eng.stage_begin(s)
            eng.stage_commit(s)
        eng.advance(1)
        assert eng.get_info().step == 2


@pytest.mark.gpu
def test_static_solve_reforms_the_per_stage_field(gf, tmp_path):
    d = gf.decks.preset_fm_demag(nx=16, ny=16, nz=8, steps=6)
    gf.decks.write_deck(d, str(tmp_path))
    with gf.Engine(str(tmp_path), device=0) as eng:
        eng.advance(5)
        h = eng.download("Hstat")
        eng.static_solve("magnetic")        # the same m: the same field, bit for bit
        assert np.array_equal(eng.download("Hstat"), h)
        eng.stage_begin(1)
        eng.stage_commit(1)
        h1 = eng.download("Hstat")
        eng.static_solve("magnetic")        # between stages: already formed by the stage
        assert np.array_equal(eng.download("Hstat"), h1)
        for s in (2, 3, 4):
            eng.stage_begin(s)
            eng.stage_commit(s)
        eng.advance(1)
        eng.static_solve("electric")        # the electrostatic solve is off: nothing to do
        with pytest.raises(gf.GFError):
            eng.static_solve("nothing")
