"""The allocation-free entry point gf_field_mean_noalloc.

It serves callers that cannot allocate device memory while they run (device
memory owned by another runtime such as the reference's OpenACC data regions
or a caller-managed pool, or code where cudaMalloc would synchronise the
device or is not allowed during stream capture).  Its partial sums live in a
fixed file-scope device array, so it takes only caller-owned pointers.

The test acts as such a caller: it owns the input and output buffers (torch
allocations made before the calls), calls the entry point through the C ABI
twice in a row, and checks each result against the engine's own gf_average
of the same field, within the parity tolerance used by the GPU tests.
This file is collected last so that a stop-at-first-failure run has already
run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def test_noalloc_mean_matches_engine_average(gf, tmp_path):
    import torch
    lib = gf.load_library()
    d = gf.decks.preset_fm_demag(nx=32, ny=24, nz=8, steps=3)
    gf.decks.write_deck(d, str(tmp_path))
    with gf.Engine(str(tmp_path), device=0) as eng:
        eng.advance(3)
        expected = eng.average("m")
        n = d.n
        buf = torch.empty(3 * n, dtype=torch.float64, device="cuda:0")     # caller-owned input
        out = torch.zeros(2, 3, dtype=torch.float64, device="cuda:0")      # caller-owned outputs
        rc = lib.gf_download_device(eng.h, gf.FIELD["m"], ctypes.c_void_p(buf.data_ptr()), 3 * n)
        assert rc == 0, lib.gf_last_error(eng.h).decode()
        eng.synchronize()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        for call in range(2):               # two calls in a row share the scratch
            for a in range(3):
                rc = lib.gf_field_mean_noalloc(ctypes.c_void_p(buf.data_ptr() + 8 * a * n), n,
                                               float(eng.info.n_fm),
                                               ctypes.c_void_p(out.data_ptr() + 8 * (3 * call + a)), stream)
                assert rc == 0, lib.gf_last_error(None).decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
    for call in range(2):
        for a in range(3):
            scale = max(abs(expected[a]), 1e-300)
            assert abs(got[call, a] - expected[a]) <= TOL * scale, (call, a, got[call, a], expected[a])
    assert np.array_equal(got[0], got[1])


def test_noalloc_rejects_oversize_and_null(gf):
    import torch
    lib = gf.load_library()
    x = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    p = ctypes.c_void_p(x.data_ptr())
    rc = lib.gf_field_mean_noalloc(p, 64 * 1024 * 1024 + 1, 1.0, p, None)
    assert rc == -1 and b"exceed the maximum" in lib.gf_last_error(None)
    rc = lib.gf_field_mean_noalloc(None, 8, 1.0, p, None)
    assert rc == -1 and b"null" in lib.gf_last_error(None)
