"""msf_probe_noalloc: the probe build for callers that may not allocate device
memory (an application that owns every device byte in its own pool, or a
running loop that must not stall on cudaMalloc).  The caller supplies the
output buffer; the entry point's scratch is a fixed device array.

Checked through the C ABI against the allocating entry point msf_probe, on
two calls in a row with different grids and optics (the second call must not
see the first call's scratch), with the same FP64 tolerance as the other
probe tests.  This file is collected last so a stop-at-first-failure run has
already run every other test; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import msf

pytestmark = pytest.mark.gpu


def _grid(nx, ny, period_x, period_y, voltage):
    return msf.Grid(nx=nx, ny=ny, voltage=voltage, xperiod=period_x, yperiod=period_y,
                    zperiod=10.0, dupe_x=1, dupe_y=1, dupe_z=1, replicate_atoms=0,
                    min_slice=2.0)


def _reference_probe(grid, optics):
    ctx = msf.Context(precision="fp64")
    spec = ctx.specimen(grid, np.zeros((0, 3)), np.zeros(0, dtype=np.uint32))
    p = ctx.probe(spec, optics)
    spec.close()
    ctx.close()
    return p


def test_noalloc_probe_matches_allocating_entry_point_twice():
    import torch

    lib = msf.lib()
    lam200, _ = msf.wavelength(200000.0)
    lam300, _ = msf.wavelength(300000.0)
    cases = [
        (_grid(256, 256, 25.0, 25.0, 200000.0),
         msf.Optics(corrected=0, cs3=1.3e7, cs5=0.0,
                    defocus=0.87 * np.sqrt(1.3e7 * lam200), alpha_max=0.010)),
        (_grid(512, 256, 50.0, 25.0, 300000.0),
         msf.Optics(corrected=1, cs3=-2000.0, cs5=5e7, defocus=-40.0, alpha_max=0.021)),
    ]
    stream = torch.cuda.current_stream().cuda_stream
    for grid, optics in cases:
        nx, ny = grid.nx, grid.ny
        out = torch.full((2 * nx * ny,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.msf_probe_noalloc(C.byref(grid), C.byref(optics), C.c_void_p(out.data_ptr()),
                                   C.c_void_p(stream))
        assert rc == 0, lib.msf_last_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(nx, ny, 2)
        want = _reference_probe(grid, optics)
        assert np.isfinite(got).all()
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
        np.testing.assert_allclose((got ** 2).sum(), 1.0, rtol=1e-12)


@pytest.mark.parametrize("nx,ny", [(2048, 2048), (2048, 64)])
def test_noalloc_probe_at_its_size_limit(nx, ny):
    """At the documented limit of 2048 samples the scratch is used in full
    and the FP64 row and column transforms need their large shared-memory
    launches; the result must still match msf_probe."""
    import torch

    lib = msf.lib()
    lam, _ = msf.wavelength(300000.0)
    grid = _grid(nx, ny, nx * 0.0977, ny * 0.0977, 300000.0)
    optics = msf.Optics(corrected=0, cs3=1.3e7, cs5=0.0,
                        defocus=0.87 * np.sqrt(1.3e7 * lam), alpha_max=0.0084)
    out = torch.full((2 * nx * ny,), float("nan"), dtype=torch.float64, device="cuda")
    rc = lib.msf_probe_noalloc(C.byref(grid), C.byref(optics), C.c_void_p(out.data_ptr()),
                               C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lib.msf_last_error().decode()
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(nx, ny, 2)
    want = _reference_probe(grid, optics)
    assert np.isfinite(got).all()
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def test_noalloc_probe_rejects_grids_beyond_its_scratch():
    import torch

    lib = msf.lib()
    grid = _grid(4096, 4096, 400.0, 400.0, 200000.0)
    optics = msf.Optics(corrected=0, cs3=1.3e7, cs5=0.0, defocus=500.0, alpha_max=0.010)
    out = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = lib.msf_probe_noalloc(C.byref(grid), C.byref(optics), C.c_void_p(out.data_ptr()),
                               None)
    assert rc == 1  # MSF_ERR_ARG
    assert b"exceeds the fixed scratch limit" in lib.msf_last_error()
