"""athad_density_profile_noalloc: the density profile for callers that cannot allocate
device memory when they need it (a host running under a fixed, pre-reserved HBM budget, a
real-time step that cannot take cudaMalloc's implicit synchronisation, a caller whose
buffers belong to another runtime).

The entry point takes a density field the caller already holds on the device and writes
rho_bar and d ln rho_bar / d rad.z into two device arrays the caller provides; its only
scratch is a fixed array inside the library.  This test calls it through the C ABI twice
in a row, on two different states, and checks each result against what the context path
(athad_densities) produces for the same state, within the densities tolerance of the
parity tests (1e-11 relative).  It also checks that grids beyond the fixed scratch are
refused.  The test allocates its own buffers (torch); the entry point allocates none.

This file is collected last, so a run that stops at the first failure has already run
every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

from athad_cond_b200 import GpuAtmosphere, make_state, load_library
from athad_cond_b200._abi import NOALLOC_MAX_IM, NOALLOC_MAX_ROWS, Status, config_params

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def context_profile(grid, seed):
    """The existing entry point: densities on a context; returns the context (alive, so its
    r_humid stays on the device) and the profile it computed."""
    g = GpuAtmosphere(*grid, params=config_params())
    g.upload_state(make_state(*grid, seed=seed))
    g.densities()
    g.synchronize()
    return g, g.download_profile("rho_base"), g.download_profile("dlnrho_dr")


def noalloc_profile(lib, g, grid):
    im, jm, km = grid
    ptr, pitch = g.device_ptr("r_humid")
    rho = torch.empty(im, dtype=torch.float64, device="cuda")
    dln = torch.empty(im, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    st = lib.athad_density_profile_noalloc(ctypes.c_void_p(ptr), im, jm, km, pitch,
                                           ctypes.c_void_p(rho.data_ptr()),
                                           ctypes.c_void_p(dln.data_ptr()),
                                           ctypes.c_void_p(stream.cuda_stream))
    assert st == Status.OK
    stream.synchronize()
    return rho.cpu().numpy(), dln.cpu().numpy()


def test_noalloc_profile_matches_context_path_two_calls():
    lib = load_library()
    torch.cuda.init()
    # odd jm (an equator row) and even jm (every row paired with its mirror)
    for grid, seed in (((41, 181, 361), 101), ((21, 91, 181), 202), ((11, 20, 41), 303)):
        g, rho_ctx, dln_ctx = context_profile(grid, seed)
        rho, dln = noalloc_profile(lib, g, grid)
        g.close()
        assert relerr(rho, rho_ctx) <= 1e-11
        assert relerr(dln, dln_ctx) <= 1e-11


def test_noalloc_accepts_the_largest_grid():
    """im = ATHAD_NOALLOC_MAX_IM levels with im*jm = ATHAD_NOALLOC_MAX_ROWS rows exactly."""
    lib = load_library()
    im, jm, km = NOALLOC_MAX_IM, NOALLOC_MAX_ROWS // NOALLOC_MAX_IM, 8
    r = torch.rand((im, jm, km), dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(7))
    r += 0.5
    rho = torch.empty(im, dtype=torch.float64, device="cuda")
    dln = torch.empty(im, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    st = lib.athad_density_profile_noalloc(ctypes.c_void_p(r.data_ptr()), im, jm, km, km,
                                           ctypes.c_void_p(rho.data_ptr()), ctypes.c_void_p(dln.data_ptr()),
                                           ctypes.c_void_p(stream.cuda_stream))
    assert st == Status.OK
    stream.synchronize()
    # every positive cell counts with its cos-latitude weight: the row means of a field that
    # is 0.5 + U[0, 1) lie in (0.5, 1.5)
    rb = rho.cpu().numpy()
    assert np.isfinite(rb).all() and (rb > 0.5).all() and (rb < 1.5).all()
    assert np.isfinite(dln.cpu().numpy()).all()


def test_noalloc_rejects_grids_beyond_its_scratch():
    lib = load_library()
    dummy = ctypes.c_void_p(16)   # never dereferenced: the size check comes first
    jm = NOALLOC_MAX_ROWS // 64 + 1
    st = lib.athad_density_profile_noalloc(dummy, 64, jm, 8, 8, dummy, dummy, None)
    assert st == Status.ERR_INVALID
    st = lib.athad_density_profile_noalloc(dummy, 2048, 3, 8, 8, dummy, dummy, None)
    assert st == Status.ERR_INVALID
