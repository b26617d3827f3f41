"""The kernels' only waits (the bucket scan's look-back, sph_kernels.cu:
k_scan_lookback) are bounded: a wait that runs out sets a device flag, the
kernel ends, and the host reports the error at its next synchronisation with
the CUDA context still usable. The test makes a wait run out with a tile that
never publishes its prefix; no GPU fault is involved.
"""
import ctypes as C

import numpy as np
import pytest

from phi_eng_b200 import _abi

F = C.POINTER(C.c_float)


def make_world(lib, nx=64, ny=64):
    w = lib.phieng_world_new()
    lib.phieng_sph_set_particle_cap(w, max(nx * ny, 4096))
    pts = np.array([(ix * 0.25, iy * 0.25) for iy in range(ny) for ix in range(nx)], np.float32)
    assert lib.phieng_world_fluid_add(w, pts.ctypes.data_as(F), len(pts)) == len(pts)
    return w


@pytest.mark.gpu
def test_scan_wait_runs_out_and_is_reported():
    lib = _abi.load()
    w = make_world(lib, 128, 128)
    lib.phieng_world_step(w, 1 / 60)
    assert lib.phieng_sph_sync(w) == 1
    st = _abi.PhiengSphStatus()
    lib.phieng_sph_status(w, C.byref(st))
    assert st.grid_buckets + 1 > 4 * 4096  # at least two look-back blocks (of up to four scan tiles)
    assert lib.phieng_sph_debug_scan_timeout(w) == 0
    lib.phieng_sph_status(w, C.byref(st))
    assert st.error == _abi.E_CUDA
    assert lib.phieng_sph_sync(w) == 0
    lib.phieng_world_free(w)
    # the context is still usable: a fresh world steps and reads back
    w2 = make_world(lib, 16, 16)
    for _ in range(3):
        lib.phieng_world_step(w2, 1 / 60)
    assert lib.phieng_sph_sync(w2) == 1
    out = np.zeros((256, 4), np.float32)
    assert lib.phieng_world_fluid_get(w2, out.ctypes.data_as(F), 256) == 256
    assert np.isfinite(out).all()
    lib.phieng_world_free(w2)
