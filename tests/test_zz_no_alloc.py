"""phieng_sph_density_noalloc: the density pass for callers that may not
allocate GPU memory (e.g. a game engine's simulation thread, where cudaMalloc
can stall the frame). It must give the same density and pressure as the
world's own density pass, on repeated calls that reuse its fixed scratch.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from phi_eng_b200 import _abi, scenes
from phi_eng_b200.world import world_from_scene

pytestmark = pytest.mark.gpu


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).mean()) / max(np.sqrt((b ** 2).mean()), 1e-30))


@pytest.mark.parametrize("make", [scenes.dam_break_4k, lambda: scenes.dam_break_scaled(256, 256)])
def test_noalloc_density_matches_world_twice(make):
    import torch

    sc = make()
    assert sc.n <= _abi.NOALLOC_MAX_PARTICLES
    # the existing path: a world's density pass on the same positions
    w = world_from_scene(sc)
    w.debug_forces()
    d_ref, p_ref = w.fluid.density_pressure()
    w.close()

    lib = _abi.load()
    xy = torch.from_numpy(np.ascontiguousarray(sc.xy)).cuda()
    dens = torch.empty(sc.n, dtype=torch.float32, device="cuda")
    pres = torch.empty(sc.n, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    cfg = sc.config
    for _ in range(2):  # the second call reuses the scratch the first one left behind
        dens.fill_(float("nan"))
        pres.fill_(float("nan"))
        rc = lib.phieng_sph_density_noalloc(C.c_void_p(xy.data_ptr()), sc.n, C.byref(cfg),
                                            C.c_void_p(dens.data_ptr()), C.c_void_p(pres.data_ptr()),
                                            C.c_void_p(stream))
        torch.cuda.synchronize()
        assert rc == _abi.OK
        d = dens.cpu().numpy()
        p = pres.cpu().numpy()
        assert rel_rms(d, d_ref) <= 1e-5 and rel_rms(p, p_ref) <= 1e-5
        assert np.array_equal(d, d_ref) and np.array_equal(p, p_ref)


def test_noalloc_rejects_too_many_particles():
    lib = _abi.load()
    cfg = scenes.si_config(0.01)
    rc = lib.phieng_sph_density_noalloc(None, _abi.NOALLOC_MAX_PARTICLES + 1, C.byref(cfg), None, None, None)
    assert rc == _abi.E_TOO_LARGE
