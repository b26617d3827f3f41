"""phieng_sph_density_noalloc: the density pass for callers that may not
allocate GPU memory (e.g. a game engine's simulation thread, where cudaMalloc
can stall the frame). It must give the same density and pressure as the
world's own density pass and as the oracle's, on repeated calls that reuse
its fixed scratch, also when the particles lie so far apart that its bucket
grid is clamped to 2^16 buckets and distant cells share buckets.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import sims
from oracle import oracle as orc
from phi_eng_b200 import _abi, scenes
from phi_eng_b200.world import world_from_scene

pytestmark = pytest.mark.gpu


def two_clusters():
    """Two 64 x 64 blocks of the 4k dam break's lattice, one shifted by
    (1500 h, 900 h): the cell bounding box needs 2^11 x 2^10 buckets, more
    than the scratch's 2^16, so the grid is clamped and cells 2^8 apart
    share a bucket."""
    sc = scenes.dam_break_4k()
    h = float(sc.config.smoothing_length)
    far = sc.xy + np.array([1500 * h, 900 * h], np.float32)
    sc.xy = np.concatenate([sc.xy, far]).astype(np.float32)
    sc.boxes = []
    return sc


def oracle_density(sc):
    o = sims.OracleSim(orc.JACOBI)
    o.config = sc.config
    assert o.add_particles(sc.xy) == sc.n
    o.w.pass_density()
    return o.density_pressure()


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).mean()) / max(np.sqrt((b ** 2).mean()), 1e-30))


@pytest.mark.parametrize("make", [scenes.dam_break_4k, lambda: scenes.dam_break_scaled(256, 256), two_clusters])
def test_noalloc_density_matches_world_twice(make):
    import torch

    sc = make()
    assert sc.n <= _abi.NOALLOC_MAX_PARTICLES
    # the existing path: a world's density pass on the same positions
    w = world_from_scene(sc)
    w.debug_forces()
    d_ref, p_ref = w.fluid.density_pressure()
    w.close()
    # and the oracle's density pass (the reference's arithmetic)
    d_o, p_o = oracle_density(sc)
    assert np.array_equal(d_ref, d_o) and np.array_equal(p_ref, p_o)

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
