"""Data-parallel training of the closure network (phieng_mlp_shard_grad,
phieng_mlp_apply_grad, closure.train_data_parallel).

Each rank takes a slice of the minibatch that a single-GPU run with the
whole batch would draw, the ranks all-reduce their gradient vectors, and every
rank takes the same Adam step. On one GPU: the slice gradient of the whole
batch equals phieng_mlp_grad bit for bit, two slices sum to the whole, and two
gloo ranks (each driving the library on the one GPU, all-reducing host
copies; no kernel waits on another rank) keep bit-identical parameters that
follow single-GPU training with the combined batch.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _blocks():
    from phi_eng_b200 import closure as cl

    o = [0, 1024, 1088, 5184, 5248, 5376, cl.NPARAMS]
    return list(zip(o[:-1], o[1:]))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _data(seed=12, npairs=40000):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((npairs, 16)).astype(np.float32)
    t = np.stack([np.tanh(x[:, 0]) * x[:, 1], np.sin(x[:, 2])], 1).astype(np.float32)
    return x, t


def _net(engine):
    """A network with every layer random (the output layer too, so every
    gradient block is nonzero)."""
    from phi_eng_b200.closure import Mlp

    m = Mlp(seed=21)
    m.train_engine = engine
    p, nrm = m.get()
    rng = np.random.default_rng(33)
    p = (rng.standard_normal(p.shape) * 0.15).astype(np.float32)
    nrm[32:] = 0.5
    m.set(p, nrm)
    return m


@pytest.mark.gpu
@pytest.mark.parametrize("engine", ["tcgen05", "mma.sync"])
def test_shard_grad_of_whole_batch_equals_grad(engine):
    import torch

    x, t = (torch.from_numpy(a).cuda() for a in _data())
    m = _net(engine)
    loss, g = m.grad(x, t, 2048, 0x99, 0)  # a fresh network's Adam step count is 0
    v = m.shard_grad(x, t, 0, 2048, 2048, 0x99).cpu().numpy()
    np.testing.assert_array_equal(v[:-1], g)
    assert abs(v[-1] / (2 * 2048) - loss) <= 1e-6 * loss
    # two slices sum to the whole
    a = m.shard_grad(x, t, 0, 1024, 2048, 0x99).cpu().numpy().astype(np.float64)
    b = m.shard_grad(x, t, 1024, 1024, 2048, 0x99).cpu().numpy().astype(np.float64)
    s = a + b
    for lo, hi in _blocks():
        assert np.linalg.norm(s[lo:hi] - v[lo:hi]) <= 1e-5 * np.linalg.norm(v[lo:hi]), (lo, hi)
    assert abs(s[-1] - v[-1]) <= 1e-5 * v[-1]
    assert m.check_waits()


@pytest.mark.gpu
def test_shard_grad_rejects_bad_slices():
    import torch

    x, t = (torch.from_numpy(a).cuda() for a in _data())
    m = _net("tcgen05")
    for first, batch, total in [(0, 100, 1024), (1024, 1024, 1024), (0, 2048, 1024)]:
        with pytest.raises(ValueError):
            m.shard_grad(x, t, first, batch, total, 1)


def _dp_worker(rank, size, port, iters, batch, lr, out):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    from phi_eng_b200.closure import train_data_parallel

    x, t = (torch.from_numpy(a).cuda() for a in _data())
    m = _net("tcgen05")
    hist = train_data_parallel(m, x, t, batch=batch, iters=iters, lr=lr, seed=0x7E)
    np.save(out + f".w{rank}.npy", m.get()[0])
    np.save(out + f".h{rank}.npy", hist)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.gpu
def test_data_parallel_training_two_ranks(tmp_path):
    import torch

    size, iters, batch, lr = 2, 6, 1024, 1e-3
    out = str(tmp_path / "dp")
    mp.start_processes(_dp_worker, args=(size, _free_port(), iters, batch, lr, out), nprocs=size,
                       start_method="spawn")
    w0, w1 = np.load(out + ".w0.npy"), np.load(out + ".w1.npy")
    np.testing.assert_array_equal(w0, w1)  # every rank applied the same all-reduced gradient
    h0, h1 = np.load(out + ".h0.npy"), np.load(out + ".h1.npy")
    np.testing.assert_array_equal(h0, h1)
    # single-GPU training on the combined batch draws the same samples
    x, t = (torch.from_numpy(a).cuda() for a in _data())
    ref = _net("tcgen05")
    start = ref.get()[0]
    hist = ref.train(x, t, batch=size * batch, iters=iters, lr=lr, seed=0x7E)
    ws = ref.get()[0]
    np.testing.assert_allclose(h0, hist, rtol=1e-4)
    d_dp, d_1 = w0 - start, ws - start
    assert np.linalg.norm(d_dp - d_1) <= 2e-2 * np.linalg.norm(d_1)
