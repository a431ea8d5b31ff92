"""The view-sharded trainer (nprush_b200.distributed.ShardedTrainer) around
the real Gaussian trainer: two ranks (processes) on cuda:0 over a gloo group
(the all-reduce goes through the host, so no kernel of one rank waits for
the other's) each render half of an 8-view step and sum their gradients.

The two replicas stay bit-identical to each other (same summed gradient, same
Adam update, same ADC), and they follow the single-process trainer that
renders all 8 views in one launch: the summed gradient equals its gradient
to float rounding (each rank sums its views first, so the additions are
associated differently: 1e-6 relative L2), and after two steps and an ADC
event the parameters agree to 1e-5."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

N, W, H, DEG = 6000, 96, 80, 1


def _scene():
    from gs_scenes import gs_scene, gs_targets, gs_views
    p = gs_scene(N, 111, deg=DEG, log_scale_mean=-3.4)
    eyes = [(4.0 * np.cos(a), 1.0, 4.0 * np.sin(a)) for a in np.linspace(0, 2 * np.pi, 8, endpoint=False)]
    vp, vpi, _ = gs_views(W, H, tuple(map(tuple, eyes)))
    tg = gs_targets(8, W, H, 112)
    return p, vp, vpi, tg, np.arange(8, dtype=np.uint32)


def _worker(rank, world, port, out_dir):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    for q in (root, root / "tests", root / "oracle"):
        sys.path.insert(0, str(q))
    import datetime

    import torch.distributed as dist

    from nprush_b200.distributed import ShardedTrainer, device_tensor
    from nprush_b200.gaussians import GaussianTrainer
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        p, vp, vpi, tg, ids = _scene()
        t = GaussianTrainer(2 * N, sh_degree=DEG, device=0, params=p)
        t.set_deterministic(True)
        t.set_targets(tg)
        st = ShardedTrainer(t)
        st.train_step(vp, vpi, ids)
        g1 = device_tensor(t.buffers()["grads"], t.count * 64, 0).cpu().numpy().copy()
        st.train_step(vp, vpi, ids)
        c = st.adc(grad_thresh=1e-6)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), grads1=g1, params=t.read_state()["params"],
                 after=c["after"])
        t.close()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_follow_the_single_process_trainer(tmp_path):
    import torch.multiprocessing as mp

    from nprush_b200 import build
    build.build()
    from nprush_b200.gaussians import GaussianTrainer
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r0, r1 = np.load(tmp_path / "rank0.npz"), np.load(tmp_path / "rank1.npz")
    for k in ("grads1", "params", "after"):
        np.testing.assert_array_equal(r0[k], r1[k])
    p, vp, vpi, tg, ids = _scene()
    t = GaussianTrainer(2 * N, sh_degree=DEG, device=0, params=p)
    t.set_deterministic(True)
    t.set_targets(tg)
    t.set_views(vp, vpi, ids)
    t.train_step()
    g1 = t.read_state()["grads"].reshape(-1)
    a, b = r0["grads1"].astype(np.float64), g1.astype(np.float64)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-6
    t.train_step()
    c = t.adc(grad_thresh=1e-6)
    assert c["after"] == int(r0["after"])
    close = np.isclose(r0["params"], t.read_state()["params"], rtol=1e-5, atol=1e-6)
    assert close.mean() > 0.999, close.mean()
