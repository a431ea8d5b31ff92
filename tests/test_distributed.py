"""View-sharded data parallelism (nprush_b200.distributed) on CPU: two gloo
ranks with a stand-in trainer (a least-squares 'renderer' whose views are
independent until their gradients are summed, like the Gaussian trainer's)
must follow the single-process trajectory, and stay identical to each other,
including steps with fewer views than ranks and the ADC statistic sum; and a
rank that fails between steps ends the survivor's next collective with an
error (short process-group timeout) instead of leaving it waiting."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

DIM, NVIEW_TABLE = 12, 16


class FakeTrainer:
    """loss = sum over the step's views v of (x . A[v] - b[v])^2 / V."""

    def __init__(self):
        rng = np.random.default_rng(3)
        self.A = rng.normal(size=(NVIEW_TABLE, DIM))
        self.b = rng.normal(size=NVIEW_TABLE)
        self.x = np.zeros(DIM)
        self.m = np.zeros(DIM)
        self.v = np.zeros(DIM)
        self.t = 0
        self.count = 1
        self.g = torch.zeros(DIM, dtype=torch.float64)
        self.ag = torch.zeros(1, dtype=torch.float64)
        self.ad = torch.zeros(1, dtype=torch.float64)
        self.lv = 0
        self.ids = None

    def grad_tensor(self):
        return self.g

    def adc_tensors(self):
        return self.ag, self.ad

    def set_accumulate(self, acc, loss_views):
        self.lv = loss_views

    def set_views(self, vp, vpi, ids):
        self.ids = np.asarray(ids)

    def forward(self):
        self.r = self.A[self.ids] @ self.x - self.b[self.ids]

    def loss(self):
        return (float((self.r ** 2).sum() / (self.lv or len(self.ids))),)

    def backward(self):
        lv = self.lv or len(self.ids)
        grad = 2.0 * (self.r[:, None] * self.A[self.ids]).sum(0) / lv
        self.g.copy_(torch.from_numpy(grad))
        # ADC statistic: per-view gradient norms and view count
        self.ag += float(np.abs(2.0 * self.r).sum())
        self.ad += float(len(self.ids))

    def adam(self):
        g = self.g.numpy()
        self.t += 1
        self.m = 0.9 * self.m + 0.1 * g
        self.v = 0.999 * self.v + 0.001 * g * g
        mh, vh = self.m / (1 - 0.9 ** self.t), self.v / (1 - 0.999 ** self.t)
        self.x -= 0.05 * mh / (np.sqrt(vh) + 1e-12)

    def adc(self):
        out = (float(self.ag[0]), float(self.ad[0]))
        self.ag.zero_()
        self.ad.zero_()
        return out


SCHEDULE = [[0, 3, 5, 7, 9], [1, 2], [4], [6, 8, 10, 11, 12, 13], [14, 15, 0]]


def run_steps(step_fn, adc_fn):
    res = []
    for k, views in enumerate(SCHEDULE):
        ids = np.array(views, np.uint32)
        vp = np.zeros((len(ids), 16), np.float32)
        step_fn(vp, vp, ids)
        if k == 3:
            res.append(adc_fn())
    return res


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from nprush_b200.distributed import ShardedTrainer
        t = FakeTrainer()
        st = ShardedTrainer(t)
        adc = run_steps(st.train_step, st.adc)
        np.save(os.path.join(out_dir, f"x{rank}.npy"), t.x)
        np.save(os.path.join(out_dir, f"adc{rank}.npy"), np.array(adc))
    finally:
        dist.destroy_process_group()


def test_two_ranks_follow_the_single_process_trajectory(tmp_path):
    ref = FakeTrainer()

    def single_step(vp, vpi, ids):
        ref.set_accumulate(False, len(ids))
        ref.set_views(vp, vpi, ids)
        ref.forward()
        ref.backward()
        ref.adam()

    adc_ref = run_steps(single_step, ref.adc)
    port = 29500 + os.getpid() % 1000
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    x0, x1 = np.load(tmp_path / "x0.npy"), np.load(tmp_path / "x1.npy")
    np.testing.assert_array_equal(x0, x1)
    np.testing.assert_allclose(x0, ref.x, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(np.load(tmp_path / "adc0.npy"), np.array(adc_ref), rtol=1e-12)
    np.testing.assert_array_equal(np.load(tmp_path / "adc0.npy"), np.load(tmp_path / "adc1.npy"))


def test_shard_views_partition():
    from nprush_b200.distributed import shard_views
    for n in range(0, 11):
        for world in (1, 2, 3, 8):
            parts = [shard_views(n, r, world) for r in range(world)]
            allv = np.sort(np.concatenate(parts)) if parts else np.array([])
            np.testing.assert_array_equal(allv, np.arange(n))


def _failing_worker(rank, world, port, out_dir):
    """Rank 1 raises between steps (after step 1, before the all-reduce of
    step 2) and leaves; rank 0 must see its next collective end with an
    error within the process group's timeout instead of waiting forever."""
    import datetime
    import time
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    from nprush_b200.distributed import ShardedTrainer
    t = FakeTrainer()
    st = ShardedTrainer(t)
    outcome = "finished"
    t0 = time.perf_counter()
    try:
        for k, views in enumerate(SCHEDULE):
            if rank == 1 and k == 2:
                raise RuntimeError("rank 1 failed between steps")
            ids = np.array(views, np.uint32)
            vp = np.zeros((len(ids), 16), np.float32)
            st.train_step(vp, vp, ids)
    except RuntimeError as e:
        outcome = "raised: " + str(e).splitlines()[0][:200]
    elapsed = time.perf_counter() - t0
    with open(os.path.join(out_dir, f"outcome{rank}.txt"), "w") as f:
        f.write(f"{outcome}\n{elapsed:.3f}\n")
    if rank == 1:
        os._exit(0)  # leaves without joining the group's teardown
    try:
        dist.destroy_process_group()
    except Exception:  # noqa: BLE001 - the peer is gone
        pass


def test_a_failed_rank_ends_the_survivors_next_collective_with_an_error(tmp_path):
    port = 30500 + os.getpid() % 1000
    ctx = mp.start_processes(_failing_worker, args=(2, port, str(tmp_path)), nprocs=2, join=False,
                             start_method="spawn")
    for p in ctx.processes:
        p.join(120)
    alive = [p for p in ctx.processes if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "a rank was still waiting after 120 s"
    o0 = (tmp_path / "outcome0.txt").read_text().splitlines()
    o1 = (tmp_path / "outcome1.txt").read_text().splitlines()
    assert o1[0].startswith("raised: rank 1 failed")
    assert o0[0].startswith("raised:"), o0  # the survivor's all-reduce of step 2 failed
    assert float(o0[1]) < 60.0
