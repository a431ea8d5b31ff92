"""View-sharded data parallelism for the Gaussian trainer (one process per GPU).

A step's V views are independent until their gradients are summed, so each
of the group's ranks renders its share of them (views rank, rank + R, ...)
on a full replica of the parameters, with the loss averaged over all V views
(so the per-rank gradients add up to the single-GPU gradient).  One
all-reduce (sum) of the N x 64-float gradient buffer per step, over NCCL
(NVLink / NVSwitch) on GPUs, then Adam on every replica; the ADC
accumulators are summed before each ADC event, which then runs replicated
(same statistics, same seed counter: the replicas stay identical).

The library owns its device buffers; they are handed to torch.distributed as
tensors that alias them (``__cuda_array_interface__``), so nothing is copied.

    torchrun --nproc-per-node 8 ... and in each process:
        t = GaussianTrainer(...); st = ShardedTrainer(t)
        st.train_step(vp[sel], vpi[sel], sel)
"""
from __future__ import annotations

import numpy as np


class _DeviceArray:
    """A float32 device buffer owned by the library, as a CUDA array interface."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f4", "data": (ptr, False), "version": 3}


def device_tensor(ptr: int, count: int, device: int = 0):
    """torch float32 tensor of `count` elements aliasing the device buffer at ptr."""
    import torch
    with torch.cuda.device(device):
        return torch.as_tensor(_DeviceArray(ptr, count), device=f"cuda:{device}")


def shard_views(n_views: int, rank: int, world: int) -> np.ndarray:
    """Indices of the step's views that this rank renders (round robin)."""
    return np.arange(rank, n_views, world)


class ShardedTrainer:
    """Wraps a trainer (GaussianTrainer, or anything with the same calls) so
    that a step's views are split over the ranks of a process group.

    The trainer side needs: count, set_accumulate, set_views, forward, loss,
    backward, adam, adc, and grad_tensor() / adc_tensors() returning tensors
    that alias its gradient and ADC buffers (defaults below build them from
    the library's device pointers)."""

    def __init__(self, trainer, group=None):
        import torch.distributed as dist
        self.t = trainer
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    # tensors aliasing the trainer's buffers
    def _grad_tensor(self):
        if hasattr(self.t, "grad_tensor"):
            return self.t.grad_tensor()
        return device_tensor(self.t.buffers()["grads"], self.t.count * 64, self.t.device)

    def _adc_tensors(self):
        if hasattr(self.t, "adc_tensors"):
            return self.t.adc_tensors()
        b = self.t.adc_buffers()
        return (device_tensor(b["adc_grad"], self.t.count, self.t.device),
                device_tensor(b["adc_denom"], self.t.count, self.t.device))

    def train_step(self, vp, vp_inv, target_ids):
        """One step over all of vp's views; returns this rank's share of the loss."""
        import torch.distributed as dist
        vp = np.asarray(vp, np.float32).reshape(-1, 16)
        vpi = np.asarray(vp_inv, np.float32).reshape(-1, 16)
        ids = np.ascontiguousarray(target_ids, np.uint32)
        mine = shard_views(vp.shape[0], self.rank, self.world)
        g = self._grad_tensor()
        loss = 0.0
        if len(mine):
            self.t.set_accumulate(False, vp.shape[0])  # loss averaged over the whole step's views
            self.t.set_views(vp[mine], vpi[mine], ids[mine])
            self.t.forward()
            loss = self.t.loss()[0]
            self.t.backward()
            self.t.set_accumulate(False, 0)
        else:
            g.zero_()  # no views here: contribute nothing to the sum
        self._sync_device()
        dist.all_reduce(g, op=dist.ReduceOp.SUM, group=self.group)
        self._sync_device()
        self.t.adam()
        return loss

    def adc(self, *args, **kwargs):
        """ADC on every replica after summing the accumulators over the ranks."""
        import torch.distributed as dist
        ag, ad = self._adc_tensors()
        self._sync_device()
        dist.all_reduce(ag, op=dist.ReduceOp.SUM, group=self.group)
        dist.all_reduce(ad, op=dist.ReduceOp.SUM, group=self.group)
        self._sync_device()
        return self.t.adc(*args, **kwargs)

    def _sync_device(self):
        # the library and torch use different streams: order them through the host
        if hasattr(self.t, "sync"):
            self.t.sync()
        try:
            import torch
            if torch.cuda.is_available():
                torch.cuda.synchronize(getattr(self.t, "device", 0))
        except Exception:
            pass
