"""FWI objective sharded over ranks (one process per GPU).

Shots are independent, so every rank evaluates the shots s = rank, rank +
world, ... (the reference's MPI loop, optimization.cpp:39) with its own
device objective; the misfit, the data norm and the gradient are summed with
one all-reduce each (FP64, torch.distributed: NCCL for device tensors, gloo
on CPU), as the reference's mpiWrapper::allReduceSum does
(optimization.cpp:191, optimization.hpp:407).
"""
from __future__ import annotations

from typing import List, Optional, Tuple

import numpy as np


def shard(nshots: int, rank: int, world: int) -> List[int]:
    """Shots of `rank` in the reference's rank-strided order."""
    return list(range(rank, nshots, world))


def reduce_objective(f_local: float, dn_local: float, g_local: Optional[np.ndarray], shape, device: str = "cpu",
                     group=None) -> Tuple[float, np.ndarray]:
    """Sum the unnormalised misfit, data norm and gradient over the ranks and
    normalise: returns (f / dnorm, g / dnorm) like FwiObjective(normalize=True)."""
    import torch
    import torch.distributed as dist

    s = torch.tensor([f_local, dn_local], dtype=torch.float64, device=device)
    g = torch.zeros(int(np.prod(shape)), dtype=torch.float64, device=device)
    if g_local is not None:
        g += torch.as_tensor(np.ascontiguousarray(g_local, dtype=np.float64).ravel(), device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(s, group=group)
        dist.all_reduce(g, group=group)
    dn = float(s[1])
    if dn < 1e-16:
        dn = 1.0
    return float(s[0]) / dn, (g / dn).to(torch.float32).cpu().numpy().reshape(shape)


class ShardedObjective:
    """Device FWI objective of this rank's shots, reduced over all ranks."""

    def __init__(self, sv, observed: np.ndarray, rank: int, world: int, batch: Optional[int] = None,
                 device: int = 0, comm_device: Optional[str] = None, group=None):
        from . import ops, synth

        self.shots = shard(len(sv.par.sxyz), rank, world)
        self.shape = (min(3, sv.nmodels), sv.ny, sv.nx, sv.nz)
        self.comm_device = comm_device or f"cuda:{device}"
        self.group = group
        obs = np.asarray(observed, dtype=np.float32)
        # the library forms dnorm with the data sampling as a float (fwi_objective_create)
        dt32 = float(np.float32(sv.dt_data))
        self.dn_local = float(np.sum(obs[self.shots].astype(np.float64) ** 2)) * dt32 if self.shots else 0.0
        self.obj = None
        if self.shots:
            par = sv.par.copy()
            par.sxyz = [sv.par.sxyz[s] for s in self.shots]
            par.rxyz = [sv.par.rxyz[s] for s in self.shots]
            par.ns = len(self.shots)
            sub = synth.Survey(sv.name, sv.nmodels, sv.nx, sv.ny, sv.nz, sv.dx, sv.dy, sv.dz, sv.model, sv.wavelet,
                               sv.dt_data, par, sv.ox, sv.oy, sv.oz)
            self.obj = ops.FwiObjective(sub, obs[self.shots], normalize=False, batch=batch, device=device)

    def evaluate(self, model: np.ndarray) -> Tuple[float, np.ndarray]:
        f, g = (0.0, None) if self.obj is None else self.obj.evaluate(model)
        return reduce_objective(f, self.dn_local, g, self.shape, self.comm_device, self.group)
