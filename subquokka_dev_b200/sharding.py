"""Batches of independent variational circuits sharded over GPUs.

One process per GPU (torch.distributed, NCCL between GPUs, gloo on CPU).
The circuits of a batch share nothing, so a rank runs its own qk_batch over
its subset and the only collective is one sum-reduction of the results at
the end -- nothing crosses NVLink on the data path.  This is the multi-GPU
form of the batch workload; the reference has no batching (its MPI runner,
src/MPI_MEM_Func.cpp, shards one state's global qubits instead).

Partition: the device cost of a circuit is its state size times its gate
count (every gate, fused or not, is paid in sweeps over the state), and the
circuits are dealt largest first to the rank with the least cost so far
(longest-processing-time greedy), ties to the lower rank.  Every rank
computes the same partition from the same items, without communicating.
"""
from __future__ import annotations

import numpy as np


def circuit_cost(pc) -> float:
    """Device work of a ParamCircuit: 2^n amplitudes x gates."""
    return float(1 << pc.n) * float(len(pc.ops))


def partition(costs, world: int) -> list[list[int]]:
    """Circuit indices per rank (ascending within a rank), LPT-balanced."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def _layout(param_counts):
    """Offsets of each circuit's gradient in the flat result vector
    [expvals (ncirc) | drift (ncirc) | gradients (sum of param counts)]."""
    ncirc = len(param_counts)
    offs = np.zeros(ncirc + 1, dtype=np.int64)
    offs[1:] = np.cumsum(param_counts)
    return 2 * ncirc + offs[:-1], 2 * ncirc + int(offs[-1])


def gather_results(mine, local, param_counts, device="cpu", group=None):
    """Combine every rank's results into the full batch, on every rank.

    mine: the global indices of this rank's circuits; local: (expvals,
    grads, drift) for them, in that order.  One all_reduce(SUM) of a vector
    in which each rank fills only its own circuits' slots (the other entries
    are zero, so the sum reproduces each value exactly).  Returns (expvals,
    [gradient of circuit c], drift) in the batch's order."""
    import torch
    import torch.distributed as dist
    ncirc = len(param_counts)
    goff, total = _layout(param_counts)
    flat = np.zeros(total, dtype=np.float64)
    ev, grads, drift = local
    for k, c in enumerate(mine):
        flat[c] = ev[k]
        flat[ncirc + c] = drift[k]
        flat[goff[c]:goff[c] + param_counts[c]] = grads[k]
    t = torch.from_numpy(flat).to(device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    flat = t.cpu().numpy()
    return (flat[:ncirc].copy(), [flat[goff[c]:goff[c] + param_counts[c]].copy() for c in range(ncirc)],
            flat[ncirc:2 * ncirc].copy())


class ShardedBatch:
    """The batch workload over all ranks of the default process group: each
    rank runs a qk_batch (one CUDA graph) over its share of `items`
    [(ParamCircuit, params, terms), ...]; run() returns every circuit's
    results on every rank."""

    def __init__(self, items, dtype="c64", autotune: bool = False, rank: int | None = None,
                 world: int | None = None, device=None, group=None):
        import torch.distributed as dist
        from .engine import Batch
        dist_on = dist.is_available() and dist.is_initialized()
        self.rank = rank if rank is not None else (dist.get_rank(group) if dist_on else 0)
        self.world = world if world is not None else (dist.get_world_size(group) if dist_on else 1)
        self.group = group
        self.device = device if device is not None else "cuda"
        self.param_counts = [pc.nparams for pc, _, _ in items]
        self.parts = partition([circuit_cost(pc) for pc, _, _ in items], self.world)
        self.mine = self.parts[self.rank]
        self.batch = Batch([items[i] for i in self.mine], dtype, autotune=autotune) if self.mine else None

    def run(self):
        if self.batch is not None:
            local = self.batch.run()
        else:
            local = (np.zeros(0), [], np.zeros(0))
        return gather_results(self.mine, local, self.param_counts, self.device, self.group)

    def device_ms(self) -> float:
        """This rank's device time of its last run (0 with no circuits)."""
        return self.batch.timing()[0] if self.batch is not None else 0.0

    def close(self) -> None:
        if self.batch is not None:
            self.batch.close()
            self.batch = None
