"""Work sharded over GPUs, one process per GPU (torch.distributed: NCCL
between GPUs, gloo on CPU).

Batches (ShardedBatch): the circuits of a batch share nothing, so a rank
runs its own qk_batch over its subset and the only collective is one
sum-reduction of the results at the end -- nothing crosses NVLink on the
data path.  The reference has no batching.

One large state (ShardedStateVector): the state's top qubits index the
ranks, as in the reference's MPI runner (src/MPI_MEM_Func.cpp); qubits move
between ranks in all-to-all exchanges between segments of the circuit.

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


# ---------------------------------------------------------------------------
# one state over several GPUs: global-qubit sharding
# ---------------------------------------------------------------------------
def _deposit(v: int, positions) -> int:
    """Bits of v placed at the given bit positions (lowest bit of v first)."""
    r = 0
    for i, p in enumerate(positions):
        if (v >> i) & 1:
            r |= 1 << p
    return r


class ShardedStateVector:
    """One n-qubit state over W = 2^g ranks, one GPU each: a rank holds the
    2^(n-g) amplitudes whose top g index bits (the global positions) equal
    its rank.  The GPU form of the reference's MPI runner
    (src/MPI_MEM_Func.cpp).

    Gates on local qubits run on each rank's shard with the engine's fused
    passes.  A gate on a global qubit needs it local first: the circuit is cut
    into segments by the light-cone segmenter of the host-resident runner
    (local set = n - g qubits), and between two segments the qubits that must
    come in are exchanged with local ones no longer needed -- the reference's
    MPI_VSWAP (src/MPI_MEM_Func.cpp:318-506) -- by one local permutation pass
    (the outgoing qubits to the top k local bits, the engine's VSWAP kernel)
    and one all-to-all of 2^k equal contiguous blocks per rank (NCCL over
    NVLink; (1 - 2^-k) of each shard crosses).  No amplitude moves for a gate
    that is already local, and the qubits' positions are tracked, not
    restored after each exchange.

    shards: the ranks this process hosts -- one (its own rank) under
    torch.distributed, or all of them in one process (ranks=range(W),
    exchanges by device copies; used to run the multi-rank logic on one
    GPU).  backend: how a shard is stored and a gate list applied to it
    (default: the engine's StateVector and fused plans)."""

    def __init__(self, nqubits: int, dtype="c128", world: int | None = None, ranks=None, group=None,
                 backend=None):
        import torch.distributed as dist
        dist_on = dist.is_available() and dist.is_initialized()
        self.world = world if world is not None else (dist.get_world_size(group) if dist_on else 1)
        if self.world & (self.world - 1):
            raise ValueError("the number of ranks must be a power of two")
        self.g = self.world.bit_length() - 1
        self.n = int(nqubits)
        self.m = self.n - self.g
        if self.m < 1:
            raise ValueError("more global qubits than qubits")
        self.ranks = list(ranks) if ranks is not None else [dist.get_rank(group) if dist_on else 0]
        self.group = group
        self.distributed = dist_on and len(self.ranks) == 1 and self.world > 1
        self.backend = backend if backend is not None else EngineShards(dtype)
        self.shards = {r: self.backend.zero(self.m, first=(r == 0)) for r in self.ranks}
        # position of logical qubit q (< m: local bit, >= m: rank bit q - m) and its inverse
        self.pos = list(range(self.n))
        self.exchanges = 0

    # -- gates ----------------------------------------------------------------
    def apply(self, circuit) -> None:
        """Apply a Circuit (logical qubits) to the sharded state."""
        from .engine import Circuit, ooc_segments
        gl = circuit.gate_list()
        for mask, idx in ooc_segments(circuit, self.n, self.m):
            need = [q for q in range(self.n) if (mask >> q) & 1]
            incoming = [q for q in need if self.pos[q] >= self.m]
            if incoming:
                self._bring_local(incoming, set(need))
            local = [self._renamed(gl[i]) for i in idx]
            circ = Circuit(local)
            for r in self.ranks:
                self.backend.apply(self.shards[r], circ, self.m)

    def _renamed(self, gate):
        """A gate on logical qubits as the same gate on their local positions.
        Multi-qubit gates take ascending targets, and renaming can reverse a
        pair: symmetric gates (CP, RZZ, SWAP) are re-sorted, a U2 (basis |a b>,
        a the high bit) also gets its two index bits exchanged; VSWAP targets
        need only be distinct."""
        from ._lib import GATE_KINDS
        g = type(gate).from_buffer_copy(gate)
        for k in range(g.nq):
            g.q[k] = self.pos[g.q[k]]
        if g.nq == 2 and g.kind != GATE_KINDS["VSWAP"] and g.kind != GATE_KINDS["MPI_VSWAP"] and g.q[0] > g.q[1]:
            g.q[0], g.q[1] = g.q[1], g.q[0]
            if g.kind == GATE_KINDS["U2"]:
                c = list(g.coeff)
                sw = lambda i: ((i & 1) << 1) | (i >> 1)
                for r in range(4):
                    for col in range(4):
                        src = 4 * sw(r) + sw(col)
                        g.coeff[2 * (4 * r + col)] = c[2 * src]
                        g.coeff[2 * (4 * r + col) + 1] = c[2 * src + 1]
        elif g.nq > 2 and g.kind != GATE_KINDS["VSWAP"] and g.kind != GATE_KINDS["MPI_VSWAP"]:
            raise ValueError("gates on more than two qubits are not renamed here")
        return g

    # -- exchanges --------------------------------------------------------------
    def _bring_local(self, incoming, need) -> None:
        """Swap the global positions of `incoming` with the highest local
        positions whose qubits the next segment does not need."""
        from .engine import Circuit, make_gate
        k = len(incoming)
        q_at = {p: q for q, p in enumerate(self.pos)}
        free = [p for p in range(self.m - 1, -1, -1) if q_at[p] not in need][:k]
        if len(free) < k:
            raise RuntimeError("no local positions free for the incoming qubits")
        # 1. the free positions to the top k local positions (one permutation
        #    pass over every shard), tracked in pos
        top = list(range(self.m - k, self.m))
        src = sorted(p for p in free if p not in top)
        dst = sorted(p for p in top if p not in free)
        if src:
            perm = Circuit([make_gate("VSWAP", src + dst)])
            for r in self.ranks:
                self.backend.apply(self.shards[r], perm, self.m)
            for a, b in zip(src, dst):
                qa, qb = q_at[a], q_at[b]
                self.pos[qa], self.pos[qb] = b, a
                q_at[a], q_at[b] = qb, qa
        # 2. block v of rank r (top-k local bits = v) goes to the rank whose
        #    bits at the incoming qubits' global positions are v; the block
        #    received from rank s lands at top-k bits = s's bits there
        G = sorted(self.pos[q] - self.m for q in incoming)   # rank bits
        self._all_to_all(k, G)
        # local position m - k + i now holds the qubit that was at rank bit G[i]
        for i, gb in enumerate(G):
            qa, qb = q_at[self.m - k + i], q_at[self.m + gb]
            self.pos[qa], self.pos[qb] = self.m + gb, self.m - k + i
            q_at[self.m - k + i], q_at[self.m + gb] = qb, qa
        self.exchanges += 1

    def _all_to_all(self, k: int, G) -> None:
        nb = 1 << k
        gmask = sum(1 << b for b in G)
        if self.distributed:
            import torch.distributed as dist
            r = self.ranks[0]
            x = self.backend.tensor(self.shards[r])
            y = self.backend.scratch(self.shards[r])
            block = x.numel() // nb
            # partners: the ranks that differ from r only in the bits G, in
            # ascending order = ascending v (deposit keeps the order)
            splits = [0] * self.world
            for v in range(nb):
                splits[(r & ~gmask) | _deposit(v, G)] = block
            # complex amplitudes as (re, im) pairs: every backend carries reals
            dist.all_to_all_single(self._real(y), self._real(x), splits, splits, group=self.group)
            self.backend.swap_in(self.shards[r])
        else:
            # every rank hosted here: the same blocks moved by device copies
            for r in self.ranks:
                y = self.backend.scratch(self.shards[r])
                block = y.numel() // nb
                v = sum(((r >> b) & 1) << i for i, b in enumerate(G))   # the block each source sends to r
                for u in range(nb):
                    s = (r & ~gmask) | _deposit(u, G)        # the source rank of block u
                    y[u * block:(u + 1) * block].copy_(self.backend.tensor(self.shards[s])[v * block:(v + 1) * block])
            for r in self.ranks:
                self.backend.swap_in(self.shards[r])

    @staticmethod
    def _real(t):
        import torch
        return torch.view_as_real(t) if t.is_complex() else t

    # -- results ---------------------------------------------------------------
    def gather(self):
        """The full state in logical qubit order as a numpy array (all
        ranks must be hosted here, or rank 0 of a process group gathers)."""
        import numpy as np
        import torch
        import torch.distributed as dist
        parts = {r: self.backend.tensor(self.shards[r]).to(torch.complex128).cpu() for r in self.ranks}
        if self.distributed:
            mine = self.backend.tensor(self.shards[self.ranks[0]]).to(torch.complex128)
            lst = [torch.empty_like(mine) for _ in range(self.world)]
            dist.all_gather([self._real(t) for t in lst], self._real(mine), group=self.group)
            parts = {r: t.cpu() for r, t in enumerate(lst)}
        phys = np.concatenate([parts[r].numpy() for r in range(self.world)])
        # physical index bit pos[q] holds logical qubit q
        shape = (2,) * self.n
        t = phys.reshape(shape)   # axis 0 = the highest physical bit
        axes = [self.n - 1 - self.pos[q] for q in range(self.n - 1, -1, -1)]
        return np.ascontiguousarray(np.transpose(t, axes)).reshape(-1)

    def close(self) -> None:
        for s in self.shards.values():
            self.backend.close(s)
        self.shards = {}


class EngineShards:
    """Shards on the GPU: an engine StateVector each (and a second one as the
    exchange buffer), gate lists run as fused plans."""

    def __init__(self, dtype="c128", fused: bool = True):
        self.dtype = dtype
        self.fused = fused
        self._plan = None
        self._plan_for = None

    def zero(self, m: int, first: bool):
        from .engine import StateVector
        a = StateVector(m, self.dtype)
        if not first:
            a.as_torch().zero_()
        return {"cur": a, "other": None, "m": m}

    def tensor(self, sh):
        return sh["cur"].as_torch()

    def scratch(self, sh):
        from .engine import StateVector
        if sh["other"] is None:
            sh["other"] = StateVector(sh["m"], self.dtype)
        return sh["other"].as_torch()

    def swap_in(self, sh):
        sh["cur"], sh["other"] = sh["other"], sh["cur"]

    def apply(self, sh, circ, m):
        from .engine import Plan
        if not circ.ngates:
            return
        if not self.fused:
            sh["cur"].apply(circ)
            return
        # the ranks hosted here run the same gate list: one plan for all of them
        if self._plan_for is not circ:
            if self._plan is not None:
                self._plan.close()
            self._plan, self._plan_for = Plan(circ, m, self.dtype), circ
        self._plan.apply(sh["cur"])

    def close(self, sh):
        for key in ("cur", "other"):
            if sh[key] is not None:
                sh[key].close()
        if self._plan is not None:
            self._plan.close()
            self._plan, self._plan_for = None, None
