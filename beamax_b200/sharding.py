"""Multi-GPU beam sharding: one process per GPU, beams partitioned, NCCL reductions.

Restates the reference's ``ShardingStrategy`` (solvers/msgb_solvers/
msgb_solver.py:128-355: beam parameters sharded along the beam axis of a
device mesh, the summed sensor data replicated) for one process per GPU under
``torch.distributed``:

* every rank runs the (cheap, deterministic) coefficient transform, top_n and
  beam initialisation, so all ranks hold the same selection without a
  broadcast;
* rank r takes the contiguous coefficient range ``shard_range(n, world, r)``
  with both branches of each coefficient: in heterogeneous media it also
  integrates only those beams, so the beam ODE is sharded with the sums;
* forward: each rank sums its beams into a partial (nt, ns) field, and one
  all-reduce (FP64, so that the ranks' Kahan-compensated FP32 partials add
  without losing bits to the reduction) gives every rank the full data;
* transpose: every rank gathers its beams against the (replicated) data, the
  per-coefficient gradients are assembled by one all-reduce of the
  zero-padded shards, and every rank applies the coefficient adjoint
  (scatter + adjoint MSWPT).
Collectives are torch.distributed's (NCCL between GPUs, gloo on CPU); no
device kernel touches another GPU's memory.
"""

from __future__ import annotations

from typing import Optional, Tuple


def shard_range(n: int, world: int, rank: int) -> Tuple[int, int]:
    """Contiguous, balanced [lo, hi) of n items for ``rank`` of ``world``
    (the first n % world ranks take one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, rem = divmod(int(n), world)
    lo = rank * base + min(rank, rem)
    return lo, lo + base + (1 if rank < rem else 0)


def _dist():
    import torch.distributed as dist

    return dist


def reduce_partials(partial, group=None):
    """Sum of every rank's partial field, returned as float64 on every rank."""
    dist = _dist()
    full = partial.double().contiguous()
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(full, op=dist.ReduceOp.SUM, group=group)
    return full


def assemble_shards(g_shard, n: int, lo: int, group=None):
    """Per-coefficient complex gradients of all ranks from each rank's shard
    [lo, lo + len(g_shard)): zero-padded to n and summed across ranks."""
    import torch

    dist = _dist()
    full = torch.zeros(n, dtype=torch.complex128, device=g_shard.device)
    full[lo:lo + g_shard.shape[0]] = g_shard
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(torch.view_as_real(full), op=dist.ReduceOp.SUM, group=group)
    return full


class ShardingStrategy:
    """Beam sharding over the ranks of a torch.distributed process group.

    ``validate_divisible``: as the reference, require the number of summed
    beams (2 n, both branches) to split evenly over the ranks
    (msgb_solver.py:145-152); the partition itself works for any n."""

    def __init__(self, group=None, *, validate_divisible: bool = True):
        dist = _dist()
        self.group = group
        if dist.is_available() and dist.is_initialized():
            self.world = dist.get_world_size(group)
            self.rank = dist.get_rank(group)
        else:
            self.world, self.rank = 1, 0
        self.validate_divisible = validate_divisible

    def _validate_beam_count(self, count: int) -> None:
        if self.validate_divisible and count % self.world != 0:
            raise ValueError(f"Beam count {count} is not divisible by {self.world} devices on mesh axis 'x'. "
                             "Adjust top_n or use batching.")

    def shard(self, n: int) -> Tuple[int, int]:
        self._validate_beam_count(2 * n)
        return shard_range(n, self.world, self.rank)


def _slice(bt, lo: int, hi: int):
    from .solvers.msgb_solver import BeamTensors

    return BeamTensors(bt.x0[lo:hi], bt.p0[lo:hi], bt.alpha[lo:hi], bt.a0[lo:hi], bt.a0_unit[lo:hi],
                       bt.omega[lo:hi], bt.modes)


class ShardedMSGB:
    """``forward`` / exact ``adjoint`` of an ``MSGBSolver`` with the beams
    sharded over the process group (same arguments and results as the
    solver's; every rank returns the full result)."""

    def __init__(self, solver, strategy: Optional[ShardingStrategy] = None):
        self.solver = solver
        self.strategy = strategy or ShardingStrategy()

    def forward(self, p0, domain, sensors, ts, wpt):
        s = self.solver
        sel = s.select(p0, domain, wpt)
        s.last_selection = sel
        s._traj_owner = None  # sharded records are not kept for the adjoint
        bt = s.beams(sel, domain, wpt)
        lo, hi = self.strategy.shard(bt.n)
        part = s.sum_forward(_slice(bt, lo, hi), domain, sensors, ts)
        return reduce_partials(part, self.strategy.group)

    def adjoint(self, data, domain, sensors, ts, wpt, *, selection=None):
        from .solvers.msgb_solver import Selection, torch_argsort

        s = self.solver
        sel = selection if selection is not None else s.last_selection
        if sel is None:
            raise ValueError("adjoint needs a beam selection: call forward first or pass selection=")
        order = torch_argsort(sel.idx)
        sel_sorted = Selection(sel.idx[order], sel.values[order], sel.total_coeffs)
        bt = s.beams(sel_sorted, domain, wpt)
        lo, hi = self.strategy.shard(bt.n)
        g = s.gather_adjoint(_slice(bt, lo, hi), domain, sensors, ts, data)
        g_all = assemble_shards(g, bt.n, lo, self.strategy.group)
        return s.coefficient_adjoint(sel_sorted, g_all, wpt)
