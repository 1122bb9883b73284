"""x-slab domain decomposition of the lattice-Boltzmann path over several GPUs.

The reference parallelises the same path over cells inside one process
(rayon chunks of the collision and of the pull gather, solver.rs:131-136,
324-328, moving/field.rs:570-611).  Here the grid is split along x, the
slowest axis of the cell order (i*ny + j)*nz + k, so that a slab is one
contiguous range of cells: rank r owns the planes [x_begin, x_end).  Each
step pulls the post-collision populations of the neighbouring planes; the
only data that crosses a slab boundary is, per step,

  forward:  the populations moving in +x (c_x = +1) of the last owned plane
            to the right neighbour, and those moving in -x of the first owned
            plane to the left neighbour (5 directions of D3Q19, 9 of D3Q27:
            ny*nz*5 values per face);
  adjoint:  the transposed pull reads x + c_q, so the cotangents of the
            directions with c_x = -1 of the last owned plane go right and
            those with c_x = +1 of the first owned plane go left.

A slab holds ghost planes beside its owned planes (one, or the design
filter's reach when it is wider); ghost cells are not stepped, and the
exchanged values land in the slots of the ghost plane next to the owned
range.  Scalars (mass, port exchange, responses, norms) are partial sums per
rank, reduced across ranks by the driver in FP64.

This module holds the partition, the halo plan and a driver over a backend
(one slab of the CUDA library, implexity_b200.solver.SlabSolver, or a test
backend) and a communicator (torch.distributed point-to-point and
all-reduce: NCCL between GPUs, gloo on CPU).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# velocity x-components in the lattice orderings of d3q19.rs:29-51 and
# moving/lattice.rs:93-121 (rest first, then lexicographic (x, y, z))
CX = {
    19: [0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1],
    27: [0] + [a for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1) if (a, b, c) != (0, 0, 0)],
}


def crossing(q: int, sign: int) -> list[int]:
    """Directions whose x velocity is `sign` (+1 or -1)."""
    return [i for i, c in enumerate(CX[q]) if c == sign]


@dataclass(frozen=True)
class Slab:
    rank: int
    world: int
    nx: int
    x_begin: int  # first owned plane (global index)
    x_end: int    # one past the last owned plane
    periodic_x: bool

    @property
    def left(self) -> int | None:
        """Rank owning the plane before x_begin (None at a closed domain end)."""
        if self.rank > 0:
            return self.rank - 1
        return self.world - 1 if self.periodic_x else None

    @property
    def right(self) -> int | None:
        if self.rank < self.world - 1:
            return self.rank + 1
        return 0 if self.periodic_x else None


def partition(nx: int, world: int, periodic_x: bool = False) -> list[Slab]:
    """Contiguous, balanced x ranges (the first nx % world ranks take one
    plane more); every rank needs at least two planes."""
    if world < 1 or nx < 2 * world:
        raise ValueError(f"cannot split {nx} x-planes over {world} ranks (two planes per rank at least)")
    base, extra = divmod(nx, world)
    out, x = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append(Slab(r, world, nx, x, x + n, periodic_x))
        x += n
    return out


@dataclass(frozen=True)
class HaloMessage:
    """One direction set of one boundary plane: which slab side it leaves
    from (to that side's neighbour) and which directions it carries."""

    side: str        # "left" or "right"
    directions: tuple


def halo_plan(q: int, kind: str) -> list[HaloMessage]:
    """The messages a slab sends per step ("state": forward, "adjoint":
    transposed step); it receives the mirror messages into its ghost planes
    (what leaves on the right arrives in the right neighbour's left ghost)."""
    plus, minus = tuple(crossing(q, +1)), tuple(crossing(q, -1))
    if kind == "state":
        return [HaloMessage("right", plus), HaloMessage("left", minus)]
    if kind == "adjoint":
        return [HaloMessage("right", minus), HaloMessage("left", plus)]
    raise ValueError(kind)


class TorchComm:
    """Point-to-point halo exchange and FP64 all-reduce over torch.distributed
    (NCCL between GPUs, gloo on CPU).  Every rank posts the same calls in the
    same order."""

    def __init__(self):
        import torch.distributed as dist

        self.dist = dist
        self.rank = dist.get_rank()
        self.world = dist.get_world_size()

    def exchange(self, sends: dict, recv_like: dict, peers: dict) -> dict:
        """sends[side] -> peers[side]; returns what arrives from each side."""
        import torch

        # tag 0: travelling right (arrives at the receiver's left), tag 1: travelling left
        tag_out = {"right": 0, "left": 1}
        tag_in = {"left": 0, "right": 1}
        mirror = {"left": "right", "right": "left"}
        ops, recvs = [], {}
        for side in ("left", "right"):
            peer = peers[side]
            if peer is None:
                continue
            if peer == self.rank:  # periodic x on one rank: the slab is its own neighbour
                recvs[side] = sends[mirror[side]].clone()
                continue
            recvs[side] = torch.empty_like(recv_like[side])
            ops.append(self.dist.P2POp(self.dist.irecv, recvs[side], peer, tag=tag_in[side]))
            ops.append(self.dist.P2POp(self.dist.isend, sends[side], peer, tag=tag_out[side]))
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
        return recvs

    def allreduce(self, values, op: str = "sum") -> np.ndarray:
        import torch

        dev = "cuda" if self.dist.get_backend() == "nccl" else "cpu"
        t = torch.as_tensor(np.asarray(values, dtype=np.float64), device=dev).clone()
        red = {"sum": self.dist.ReduceOp.SUM, "min": self.dist.ReduceOp.MIN, "max": self.dist.ReduceOp.MAX}[op]
        self.dist.all_reduce(t, op=red)
        return t.cpu().numpy()


class SlabDriver:
    """Runs the decomposed forward trajectory with admission, the responses and
    the steady adjoint over one slab backend and a communicator.

    Backend interface (one slab):
      q, slab                         lattice size and Slab
      halo_pack(kind, msg) -> tensor  the values `msg` sends from the owned boundary plane
      halo_unpack(kind, msg, tensor)  values arriving from msg.side into the ghost plane
      forward_begin()                 the initial state
      forward_stage(t)                work of step t before the exchange (may be none)
      forward_finish(t)               the rest of step t
      exchange_before_end, forward_end()  (optional) a last exchange and a read of the final state
      exchange_before_first_step      (optional, default True) False when forward_begin already
                                      leaves the ghost slots of the initial state filled
      diagnostics() -> (n_states, 5)  partial admission sums of every state: mass, exchange,
                                      min population, max |u|^2, non-finite flag
      responses() -> 8                partial responses of the final state
      adjoint_begin(weights) -> |lambda_0|^2 partial
      adjoint_stage()                 work of a transposed step before the exchange (may be none)
      adjoint_finish(want_norm) -> |lambda_k|^2 partial
      gradient() -> array             this rank's share of the design gradient (whole-problem size)
    """

    def __init__(self, backend, comm, mach_limit: float, mass_drift_limit: float = 1e-6):
        self.b = backend
        self.c = comm
        self.mach_limit = mach_limit
        self.mass_drift_limit = mass_drift_limit
        s = backend.slab
        self.peers = {"left": s.left, "right": s.right}

    def _exchange(self, kind: str):
        full = halo_plan(self.b.q, kind)
        plan = [m for m in full if self.peers[m.side] is not None]
        if not plan:
            return
        sends = {m.side: self.b.halo_pack(kind, m) for m in plan}
        # both messages of a plan have the same size (as many +x as -x directions)
        like = next(iter(sends.values()))
        arrived = self.c.exchange(sends, {"left": like, "right": like}, self.peers)
        mirror = {"left": "right", "right": "left"}
        for m in full:
            src = mirror[m.side]  # the neighbour on src sent its m.side message to us
            if src in arrived:
                self.b.halo_unpack(kind, HaloMessage(src, m.directions), arrived[src])

    def forward(self, steps: int) -> dict:
        self.b.forward_begin()
        first = getattr(self.b, "exchange_before_first_step", True)
        for t in range(steps):
            self.b.forward_stage(t)
            if t > 0 or first:
                self._exchange("state")
            self.b.forward_finish(t)
        if getattr(self.b, "exchange_before_end", False):
            # a backend that reduces a state while reading it needs the last halos too
            self._exchange("state")
        if hasattr(self.b, "forward_end"):
            self.b.forward_end()
        d = np.asarray(self.b.diagnostics(), dtype=np.float64)
        sums = self.c.allreduce(d[:, :2].ravel(), "sum").reshape(-1, 2)
        mins = self.c.allreduce(d[:, 2], "min")
        maxs = self.c.allreduce(d[:, 3:5].ravel(), "max").reshape(-1, 2)
        return self._admit(sums[:, 0], sums[:, 1], mins, maxs[:, 0], maxs[:, 1])

    def _admit(self, mass, exchange, min_f, max_u2, nonfinite) -> dict:
        """LbmProblem::admit (solver.rs:708-793) on the reduced per-state sums."""
        mach = float(np.sqrt(np.max(max_u2)) * np.sqrt(3.0))
        cum = np.concatenate([[0.0], np.cumsum(exchange[1:])])
        drift = float(np.max(np.abs(mass - (mass[0] + cum))) / mass[0])
        bad = bool(np.any(nonfinite > 0)) or not float(np.min(min_f)) > 0
        return {"maximum_mach": mach, "relative_mass_drift": drift, "minimum_population": float(np.min(min_f)),
                "admitted": (not bad) and mach <= self.mach_limit and drift <= self.mass_drift_limit,
                "mass": mass, "exchange": exchange}

    def responses(self) -> np.ndarray:
        return self.c.allreduce(self.b.responses(), "sum")

    def gradient_steady(self, weights, tolerance: float = 1e-8, max_iterations: int = 100000,
                        check_every: int = 50) -> tuple[np.ndarray, dict]:
        n0 = float(np.sqrt(self.c.allreduce([self.b.adjoint_begin(weights)], "sum")[0]))
        resid, it = (0.0 if n0 == 0 else 1.0), 0
        while n0 > 0 and it < max_iterations:
            self.b.adjoint_stage()
            self._exchange("adjoint")
            nrm2 = self.b.adjoint_finish(want_norm=(it + 1) % check_every == 0)
            it += 1
            if (it % check_every) == 0:
                resid = float(np.sqrt(self.c.allreduce([nrm2], "sum")[0])) / n0
                if resid <= tolerance:
                    break
        return self.c.allreduce(self.b.gradient(), "sum"), {"iterations": it, "residual": resid,
                                                          "converged": resid <= tolerance}
