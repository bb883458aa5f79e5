"""Slab-decomposed 2-D stepping: a grid split into y slabs, one per rank.

Each rank advances the rows it owns plus W overlap rows on each side that it
shares with its y neighbours, with one bound FP64 Stepper on that extended
slab, and every K steps swaps W rows with its neighbours.  Values next to the
extended slab's y edges are wrong (its y sides carry no neighbour data), and
the error moves inward by the stencil reach of one time step per step (H
rows: 1 for Allen-Cahn Euler, 2 for Cahn-Hilliard Euler, 4 for Allen-Cahn
RK4, 8 for Cahn-Hilliard RK4).  With W >= K * H the owned rows after K steps
are exactly the cells of a whole-grid run, bit for bit, since every cell sees
the same neighbours and the same arithmetic.  One exchange of W rows per K
steps replaces the per-stage halo exchange of the reference's sequence.

The y sides of an extended slab that border a neighbour take any boundary
condition (only rows that the next exchange overwrites read them): both
periodic when x is periodic and both y sides border neighbours, so the
Cahn-Hilliard pair kernels still apply; zero-flux otherwise.  With
poison=True they take none and their stored ghost rows hold NaN instead, so
that any row read before its exchange turns NaN (the check that the overlap
and the exchanges cover every owned row: the edge error itself often decays
below one ulp before it arrives).  A slab on a non-periodic global y edge
keeps the true condition there and has no overlap on that side.

Exchanges: DistExchange (torch.distributed point-to-point: NCCL across GPUs,
gloo on CPU) or LocalExchange (several slabs in one process, direct copies).
Per exchange, between a pair of ranks the upward message (the sender's top
owned rows, the receiver's lower overlap) goes first, then the downward one,
so that two ranks that are each other's lower and upper neighbour (two slabs
of a periodic grid) still match.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Sequence

from . import BC_NONE, BC_NOFLUX, BC_PERIODIC, EULER, F64, PHYS_AC, PHYS_CH, RK4, Stepper, make_grid

# rows of a field a time step reads beyond a cell (the stencil reach of the step)
HALO_PER_STEP = {(PHYS_AC, EULER): 1, (PHYS_CH, EULER): 2, (PHYS_AC, RK4): 4, (PHYS_CH, RK4): 8}


@dataclass
class Slab:
    rank: int
    nranks: int
    y0: int  # first owned global row
    y1: int  # one past the last owned global row
    lo: int  # overlap rows below (0 on a non-periodic global edge)
    hi: int  # overlap rows above

    @property
    def owned(self) -> int:
        return self.y1 - self.y0

    @property
    def ny_ext(self) -> int:
        return self.owned + self.lo + self.hi

    @property
    def lo_rank(self) -> int:
        return (self.rank - 1) % self.nranks

    @property
    def hi_rank(self) -> int:
        return (self.rank + 1) % self.nranks


def slabs(ny: int, nranks: int, overlap: int, periodic_y: bool) -> list[Slab]:
    """Balanced split of ny rows over nranks; every slab owns at least
    `overlap` rows (its neighbours' overlaps come from them)."""
    if nranks < 1 or overlap < 0:
        raise ValueError("slabs: nranks >= 1 and overlap >= 0")
    out = []
    for r in range(nranks):
        y0, y1 = r * ny // nranks, (r + 1) * ny // nranks
        if nranks > 1 and y1 - y0 < overlap:
            raise ValueError(f"slabs: slab {r} owns {y1 - y0} rows, fewer than the overlap {overlap}")
        lo = overlap if nranks > 1 and (periodic_y or r > 0) else 0
        hi = overlap if nranks > 1 and (periodic_y or r < nranks - 1) else 0
        out.append(Slab(r, nranks, y0, y1, lo, hi))
    return out


def overlap_for(phys: int, scheme: int, steps_per_exchange: int) -> int:
    """Overlap rows that keep the owned rows exact for steps_per_exchange steps."""
    try:
        return HALO_PER_STEP[(phys, scheme)] * steps_per_exchange
    except KeyError:
        raise ValueError("slab stepping covers 2-D AC and CH with Euler or RK4") from None


class GpuEngine:
    """A bound FP64 Stepper on one extended slab (the state stays in the
    caller's two device buffers, so rows can be swapped in place)."""

    def __init__(self, phys, scheme, prm, dt, grid, init, torch, steps_per_graph=0):
        self.st = Stepper(phys, scheme, F64, prm, dt, grid)
        self.buf = [torch.as_tensor(init, dtype=torch.float64).cuda().contiguous()]
        self.buf.append(self.buf[0].clone())
        self.st.bind([self.buf[0]], [self.buf[1]])
        if steps_per_graph:
            self.st.set_graph(steps_per_graph)

    def advance(self, k: int):
        self.st.advance(k)

    def state(self):
        return self.buf[self.st.current()]

    def close(self):
        self.st.close()


class SlabStepper:
    """One rank's slab of a 2-D field (stored layout, ghost 1).

    `engine_factory(grid, init)` returns an object with advance(k) and
    state() (a torch tensor of the extended slab's stored array, updated in
    place); by default a GpuEngine."""

    def __init__(self, phys: int, scheme: int, prm: Sequence[float], dt: float, n: Sequence[int], slab: Slab,
                 global_stored, d=(1.0, 1.0), bc=(BC_PERIODIC,) * 4, bc_val=(0.0,) * 4,
                 engine_factory: Callable | None = None, torch=None, steps_per_graph: int = 0,
                 poison: bool = False):
        import torch as _torch
        self.torch = torch or _torch
        self.slab, self.n = slab, (int(n[0]), int(n[1]))
        nx, ny = self.n
        periodic_y = bc[2] == BC_PERIODIC
        bcs = list(bc[:4]) + [BC_PERIODIC, BC_PERIODIC]
        vals = list(bc_val[:4]) + [0.0, 0.0]
        if slab.lo or slab.hi:
            both = slab.lo and slab.hi
            side = BC_PERIODIC if both and bc[0] == BC_PERIODIC else BC_NOFLUX
            if poison:
                side = BC_NONE  # the stored ghost row, NaN: wrong rows become NaN
            if slab.lo:
                bcs[2], vals[2] = side, 0.0
            if slab.hi:
                bcs[3], vals[3] = side, 0.0
        self.bcs, self.vals = tuple(bcs), tuple(vals)
        self.grid = make_grid((nx, slab.ny_ext), tuple(d[:2]), 1, self.bcs, self.vals)
        # the extended slab's rows: global rows y0 - lo .. y1 + hi (wrapped when periodic)
        g = self.torch.as_tensor(global_stored)
        init = self.torch.zeros((3, slab.ny_ext + 2, nx + 2), dtype=self.torch.float64)
        for j in range(-1, slab.ny_ext + 1):
            gy = slab.y0 - slab.lo + j
            if periodic_y:
                gy %= ny
            elif gy < -1 or gy > ny:
                continue
            init[:, j + 1, :] = g[:, gy + 1, :]
        if poison:
            if slab.lo:
                init[:, 0, :] = float("nan")
            if slab.hi:
                init[:, slab.ny_ext + 1, :] = float("nan")
        if engine_factory is None:
            engine_factory = lambda grid, a: GpuEngine(phys, scheme, prm, dt, grid, a, self.torch, steps_per_graph)
        self.engine = engine_factory(self.grid, init)

    # stored-row ranges (physical plane index 1, stored row = local row + 1)
    def _rows(self, a, j0, j1):
        return a[1, j0 + 1:j1 + 1, :]

    def send_rows(self):
        """(rows for the lower neighbour's upper overlap, rows for the upper
        neighbour's lower overlap): this slab's first and last W owned rows
        (every overlapped side is W rows wide)."""
        s, a = self.slab, self.engine.state()
        w = max(s.lo, s.hi)
        down = self._rows(a, s.lo, s.lo + w).contiguous() if s.lo else None
        up = self._rows(a, s.lo + s.owned - w, s.lo + s.owned).contiguous() if s.hi else None
        return down, up

    def recv_into(self, from_lo, from_hi):
        s, a = self.slab, self.engine.state()
        if from_lo is not None:
            self._rows(a, 0, s.lo).copy_(from_lo)
        if from_hi is not None:
            self._rows(a, s.lo + s.owned, s.ny_ext).copy_(from_hi)

    def owned_rows(self):
        """The owned physical rows, (owned, nx)."""
        s = self.slab
        return self._rows(self.engine.state(), s.lo, s.lo + s.owned)[:, 1:-1]

    def advance(self, k: int):
        self.engine.advance(k)

    def close(self):
        if hasattr(self.engine, "close"):
            self.engine.close()


class LocalExchange:
    """Row swaps between slabs held by one process (direct tensor copies)."""

    def __init__(self, steppers: Sequence[SlabStepper]):
        self.s = list(steppers)

    def __call__(self):
        out = [st.send_rows() for st in self.s]
        for st in self.s:
            sl = st.slab
            from_lo = out[sl.lo_rank][1] if sl.lo else None
            from_hi = out[sl.hi_rank][0] if sl.hi else None
            st.recv_into(from_lo, from_hi)


class DistExchange:
    """Row swaps with the y neighbours over torch.distributed point-to-point
    operations (one slab per rank)."""

    def __init__(self, stepper: SlabStepper, dist):
        self.st, self.dist = stepper, dist

    def __call__(self):
        dist, st, sl = self.dist, self.st, self.st.slab
        down, up = st.send_rows()
        torch = st.torch
        a = st.engine.state()
        from_lo = torch.empty_like(a[1, 1:sl.lo + 1, :]) if sl.lo else None
        from_hi = torch.empty_like(a[1, 1:sl.hi + 1, :]) if sl.hi else None
        ops = []
        # upward messages first, then downward ones (see the module note)
        if sl.hi:
            ops.append(dist.P2POp(dist.isend, up, sl.hi_rank))
        if sl.lo:
            ops.append(dist.P2POp(dist.irecv, from_lo, sl.lo_rank))
        if sl.lo:
            ops.append(dist.P2POp(dist.isend, down, sl.lo_rank))
        if sl.hi:
            ops.append(dist.P2POp(dist.irecv, from_hi, sl.hi_rank))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        st.recv_into(from_lo, from_hi)


def run(steppers: Sequence[SlabStepper], exchange: Callable, nsteps: int, steps_per_exchange: int):
    """Advance every slab nsteps time steps, swapping rows every
    steps_per_exchange steps (and after the last group)."""
    done = 0
    while done < nsteps:
        k = min(steps_per_exchange, nsteps - done)
        for st in steppers:
            st.advance(k)
        done += k
        exchange()
