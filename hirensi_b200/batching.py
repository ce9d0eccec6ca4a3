"""Batches of shots with uneven record lengths and receiver sets.

The reference solves one source at a time, each with its own NSTEP and EqDis /
Dis_meas (S4/Program_Main.F90:379-470).  The GPU path advances up to
HRN_MAX_SHOTS shots together so that the operator is streamed once per stage
for all of them.  This module plans the batches and packs the shots of a batch
into the arrays of one context:

* ``plan``: shots sorted by record length, longest first, cut into batches, so
  that a batch steps little past its shorter shots;
* ``pack``: one batch's union receiver list, the mask of each shot's receivers,
  the per-shot record lengths, and sources and data padded to the batch length;
* ``unpack_traces``: each shot's own traces out of the batch traces.

Duplicate receiver equations inside a shot's list are kept: the union holds
each equation as many times as the shot that lists it most, and shot s uses the
first m_s copies in its own order, so the residuals of duplicates still add
before squaring as in Compute_Misfit (S4/Solver_PETSc_Inverse.F90:591-657).
"""
from __future__ import annotations

import dataclasses
from collections import Counter

import numpy as np

MAX_SHOTS = 8


@dataclasses.dataclass
class Shot:
    src_eq: np.ndarray        # [nsrc] equations of the force entries
    src_b: np.ndarray         # [nsrc] unscaled force values
    ftab: np.ndarray          # [nstep + 1, 3] TIME_FUNCTION samples (t, t + dt, t + dt/2)
    eqdis: np.ndarray         # [nrec3] receiver equations (EqDis)
    dis: np.ndarray | None = None   # [nrec3, nstep + 1] measured data (Dis_meas transposed)

    @property
    def nstep(self) -> int:
        return int(self.ftab.shape[0]) - 1


@dataclasses.dataclass
class Batch:
    shots: list               # indices into the planned shot list
    nstep: int                # steps of the batch (its longest shot)
    src_eq: np.ndarray        # [nsrc] union of the force equations
    src_b: np.ndarray         # [nsrc, nshot]
    ftab: np.ndarray          # [nshot, nstep + 1, 3], zero past each shot's length
    eqdis: np.ndarray         # [nrec3] union receiver list
    nstep_shot: np.ndarray    # [nshot] int32
    rec_mask: np.ndarray      # [nshot, nrec3] uint8
    slots: list               # per shot: positions of its receiver entries in the union, in its order
    dis: np.ndarray | None    # [nshot, nrec3, nstep + 1] data padded with zeros, or None


def plan(lengths, max_shots: int = MAX_SHOTS) -> list[list[int]]:
    """Shot indices grouped into batches of at most max_shots, longest records first."""
    if not 1 <= max_shots <= MAX_SHOTS:
        raise ValueError(f"max_shots must be 1..{MAX_SHOTS}")
    order = sorted(range(len(lengths)), key=lambda i: (-int(lengths[i]), i))
    return [order[i:i + max_shots] for i in range(0, len(order), max_shots)]


def pack(shots: list[Shot], ids: list[int]) -> Batch:
    """The arrays of one context for the shots ``ids``."""
    sel = [shots[i] for i in ids]
    S = len(sel)
    if not 1 <= S <= MAX_SHOTS:
        raise ValueError(f"a batch holds 1..{MAX_SHOTS} shots")
    nstep = max(s.nstep for s in sel)
    # sources: union of equations, one column per shot
    src_eq = sorted({int(e) for s in sel for e in s.src_eq})
    col = {e: i for i, e in enumerate(src_eq)}
    src_b = np.zeros((len(src_eq), S))
    ftab = np.zeros((S, nstep + 1, 3))
    for k, s in enumerate(sel):
        for e, b in zip(np.asarray(s.src_eq), np.asarray(s.src_b, dtype=np.float64)):
            src_b[col[int(e)], k] += b
        ftab[k, : s.nstep + 1] = s.ftab
    # receivers: each equation as often as the shot that lists it most, in order of first use
    need: dict[int, int] = {}
    first: list[int] = []
    for s in sel:
        for e, m in Counter(int(e) for e in s.eqdis).items():
            if e not in need:
                first.append(e)
                need[e] = 0
            need[e] = max(need[e], m)
    union = [e for e in first for _ in range(need[e])]
    start = {}
    for q, e in enumerate(union):
        start.setdefault(e, q)
    mask = np.zeros((S, len(union)), np.uint8)
    slots = []
    for k, s in enumerate(sel):
        seen: Counter = Counter()
        pos = []
        for e in (int(v) for v in s.eqdis):
            q = start[e] + seen[e]
            seen[e] += 1
            mask[k, q] = 1
            pos.append(q)
        slots.append(np.asarray(pos, dtype=np.int64))
    dis = None
    if all(s.dis is not None for s in sel):
        dis = np.zeros((S, len(union), nstep + 1))
        for k, s in enumerate(sel):
            d = np.asarray(s.dis, dtype=np.float64)
            if d.shape != (len(s.eqdis), s.nstep + 1):
                raise ValueError("a shot's data must be [nrec3, nstep + 1]")
            dis[k][slots[k], : s.nstep + 1] = d
    return Batch(list(ids), nstep, np.asarray(src_eq, dtype=np.int32), src_b, ftab,
                 np.asarray(union, dtype=np.int32), np.asarray([s.nstep for s in sel], dtype=np.int32),
                 mask, slots, dis)


def unpack_traces(batch: Batch, traces: np.ndarray) -> list[np.ndarray]:
    """Each shot's traces [its nrec3, its nstep + 1] from the batch traces [nshot, nrec3, nstep + 1]."""
    return [np.ascontiguousarray(traces[k][batch.slots[k], : int(batch.nstep_shot[k]) + 1])
            for k in range(len(batch.shots))]


def configure(solver, batch: Batch, dt: float, store_position) -> None:
    """Set the shots, receivers and per-shot records of ``solver`` for ``batch``;
    store_position maps receiver equations to history positions (Mesh.store_position)."""
    solver.set_shots(batch.nstep, dt, batch.src_eq, batch.src_b, batch.ftab)
    solver.set_receivers(batch.eqdis, store_position(batch.eqdis))
    solver.set_shot_records(batch.nstep_shot, batch.rec_mask)
