"""Batched probe updates: several fields (independent scenes) and cascades of
different divisions through one launch per stage (sb_solve_batch).

The reference updates one field's cascades with one compute pass each
(gi_probes.js:3732-3840); there is no cross-scene batching in it. Here a frame
of many fields runs every field's tick lanes (beginTick), one batched solve of
all their probe ranges plus any extra cascades, then endTick on each. The
per-item arithmetic is the per-solve arithmetic, so a batched frame produces
the same atlases as the same solves run one by one.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import _abi
from .field import ProbeField


@dataclass
class SolveItem:
    field: ProbeField
    cascade: int
    probeOffset: int
    updatedCount: int


def solveBatch(items) -> None:
    """One sb_solve_batch over `items` (SolveItem); the first item's field
    owns the launch's stream and queues."""
    items = list(items)
    if not items:
        return
    arr = (_abi.sb_solve_item * len(items))()
    for i, it in enumerate(items):
        arr[i].ctx = it.field.ctx
        arr[i].cascade = it.cascade
        arr[i].probeOffset = it.probeOffset
        arr[i].updatedCount = it.updatedCount
    lead = items[0].field
    _abi.check(lead._lib.sb_solve_batch(arr, len(items)), lead.ctx)


class BatchedFrame:
    """Per-frame driver of several fields: each field's C0 tick range, plus
    extra cascades (field, ci) solved in full every frame."""

    def __init__(self, fields, extra=()):
        self.fields = list(fields)
        self.extra = list(extra)

    def items(self, frames) -> list:
        out = [SolveItem(f, fr["cascade"], fr["probeOffset"], fr["updatedCount"])
               for f, fr in zip(self.fields, frames)]
        out += [SolveItem(f, ci, 0, f.cascadeProbes(ci)) for f, ci in self.extra]
        return out

    def tick(self) -> list:
        """All solves of the frame in one batched launch."""
        frames = [f.beginTick() for f in self.fields]
        solveBatch(self.items(frames))
        for f, fr in zip(self.fields, frames):
            f.endTick(fr)
        return frames

    def tickPlain(self) -> list:
        """The same solves as per-field launches, one after another."""
        frames = [f.beginTick() for f in self.fields]
        for it in self.items(frames):
            _abi.check(it.field._lib.sb_solve(it.field.ctx, it.cascade, it.probeOffset, it.updatedCount),
                       it.field.ctx)
        for f, fr in zip(self.fields, frames):
            f.endTick(fr)
        return frames

    def setStream(self, stream) -> None:
        """Put every field on one CUDA stream (an int handle)."""
        for f in self.fields:
            _abi.check(f._lib.sb_set_stream(f.ctx, C.c_void_p(int(stream))), f.ctx)


def autotune(field: ProbeField, cascade: int = 0) -> dict:
    """sb_autotune on one field: the fastest of the candidate traversal
    tunings for its scene, kept on its context; the probe state is restored."""
    t = _abi.sb_tuning()
    _abi.check(field._lib.sb_autotune(field.ctx, cascade, C.byref(t)), field.ctx)
    return dict(traceBlock=t.traceBlock, sortKey=t.sortKey, smemTlasNodes=t.smemTlasNodes, bvhKind=t.bvhKind,
                smemWideNodes=t.smemWideNodes)


def autotuneBatch(items) -> dict:
    """sb_autotune_batch: the batched launches' block size and ray order timed
    on the batch itself, kept on the lead context."""
    items = list(items)
    arr = (_abi.sb_solve_item * len(items))()
    for i, it in enumerate(items):
        arr[i].ctx = it.field.ctx
        arr[i].cascade = it.cascade
        arr[i].probeOffset = it.probeOffset
        arr[i].updatedCount = it.updatedCount
    t = _abi.sb_tuning()
    lead = items[0].field
    _abi.check(lead._lib.sb_autotune_batch(arr, len(items), C.byref(t)), lead.ctx)
    return dict(traceBlock=t.traceBlock, sortKey=t.sortKey)


@dataclass
class Lane:
    """A field's device-side motion lane in a captured frame."""
    field: ProbeField
    refits: list          # [(root, end)] BLAS node ranges refit every frame
    refitTlas: bool = True


class GraphFrame:
    """A BatchedFrame whose per-frame chain (every lane's refits and TLAS
    refit, then the batched solve) is one CUDA graph (sb_graph_capture_batch,
    sb_graph_launch). Each launch takes the fields' current uniforms (jitter
    epoch, hysteresis exponent); a changed probe range captures again."""

    def __init__(self, frame: BatchedFrame, lanes):
        self.frame = frame
        self.lanes = list(lanes)
        self._captured = None
        self._keep = []

    def _capture(self, items) -> None:
        lanes = (_abi.sb_frame_lane * max(1, len(self.lanes)))()
        self._keep = []
        for i, l in enumerate(self.lanes):
            roots = (C.c_uint32 * max(1, len(l.refits)))(*[r for r, _ in l.refits])
            ends = (C.c_uint32 * max(1, len(l.refits)))(*[e for _, e in l.refits])
            self._keep += [roots, ends]
            lanes[i].ctx = l.field.ctx
            lanes[i].refitRoots = C.cast(roots, C.c_void_p)
            lanes[i].refitEnds = C.cast(ends, C.c_void_p)
            lanes[i].refitCount = len(l.refits)
            lanes[i].refitTlas = 1 if l.refitTlas else 0
        arr = (_abi.sb_solve_item * len(items))()
        for i, it in enumerate(items):
            arr[i].ctx = it.field.ctx
            arr[i].cascade = it.cascade
            arr[i].probeOffset = it.probeOffset
            arr[i].updatedCount = it.updatedCount
        lead = items[0].field
        _abi.check(lead._lib.sb_graph_capture_batch(lanes, len(self.lanes), arr, len(items)), lead.ctx)
        self._captured = [(it.field.ctx, it.cascade, it.probeOffset, it.updatedCount) for it in items]

    def tick(self) -> list:
        """One frame: captured (and run) the first time or when a probe range
        changed, replayed otherwise."""
        fr = self.frame
        frames = [f.beginTick() for f in fr.fields]
        items = fr.items(frames)
        key = [(it.field.ctx, it.cascade, it.probeOffset, it.updatedCount) for it in items]
        if key != self._captured:
            self._capture(items)
        else:
            lead = items[0].field
            _abi.check(lead._lib.sb_graph_launch(lead.ctx), lead.ctx)
        for f, x in zip(fr.fields, frames):
            f.endTick(x)
        return frames

    def dispose(self) -> None:
        if self._captured:
            lead = self.frame.fields[0]
            lead._lib.sb_graph_destroy(lead.ctx)
        self._captured = None
