"""Batched PSTM over offset/azimuth classes: one persistent launch, captured
in a CUDA graph.

A survey is split into classes (offset x azimuth bins, the selection of
``MigrationGeometry.get_indices_for_bin``, models/migration_geometry.py:256-283).
Each class gets its own plan (trace list per output tile) and its own output
image (common-image-gather volumes), and ``BatchedPSTM.migrate`` runs all classes
in one launch of the persistent kernel.  ``capture`` records the per-class trace
staging plus the batched launch into a ``torch.cuda.CUDAGraph``; ``replay``
re-runs it with the current contents of the captured input buffers.

The reference has no batched path: its worker migrates bin after bin in a
Python loop (views/migration_monitor_dialog.py:201-430).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib, autotune
from .kirchhoff import PSTMPlan, velocity_strides


@dataclass
class OffsetAzimuthBin:
    """One offset/azimuth class, as the reference's binning table defines it
    (models/binning.py:34-60): offsets in [offset_min, offset_max), azimuths in
    [azimuth_min, azimuth_max) degrees clockwise from north, wrapping through
    360 when azimuth_max < azimuth_min."""
    name: str
    offset_min: float
    offset_max: float
    azimuth_min: float = 0.0
    azimuth_max: float = 360.0
    enabled: bool = True
    metadata: Dict[str, Any] = field(default_factory=dict)

    def __post_init__(self):
        if self.offset_min < 0 or self.offset_max <= self.offset_min:
            raise ValueError(f"bin {self.name}: need 0 <= offset_min < offset_max")
        if not (0.0 <= self.azimuth_min <= 360.0 and 0.0 <= self.azimuth_max <= 360.0):
            raise ValueError(f"bin {self.name}: azimuths must lie in [0, 360]")


def offset_azimuth(source_x: torch.Tensor, source_y: torch.Tensor, receiver_x: torch.Tensor,
                   receiver_y: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
    """Offset (float32, m) and source-to-receiver azimuth (degrees in [0, 360),
    clockwise from north) on the coordinates' device, in the coordinates'
    precision as the reference forms them (models/migration_geometry.py:88-116):
    dx, dy and dx^2 + dy^2 in that precision, the square root correctly
    rounded (taken in float64 and rounded once, which equals numpy's IEEE
    square root; torch's CPU float32 sqrt is not correctly rounded), and
    (degrees + 360) % 360 in that precision.  The arctangent is taken in
    float64 and rounded once: numpy's float32 arctan2 is a vectorised
    approximation whose last bit depends on the CPU it runs on, so only a
    trace within an ulp or two of an azimuth edge could be classed
    differently from a given numpy build."""
    dx = receiver_x - source_x
    dy = receiver_y - source_y
    off = torch.sqrt((dx * dx + dy * dy).to(torch.float64)).to(torch.float32)
    deg = torch.rad2deg(torch.atan2(dx.to(torch.float64), dy.to(torch.float64))).to(dx.dtype)
    az = torch.remainder(deg + 360.0, 360.0)
    return off, az


def bin_indices(source_x: torch.Tensor, source_y: torch.Tensor, receiver_x: torch.Tensor,
                receiver_y: torch.Tensor, bins: Sequence[OffsetAzimuthBin],
                inclusive: bool = False) -> List[torch.Tensor]:
    """Trace indices (on the coordinates' device) of every enabled bin.

    Membership is the binning table's (models/binning.py:136-158): offsets in
    [offset_min, offset_max), azimuths in [azimuth_min, azimuth_max), wrapping
    through north when azimuth_max < azimuth_min.  ``inclusive=True`` takes
    MigrationGeometry.get_indices_for_bin's closed intervals instead
    (models/migration_geometry.py:256-283), under which neighbouring bins
    share their edges.

    The reference assigns traces bin by bin on the host and the worker then
    migrates bin after bin (models/binning.py:304-325,
    views/migration_monitor_dialog.py:201-254).  Here the class of each trace is
    found on the device and one stable sort groups the classes, so the whole
    binning costs one device-to-host copy of the class sizes.  Bins that
    overlap are resolved bin by bin instead (a trace may then belong to several).
    """
    bins = [b for b in bins if b.enabled]
    off, az = offset_azimuth(source_x, source_y, receiver_x, receiver_y)

    def member(b):
        if inclusive:
            ok = (off >= b.offset_min) & (off <= b.offset_max)
            if b.azimuth_max < b.azimuth_min:
                return ok & ((az >= b.azimuth_min) | (az <= b.azimuth_max))
            return ok & (az >= b.azimuth_min) & (az <= b.azimuth_max)
        ok = (off >= b.offset_min) & (off < b.offset_max)
        if b.azimuth_max < b.azimuth_min:
            return ok & ((az >= b.azimuth_min) | (az < b.azimuth_max))
        return ok & (az >= b.azimuth_min) & (az < b.azimuth_max)

    masks = [member(b) for b in bins]
    if not masks:
        return []
    count = torch.stack(masks).sum(0)
    if bool((count > 1).any()):  # overlapping bins
        return [torch.nonzero(m).flatten() for m in masks]
    cls = torch.full(off.shape, len(bins), dtype=torch.int64, device=off.device)
    for i, m in enumerate(masks):
        cls = torch.where(m, torch.full_like(cls, i), cls)
    order = torch.argsort(cls, stable=True)
    sizes = torch.bincount(cls, minlength=len(bins) + 1)[:len(bins)].tolist()
    out, start = [], 0
    for n in sizes:
        out.append(order[start:start + n])
        start += n
    return out


def class_indices(offset: np.ndarray, azimuth: np.ndarray, n_offset_bins: int,
                  n_azimuth_bins: int, max_offset: float) -> List[np.ndarray]:
    """Trace indices of each (offset bin, azimuth sector) class, offset-major."""
    ob = np.minimum((offset / max_offset * n_offset_bins).astype(np.int64), n_offset_bins - 1)
    ab = np.minimum((azimuth / 360.0 * n_azimuth_bins).astype(np.int64), n_azimuth_bins - 1)
    key = ob * n_azimuth_bins + ab
    order = np.argsort(key, kind="stable")
    bounds = np.searchsorted(key[order], np.arange(n_offset_bins * n_azimuth_bins + 1))
    return [order[bounds[i]:bounds[i + 1]] for i in range(n_offset_bins * n_azimuth_bins)]


class BatchedPSTM:
    """All classes of a survey in one persistent launch per kernel shape.

    ``plans`` share grid, parameters and storage; ``velocity`` is V_rms for all
    classes.  Images (and folds) are allocated here, one per class.  Classes
    whose plans have different kernel shapes (per-class tuning) are grouped by
    shape, one persistent launch per group; ``shapes`` lists each class's
    shape id and ``capture`` records every group's launch in the same graph.
    """

    def __init__(self, plans: Sequence[PSTMPlan], velocity: torch.Tensor, with_fold: bool = True):
        if not plans:
            raise ValueError("empty batch")
        self.plans = list(plans)
        p0 = self.plans[0]
        self.device = p0.device
        self.velocity, vst, vsc = velocity_strides(velocity.to(self.device), p0.n_times,
                                                   p0.n_cols)
        shape = (p0.n_times, p0.n_il, p0.n_xl)
        self.images = [torch.zeros(shape, device=self.device) for _ in self.plans]
        self.folds = [torch.zeros(shape, device=self.device) for _ in self.plans] \
            if with_fold else None
        self.shapes = [int(p.stats()["variant"]) for p in self.plans]
        self._lib = _lib.lib()
        self._handles: List[C.c_void_p] = []
        try:
            for sid in sorted(set(self.shapes)):
                idx = [i for i, v in enumerate(self.shapes) if v == sid]
                P = C.c_void_p * len(idx)
                plans_arr = P(*[self.plans[i]._handle.value for i in idx])
                imgs = P(*[self.images[i].data_ptr() for i in idx])
                folds = P(*[self.folds[i].data_ptr() for i in idx]) if with_fold else None
                h = C.c_void_p(None)
                _lib.check(self._lib.pstm_batch_create(
                    C.byref(h), plans_arr, len(idx), imgs, folds, self.velocity.data_ptr(),
                    vst, vsc, torch.cuda.current_stream().cuda_stream))
                self._handles.append(h)
        except Exception:
            self.close()
            raise
        self._graph: Optional[torch.cuda.CUDAGraph] = None
        self._inputs: List[torch.Tensor] = []
        self.launches_per_replay = 0

    def close(self):
        if getattr(self, "_handles", None):
            self._graph = None
            for h in self._handles:
                if h.value:
                    self._lib.pstm_batch_destroy(h)
            self._handles = []
        if getattr(self, "_own_plans", False):
            for p in self.plans:
                p.close()
            self._own_plans = False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, traces: Sequence[torch.Tensor]) -> None:
        for p, t in zip(self.plans, traces):
            p.load_traces(t)

    def migrate(self) -> None:
        for h in self._handles:
            _lib.check(self._lib.pstm_batch_migrate(h, torch.cuda.current_stream().cuda_stream))

    def check(self) -> None:
        for p in self.plans:
            p.check()

    # ------------------------------------------------------- from a survey
    @classmethod
    def from_survey(cls, traces: torch.Tensor, source_x: torch.Tensor, source_y: torch.Tensor,
                    receiver_x: torch.Tensor, receiver_y: torch.Tensor,
                    bins: Sequence[OffsetAzimuthBin], velocity: torch.Tensor,
                    with_fold: bool = True, **plan_kwargs) -> "BatchedPSTM":
        """Bins a whole survey on the device and builds one plan per non-empty
        class (``plan_kwargs`` as for ``PSTMPlan``: grid, axes, aperture ...).
        ``traces`` (n_samples, n_traces) stay on the device; each class's traces
        are gathered into ``self.class_traces`` and loaded.  ``self.bins`` and
        ``self.indices`` name the classes and their traces.  ``variant="auto"``
        picks each class's kernel shape with the autotuner (cached per problem
        class)."""
        dev = traces.device
        idx = bin_indices(source_x.to(dev), source_y.to(dev), receiver_x.to(dev),
                          receiver_y.to(dev), bins)
        keep = [(b, i) for b, i in zip([b for b in bins if b.enabled], idx) if i.numel() > 0]
        if not keep:
            raise ValueError("no trace falls in an enabled bin")
        plans, class_traces = [], []
        for _, i in keep:
            coords = [a.to(dev).index_select(0, i).contiguous()
                      for a in (source_x, source_y, receiver_x, receiver_y)]
            kw = dict(plan_kwargs)
            if kw.get("variant") == "auto":
                kw["variant"] = autotune.choose_variant(coords, velocity=velocity.to(dev),
                                                        **{k: v for k, v in kw.items()
                                                           if k != "variant"})
            plans.append(PSTMPlan(*coords, **kw))
            class_traces.append(traces.index_select(1, i).contiguous())
        batch = cls(plans, velocity, with_fold=with_fold)
        batch._own_plans = True
        batch.bins = [b for b, _ in keep]
        batch.indices = [i for _, i in keep]
        batch.class_traces = class_traces
        batch.load(class_traces)
        return batch

    # ------------------------------------------------------------ CUDA graph
    def capture(self, traces: Sequence[torch.Tensor]) -> None:
        """Capture [stage every class's traces, batched migration] in a CUDA graph.

        ``traces`` are device buffers whose contents are read at every replay.
        One eager run precedes the capture (it allocates the plans' staging
        copies, which must not happen inside the capture)."""
        self._inputs = [t.contiguous() for t in traces]
        self.load(self._inputs)
        self.migrate()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        n0 = self._lib.pstm_launch_count()
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.load(self._inputs)
                self.migrate()
        # kernels recorded in the graph (each replay launches them all)
        self.launches_per_replay = int(self._lib.pstm_launch_count() - n0)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        self._graph = g

    def replay(self) -> None:
        if self._graph is None:
            raise RuntimeError("capture() first")
        self._graph.replay()
