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
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from .kirchhoff import PSTMPlan, velocity_strides


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
    """All classes of a survey in one persistent launch.

    ``plans`` share grid, parameters and storage; ``velocity`` is V_rms for all
    classes.  Images (and folds) are allocated here, one per class.
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
        n = len(self.plans)
        P = C.c_void_p * n
        plans_arr = P(*[p._handle.value for p in self.plans])
        imgs = P(*[t.data_ptr() for t in self.images])
        folds = P(*[t.data_ptr() for t in self.folds]) if with_fold else None
        self._lib = _lib.lib()
        self._handle = C.c_void_p(None)
        _lib.check(self._lib.pstm_batch_create(C.byref(self._handle), plans_arr, n, imgs, folds,
                                               self.velocity.data_ptr(), vst, vsc,
                                               torch.cuda.current_stream().cuda_stream))
        self._graph: Optional[torch.cuda.CUDAGraph] = None
        self._inputs: List[torch.Tensor] = []
        self.launches_per_replay = 0

    def close(self):
        if getattr(self, "_handle", None) is not None and self._handle.value:
            self._graph = None
            self._lib.pstm_batch_destroy(self._handle)
            self._handle = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, traces: Sequence[torch.Tensor]) -> None:
        for p, t in zip(self.plans, traces):
            p.load_traces(t)

    def migrate(self) -> None:
        _lib.check(self._lib.pstm_batch_migrate(self._handle,
                                                torch.cuda.current_stream().cuda_stream))

    def check(self) -> None:
        for p in self.plans:
            p.check()

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
