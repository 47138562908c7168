"""MigrationEngine: the PSTM entry point called per bin by the batch worker.

``migrate_bin_full`` keeps the signature of the reference
(processors/migration/migration_engine.py:225-360) and adds ``velocity_model``
(V_rms varying with t0, x, y) and ``kernel_backend``.  The work runs on the
sm_100a kernels through libseispstm; numpy arrays go in and come out.

Reference behaviour kept:
* output grid x = origin_x + il * il_spacing, y = origin_y + xl * xl_spacing,
  ``azimuth_deg`` ignored (:295-301);
* output time axis t = t_min_ms + k * dt_ms with ``n_times`` samples (default:
  the input trace length), depth z = V t / 2 (:305-306);
* optional fold normalisation image / fold where fold >= min_fold (:347-348);
* progress reported as (fraction, message) with the 0.0 / 0.1 / 0.9 / 1.0
  milestones of the reference.
Coordinates given as float64 keep their precision: the grid origin is
subtracted in float64 on the device before rounding to float32.

``migrate_bin_time_domain_rms`` (:633-802) is the reference's time-domain RMS
operator, a different operator, on its own kernel (``time_domain``); the other
time-domain and own-midpoint entries raise ``NotImplementedError``.
"""
from __future__ import annotations

import logging
import time
from typing import Callable, Optional, Tuple

import numpy as np
import torch

from . import autotune
from .kernel_backend import require_cuda
from .kirchhoff import PSTMPlan, normalize_by_fold
from . import models as _models
from . import velocity as _velocity
from .velocity_io import velocity_grid

logger = logging.getLogger(__name__)


def velocity_at_outputs(velocity_mps: float, velocity_model, t_ms: np.ndarray,
                        col_x: np.ndarray, col_y: np.ndarray) -> np.ndarray:
    """V_rms at the output samples: shape (1,), (n_t,) or (n_t, n_cols)."""
    if velocity_model is None:
        return np.array([velocity_mps], np.float32)
    if isinstance(velocity_model, _velocity.VelocityModel):
        return np.asarray(velocity_model.rms_velocity_at_time(t_ms), np.float32).reshape(-1)
    if isinstance(velocity_model, _models.VelocityModel):
        if not velocity_model.is_time:
            raise ValueError("PSTM needs a time-domain velocity model (is_time=True)")
        return velocity_model.rms_grid(np.asarray(t_ms, np.float64) / 1000.0, col_x, col_y)
    arr = np.asarray(velocity_model, np.float32)
    n_t = t_ms.shape[0]
    if arr.ndim == 0:
        return arr.reshape(1)
    if arr.ndim == 1 and arr.shape[0] == n_t:
        return arr
    return arr.reshape(n_t, -1)


class MigrationEngine:
    """PSTM engine on the CUDA sm_100a kernels (the reference picks MPS > CUDA >
    CPU; this engine only runs on CUDA and raises otherwise)."""

    def __init__(self, device: Optional[torch.device] = None, kernel_backend=None,
                 storage: str = "f32", variant="auto"):
        """``variant``: the kernel shape id, 0 for the library's heuristic, or
        "auto" (default) for the autotuner's choice per problem class (cached;
        a miss costs one timing run on a crop of the grid)."""
        require_cuda(kernel_backend)
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        if torch.device(device).type != "cuda":
            raise ValueError("MigrationEngine runs on a CUDA device only")
        self.device = torch.device(device)
        self.kernel_backend = kernel_backend
        self.storage = storage
        self.variant = variant
        self.last_stats = {}
        self._stage, self._stage_key, self._pool = [], None, None
        self._copy_stream = None
        self._plan_stream = None
        self._result_stream = None
        # bins migrated together run in up to batch_groups batched launches, the
        # results of one downloaded while the next runs
        self.batch_groups = 8
        # bins of at least 2 x block_traces traces are uploaded and migrated in
        # up to max_blocks blocks (one plan each), pipelining the copies
        self.block_traces = 100_000
        self.max_blocks = 4

    def migrate_bin_full(
        self,
        traces: np.ndarray,
        source_x: np.ndarray,
        source_y: np.ndarray,
        receiver_x: np.ndarray,
        receiver_y: np.ndarray,
        origin_x: float,
        origin_y: float,
        il_spacing: float,
        xl_spacing: float,
        azimuth_deg: float,
        n_il: int,
        n_xl: int,
        dt_ms: float,
        t_min_ms: float,
        n_times: int = None,
        velocity_mps: float = 2500.0,
        max_aperture_m: float = 5000.0,
        max_angle_deg: float = 60.0,
        normalize: bool = True,
        min_fold: int = 1,
        progress_callback: Optional[Callable[[float, str], None]] = None,
        enable_profiling: bool = False,
        use_time_dependent_aperture: bool = False,
        velocity_model=None,
        kernel_backend=None,
        antialias: bool = False,
        aa_max_halfwidth: float = 32.0,
    ) -> Tuple[np.ndarray, np.ndarray]:
        """Full Kirchhoff migration of one bin; returns (image, fold) as
        (n_times, n_il, n_xl) float32 numpy arrays.

        ``antialias`` applies the causal-integrated triangle filter whose
        half-width follows the operator dip times the bin spacing (capped at
        ``aa_max_halfwidth`` input samples)."""
        require_cuda(kernel_backend if kernel_backend is not None else self.kernel_backend)
        traces = np.asarray(traces)
        if traces.ndim != 2:
            raise ValueError(f"traces must be (n_samples, n_traces), got {traces.shape}")
        n_s, n_tr = traces.shape

        host_tr = np.ascontiguousarray(traces, dtype=np.float32)

        def upload(stream, blocks):
            # one strided copy per block of traces, each with its own event, so
            # block b can be migrated while the later blocks are in flight; the
            # host array outlives the copies (the call ends synchronised)
            from . import _lib
            L = _lib.lib()
            waits = []
            for first, count in blocks:
                with torch.cuda.stream(stream):
                    dst = torch.empty((n_s, count), dtype=torch.float32, device=self.device)
                    _lib.check(L.pstm_copy_trace_columns(
                        dst.data_ptr(), host_tr.ctypes.data, n_s, n_tr, first, count,
                        stream.cuda_stream))
                    ev = torch.cuda.Event()
                    ev.record(stream)

                def wait(dst=dst, ev=ev):
                    cur = torch.cuda.current_stream(self.device)
                    cur.wait_event(ev)
                    dst.record_stream(cur)
                    return dst, False
                waits.append(wait)
            return waits

        return self._migrate(upload, n_s, n_tr, source_x, source_y, receiver_x, receiver_y,
                             origin_x, origin_y, il_spacing, xl_spacing, n_il, n_xl, dt_ms,
                             t_min_ms, n_times, velocity_mps, max_aperture_m, max_angle_deg,
                             normalize, min_fold, progress_callback, enable_profiling,
                             use_time_dependent_aperture, velocity_model, kernel_backend,
                             antialias, aa_max_halfwidth)

    def migrate_bin_from_reader(
        self,
        reader,
        trace_numbers: np.ndarray,
        source_x: np.ndarray,
        source_y: np.ndarray,
        receiver_x: np.ndarray,
        receiver_y: np.ndarray,
        origin_x: float,
        origin_y: float,
        il_spacing: float,
        xl_spacing: float,
        azimuth_deg: float,
        n_il: int,
        n_xl: int,
        dt_ms: float,
        t_min_ms: float,
        n_times: int = None,
        velocity_mps: float = 2500.0,
        max_aperture_m: float = 5000.0,
        max_angle_deg: float = 60.0,
        normalize: bool = True,
        min_fold: int = 1,
        progress_callback: Optional[Callable[[float, str], None]] = None,
        enable_profiling: bool = False,
        use_time_dependent_aperture: bool = False,
        velocity_model=None,
        kernel_backend=None,
        antialias: bool = False,
        aa_max_halfwidth: float = 32.0,
        chunk_traces: int = 16384,
        reader_threads: int = 8,
    ) -> Tuple[np.ndarray, np.ndarray]:
        """``migrate_bin_full`` with the traces ``trace_numbers`` taken from a
        ``DataReader`` (``read_traces`` -> (n, n_samples); seisio/gather_readers.py:102-142)
        instead of a transposed host array: they stream into device memory
        through page-locked chunks while the plans are built (a large bin in
        blocks, each migrated while the next is read), and are staged from
        their trace-major layout.  Coordinates are those of the selected
        traces, in the same order."""
        from .ingest import TraceUpload
        require_cuda(kernel_backend if kernel_backend is not None else self.kernel_backend)
        idx = np.asarray(trace_numbers, np.int64)
        n_s, n_tr = int(reader.get_n_samples()), int(idx.size)

        def upload(stream, blocks):
            up = TraceUpload(reader, idx, self.device, stream, chunk_traces=chunk_traces,
                             threads=reader_threads, blocks=blocks)
            return [lambda b=b: (up.block(b), True) for b in range(len(blocks))]

        return self._migrate(upload, n_s, n_tr, source_x, source_y, receiver_x, receiver_y,
                             origin_x, origin_y, il_spacing, xl_spacing, n_il, n_xl, dt_ms,
                             t_min_ms, n_times, velocity_mps, max_aperture_m, max_angle_deg,
                             normalize, min_fold, progress_callback, enable_profiling,
                             use_time_dependent_aperture, velocity_model, kernel_backend,
                             antialias, aa_max_halfwidth)

    def migrate_bins_full(
        self,
        bins,
        origin_x: float,
        origin_y: float,
        il_spacing: float,
        xl_spacing: float,
        azimuth_deg: float,
        n_il: int,
        n_xl: int,
        dt_ms: float,
        t_min_ms: float,
        n_times: int = None,
        velocity_mps: float = 2500.0,
        max_aperture_m: float = 5000.0,
        max_angle_deg: float = 60.0,
        normalize: bool = True,
        min_fold: int = 1,
        progress_callback: Optional[Callable[[float, str], None]] = None,
        use_time_dependent_aperture: bool = False,
        velocity_model=None,
        kernel_backend=None,
        out=None,
    ):
        """``migrate_bin_full`` for many bins (offset/azimuth classes) at once.

        The reference's worker migrates the classes of a survey one bin after
        another (views/migration_monitor_dialog.py:201-430); here every bin
        gets its own plan and the bins run in up to ``batch_groups`` persistent
        launches of the batched kernel (``BatchedPSTM``), each into its own image
        (common-image gathers), queued back to back: a group's images are
        normalised and downloaded while the later groups migrate.  ``bins`` is a
        sequence of mappings with ``traces``
        ((n_samples, n_traces) float32), ``source_x``, ``source_y``,
        ``receiver_x`` and ``receiver_y``; the grid, time axis, velocity and
        aperture arguments are shared and mean what they mean for
        ``migrate_bin_full``.  Returns one (image, fold) pair per bin, each
        (n_times, n_il, n_xl) float32: new numpy arrays, or the buffers of
        ``out`` (a sequence of (image, fold) host arrays or CPU tensors; page-
        locked tensors receive the copies at full bus speed)."""
        from . import _lib
        from .batched import BatchedPSTM
        require_cuda(kernel_backend if kernel_backend is not None else self.kernel_backend)
        bins = list(bins)
        if not bins:
            raise ValueError("no bins to migrate")
        if out is not None and len(out) != len(bins):
            raise ValueError("out must hold one (image, fold) pair per bin")
        n_s = int(np.asarray(bins[0]["traces"]).shape[0])
        n_t = int(n_times) if n_times is not None else n_s
        if progress_callback:
            progress_callback(0.0, "Preparing data...")
        L = _lib.lib()
        with torch.cuda.device(self.device):
            cur = torch.cuda.current_stream(self.device)
            t_ms = np.arange(n_t, dtype=np.float32) * np.float32(dt_ms) + np.float32(t_min_ms)
            il = np.arange(n_il)[:, None]
            xl = np.arange(n_xl)[None, :]
            col_x = (origin_x + il * il_spacing + 0 * xl).ravel()
            col_y = (origin_y + 0 * il + xl * xl_spacing).ravel()
            vel_t = self._velocity_grid(velocity_mps, velocity_model, t_ms, col_x, col_y)
            kw = dict(n_il=n_il, n_xl=n_xl, n_times=n_t, origin_x=origin_x, origin_y=origin_y,
                      il_dx=il_spacing, il_dy=0.0, xl_dx=0.0, xl_dy=xl_spacing, t0_ms=t_min_ms,
                      dt_ms=dt_ms, n_samples=n_s, in_t0_ms=t_min_ms, in_dt_ms=dt_ms,
                      max_aperture_m=max_aperture_m, max_angle_deg=max_angle_deg,
                      time_dependent_aperture=use_time_dependent_aperture,
                      storage=self.storage, variant=self.variant,
                      kernel_backend=kernel_backend or self.kernel_backend, forward_only=True)
            # every bin's coordinates and kernel shape first: the tuner times its
            # candidates on an idle device
            coords_all, variants = [], []
            for b in bins:
                tr = np.asarray(b["traces"])
                if tr.ndim != 2 or tr.shape[0] != n_s:
                    raise ValueError("every bin's traces must be (n_samples, n_traces) with "
                                     f"n_samples = {n_s}")
                coords = []
                for key in ("source_x", "source_y", "receiver_x", "receiver_y"):
                    a = np.asarray(b[key])
                    a = a.astype(np.float64 if a.dtype == np.float64 else np.float32)
                    coords.append(torch.from_numpy(np.ascontiguousarray(a)).to(self.device))
                v = kw["variant"]
                if v == "auto":
                    v = autotune.choose_variant(coords, velocity=vel_t,
                                                **{k: x for k, x in kw.items() if k != "variant"})
                coords_all.append(coords)
                variants.append(v)
            out_s = self._out_stream()
            # The bins run in groups, one batched launch each, all queued back to
            # back once every plan is built and every batch created (both
            # synchronise the stream); group g's images are then normalised and
            # downloaded on the output stream while the later groups migrate.
            # (Building a group's plans on a side stream while the previous
            # group ran was slower: 1232 against 981 ms for 64 classes.)
            # Groups hold the bins in ascending order of trace count: the first
            # group's short launch lets the downloads, which take longer than
            # the kernels when every image and fold comes back, start early.
            n_groups = max(1, min(self.batch_groups, len(bins)))
            cuts = np.linspace(0, len(bins), n_groups + 1).astype(np.int64)
            order = np.argsort([np.asarray(b["traces"]).shape[1] for b in bins], kind="stable")
            results = [None] * len(bins)
            plans, batches = [], []
            try:
                for i in order:
                    b = bins[i]
                    plan = PSTMPlan(*coords_all[i], **dict(kw, variant=variants[i]))
                    plans.append(plan)
                    host = np.ascontiguousarray(b["traces"], dtype=np.float32)
                    dev_tr = torch.empty((n_s, host.shape[1]), dtype=torch.float32,
                                         device=self.device)
                    if host.shape[1] > 0:
                        _lib.check(L.pstm_copy_trace_columns(
                            dev_tr.data_ptr(), host.ctypes.data, n_s, host.shape[1], 0,
                            host.shape[1], cur.cuda_stream))
                    plan.load_traces(dev_tr)
                for g in range(n_groups):
                    batches.append(BatchedPSTM(plans[int(cuts[g]):int(cuts[g + 1])], vel_t))
                if progress_callback:
                    progress_callback(0.1, "Running Kirchhoff migration...")
                done = []
                for batch in batches:
                    for t in batch.images + batch.folds:
                        t.record_stream(out_s)
                    batch.migrate()
                    ev = torch.cuda.Event()
                    ev.record(cur)
                    done.append(ev)
                for g, batch in enumerate(batches):
                    out_s.wait_event(done[g])
                    with torch.cuda.stream(out_s):
                        for j, i in enumerate(order[int(cuts[g]):int(cuts[g + 1])]):
                            img, fold = batch.images[j], batch.folds[j]
                            if normalize:
                                img = normalize_by_fold(img, fold, min_fold)
                            if out is not None:
                                for dst, src in zip(out[i], (img, fold)):
                                    if isinstance(dst, torch.Tensor):
                                        dst.copy_(src.reshape(dst.shape),
                                                  non_blocking=dst.is_pinned())
                                    else:
                                        np.copyto(dst, src.reshape(dst.shape).cpu().numpy())
                                results[i] = tuple(out[i])
                            else:
                                results[i] = self._download(img, fold)
                out_s.synchronize()
                cur.synchronize()
                for batch in batches:
                    batch.check()
            finally:
                for batch in batches:
                    batch.close()
                for plan in plans:
                    plan.close()
        if progress_callback:
            progress_callback(1.0, "Complete")
        return results

    def _velocity_grid(self, velocity_mps, velocity_model, t_ms, col_x, col_y) -> torch.Tensor:
        """V_rms at the output samples on the device (constant, V(t0) or V(t0, column))."""
        if isinstance(velocity_model, _models.VelocityModel) and \
                velocity_model.velocity_type in (_models.VelocityType.V_OF_XZ,
                                                 _models.VelocityType.V_OF_XYZ):
            return velocity_grid(velocity_model, np.asarray(t_ms, np.float64) / 1000.0, col_x,
                                 col_y, self.device)
        vel = np.ascontiguousarray(velocity_at_outputs(velocity_mps, velocity_model, t_ms, col_x,
                                                       col_y))
        return torch.from_numpy(vel).to(self.device)

    def _migrate(self, upload, n_s, n_tr, source_x, source_y, receiver_x, receiver_y, origin_x,
                 origin_y, il_spacing, xl_spacing, n_il, n_xl, dt_ms, t_min_ms, n_times,
                 velocity_mps, max_aperture_m, max_angle_deg, normalize, min_fold,
                 progress_callback, enable_profiling, use_time_dependent_aperture,
                 velocity_model, kernel_backend, antialias, aa_max_halfwidth, blocks=None):
        """The body shared by the entry points.  ``upload(stream, blocks)``
        starts the copies of the blocks of traces (first, count) on ``stream``
        and returns one wait() -> (device tensor, trace_major) per block, which
        also orders the current stream after that block's copy.

        A large bin is split into up to four blocks of traces, each with its
        own plan: the plans are built while the first block is in flight, and
        block b is migrated while blocks b + 1 ... are uploaded, hiding most of
        the host-to-device copy behind the kernels.  The partial images and
        folds are summed on the device."""
        if blocks is None:
            blocks = self._trace_blocks(n_tr)
        t_start = time.perf_counter()
        n_t = int(n_times) if n_times is not None else n_s
        # the result arrays are allocated now and their pages faulted in by
        # host threads while the kernels run
        outs, faults = self._output_arrays((n_t, n_il, n_xl))
        if progress_callback:
            progress_callback(0.0, "Preparing data...")
        with torch.cuda.device(self.device):
            cur = torch.cuda.current_stream(self.device)
            # The traces (the bulk of the input) go up on a side stream while the
            # plans, which need only the coordinates, are built on this one.
            if self._copy_stream is None:
                self._copy_stream = torch.cuda.Stream(self.device)
            self._copy_stream.wait_stream(cur)
            coords = []
            for a in (source_x, source_y, receiver_x, receiver_y):
                a = np.asarray(a)
                a = a.astype(np.float64 if a.dtype == np.float64 else np.float32)
                coords.append(torch.from_numpy(np.ascontiguousarray(a)).to(self.device))
            t_ms = np.arange(n_t, dtype=np.float32) * np.float32(dt_ms) + np.float32(t_min_ms)
            il = np.arange(n_il)[:, None]
            xl = np.arange(n_xl)[None, :]
            col_x = (origin_x + il * il_spacing + 0 * xl).ravel()
            col_y = (origin_y + 0 * il + xl * xl_spacing).ravel()
            if isinstance(velocity_model, _models.VelocityModel) and \
                    velocity_model.velocity_type in (_models.VelocityType.V_OF_XZ,
                                                     _models.VelocityType.V_OF_XYZ):
                # laterally varying: resampled onto the output grid on the device
                vel_t = velocity_grid(velocity_model, np.asarray(t_ms, np.float64) / 1000.0,
                                      col_x, col_y, self.device)
            else:
                vel = np.ascontiguousarray(
                    velocity_at_outputs(velocity_mps, velocity_model, t_ms, col_x, col_y))
                # on the copy stream ahead of the traces (asynchronous from
                # page-locked memory; ``vel`` lives until the call returns)
                with torch.cuda.stream(self._copy_stream):
                    vel_t = torch.from_numpy(vel).to(self.device, non_blocking=True)
                vel_t.record_stream(cur)
            # The small uploads (coordinates, velocity) go first: queued behind the
            # traces on the copy engine, a synchronous one would hold the host
            # until the whole bin had crossed the bus, and the plans could not be
            # built meanwhile.  Block 0's event follows the velocity's copy on the
            # copy stream, so the first migration waits for both.
            waits = upload(self._copy_stream, blocks)
            kw = dict(n_il=n_il, n_xl=n_xl, n_times=n_t, origin_x=origin_x, origin_y=origin_y,
                      il_dx=il_spacing, il_dy=0.0, xl_dx=0.0, xl_dy=xl_spacing, t0_ms=t_min_ms,
                      dt_ms=dt_ms, n_samples=n_s, in_t0_ms=t_min_ms, in_dt_ms=dt_ms,
                      max_aperture_m=max_aperture_m, max_angle_deg=max_angle_deg,
                      time_dependent_aperture=use_time_dependent_aperture,
                      storage=self.storage, variant=self.variant,
                      kernel_backend=kernel_backend or self.kernel_backend,
                      antialias=antialias, aa_dx=il_spacing, aa_dy=xl_spacing,
                      aa_max_halfwidth=aa_max_halfwidth, forward_only=True)
            if kw["variant"] == "auto":
                kw["variant"] = autotune.choose_variant(coords, velocity=vel_t,
                                                        **{k: v for k, v in kw.items()
                                                           if k != "variant"})
            plans = []
            try:
                # Block 0's plan is built on this stream before the first launch;
                # the plan of block b + 1 is built on a side stream while block b
                # migrates (a build synchronises the stream it runs on, so on
                # this stream it would wait for the kernels queued before it).
                coords_ready = torch.cuda.Event()
                coords_ready.record(cur)
                self._side_stream()

                def build(b):
                    first, count = blocks[b]
                    part = [c[first:first + count] for c in coords]
                    if b == 0:
                        return PSTMPlan(*part, **kw)
                    self._plan_stream.wait_event(coords_ready)
                    with torch.cuda.stream(self._plan_stream):
                        plan = PSTMPlan(*part, **kw)
                    for c in part:
                        c.record_stream(self._plan_stream)
                    return plan

                plans.append(build(0))
                if progress_callback:
                    progress_callback(0.1, "Running Kirchhoff migration...")
                ev0 = torch.cuda.Event(enable_timing=True)
                ev1 = torch.cuda.Event(enable_timing=True)
                image = fold = None
                for b, wait in enumerate(waits):
                    tr, trace_major = wait()
                    if image is None:
                        ev0.record()
                    img_b, fold_b = plans[b].migrate(tr, vel_t, trace_major=trace_major)
                    if image is None:
                        image, fold = img_b, fold_b
                    else:
                        image.add_(img_b)
                        fold.add_(fold_b)
                    if b + 1 < len(blocks):
                        plans.append(build(b + 1))
                ev1.record()
                for plan in plans:
                    plan.check()
                self.last_stats = {k: sum(p.stats()[k] for p in plans)
                                   for k in ("n_traces", "list_entries", "device_bytes")}
                self.last_stats["blocks"] = len(plans)
                self.last_stats["variant"] = plans[0].stats()["variant"]
                self.last_stats["kernel_ms"] = ev0.elapsed_time(ev1)
                if enable_profiling:
                    pairs = float(fold.double().sum().item())
                    self.last_stats["pairs"] = pairs
                    logger.info("PSTM bin: %d traces, %.3e pairs, %.2f ms, %.2f Gpairs/s",
                                n_tr, pairs, self.last_stats["kernel_ms"],
                                pairs / max(self.last_stats["kernel_ms"], 1e-9) / 1e6)
            finally:
                for plan in plans:
                    plan.close()
            if progress_callback:
                progress_callback(0.9, "Normalizing...")
            if normalize:
                from .kirchhoff import normalize_by_fold
                image = normalize_by_fold(image, fold, min_fold)
            image_np, fold_np = self._download(image, fold, outs, faults)
        logger.info("Full migration complete: %.2fs", time.perf_counter() - t_start)
        if progress_callback:
            progress_callback(1.0, "Complete")
        return image_np, fold_np

    def _side_stream(self) -> torch.cuda.Stream:
        """High-priority stream for plan builds that overlap running kernels
        (their small kernels take SMs as soon as CTAs of the migration retire)."""
        if self._plan_stream is None:
            self._plan_stream = torch.cuda.Stream(self.device, priority=-1)
        return self._plan_stream

    def _out_stream(self) -> torch.cuda.Stream:
        """High-priority stream for normalising and downloading results while
        later kernels run."""
        if self._result_stream is None:
            self._result_stream = torch.cuda.Stream(self.device, priority=-1)
        return self._result_stream

    def _trace_blocks(self, n_tr: int):
        """Blocks of traces (first, count) for a bin: up to ``max_blocks``, the
        first one an eighth of the bin when there are several, so that the
        first launch waits for a small upload; the rest split the remainder."""
        n_blk = min(self.max_blocks, max(1, n_tr // self.block_traces))
        if n_blk == 1:
            return [(0, n_tr)]
        first = n_tr // (2 * n_blk)
        cuts = first + np.linspace(0, n_tr - first, n_blk).astype(np.int64)
        cuts = np.concatenate([[0], cuts])
        return [(int(a), int(b - a)) for a, b in zip(cuts[:-1], cuts[1:])]

    def _workers(self):
        if self._pool is None:
            import concurrent.futures as cf
            self._pool = cf.ThreadPoolExecutor(max_workers=8)
        return self._pool

    def _output_arrays(self, shape):
        """Two new float32 arrays of ``shape`` (image, fold) and the futures of
        the host threads that touch every page of them (a first touch faults
        the page in, which costs more than the bus transfer into it)."""
        outs = [np.empty(shape, np.float32) for _ in range(2)]
        flat = [o.reshape(-1) for o in outs]
        cuts = np.linspace(0, flat[0].shape[0], 5).astype(np.int64)
        pool = self._workers()
        faults = [pool.submit(f[a:b].fill, 0.0) for f in flat for a, b in zip(cuts[:-1], cuts[1:])]
        return outs, faults

    def _download(self, image: torch.Tensor, fold: torch.Tensor, outs=None,
                  faults=()) -> Tuple[np.ndarray, np.ndarray]:
        """Device results to numpy arrays (new ones unless ``outs`` is given,
        whose page faulting ``faults`` are the futures of).

        Both come back through page-locked staging buffers kept by the engine
        (a copy straight into pageable memory runs at a fraction of the bus
        bandwidth), in four slices each: host threads copy a slice out of
        staging as soon as its transfer has landed, while the next ones cross
        the bus."""
        key = tuple(image.shape)
        if self._stage_key != key:
            self._stage = [torch.empty(key, dtype=torch.float32, pin_memory=True) for _ in range(2)]
            self._stage_key = key
        if outs is None:
            outs, faults = self._output_arrays(key)
        n = outs[0].size
        cuts = np.linspace(0, n, 5).astype(np.int64)
        dev = [image.reshape(-1), fold.reshape(-1)]
        stage = [h.reshape(-1) for h in self._stage]
        src = [h.numpy().reshape(-1) for h in self._stage]
        dst = [o.reshape(-1) for o in outs]
        pool = self._workers()
        for f in faults:
            f.result()

        def copy_out(ev, i, a, b):
            while not ev.query():  # polls, so the waiting threads hold no lock
                time.sleep(2e-4)
            np.copyto(dst[i][a:b], src[i][a:b])

        jobs = []
        for a, b in zip(cuts[:-1], cuts[1:]):
            for i in range(2):
                stage[i][a:b].copy_(dev[i][a:b], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record()
                jobs.append(pool.submit(copy_out, ev, i, int(a), int(b)))
        for j in jobs:
            j.result()
        torch.cuda.current_stream().synchronize()
        return outs[0], outs[1]

    def _not_this_operator(self, name: str):
        raise NotImplementedError(
            f"MigrationEngine.{name} is the reference's scatter-to-own-midpoint / time-domain "
            "operator, a different operator from the Kirchhoff summation; use migrate_bin_full")

    def migrate_bin(self, *a, **k):
        self._not_this_operator("migrate_bin")

    def migrate_bin_batched(self, *a, **k):
        self._not_this_operator("migrate_bin_batched")

    def migrate_bin_time_domain(self, *a, **k):
        self._not_this_operator("migrate_bin_time_domain")

    def migrate_bin_time_domain_rms(
        self,
        traces: np.ndarray,
        source_x: np.ndarray,
        source_y: np.ndarray,
        receiver_x: np.ndarray,
        receiver_y: np.ndarray,
        origin_x: float,
        origin_y: float,
        il_spacing: float,
        xl_spacing: float,
        azimuth_deg: float,
        n_il: int,
        n_xl: int,
        dt_ms: float,
        t_min_ms: float,
        n_times: int,
        velocity_model,
        max_aperture_m: float = 5000.0,
        max_angle_deg: float = 60.0,
        tile_size: int = 100,
        sample_batch_size: int = 200,
        max_traces_per_tile: int = 5000,
        normalize: bool = True,
        min_fold: int = 1,
        progress_callback: Optional[Callable[[float, str], None]] = None,
        enable_profiling: bool = False,
        use_time_dependent_aperture: bool = True,
    ) -> Tuple[np.ndarray, np.ndarray]:
        """The reference's time-domain RMS operator (migration_engine.py:633-802):
        each trace's samples moved by t_out = sqrt(t_in^2 + 4 h_eff^2 / V_rms^2)
        into its own midpoint column, on the ``pstm_time_rms_migrate`` kernel.
        A different operator from ``migrate_bin_full``; same arguments and
        results as the reference, (image, fold) (n_times, n_il, n_xl) float32."""
        from .time_domain import migrate_kirchhoff_time_domain_rms
        dev = self.device
        f32 = torch.float32
        if progress_callback:
            progress_callback(0.0, "Preparing data...")
        with torch.cuda.device(dev):
            tr = torch.from_numpy(np.ascontiguousarray(traces, np.float32)).to(dev)
            sx, sy, rx, ry = (torch.from_numpy(np.asarray(a, np.float32)).to(dev)
                              for a in (source_x, source_y, receiver_x, receiver_y))
            # output grid as migration_engine.py:727-737 builds it
            cos_az = np.cos(np.radians(azimuth_deg))
            sin_az = np.sin(np.radians(azimuth_deg))
            il = torch.arange(n_il, device=dev, dtype=f32) * il_spacing
            xl = torch.arange(n_xl, device=dev, dtype=f32) * xl_spacing
            xl_g, il_g = torch.meshgrid(xl, il, indexing="xy")
            out_x = origin_x + il_g.flatten() * cos_az - xl_g.flatten() * sin_az
            out_y = origin_y + il_g.flatten() * sin_az + xl_g.flatten() * cos_az
            t_axis = torch.arange(n_times, device=dev, dtype=f32) * dt_ms + t_min_ms

            def kernel_progress(pct: float, msg: str):
                if progress_callback:
                    progress_callback(0.1 + pct * 0.8, msg)

            image, fold = migrate_kirchhoff_time_domain_rms(
                tr, sx, sy, rx, ry, out_x, out_y, t_axis, velocity_model, dt_ms, t_min_ms,
                max_aperture_m, max_angle_deg, n_il, n_xl, origin_x, origin_y, il_spacing,
                xl_spacing, azimuth_deg, tile_size=tile_size,
                sample_batch_size=sample_batch_size, max_traces_per_tile=max_traces_per_tile,
                progress_callback=kernel_progress, enable_profiling=enable_profiling,
                use_time_dependent_aperture=use_time_dependent_aperture)
            if normalize:
                image = normalize_by_fold(image, fold, min_fold)
            out = image.cpu().numpy(), fold.cpu().numpy()
        if progress_callback:
            progress_callback(1.0, "Complete")
        return out
