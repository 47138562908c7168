"""Multi-GPU PSTM: one process per GPU, output inline slabs per rank.

Every output column is independent, so the forward migration shards without a
collective: rank r migrates inlines [il0, il1) of the output grid from the
traces whose two legs reach that slab (its aperture halo), and the slabs are
gathered only when the caller wants the whole image on one rank.

The adjoint (demigration) is where the ranks exchange data: every rank scatters
its slab of the image into the traces of its halo, and the partial traces are
summed over the ranks (an all-reduce over NVLink for NCCL groups).  Least-squares
migration by CGLS then needs one such sum per iteration plus FP64 all-reduces of
the image-space inner products; data-space inner products are local because the
data are replicated after the sum.

The partition and the communication here are operator-agnostic (callables), so
the same code drives the CUDA operators of ``ShardedPSTM`` and any other
implementation of the pair (L, L^T).

The reference has no multi-device path: its worker migrates bin after bin on
one device (views/migration_monitor_dialog.py:201-430); the per-bin operator is
migrate_bin_full (processors/migration/migration_engine.py:225-360).
"""
from __future__ import annotations

import time
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np
import torch
import torch.distributed as dist


# --------------------------------------------------------------- partition ---
def inline_slabs(n_il: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous inline ranges [il0, il1), one per rank, sizes differing by <= 1."""
    if n_il < 1 or world < 1:
        raise ValueError("n_il and world must be positive")
    base, extra = divmod(n_il, world)
    out, il0 = [], 0
    for r in range(world):
        il1 = il0 + base + (1 if r < extra else 0)
        out.append((il0, il1))
        il0 = il1
    return out


def slab_bbox(origin_x: float, origin_y: float, il_dx: float, il_dy: float, xl_dx: float,
              xl_dy: float, n_xl: int, il0: int, il1: int) -> Tuple[float, float, float, float]:
    """Axis-aligned box (xmin, xmax, ymin, ymax) of the slab's output columns.

    Column (il, xl) sits at origin + il * (il_dx, il_dy) + xl * (xl_dx, xl_dy);
    the box of the slab's four corner columns contains all of them (also for a
    rotated grid)."""
    if il1 <= il0:
        return (np.inf, -np.inf, np.inf, -np.inf)
    ils = np.array([il0, il0, il1 - 1, il1 - 1], np.float64)
    xls = np.array([0, n_xl - 1, 0, n_xl - 1], np.float64)
    x = origin_x + ils * il_dx + xls * xl_dx
    y = origin_y + ils * il_dy + xls * xl_dy
    return float(x.min()), float(x.max()), float(y.min()), float(y.max())


def _dist_to_box(x: np.ndarray, y: np.ndarray, box) -> np.ndarray:
    xmin, xmax, ymin, ymax = box
    dx = np.maximum(np.maximum(xmin - x, 0.0), x - xmax)
    dy = np.maximum(np.maximum(ymin - y, 0.0), y - ymax)
    return np.hypot(dx, dy)


def halo_traces(source_x, source_y, receiver_x, receiver_y, box, aperture_m: float) -> np.ndarray:
    """Indices of the traces whose source and receiver both lie within
    ``aperture_m`` of the box: every trace that can pass the per-leg aperture
    test (h_s < A and h_r < A) at some column of the slab (a superset)."""
    sx, sy, rx, ry = (np.asarray(a, np.float64) for a in (source_x, source_y, receiver_x,
                                                           receiver_y))
    reach = aperture_m * (1.0 + 1e-9) + 1e-6
    keep = (_dist_to_box(sx, sy, box) <= reach) & (_dist_to_box(rx, ry, box) <= reach)
    return np.nonzero(keep)[0]


# ----------------------------------------------------------- communication ---
def _world(group) -> Tuple[int, int]:
    if group is None and not (dist.is_available() and dist.is_initialized()):
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def allreduce_sum_(t: torch.Tensor, group=None) -> torch.Tensor:
    """In-place sum over the ranks (no-op on one rank)."""
    if _world(group)[1] > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def allreduce_scalar(v: float, device, group=None) -> float:
    """Sum of a float64 scalar over the ranks."""
    if _world(group)[1] == 1:
        return float(v)
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())


def gather_slabs(local: torch.Tensor, slabs: Sequence[Tuple[int, int]], group=None) -> torch.Tensor:
    """Whole image (n_t, n_il, n_xl) on every rank from the local slabs
    (n_t, il1 - il0, n_xl).  Slabs are padded to the largest one for the
    all-gather and trimmed afterwards."""
    rank, world = _world(group)
    if world == 1:
        return local
    n_t, _, n_xl = local.shape
    width = max(b - a for a, b in slabs)
    pad = torch.zeros((n_t, width, n_xl), dtype=local.dtype, device=local.device)
    pad[:, :local.shape[1]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad.contiguous(), group=group)
    return torch.cat([p[:, :b - a] for p, (a, b) in zip(parts, slabs)], dim=1)


# ------------------------------------------------------------ distributed CG ---
def distributed_cgls(apply_L: Callable[[torch.Tensor], torch.Tensor],
                     apply_Lt: Callable[[torch.Tensor], torch.Tensor], data: torch.Tensor,
                     m_shape: Sequence[int], n_iter: int = 10, damp: float = 0.0, group=None,
                     callback: Optional[Callable[[int, float, float], None]] = None):
    """CGLS for min_m ||L m - d||^2 + damp ||m||^2 with the image m split over
    the ranks.

    ``apply_L(m_local)`` returns this rank's partial data (full data shape; the
    ranks' partials are summed here); ``apply_Lt(r)`` maps the full residual to
    this rank's image part.  ``data`` is the same on every rank.  Inner products
    are accumulated in float64: image-space ones are all-reduced, data-space
    ones are computed locally on the replicated data.  Returns (m_local,
    history) with history entries (iteration, ||r|| / ||d||, seconds).
    """
    dev = data.device

    def sync():
        if dev.type == "cuda":
            torch.cuda.synchronize(dev)

    def img_dot(a, b):
        return allreduce_scalar(float((a.double() * b.double()).sum()), dev, group)

    def L(m):
        return allreduce_sum_(apply_L(m), group)

    d = data
    m = torch.zeros(tuple(m_shape), dtype=d.dtype, device=dev)
    r = d.clone()
    s = apply_Lt(r) - damp * m
    p = s.clone()
    gamma = img_dot(s, s)
    dnorm = float(torch.linalg.vector_norm(d.double()))
    hist: List[Tuple[int, float, float]] = [(0, 1.0, 0.0)]
    for it in range(1, n_iter + 1):
        sync()
        t0 = time.perf_counter()
        q = L(p)
        delta = float((q.double() ** 2).sum()) + (damp * img_dot(p, p) if damp else 0.0)
        if delta <= 0.0:
            break
        alpha = gamma / delta
        m = m + alpha * p
        r = r - alpha * q
        s = apply_Lt(r) - damp * m
        gamma_new = img_dot(s, s)
        beta = gamma_new / gamma
        gamma = gamma_new
        p = s + beta * p
        sync()
        el = time.perf_counter() - t0
        res = float(torch.linalg.vector_norm(r.double())) / max(dnorm, 1e-300)
        hist.append((it, res, el))
        if callback:
            callback(it, res, el)
        if gamma == 0.0:
            break
    return m, hist


# ------------------------------------------------------- CUDA operator pair ---
class ShardedPSTM:
    """This rank's slab of a multi-GPU PSTM on the sm_100a kernels.

    Geometry is given for the whole survey (world coordinates, float64 kept);
    the slab of inlines and its halo traces are selected here and a
    ``PSTMPlan`` is built for them on the current CUDA device.  ``velocity`` is
    a scalar, a (n_times,) V_rms(t0) or the whole (n_times, n_il, n_xl) grid
    (the slab's part is taken).  ``plan_kwargs`` are passed to ``PSTMPlan``
    (max_aperture_m, max_angle_deg, storage, weight, clamp, antialias ...).

    ``rank``/``world`` select the slab explicitly; without a process group this
    runs one slab of a slab-by-slab migration in a single process (the caller
    concatenates the slabs and sums the demigration partials).
    """

    def __init__(self, source_x, source_y, receiver_x, receiver_y, *, n_il: int, n_xl: int,
                 n_times: int, origin_x: float, origin_y: float, il_dx: float, il_dy: float,
                 xl_dx: float, xl_dy: float, t0_ms: float, dt_ms: float, n_samples: int,
                 in_t0_ms: float, in_dt_ms: float, max_aperture_m: float, velocity,
                 group=None, device: Optional[torch.device] = None, rank: Optional[int] = None,
                 world: Optional[int] = None, **plan_kwargs):
        from .kirchhoff import PSTMPlan

        self.group = group
        g_rank, g_world = _world(group)
        self.rank = g_rank if rank is None else int(rank)
        self.world = g_world if world is None else int(world)
        if not 0 <= self.rank < self.world:
            raise ValueError(f"rank {self.rank} outside world {self.world}")
        if n_il < self.world:
            raise ValueError(f"{n_il} inlines cannot be split over {self.world} ranks")
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        self.n_il, self.n_xl, self.n_times, self.n_samples = n_il, n_xl, n_times, n_samples
        self.n_traces = int(np.asarray(source_x).shape[0])
        self.slabs = inline_slabs(n_il, self.world)
        self.il0, self.il1 = self.slabs[self.rank]
        box = slab_bbox(origin_x, origin_y, il_dx, il_dy, xl_dx, xl_dy, n_xl, self.il0, self.il1)
        self.halo = halo_traces(source_x, source_y, receiver_x, receiver_y, box, max_aperture_m)
        self._halo_dev = torch.from_numpy(self.halo).to(self.device)
        coords = [torch.from_numpy(np.ascontiguousarray(np.asarray(a)[self.halo])).to(self.device)
                  for a in (source_x, source_y, receiver_x, receiver_y)]
        self.local_il = self.il1 - self.il0
        v = velocity if torch.is_tensor(velocity) else torch.as_tensor(
            np.asarray(velocity, np.float32))
        v = v.to(self.device, torch.float32)
        if v.dim() == 3:
            v = v[:, self.il0:self.il1, :].contiguous()
        elif v.dim() == 2:
            v = v.reshape(n_times, n_il, n_xl)[:, self.il0:self.il1, :].contiguous()
        self.velocity = v.reshape(-1) if v.dim() == 0 else v
        self.plan = PSTMPlan(*coords, n_il=max(self.local_il, 1), n_xl=n_xl, n_times=n_times,
                             origin_x=origin_x + self.il0 * il_dx,
                             origin_y=origin_y + self.il0 * il_dy, il_dx=il_dx, il_dy=il_dy,
                             xl_dx=xl_dx, xl_dy=xl_dy, t0_ms=t0_ms, dt_ms=dt_ms,
                             n_samples=n_samples, in_t0_ms=in_t0_ms, in_dt_ms=in_dt_ms,
                             max_aperture_m=max_aperture_m, **plan_kwargs)

    def close(self):
        self.plan.close()

    def local_traces(self, traces: torch.Tensor) -> torch.Tensor:
        """The halo traces (n_samples, n_halo) of the whole survey's traces."""
        return traces.to(self.device).index_select(1, self._halo_dev).contiguous()

    def migrate(self, traces: torch.Tensor, with_fold: bool = True):
        """This rank's slab image (and fold) from the survey's traces."""
        self.plan.load_traces(self.local_traces(traces))
        img, fold = self.plan.migrate_loaded(self.velocity, with_fold=with_fold)
        return img[:, :self.local_il], (fold[:, :self.local_il] if fold is not None else None)

    def gather(self, local: torch.Tensor) -> torch.Tensor:
        return gather_slabs(local, self.slabs, self.group)

    def demigrate_partial(self, m_local: torch.Tensor) -> torch.Tensor:
        """This rank's contribution to the survey's traces (zero outside the halo)."""
        part = self.plan.demigrate(m_local.contiguous(), self.velocity)
        out = torch.zeros((self.n_samples, self.n_traces), device=self.device)
        out.index_copy_(1, self._halo_dev, part)
        return out

    def demigrate(self, m_local: torch.Tensor) -> torch.Tensor:
        """Survey traces from the whole image (summed over the ranks)."""
        return allreduce_sum_(self.demigrate_partial(m_local), self.group)

    def cgls(self, data: torch.Tensor, n_iter: int = 10, damp: float = 0.0, callback=None):
        data = data.to(self.device, torch.float32)

        def Lt(r):
            self.plan.load_traces(self.local_traces(r))
            out, _ = self.plan.migrate_loaded(self.velocity, with_fold=False)
            return out

        m, hist = distributed_cgls(self.demigrate_partial, Lt, data,
                                   (self.n_times, self.local_il, self.n_xl), n_iter=n_iter,
                                   damp=damp, group=self.group, callback=callback)
        self.plan.check()
        return m, hist
