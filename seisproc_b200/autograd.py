"""Differentiable PSTM and least-squares migration.

``PSTMMigrate`` is a ``torch.autograd.Function`` for the migration operator
m = L^T(V) d (data -> image, the forward gather kernel):

* d m / d d is the hand-written demigration kernel L (the exact transpose of the
  gather: it scatters w * m into samples i0, i0+1 of each trace);
* d m / d V is the V_rms-gradient kernel, which recomputes traveltimes and
  weights instead of storing them (masks held fixed, zero derivative where the
  sample index is clamped).

``dot_product_test`` checks <L m, d> = <m, L^T d> with float64 inner products.
``cgls`` solves min_m ||L m - d||^2 (+ damp ||m||^2) by conjugate gradients on
the normal equations (CGLS, Hestenes-Stiefel / Paige-Saunders), each iteration
one demigration and one migration; scalars are accumulated in float64.

None of this exists in the reference (it has no adjoint); the operators follow
the forward semantics of migrate_kirchhoff_full (kirchhoff_kernel.py:459-854).
"""
from __future__ import annotations

import time
from typing import Callable, List, Optional, Tuple

import torch

from .kirchhoff import PSTMPlan


class PSTMMigrate(torch.autograd.Function):
    """image = migrate(traces; velocity) with gradients for traces and velocity.

    ``traces`` (n_samples, n_traces) float32 CUDA; ``velocity`` a CUDA float32
    tensor (1,), (n_times,) or (n_times, n_il, n_xl).  The gradient w.r.t.
    velocity is returned with the velocity's shape; for a constant or V(t0)
    velocity the per-sample gradient is summed accordingly.
    """

    @staticmethod
    def forward(ctx, traces: torch.Tensor, velocity: torch.Tensor, plan: PSTMPlan):
        plan.load_traces(traces)
        image, _ = plan.migrate_loaded(velocity, with_fold=False)
        ctx.plan = plan
        ctx.save_for_backward(traces, velocity)
        return image

    @staticmethod
    def backward(ctx, grad_image: torch.Tensor):
        traces, velocity = ctx.saved_tensors
        plan: PSTMPlan = ctx.plan
        g_tr = g_v = None
        if ctx.needs_input_grad[0]:
            g_tr = plan.demigrate(grad_image, velocity)
        if ctx.needs_input_grad[1]:
            plan.load_traces(traces)
            gv = plan.velocity_gradient(grad_image, velocity)
            if velocity.numel() == 1:
                g_v = gv.sum().reshape(velocity.shape)
            elif velocity.dim() == 1:
                g_v = gv.reshape(gv.shape[0], -1).sum(1)
            else:
                g_v = gv.reshape(velocity.shape)
        return g_tr, g_v, None


def migrate(traces: torch.Tensor, velocity: torch.Tensor, plan: PSTMPlan) -> torch.Tensor:
    return PSTMMigrate.apply(traces, velocity, plan)


def dot_product_test(plan: PSTMPlan, velocity: torch.Tensor, seed: int = 7) -> Tuple[float, float, float]:
    """Returns (<L m, d>, <m, L^T d>, relative mismatch) for random m and d."""
    g = torch.Generator(device=plan.device).manual_seed(seed)
    d = torch.randn((plan.n_samples, plan.n_traces), generator=g, device=plan.device)
    m = torch.randn((plan.n_times, plan.n_il, plan.n_xl), generator=g, device=plan.device)
    Lm = plan.demigrate(m, velocity)
    plan.load_traces(d)
    Ltd, _ = plan.migrate_loaded(velocity, with_fold=False)
    plan.check()
    a = float((Lm.double() * d.double()).sum())
    b = float((m.double() * Ltd.double()).sum())
    return a, b, abs(a - b) / max(abs(a), abs(b), 1e-300)


def cgls(plan: PSTMPlan, data: torch.Tensor, velocity: torch.Tensor, n_iter: int = 10,
         damp: float = 0.0, callback: Optional[Callable[[int, float, float], None]] = None):
    """Least-squares PSTM: min_m ||L m - d||^2 + damp ||m||^2 by CGLS.

    Returns (m, history) where history holds (iteration, ||r||/||d||, seconds).
    """
    dev = plan.device

    def Lt(r):  # migration
        plan.load_traces(r)
        out, _ = plan.migrate_loaded(velocity, with_fold=False)
        return out

    def L(m):  # demigration
        return plan.demigrate(m, velocity)

    d = data.to(dev, torch.float32)
    m = torch.zeros((plan.n_times, plan.n_il, plan.n_xl), device=dev)
    r = d.clone()
    s = Lt(r) - damp * m
    p = s.clone()
    gamma = float((s.double() ** 2).sum())
    dnorm = float(torch.linalg.vector_norm(d.double()))
    hist: List[Tuple[int, float, float]] = [(0, 1.0, 0.0)]
    for it in range(1, n_iter + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        q = L(p)
        delta = float((q.double() ** 2).sum()) + damp * float((p.double() ** 2).sum())
        if delta <= 0.0:
            break
        alpha = gamma / delta
        m = m + alpha * p
        r = r - alpha * q
        s = Lt(r) - damp * m
        gamma_new = float((s.double() ** 2).sum())
        beta = gamma_new / gamma
        gamma = gamma_new
        p = s + beta * p
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        res = float(torch.linalg.vector_norm(r.double())) / max(dnorm, 1e-300)
        hist.append((it, res, el))
        if callback:
            callback(it, res, el)
        if gamma == 0.0:
            break
    plan.check()
    return m, hist
