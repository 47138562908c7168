"""Golden vectors for the aperture tapers, made by running the reference's
ApertureController (processors/migration/aperture.py) itself.

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_taper_golden.py /path/to/reference

Writes ``aperture_taper.npz``: a few traces and image points at several depths,
the reference's combined mask from ``compute_aperture_mask`` (offset, distance
and angle cosine tapers, :65-147) and its offset mask alone (:197-226), for two
taper widths.  The reference is imported through the namespace-package shim of
``make_golden.py``; nothing is written into its tree.
"""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import import_reference  # noqa: E402


def main(ref_root: str):
    import_reference(ref_root)
    ap = importlib.import_module("processors.migration.aperture")
    rs = np.random.RandomState(77)
    n_tr = 40
    mx, my = rs.uniform(-600, 600, n_tr), rs.uniform(-600, 600, n_tr)
    off, az = rs.uniform(0, 1500, n_tr), rs.uniform(0, 2 * np.pi, n_tr)
    sx, sy = mx - 0.5 * off * np.cos(az), my - 0.5 * off * np.sin(az)
    rx, ry = mx + 0.5 * off * np.cos(az), my + 0.5 * off * np.sin(az)
    ix = np.array([-150.0, 0.0, 80.0, 400.0])
    iy = np.array([60.0, -20.0, 300.0, -250.0])
    iz = np.array([5.0, 150.0, 400.0, 900.0, 1600.0])
    out = dict(sx=sx, sy=sy, rx=rx, ry=ry, ix=ix, iy=iy, iz=iz)
    f = lambda a: torch.from_numpy(np.asarray(a, np.float32))
    for k, (tw, a, th, omin, omax) in enumerate([(0.1, 1000.0, 60.0, 100.0, 1300.0),
                                                 (0.3, 700.0, 45.0, 0.0, 10000.0)]):
        c = ap.ApertureController(max_aperture_m=a, max_angle_deg=th, min_offset_m=omin,
                                  max_offset_m=omax, taper_width=tw, device=torch.device("cpu"))
        m = c.compute_aperture_mask(f(sx), f(sy), f(rx), f(ry), f(ix), f(iy), f(iz))
        o = c._compute_offset_mask(f(np.hypot(rx - sx, ry - sy)))
        out[f"params{k}"] = np.array([tw, a, th, omin, omax])
        out[f"mask{k}"] = m.numpy()          # (n_z, n_traces, n_xy)
        out[f"offset_mask{k}"] = o.numpy()  # (n_traces,)
    np.savez_compressed(os.path.join(HERE, "aperture_taper.npz"), **out)
    print("wrote", os.path.join(HERE, "aperture_taper.npz"))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SEISPROC_REFERENCE")
    if not ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path to the SeisProc checkout> "
                 "(or set SEISPROC_REFERENCE)")
    main(ref)
