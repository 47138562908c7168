"""Generate the offset/azimuth class fixture by running the reference's binning.

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_binning_golden.py /path/to/reference

Seeded float32 geometry (the precision the reference worker passes,
views/migration_monitor_dialog.py:245-249) with extra traces placed exactly on
offset and azimuth edges (axis-aligned offsets that are multiples of the bin
width, zero offset).  For three of the reference's binning tables -- OVT (8
offset ranges x 8 azimuth sectors), narrow azimuth (sectors wrapping through
north) and common offset with a disabled bin -- the fixture stores the
reference's offsets and azimuths (MigrationGeometry.offset / .azimuth,
models/migration_geometry.py:88-116), the trace indices of every enabled bin
from BinningTable.assign_traces_batch (models/binning.py:304-325), and, for
the OVT table, MigrationGeometry.get_indices_for_bin (closed intervals,
models/migration_geometry.py:256-283).  Nothing is written into the reference
tree.
"""
from __future__ import annotations

import importlib
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def import_binning(ref_root: str):
    sys.dont_write_bytecode = True
    m = types.ModuleType("models")
    m.__path__ = [os.path.join(ref_root, "models")]
    sys.modules["models"] = m
    return (importlib.import_module("models.binning"),
            importlib.import_module("models.migration_geometry"))


def geometry(seed: int = 17, n: int = 20000):
    """float32 source/receiver coordinates: random traces plus edge cases."""
    rs = np.random.RandomState(seed)
    mx, my = rs.uniform(0, 5000, n), rs.uniform(0, 5000, n)
    off, az = rs.uniform(0, 3000, n), rs.uniform(0, 2 * np.pi, n)
    hx, hy = 0.5 * off * np.sin(az), 0.5 * off * np.cos(az)
    sx, sy, rx, ry = mx - hx, my - hy, mx + hx, my + hy
    # edge cases: offsets k * 375 m (and 250 m multiples) along +-x and +-y,
    # and zero offset, from integer midpoints so the float32 offset is exact
    ex, ey = [], []
    for k in range(0, 9):
        for d in (375.0 * k, 250.0 * k):
            for vx, vy in ((0.0, 1.0), (1.0, 0.0), (0.0, -1.0), (-1.0, 0.0)):
                ex.append(d * vx)
                ey.append(d * vy)
    ex, ey = np.array(ex), np.array(ey)
    cx = rs.randint(1000, 4000, ex.size).astype(np.float64)
    cy = rs.randint(1000, 4000, ex.size).astype(np.float64)
    sx = np.concatenate([sx, cx])
    sy = np.concatenate([sy, cy])
    rx = np.concatenate([rx, cx + ex])
    ry = np.concatenate([ry, cy + ey])
    return [a.astype(np.float32) for a in (sx, sy, rx, ry)]


def tables(B):
    ovt = B.create_ovt_binning([(375.0 * i, 375.0 * (i + 1)) for i in range(8)],
                               n_azimuth_sectors=8)
    narrow = B.create_narrow_azimuth_binning(0.0, 3000.0, inline_azimuth=0.0,
                                             azimuth_width=30.0)
    co = B.create_uniform_offset_binning(0.0, 3000.0, 6)
    co.bins[2].enabled = False
    return {"ovt": ovt, "narrow": narrow, "common_offset": co}


def main(ref_root: str):
    B, G = import_binning(ref_root)
    sx, sy, rx, ry = geometry()
    geom = G.MigrationGeometry(source_x=sx, source_y=sy, receiver_x=rx, receiver_y=ry)
    off, az = geom.offset, geom.azimuth
    out = dict(source_x=sx, source_y=sy, receiver_x=rx, receiver_y=ry, offset=off, azimuth=az)
    for tname, t in tables(B).items():
        masks = t.assign_traces_batch(off, az)
        rows = np.array([[b.offset_min, b.offset_max, b.azimuth_min, b.azimuth_max,
                          float(b.enabled)] for b in t.bins], dtype=np.float64)
        idx = [np.nonzero(masks[b.name])[0].astype(np.int64) for b in t.bins if b.enabled]
        out[f"{tname}_bins"] = rows
        out[f"{tname}_counts"] = np.array([i.size for i in idx], np.int64)
        out[f"{tname}_indices"] = np.concatenate(idx) if idx else np.zeros(0, np.int64)
    ovt = tables(B)["ovt"]
    closed = [geom.get_indices_for_bin(b.offset_min, b.offset_max, b.azimuth_min, b.azimuth_max)
              for b in ovt.bins]
    out["ovt_closed_counts"] = np.array([c.size for c in closed], np.int64)
    out["ovt_closed_indices"] = np.concatenate(closed).astype(np.int64)
    np.savez_compressed(os.path.join(HERE, "binning.npz"), **out)
    print({k: int(v.sum()) for k, v in out.items() if k.endswith("_counts")})


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SEISPROC_REFERENCE")
    if not ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path to the SeisProc checkout> "
                 "(or set SEISPROC_REFERENCE)")
    main(ref)
