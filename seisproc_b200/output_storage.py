"""Migrated-cube storage in the reference's on-disk layout, without zarr.

The reference writes each migrated bin through ``MigrationOutputStorage``
(utils/migration_output_storage.py:30-485) into the layout of its SEG-Y
import, which its application and ``ZarrDataReader`` (seisio/gather_readers.py:
145-262) read back:

    output_dir/
        traces.zarr/            image, (n_time, n_inline * n_xline) float32,
                                zarr format 2, no compressor, chunks
                                (n_time, chunk_size), inline-major traces
        headers.parquet         trace_index, inline, xline, cdp_x, cdp_y,
                                ensemble_number, trace_in_ensemble
        ensemble_index.parquet  one row per inline
        trace_index.parquet     trace_index, global_trace_id
        fold.npy                fold, (n_time, n_traces) float32
        metadata.json           grid, processing stats, storage info

The zarr package is not installed here, so ``ZarrV2Array`` writes and reads the
uncompressed zarr format-2 array directly from the format's specification: a
``.zarray`` JSON document (shape, chunks, dtype "<f4", compressor null,
fill_value, C order, "." chunk-key separator), an empty ``.zattrs``, and one
file of raw little-endian C-order bytes per chunk named "i.j" (edge chunks are
stored at full chunk size, padded with the fill value).  The parquet tables are
written with pandas/pyarrow, snappy-compressed, as the reference writes them.
"""
from __future__ import annotations

import concurrent.futures as cf
import json
import math
import os
from datetime import datetime
from pathlib import Path
from typing import Dict, Optional, Sequence, Tuple

import numpy as np


class ZarrV2Array:
    """A 2-D uncompressed zarr (format 2) float32 array on disk."""

    def __init__(self, path, shape: Tuple[int, int], chunks: Tuple[int, int],
                 fill_value: float = 0.0):
        self.path = Path(path)
        self.shape = tuple(int(v) for v in shape)
        self.chunks = tuple(int(v) for v in chunks)
        self.fill_value = float(fill_value)
        self.dtype = np.dtype("<f4")

    # ------------------------------------------------------------ creation --
    @classmethod
    def create(cls, path, shape, chunks, fill_value: float = 0.0) -> "ZarrV2Array":
        a = cls(path, shape, chunks, fill_value)
        a.path.mkdir(parents=True, exist_ok=True)
        meta = {"zarr_format": 2, "shape": list(a.shape), "chunks": list(a.chunks),
                "dtype": "<f4", "compressor": None, "fill_value": a.fill_value, "order": "C",
                "filters": None, "dimension_separator": "."}
        (a.path / ".zarray").write_text(json.dumps(meta, indent=4))
        (a.path / ".zattrs").write_text("{}")
        return a

    @classmethod
    def open(cls, path) -> "ZarrV2Array":
        path = Path(path)
        meta = json.loads((path / ".zarray").read_text())
        if meta.get("zarr_format") != 2:
            raise ValueError(f"{path}: not a zarr format-2 array")
        if meta.get("compressor") is not None or meta.get("filters"):
            raise ValueError(f"{path}: compressed or filtered zarr arrays need the zarr "
                             "package; this reader handles uncompressed arrays only")
        if np.dtype(meta["dtype"]) not in (np.dtype("<f4"), np.dtype("float32")) or \
                meta.get("order", "C") != "C" or len(meta["shape"]) != 2:
            raise ValueError(f"{path}: only 2-D little-endian float32 C-order arrays are "
                             "supported")
        fv = meta.get("fill_value")
        a = cls(path, meta["shape"], meta["chunks"], 0.0 if fv is None else float(fv))
        a._sep = meta.get("dimension_separator", ".")
        return a

    # ------------------------------------------------------------- chunks --
    @property
    def n_chunks(self) -> Tuple[int, int]:
        return tuple(max(1, math.ceil(s / c)) for s, c in zip(self.shape, self.chunks))

    def _key(self, i: int, j: int) -> Path:
        return self.path / f"{i}{getattr(self, '_sep', '.')}{j}"

    def _read_chunk(self, i: int, j: int) -> np.ndarray:
        p = self._key(i, j)
        if not p.exists():
            return np.full(self.chunks, self.fill_value, np.float32)
        return np.fromfile(p, dtype=self.dtype).reshape(self.chunks)

    def _write_chunk(self, i: int, j: int, block: np.ndarray) -> None:
        full = np.full(self.chunks, self.fill_value, np.float32)
        full[:block.shape[0], :block.shape[1]] = block
        key = self._key(i, j)
        tmp = key.parent / (key.name + ".tmp")  # one temporary per chunk
        full.astype(self.dtype, copy=False).tofile(tmp)
        os.replace(tmp, key)

    def write(self, data: np.ndarray, col0: int = 0, threads: int = 8) -> None:
        """Writes columns [col0, col0 + data.shape[1]) (all rows): every chunk
        the range touches is rewritten whole (chunks partly outside the range
        keep their other columns)."""
        data = np.asarray(data, np.float32)
        n0, n1 = self.shape
        c0, c1 = self.chunks
        if data.shape[0] != n0 or col0 < 0 or col0 + data.shape[1] > n1:
            raise ValueError("write outside the array")
        j_lo, j_hi = col0 // c1, (col0 + data.shape[1] - 1) // c1

        def one(ij):
            i, j = ij
            r0, r1 = i * c0, min(n0, (i + 1) * c0)
            a0, a1 = j * c1, min(n1, (j + 1) * c1)
            lo, hi = max(a0, col0), min(a1, col0 + data.shape[1])
            block = self._read_chunk(i, j)[:r1 - r0, :a1 - a0].copy() \
                if (lo > a0 or hi < a1) else np.empty((r1 - r0, a1 - a0), np.float32)
            block[:, lo - a0:hi - a0] = data[r0:r1, lo - col0:hi - col0]
            self._write_chunk(i, j, block)

        jobs = [(i, j) for i in range(self.n_chunks[0]) for j in range(j_lo, j_hi + 1)]
        with cf.ThreadPoolExecutor(max_workers=max(1, min(threads, len(jobs)))) as ex:
            list(ex.map(one, jobs))

    def read_rows(self, rows) -> np.ndarray:
        """The rows ``rows`` (an index array), all columns."""
        n0, n1 = self.shape
        c0, c1 = self.chunks
        idx = np.asarray(rows, np.int64)
        out = np.empty((idx.size, n1), np.float32)
        for i in np.unique(idx // c0):
            sel = np.nonzero(idx // c0 == i)[0]
            for j in range(self.n_chunks[1]):
                a0, a1 = j * c1, min(n1, (j + 1) * c1)
                out[sel, a0:a1] = self._read_chunk(int(i), j)[idx[sel] - i * c0, :a1 - a0]
        return out

    def read(self, cols=None) -> np.ndarray:
        """All rows of the columns ``cols`` (a slice, an index array, or all)."""
        n0, n1 = self.shape
        c0, c1 = self.chunks
        if cols is None:
            cols = slice(0, n1)
        if isinstance(cols, slice):
            idx = np.arange(n1)[cols]
        else:
            idx = np.asarray(cols, np.int64)
        out = np.empty((n0, idx.size), np.float32)
        for j in np.unique(idx // c1):
            sel = np.nonzero(idx // c1 == j)[0]
            for i in range(self.n_chunks[0]):
                r0, r1 = i * c0, min(n0, (i + 1) * c0)
                out[r0:r1, sel] = self._read_chunk(i, int(j))[:r1 - r0, idx[sel] - j * c1]
        return out


class MigrationOutputStorage:
    """Writes a migrated cube in the reference's layout (module docstring).

    Same interface as the reference's class: ``initialize_output`` (creates
    the zero-filled ``traces.zarr``), ``write_inline`` / ``write_full_cube``
    (image into the zarr array, fold kept in memory), ``finalize`` (optional
    fold normalisation where fold > 0, then ``fold.npy``, the parquet tables
    and ``metadata.json``; returns the metadata) and ``get_output_path``.  The
    3-D cube (time, inline, xline) is stored as (time, traces), inline-major.
    """

    def __init__(self, output_dir):
        self.output_dir = Path(output_dir)
        self.output_dir.mkdir(parents=True, exist_ok=True)
        self.traces_path = self.output_dir / "traces.zarr"
        self.fold_path = self.output_dir / "fold.npy"
        self.headers_path = self.output_dir / "headers.parquet"
        self.ensemble_index_path = self.output_dir / "ensemble_index.parquet"
        self.trace_index_path = self.output_dir / "trace_index.parquet"
        self.metadata_path = self.output_dir / "metadata.json"
        self._source_file = None
        self._traces = None
        self._image = None
        self._fold = None
        self._stats = {"inlines_written": 0, "traces_written": 0, "max_fold": 0,
                       "start_time": None, "end_time": None}

    def initialize_output(self, n_time: int, n_inline: int, n_xline: int, dt_ms: float = 4.0,
                          t0_ms: float = 0.0, d_inline: float = 25.0, d_xline: float = 25.0,
                          inline_start: int = 1, xline_start: int = 1, x_origin: float = 0.0,
                          y_origin: float = 0.0, grid_azimuth_deg: float = 0.0,
                          chunk_size: int = 1000, source_file: Optional[str] = None):
        self._n_time, self._n_inline, self._n_xline = int(n_time), int(n_inline), int(n_xline)
        self._n_traces = self._n_inline * self._n_xline
        self._dt_ms, self._t0_ms = float(dt_ms), float(t0_ms)
        self._d_inline, self._d_xline = float(d_inline), float(d_xline)
        self._inline_start, self._xline_start = int(inline_start), int(xline_start)
        self._x_origin, self._y_origin = float(x_origin), float(y_origin)
        self._grid_azimuth_deg = float(grid_azimuth_deg)
        self._source_file = source_file
        self._stats["start_time"] = datetime.now().isoformat()
        self._traces = ZarrV2Array.create(self.traces_path, (self._n_time, self._n_traces),
                                          (self._n_time, min(int(chunk_size), self._n_traces)))
        self._image = np.zeros((self._n_time, self._n_traces), np.float32)
        self._fold = np.zeros((self._n_time, self._n_traces), np.float32)
        self._traces.write(self._image)  # the array starts as zeros on disk

    def _require(self):
        if self._traces is None:
            raise RuntimeError("Output not initialized. Call initialize_output first.")

    def write_inline(self, inline_idx: int, image_data: np.ndarray, fold_data: np.ndarray):
        """One inline (0-based index): image and fold (n_time, n_xline)."""
        self._require()
        a = int(inline_idx) * self._n_xline
        img = np.asarray(image_data, np.float32).reshape(self._n_time, self._n_xline)
        self._image[:, a:a + self._n_xline] = img
        self._fold[:, a:a + self._n_xline] = np.asarray(fold_data, np.float32).reshape(
            self._n_time, self._n_xline)
        self._traces.write(img, col0=a)
        self._stats["inlines_written"] += 1
        self._stats["traces_written"] += self._n_xline
        self._stats["max_fold"] = max(self._stats["max_fold"], float(np.max(fold_data)))

    def write_full_cube(self, image_cube: np.ndarray, fold_cube: np.ndarray):
        """The whole cube, (n_time, n_inline, n_xline)."""
        self._require()
        shape = (self._n_time, self._n_inline, self._n_xline)
        if tuple(image_cube.shape) != shape:
            raise ValueError(f"Shape mismatch: expected {shape}, got {tuple(image_cube.shape)}")
        self._image[:] = np.asarray(image_cube, np.float32).reshape(self._n_time, -1)
        self._fold[:] = np.asarray(fold_cube, np.float32).reshape(self._n_time, -1)
        self._traces.write(self._image)
        self._stats["inlines_written"] = self._n_inline
        self._stats["traces_written"] = self._n_traces
        self._stats["max_fold"] = float(self._fold.max()) if self._fold.size else 0.0

    def headers(self):
        """Trace headers: inline-major traces, coordinates rotated by the grid
        azimuth (inline direction from north), as the reference builds them."""
        import pandas as pd
        az = math.radians(self._grid_azimuth_deg)
        il = np.repeat(np.arange(self._n_inline), self._n_xline)
        xl = np.tile(np.arange(self._n_xline), self._n_inline)
        di, dx = il * self._d_inline, xl * self._d_xline
        return pd.DataFrame({
            "trace_index": np.arange(self._n_traces, dtype=np.int64),
            "inline": (self._inline_start + il).astype(np.int64),
            "xline": (self._xline_start + xl).astype(np.int64),
            "cdp_x": self._x_origin + di * math.sin(az) + dx * math.cos(az),
            "cdp_y": self._y_origin + di * math.cos(az) - dx * math.sin(az),
            "ensemble_number": (self._inline_start + il).astype(np.int64),
            "trace_in_ensemble": xl.astype(np.int64)})

    def ensemble_index(self):
        import pandas as pd
        il = np.arange(self._n_inline, dtype=np.int64)
        start = il * self._n_xline
        return pd.DataFrame({"ensemble_id": il, "ensemble_value": self._inline_start + il,
                             "inline": self._inline_start + il, "start_trace": start,
                             "end_trace": start + self._n_xline - 1,
                             "n_traces": np.full(self._n_inline, self._n_xline, np.int64)})

    def metadata(self, extra_metadata: Optional[Dict] = None) -> Dict:
        self._stats["end_time"] = datetime.now().isoformat()
        n, dt = self._n_time, self._dt_ms
        meta = {
            "shape": [n, self._n_traces], "sample_rate": dt, "n_samples": n,
            "n_traces": self._n_traces, "duration_ms": (n - 1) * dt,
            "nyquist_freq": 1000.0 / (2 * dt), "data_type": "migration",
            "migration_info": {
                "n_inline": self._n_inline, "n_xline": self._n_xline, "n_time": n, "dt_ms": dt,
                "t0_ms": self._t0_ms, "d_inline": self._d_inline, "d_xline": self._d_xline,
                "inline_start": self._inline_start, "xline_start": self._xline_start,
                "inline_end": self._inline_start + self._n_inline - 1,
                "xline_end": self._xline_start + self._n_xline - 1,
                "x_origin": self._x_origin, "y_origin": self._y_origin,
                "grid_azimuth_deg": self._grid_azimuth_deg},
            "processing_stats": dict(self._stats),
            "storage_info": {"zarr_chunks": f"({n}, chunk_size)",
                             "parquet_compression": "snappy", "zarr_compression": "none",
                             "fold_available": True},
            "seismic_metadata": {
                "source_file": self._source_file or str(self.output_dir),
                "source_type": "migration",
                "processing_history": ["PSTM Kirchhoff Migration"],
                "file_info": {"filename": self._source_file or "PSTM Migration Output",
                              "n_traces": self._n_traces, "n_samples": n,
                              "sample_interval": dt, "trace_length_ms": (n - 1) * dt}}}
        if extra_metadata:
            meta["migration_params"] = extra_metadata
        return meta

    def finalize(self, normalize: bool = True, extra_metadata: Optional[Dict] = None) -> Dict:
        """Normalises by fold (where fold > 0, else 0) if asked, then writes
        fold.npy, the parquet tables and metadata.json; returns the metadata."""
        import pandas as pd
        self._require()
        if normalize:
            with np.errstate(divide="ignore", invalid="ignore"):
                self._image = np.where(self._fold > 0, self._image / self._fold,
                                       0.0).astype(np.float32)
            self._traces.write(self._image)
        np.save(self.fold_path, self._fold)
        self.headers().to_parquet(self.headers_path, engine="pyarrow", compression="snappy",
                                  index=False)
        self.ensemble_index().to_parquet(self.ensemble_index_path, engine="pyarrow",
                                         compression="snappy", index=False)
        pd.DataFrame({"trace_index": np.arange(self._n_traces, dtype=np.int64),
                      "global_trace_id": np.arange(self._n_traces, dtype=np.int64)}).to_parquet(
            self.trace_index_path, engine="pyarrow", compression="snappy", index=False)
        meta = self.metadata(extra_metadata)
        with open(self.metadata_path, "w") as f:
            json.dump(meta, f, indent=2)
        return meta

    def get_output_path(self) -> Path:
        return self.output_dir


def create_migration_output_storage(output_dir, n_time: int, n_inline: int, n_xline: int,
                                    dt_ms: float = 4.0, **kwargs) -> MigrationOutputStorage:
    """A storage with ``initialize_output`` already called (the reference's factory)."""
    s = MigrationOutputStorage(output_dir)
    s.initialize_output(n_time=n_time, n_inline=n_inline, n_xline=n_xline, dt_ms=dt_ms, **kwargs)
    return s
