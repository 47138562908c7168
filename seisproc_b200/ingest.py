"""Trace ingest: a reader's traces streamed into device memory.

The reference's batch worker reads each bin's traces with
``DataReader.read_traces(trace_numbers)`` -> (n_traces, n_samples)
(seisio/gather_readers.py:102-142; ``ZarrDataReader`` :145-262), transposes
them on the host to (n_samples, n_traces) (views/migration_monitor_dialog.py:254)
and hands them to the engine, which copies them to the device from pageable
memory.  Here the reader fills page-locked chunks on host threads while the
previous chunk is in flight to the device, and the traces stay trace-major:
the plan stages them from that layout directly, so the host transpose and the
pageable copy disappear and reading overlaps the upload.

``NumpyDataReader`` keeps the reference's interface; ``SegyDataReader`` reads a
SEG-Y file through a memory map (IEEE or IBM float samples); ``ZarrDataReader``
reads an uncompressed zarr format-2 trace array (the layout the reference's
import and ``MigrationOutputStorage`` write) without the zarr package, which is
not installed here.  Any object with ``read_traces`` and ``get_n_samples`` can
be streamed.
"""
from __future__ import annotations

import concurrent.futures as cf
from abc import ABC, abstractmethod
from pathlib import Path
from typing import Optional, Union

import numpy as np
import torch


class DataReader(ABC):
    """Trace source: ``read_traces(trace_numbers)`` -> (n, n_samples) float32."""

    @abstractmethod
    def read_traces(self, trace_numbers: np.ndarray) -> np.ndarray:
        ...

    @abstractmethod
    def get_n_samples(self) -> int:
        ...


class NumpyDataReader(DataReader):
    """Traces held in an (n_traces, n_samples) array."""

    def __init__(self, data: np.ndarray):
        self._data = data

    def read_traces(self, trace_numbers: np.ndarray) -> np.ndarray:
        return self._data[trace_numbers]

    def get_n_samples(self) -> int:
        return self._data.shape[1]

    @property
    def n_traces(self) -> int:
        return self._data.shape[0]


class SegyDataReader(DataReader):
    """SEG-Y traces through a memory map: the 240-byte headers are skipped and
    only the requested traces are decoded (big-endian IEEE or IBM float)."""

    def __init__(self, path: Union[str, Path]):
        from .velocity_io import _be
        head = np.fromfile(str(path), np.uint8, count=3600)
        if head.size < 3600:
            raise ValueError(f"{path}: too short for a SEG-Y file")
        n_s = _be(head, 3220, 2) & 0xFFFF
        fmt = _be(head, 3224, 2)
        n_ext = max(_be(head, 3504, 2), 0)
        if fmt not in (1, 5):
            raise ValueError(f"{path}: SegyDataReader reads IBM (1) or IEEE (5) float samples")
        start = 3600 + 3200 * n_ext
        size = Path(path).stat().st_size
        if n_s == 0 and size >= start + 240:
            th = np.fromfile(str(path), np.uint8, count=240, offset=start)
            n_s = _be(th, 114, 2) & 0xFFFF
        rec = 240 + 4 * n_s
        n_tr = (size - start) // rec
        self._fmt = fmt
        self._n_s = n_s
        self._map = np.memmap(str(path), dtype=np.uint8, mode="r", offset=start,
                              shape=(n_tr, rec))

    def read_traces(self, trace_numbers: np.ndarray) -> np.ndarray:
        from .velocity_io import ibm_to_ieee
        body = np.ascontiguousarray(self._map[np.asarray(trace_numbers, np.int64), 240:])
        if self._fmt == 1:
            return ibm_to_ieee(body.view(">u4"))
        return body.view(">f4").astype(np.float32)

    def get_n_samples(self) -> int:
        return self._n_s

    @property
    def n_traces(self) -> int:
        return self._map.shape[0]


class ZarrDataReader(DataReader):
    """Traces from a zarr format-2 array, as the reference's reader takes them
    (seisio/gather_readers.py:145-262): ``zarr_path`` is the array or a
    directory holding ``traces.zarr``; the array is (n_samples, n_traces)
    ("transposed", the reference's import layout) when ``metadata.json`` beside
    it gives n_samples and n_traces matching its shape, else (n_traces,
    n_samples).  Uncompressed float32 arrays only (no zarr package here):
    compressed arrays raise ``ValueError``."""

    def __init__(self, zarr_path: Union[str, Path]):
        import json
        from .output_storage import ZarrV2Array
        zarr_path = Path(zarr_path)
        if zarr_path.name == "traces.zarr" or (zarr_path / ".zarray").exists():
            array_path, meta_path = zarr_path, zarr_path.parent / "metadata.json"
        elif (zarr_path / "traces.zarr").exists():
            array_path, meta_path = zarr_path / "traces.zarr", zarr_path / "metadata.json"
        else:
            raise ValueError(f"No valid Zarr array found at {zarr_path}")
        self._z = ZarrV2Array.open(array_path)
        self._transposed = False
        self._n_traces, self._n_samples = self._z.shape
        if meta_path.exists():
            meta = json.loads(meta_path.read_text())
            ns, nt = meta.get("n_samples"), meta.get("n_traces")
            if ns and nt and tuple(self._z.shape) == (ns, nt):
                self._transposed = True
                self._n_samples, self._n_traces = ns, nt

    def read_traces(self, trace_numbers: np.ndarray) -> np.ndarray:
        idx = np.asarray(trace_numbers, np.int64)
        return self._z.read(idx).T if self._transposed else self._z.read_rows(idx)

    def get_n_samples(self) -> int:
        return self._n_samples

    @property
    def n_traces(self) -> int:
        return self._n_traces

    @property
    def shape(self):
        return (self._n_traces, self._n_samples)

    @property
    def is_transposed(self) -> bool:
        return self._transposed


class TraceUpload:
    """Streams ``reader``'s traces ``trace_numbers`` into (count, n_samples)
    float32 device tensors on ``stream``, in the background, one per block
    (first, count) of ``trace_numbers`` (default: one block): host threads fill
    one page-locked chunk while the other is being copied.  ``block(b)`` waits
    for block b and orders the caller's current stream after its copies, so
    block b can be used while the later blocks are still being read."""

    def __init__(self, reader: DataReader, trace_numbers: np.ndarray, device: torch.device,
                 stream: torch.cuda.Stream, chunk_traces: int = 16384, threads: int = 8,
                 blocks=None):
        self.reader = reader
        self.idx = np.asarray(trace_numbers, np.int64)
        self.device = torch.device(device)
        self.stream = stream
        self.chunk = max(1, int(chunk_traces))
        self.threads = max(1, int(threads))
        self.blocks = list(blocks) if blocks is not None else [(0, int(self.idx.size))]
        self._done = [cf.Future() for _ in self.blocks]
        self._pool = cf.ThreadPoolExecutor(max_workers=self.threads + 1)
        self._pool.submit(self._run)

    def _fill(self, buf: np.ndarray, sel: np.ndarray) -> None:
        """Read ``sel`` into ``buf`` on the pool's threads, split by traces."""
        def work(a: int, b: int) -> None:
            np.copyto(buf[a:b], self.reader.read_traces(sel[a:b]), casting="unsafe")

        cuts = np.linspace(0, sel.size, min(self.threads, max(1, sel.size // 256)) + 1)
        cuts = np.unique(cuts.astype(np.int64))
        jobs = [self._pool.submit(work, int(a), int(b)) for a, b in zip(cuts[:-1], cuts[1:])]
        for j in jobs:
            j.result()

    def _run(self) -> None:
        try:
            n_s = int(self.reader.get_n_samples())
            with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
                m = max(1, min(self.chunk, max(c for _, c in self.blocks)))
                bufs = [torch.empty((m, n_s), dtype=torch.float32, pin_memory=True)
                        for _ in range(2)]
                used = [None, None]  # the copy that last read each buffer
                k = 0
                for bi, (first, count) in enumerate(self.blocks):
                    out = torch.empty((count, n_s), dtype=torch.float32, device=self.device)
                    for c0 in range(0, count, m):
                        c1 = min(c0 + m, count)
                        b = k % 2
                        k += 1
                        if used[b] is not None:
                            used[b].synchronize()  # its previous copy has finished
                        self._fill(bufs[b].numpy(), self.idx[first + c0:first + c1])
                        out[c0:c1].copy_(bufs[b][:c1 - c0], non_blocking=True)
                        used[b] = torch.cuda.Event()
                        used[b].record(self.stream)
                    ready = torch.cuda.Event()
                    ready.record(self.stream)
                    self._done[bi].set_result((out, ready))
                # the pinned buffers go back to torch's host cache once the copies end
                for e in used:
                    if e is not None:
                        e.synchronize()
        except BaseException as exc:  # reported by block()
            for f in self._done:
                if not f.done():
                    f.set_exception(exc)
        finally:
            self._pool.shutdown(wait=False)

    def block(self, b: int) -> torch.Tensor:
        out, ready = self._done[b].result()
        cur = torch.cuda.current_stream(self.device)
        cur.wait_event(ready)
        out.record_stream(cur)
        return out

    def result(self) -> torch.Tensor:
        """All the traces (a one-block upload)."""
        if len(self.blocks) != 1:
            raise ValueError("result() is for a one-block upload; use block(b)")
        return self.block(0)


def upload_traces(reader: DataReader, trace_numbers: np.ndarray,
                  device: Optional[torch.device] = None,
                  stream: Optional[torch.cuda.Stream] = None, **kw) -> torch.Tensor:
    """The traces as an (n, n_samples) float32 device tensor (blocking form of
    ``TraceUpload``)."""
    dev = torch.device(device) if device is not None else torch.device("cuda")
    s = stream if stream is not None else torch.cuda.Stream(dev)
    return TraceUpload(reader, trace_numbers, dev, s, **kw).result()
