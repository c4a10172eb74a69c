"""VTU export of cell fields (gridfoam ``io/vtu.py``).

The reference builds a ``pyvista.UnstructuredGrid`` of one hexahedron per
cell (8 unshared points per cell, io/vtu.py:7-85), fills ``cell_data`` with
every exported cell field (io/vtu.py:88-110) and saves it
(io/vtu.py:113-134).  pyvista is not a dependency here: ``UnstructuredGrid``
is a small container with the same points, connectivity, cell types and
cell data, and ``save`` writes the VTK XML UnstructuredGrid format itself
(raw appended binary, UInt64 block headers), which ParaView and VTK read.

``AsyncVtuExporter`` keeps the export off the step loop: ``snapshot``
copies the exported fields into device staging buffers on the solver's
stream, a side stream copies those into pinned host buffers, and a writer
thread waits for that copy and writes the file while the solver runs on.
"""

from __future__ import annotations

import threading
from collections import deque
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import torch

VTK_HEXAHEDRON = 12

# Hexahedron corner order (io/vtu.py:33-41): sign of (x, y, z) offsets.
_CORNERS = np.array(
    [[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1], [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]],
    dtype=np.float64,
)


@dataclass
class UnstructuredGrid:
    """Points [P, 3], hexahedral connectivity [C, 8], cell types [C] and
    named cell data arrays ([C] or [C, k])."""

    points: np.ndarray
    connectivity: np.ndarray
    cell_types: np.ndarray
    cell_data: dict[str, np.ndarray] = field(default_factory=dict)

    @property
    def n_cells(self) -> int:
        return int(self.connectivity.shape[0])

    @property
    def n_points(self) -> int:
        return int(self.points.shape[0])

    def save(self, path: str | Path) -> None:
        write_vtu(path, self)


def hex_points(centers: np.ndarray, sizes: np.ndarray) -> np.ndarray:
    """Eight corners per cell, ``center + sign * size / 2`` (io/vtu.py:23-78)."""
    half = 0.5 * np.asarray(sizes, dtype=np.float64)
    pts = np.asarray(centers, dtype=np.float64)[:, None, :] + _CORNERS[None, :, :] * half[:, None, :]
    return pts.reshape(-1, 3)


def to_unstructured_grid(grid) -> UnstructuredGrid:
    """io/vtu.py:7-85: one hexahedron per cell, points not shared."""
    n = grid.num_cells
    pts = hex_points(grid.cell_centers.detach().cpu().numpy(), grid.cell_sizes.detach().cpu().numpy())
    conn = np.arange(8 * n, dtype=np.int64).reshape(n, 8)
    types = np.full(n, VTK_HEXAHEDRON, dtype=np.uint8)
    return UnstructuredGrid(pts, conn, types)


def _exported_fields(grid):
    for name in grid.cellfield_names():
        f = grid.get_cellfield(name)
        if f is not None and f.export:
            yield f


def _cell_values(store_host: np.ndarray, ncomp: int, n: int) -> np.ndarray:
    """A field's [ncomp, C] store as the reference's cell data: [C] for a
    scalar, [C, ncomp] otherwise."""
    if ncomp == 1:
        return np.ascontiguousarray(store_host.reshape(n))
    return np.ascontiguousarray(store_host.reshape(ncomp, n).T)


def update_export_cell_data(ugrid: UnstructuredGrid, grid) -> None:
    """io/vtu.py:88-110 (synchronous: copies every exported field now)."""
    n = grid.num_cells
    for f in _exported_fields(grid):
        ugrid.cell_data[f.name] = _cell_values(f.store.detach().cpu().numpy(), f.num_components, n)


def save_export_fields_as_vtu(grid, output_path: str, *, ugrid: UnstructuredGrid | None = None) -> UnstructuredGrid:
    """io/vtu.py:113-134."""
    target = ugrid if ugrid is not None else to_unstructured_grid(grid)
    update_export_cell_data(target, grid)
    target.save(output_path)
    return target


# ---------------------------------------------------------------------------
# VTK XML writer (UnstructuredGrid, raw appended data, UInt64 headers)

_VTK_TYPES = {
    np.dtype(np.float64): "Float64",
    np.dtype(np.float32): "Float32",
    np.dtype(np.int64): "Int64",
    np.dtype(np.int32): "Int32",
    np.dtype(np.uint8): "UInt8",
}


def write_vtu(path: str | Path, ug: UnstructuredGrid) -> None:
    arrays: list[tuple[str, str, np.ndarray, int]] = []  # (section, name, data, ncomp)
    arrays.append(("Points", "Points", np.ascontiguousarray(ug.points, dtype=np.float64), 3))
    arrays.append(("Cells", "connectivity", np.ascontiguousarray(ug.connectivity.reshape(-1), dtype=np.int64), 1))
    offsets = np.arange(1, ug.n_cells + 1, dtype=np.int64) * ug.connectivity.shape[1]
    arrays.append(("Cells", "offsets", offsets, 1))
    arrays.append(("Cells", "types", np.ascontiguousarray(ug.cell_types, dtype=np.uint8), 1))
    for name, values in ug.cell_data.items():
        v = np.ascontiguousarray(values)
        arrays.append(("CellData", name, v, 1 if v.ndim == 1 else int(v.shape[1])))

    offset = 0
    tags: dict[str, list[str]] = {"Points": [], "Cells": [], "CellData": []}
    blobs = []
    for section, name, data, ncomp in arrays:
        vtype = _VTK_TYPES[data.dtype]
        comp = f' NumberOfComponents="{ncomp}"' if section in ("Points", "CellData") else ""
        tags[section].append(f'        <DataArray type="{vtype}" Name="{name}"{comp} format="appended" '
                             f'offset="{offset}"/>')
        raw = data.tobytes(order="C")
        blobs.append(np.uint64(len(raw)).tobytes() + raw)
        offset += 8 + len(raw)

    head = [
        '<?xml version="1.0"?>',
        '<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">',
        "  <UnstructuredGrid>",
        f'    <Piece NumberOfPoints="{ug.n_points}" NumberOfCells="{ug.n_cells}">',
        "      <Points>", *tags["Points"], "      </Points>",
        "      <Cells>", *tags["Cells"], "      </Cells>",
        "      <CellData>", *tags["CellData"], "      </CellData>",
        "    </Piece>",
        "  </UnstructuredGrid>",
        '  <AppendedData encoding="raw">',
    ]
    with open(path, "wb") as fh:
        fh.write(("\n".join(head) + "\n   _").encode())
        for b in blobs:
            fh.write(b)
        fh.write(b"\n  </AppendedData>\n</VTKFile>\n")


def read_vtu(path: str | Path) -> UnstructuredGrid:
    """Read back a file written by ``write_vtu`` (raw appended, UInt64
    headers) -- for tests and tools."""
    import re

    data = Path(path).read_bytes()
    start = data.index(b'<AppendedData encoding="raw">')
    xml = data[:start].decode()
    base = data.index(b"_", start) + 1
    rev = {v: k for k, v in _VTK_TYPES.items()}

    def block(off: int, dtype) -> np.ndarray:
        n = int(np.frombuffer(data, dtype=np.uint64, count=1, offset=base + off)[0])
        return np.frombuffer(data, dtype=dtype, count=n // np.dtype(dtype).itemsize, offset=base + off + 8).copy()

    out: dict[str, tuple[np.ndarray, int]] = {}
    for m in re.finditer(r'<DataArray type="(\w+)" Name="([^"]+)"(?: NumberOfComponents="(\d+)")? '
                         r'format="appended" offset="(\d+)"/>', xml):
        vtype, name, ncomp, off = m.group(1), m.group(2), int(m.group(3) or 1), int(m.group(4))
        out[name] = (block(off, rev[vtype]), ncomp)
    pts = out.pop("Points")[0].reshape(-1, 3)
    conn = out.pop("connectivity")[0]
    offsets = out.pop("offsets")[0]
    types = out.pop("types")[0]
    per = int(offsets[0]) if offsets.size else 8
    cell_data = {name: (v if nc == 1 else v.reshape(-1, nc)) for name, (v, nc) in out.items()}
    return UnstructuredGrid(pts, conn.reshape(-1, per), types, cell_data)


# ---------------------------------------------------------------------------
# Export off the step loop


@dataclass
class _Snapshot:
    path: Path
    fields: list[tuple[str, int, torch.Tensor, torch.Tensor]]  # (name, ncomp, device staging, pinned host)
    event: torch.cuda.Event


class AsyncVtuExporter:
    """Write VTU snapshots of the exported cell fields without stalling the
    solver.  ``snapshot(path)`` copies every exported field into a device
    staging buffer on the current stream (a device-to-device copy, ~10 us
    for a million-cell U and p), then a side stream copies the staging
    buffers into pinned host memory and a writer thread waits for that copy
    and writes the file, while the solver's stream runs on.  At most
    ``depth`` snapshots are in flight (their buffers); a further
    ``snapshot`` waits for the oldest.  ``close`` waits for all."""

    def __init__(self, grid, depth: int = 2):
        self.grid = grid
        self.ugrid = to_unstructured_grid(grid)
        self.depth = max(1, int(depth))
        self._stream = torch.cuda.Stream(device=grid.device)
        self._queue: deque[_Snapshot] = deque()
        self._cv = threading.Condition()
        self._inflight = 0
        self._closed = False
        self._error: BaseException | None = None
        self._free: list[dict[str, tuple[torch.Tensor, torch.Tensor]]] = []
        self._thread = threading.Thread(target=self._run, name="vtu-writer", daemon=True)
        self._thread.start()

    def snapshot(self, path: str | Path) -> None:
        with self._cv:
            if self._error is not None:
                raise RuntimeError("VTU writer failed") from self._error
            while self._inflight >= self.depth:
                self._cv.wait()
            self._inflight += 1
            bufs = self._free.pop() if self._free else {}
        cur = torch.cuda.current_stream(self.grid.device)
        out = []
        for f in _exported_fields(self.grid):
            src = f.store.detach()
            dev, host = bufs.get(f.name, (None, None))
            if dev is None or dev.shape != src.shape:
                dev = torch.empty_like(src)
                host = torch.empty(src.shape, dtype=src.dtype, pin_memory=True)
            dev.copy_(src)
            out.append((f.name, f.num_components, dev, host))
        ready = torch.cuda.Event()
        ready.record(cur)
        with torch.cuda.stream(self._stream):
            self._stream.wait_event(ready)
            for _, _, dev, host in out:
                host.copy_(dev, non_blocking=True)
            done = torch.cuda.Event()
            done.record(self._stream)
        with self._cv:
            self._queue.append(_Snapshot(Path(path), out, done))
            self._cv.notify_all()

    def _run(self) -> None:
        n = self.grid.num_cells
        while True:
            with self._cv:
                while not self._queue and not self._closed:
                    self._cv.wait()
                if not self._queue:
                    return
                snap = self._queue.popleft()
            try:
                snap.event.synchronize()
                ug = UnstructuredGrid(self.ugrid.points, self.ugrid.connectivity, self.ugrid.cell_types)
                for name, ncomp, _, host in snap.fields:
                    ug.cell_data[name] = _cell_values(host.numpy(), ncomp, n)
                write_vtu(snap.path, ug)
            except BaseException as exc:  # reported to the next snapshot/close
                with self._cv:
                    self._error = exc
            with self._cv:
                self._free.append({name: (dev, host) for name, _, dev, host in snap.fields})
                self._inflight -= 1
                self._cv.notify_all()

    def close(self) -> None:
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        self._thread.join()
        if self._error is not None:
            raise RuntimeError("VTU writer failed") from self._error

    def __enter__(self) -> AsyncVtuExporter:
        return self

    def __exit__(self, exc_type, exc, tb) -> None:
        self.close()
