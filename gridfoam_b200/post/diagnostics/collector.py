"""Streaming CSV diagnostics (gridfoam ``post/diagnostics/collector.py``).

``DiagnosticsCollector`` keeps the reference's constructor, ``from_config``,
``record_step``, ``get_phi_field``, ``close`` and context-manager API, the
two files (``continuity_error.csv``: time, local, global, cumulative;
``solver_info.csv``: time and per field component solver, initial, final,
iters, converged), the record rule (every ``writeInterval`` steps and the
last step) and the values.

What differs is where the host waits.  The reference calls ``.item()`` on
every recorded step.  Here ``record_step`` only enqueues: the continuity
sums are reduced on the device into a ring slot and copied to pinned host
memory on a side stream, the solver statistics already travel the same way
(``SolveStats``), and rows are written, in step order, once their copies
have landed.  ``close`` (or a full ring) waits for the rest.  The step loop
never blocks on the diagnostics.
"""

from __future__ import annotations

import csv
from collections import deque
from dataclasses import dataclass
from pathlib import Path
from typing import Any

import torch

from gridfoam_b200.core.field import get_or_create_facefield
from gridfoam_b200.meta.config import PostProcessingConfig
from gridfoam_b200.post.diagnostics.continuity import continuity_sums_async, scratch_doubles

RING = 64


@dataclass(frozen=True)
class SolverInfoColumn:
    """One solverInfo CSV column group for a field component."""

    csv_key: str
    field_name: str
    component_index: int


@dataclass
class _Pending:
    step: int
    time: float
    slot: int | None  # continuity ring slot (None: no continuity row)
    done: Any  # CUDA event of the slot's host copy
    stats: dict | None  # solverInfo stats (None: no solverInfo row)


def _stats_ready(stats_tuple) -> bool:
    return all(s.ready() for s in stats_tuple)


class DiagnosticsCollector:
    """Stream post-processing diagnostics to CSV files during a simulation."""

    def __init__(self, *, grid, config: PostProcessingConfig | dict, output_dir: Path, n_steps: int,
                 delta_t: float, phase: str | None = None) -> None:
        if isinstance(config, dict):
            config = PostProcessingConfig.model_validate(config)
        self._grid = grid
        self._config = config
        self._output_dir = Path(output_dir)
        self._n_steps = n_steps
        self._delta_t = delta_t
        self._phase = phase
        self._cumulative_continuity = 0.0
        self._closed = False
        self._pending: deque[_Pending] = deque()
        self._continuity_file = self._continuity_writer = None
        self._solver_info_file = self._solver_info_writer = None
        self._solver_info_columns: list[SolverInfoColumn] = []
        self._output_dir.mkdir(parents=True, exist_ok=True)

        if config.continuityError is not None:
            dev = grid.device
            self._sums = torch.zeros((RING, 3), dtype=torch.float64, device=dev)
            self._scratch = torch.empty(scratch_doubles(), dtype=torch.float64, device=dev)
            self._host = torch.empty((RING, 3), dtype=torch.float64, pin_memory=True)
            self._copied: list[Any] = [None] * RING
            self._copy_stream = torch.cuda.Stream(device=dev)
            self._next_slot = 0
            self._continuity_file = (self._output_dir / "continuity_error.csv").open("w", newline="")
            self._continuity_writer = csv.writer(self._continuity_file)
            self._continuity_writer.writerow(["time", "local", "global", "cumulative"])
            self._continuity_file.flush()

        if config.solverInfo is not None:
            self._solver_info_columns = self._build_solver_info_columns(config)
            self._solver_info_file = (self._output_dir / "solver_info.csv").open("w", newline="")
            self._solver_info_writer = csv.writer(self._solver_info_file)
            header = ["time"]
            for column in self._solver_info_columns:
                k = column.csv_key
                header.extend([f"{k}_solver", f"{k}_initial", f"{k}_final", f"{k}_iters", f"{k}_converged"])
            self._solver_info_writer.writerow(header)
            self._solver_info_file.flush()

    @classmethod
    def from_config(cls, grid, post_processing, output_dir: Path, *, n_steps: int, delta_t: float,
                    phase: str | None = None) -> DiagnosticsCollector | None:
        """collector.py:103-142: a collector when any diagnostic is enabled."""
        if post_processing is None:
            return None
        if isinstance(post_processing, dict):
            post_processing = PostProcessingConfig.model_validate(post_processing)
        if post_processing.continuityError is None and post_processing.solverInfo is None:
            return None
        return cls(grid=grid, config=post_processing, output_dir=output_dir, n_steps=n_steps, delta_t=delta_t,
                   phase=phase)

    # -- columns (collector.py:144-188) -----------------------------------
    def _resolve_solver_info_fields(self, config: PostProcessingConfig) -> list[str]:
        if config.solverInfo.fields is not None:
            return list(config.solverInfo.fields)
        return ["U", "p"]

    def _resolve_field_num_components(self, field_name: str) -> int:
        field = self._grid.get_cellfield(field_name)
        if field is not None:
            return field.num_components
        cond = self._grid.sim_config.conditions.get(field_name)
        if cond is not None:
            return torch.as_tensor(cond.internal).numel()
        return 1

    def _build_solver_info_columns(self, config: PostProcessingConfig) -> list[SolverInfoColumn]:
        columns: list[SolverInfoColumn] = []
        for name in self._resolve_solver_info_fields(config):
            nc = self._resolve_field_num_components(name)
            if nc == 1:
                columns.append(SolverInfoColumn(name, name, 0))
                continue
            columns.extend(SolverInfoColumn(f"{name}_{k}", name, k) for k in range(nc))
        return columns

    def _should_record(self, step: int, write_interval: int) -> bool:
        return step % write_interval == 0 or step == self._n_steps

    # -- recording ---------------------------------------------------------
    def record_step(self, step: int, phi, solve_stats: dict) -> None:
        """collector.py:190-256: enqueue the rows of this step (1-based)."""
        if self._closed:
            return
        cont = self._config.continuityError
        info = self._config.solverInfo
        want_cont = cont is not None and self._should_record(step, cont.writeInterval)
        want_info = info is not None and self._should_record(step, info.writeInterval)
        if not (want_cont or want_info):
            return
        if len(self._pending) >= RING:
            self._drain(block_head=True)
        slot = done = None
        if want_cont:
            slot = self._next_slot
            self._next_slot = (slot + 1) % RING
            cur = torch.cuda.current_stream(self._grid.device)
            if self._copied[slot] is not None:
                cur.wait_event(self._copied[slot])  # the slot's last copy has left the device
            continuity_sums_async(phi, self._grid.cell_volumes, self._sums[slot], self._scratch)
            ready = torch.cuda.Event()
            ready.record(cur)
            done = torch.cuda.Event()
            with torch.cuda.stream(self._copy_stream):
                self._copy_stream.wait_event(ready)
                self._host[slot].copy_(self._sums[slot], non_blocking=True)
                done.record(self._copy_stream)
            self._copied[slot] = done
        stats = dict(solve_stats) if want_info else None
        self._pending.append(_Pending(step, step * self._delta_t, slot, done, stats))
        self._drain(block_head=False)

    def _row_ready(self, row: _Pending) -> bool:
        if row.done is not None and not row.done.query():
            return False
        if row.stats is not None:
            return all(_stats_ready(v) for v in row.stats.values() if v)
        return True

    def _drain(self, block_head: bool) -> None:
        """Write every leading pending row whose copies have landed (and the
        head row in any case when ``block_head``)."""
        first = True
        while self._pending:
            row = self._pending[0]
            if not self._row_ready(row):
                if not (block_head and first):
                    return
                if row.done is not None:
                    row.done.synchronize()
            self._pending.popleft()
            self._write(row)
            first = False

    def _write(self, row: _Pending) -> None:
        if row.slot is not None and self._continuity_writer is not None:
            a, g, v = self._host[row.slot].tolist()
            local_error, global_error = self._delta_t * (a / v), self._delta_t * (g / v)
            self._cumulative_continuity += global_error
            self._continuity_writer.writerow([row.time, local_error, global_error, self._cumulative_continuity])
            self._continuity_file.flush()
        if row.stats is not None and self._solver_info_writer is not None:
            out: list = [row.time]
            for column in self._solver_info_columns:
                st = row.stats.get(column.field_name)
                if not st or column.component_index >= len(st):
                    out.extend(["", "", "", "", ""])
                    continue
                s = st[column.component_index]
                out.extend([s.solver, s.initial_residual, s.final_residual, s.iterations, int(s.converged)])
            self._solver_info_writer.writerow(out)
            self._solver_info_file.flush()

    def get_phi_field(self):
        """collector.py:258-277: the flux field named by ``continuityError.phi``."""
        name = self._config.continuityError.phi
        if self._phase is not None:
            name = f"{name}.{self._phase}"
        return get_or_create_facefield(self._grid, name, "local", ())

    def close(self) -> None:
        """Write every pending row, then flush and close the files."""
        if self._closed:
            return
        while self._pending:
            self._drain(block_head=True)
        for attr in ("_continuity_file", "_solver_info_file"):
            fh = getattr(self, attr)
            if fh is not None:
                fh.flush()
                fh.close()
                setattr(self, attr, None)
        self._continuity_writer = self._solver_info_writer = None
        self._closed = True

    def __enter__(self) -> DiagnosticsCollector:
        return self

    def __exit__(self, exc_type, exc, tb) -> None:
        self.close()
