"""Batched H|psi> over many independent systems, CUDA-graph replay and option autotuning.

The reference applies one ks_hamiltonian per call (ks_hamiltonian.hpp:137-156) and
syncs after every kernel; serving many small systems that way is launch-bound.  Here
a :class:`Batch` holds the resident (Hamiltonian, input, output) triples of many
systems on one context:

* :meth:`Batch.apply` forks the systems' operator chains over auxiliary streams and
  joins them (``inqb_batch_apply``), so small systems overlap on the device;
* :meth:`Batch.capture` records that fork/join into one CUDA graph
  (``inqb_graph_capture_*``) which :meth:`Batch.launch` replays with a single
  launch per batch.

:func:`autotune` picks, per system shape, the kernel options (specialised TMA or generic
FFT kernel, FFT row width and ring depth, nonlocal kernel form and batch sizes) by coordinate
descent over CUDA-event timings on the context's stream, and sets them on each system's
Hamiltonian, so one batched call runs every system with its own options.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

from . import _lib
from .core import Context, KSHamiltonian, OrbitalSet

DEFAULT_OPTIONS = {"fft_impl": 0, "fft_wide": 1, "fft_flat": 1, "fft_stages": 0, "nl_bulk": 0, "nl_apply_points": 0,
                   "nl_project_points": 0, "nl_project_ranges": 0}

# The knobs the autotuner searches, each with its candidate values (the first is the default):
#   fft_impl           specialised persistent TMA kernels (0) or the generic kernel (1)
#   fft_wide           512-byte (64-state) rows in the single-precision streaming passes (1) or 256-byte (0)
#   fft_flat           y and x passes over flattened (point, state) columns (1) or line x state-block tiles (0)
#   fft_stages         ring depth of the TMA passes (0: from their shared-memory budget)
#   nl_bulk            bulk-copy nonlocal kernels by size (0), wherever rows allow (1), never (-1)
#   nl_apply_points    hit points per batch of the bulk-copy nonlocal apply (0: 8)
#   nl_project_points  sphere points per stage of the bulk-copy projection (0: about 16 KB of rows)
#   nl_project_ranges  ranges of each sphere's points, one CTA each, in the projection (0: 16)
SEARCH_SPACE = (("fft_impl", (0, 1)), ("fft_wide", (1, 0)), ("fft_flat", (1, 0)), ("fft_stages", (0, 2, 3, 4)),
                ("nl_bulk", (0, 1, -1)),
                ("nl_apply_points", (0, 4, 16)), ("nl_project_points", (0, 4, 8, 16)),
                ("nl_project_ranges", (0, 8, 24)))


@dataclass
class Tuning:
    """Best kernel options per (grid, states, precision) found by :func:`autotune`."""
    table: dict = field(default_factory=dict)

    def key(self, phi: OrbitalSet):
        return (tuple(phi.basis.sizes), phi.nst, phi.precision)

    def options(self, phi: OrbitalSet) -> dict:
        return self.table.get(self.key(phi), dict(DEFAULT_OPTIONS))


def _time_apply(ctx: Context, ham: KSHamiltonian, phi: OrbitalSet, out: OrbitalSet, reps: int) -> float:
    import torch
    stream = torch.cuda.ExternalStream(ctx.stream())
    for _ in range(2):
        ham.apply(phi, out)
    ctx.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        ham.apply(phi, out)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def _set_all(ham: KSHamiltonian, opts: dict):
    for k, v in opts.items():
        ham.set_option(k, v)


def autotune(systems, tuning: Tuning | None = None, reps: int = 3, search=SEARCH_SPACE,
             min_gain: float = 0.02) -> Tuning:
    """Per system shape, choose the kernel options by coordinate descent: each knob of ``search`` in turn
    takes the candidate value that times fastest with the other knobs at their best so far (a candidate
    must beat the current choice by ``min_gain`` relative).  Times are CUDA-event times of H applications
    on the context's stream.

    ``systems`` is a sequence of (ham, phi) pairs.  The result is stored in ``tuning`` and set on each
    Hamiltonian as its option overrides (inqb_hamiltonian_set_option), so a batch runs every system with
    its own options in one call.  Candidates a shape cannot use (a ring too deep for shared memory, for
    example) are skipped."""
    tuning = tuning or Tuning()
    for ham, phi in systems:
        key = tuning.key(phi)
        if key not in tuning.table:
            ctx = ham.ctx
            out = phi.skeleton()
            best = dict(DEFAULT_OPTIONS)
            _set_all(ham, best)
            best_ms = _time_apply(ctx, ham, phi, out, reps)
            for knob, values in search:
                for v in values:
                    if v == best[knob]:
                        continue
                    cand = dict(best)
                    cand[knob] = v
                    try:
                        _set_all(ham, cand)
                        ms = _time_apply(ctx, ham, phi, out, reps)
                    except _lib.InqbError:
                        continue
                    if ms < best_ms * (1.0 - min_gain):
                        best, best_ms = cand, ms
            tuning.table[key] = best
        _set_all(ham, tuning.table[key])
    return tuning


class Batch:
    """Resident systems applied together; see the module docstring."""

    def __init__(self, ctx: Context, hams, ins, outs, nstreams: int = 8, tuning: Tuning | None = None):
        assert len(hams) == len(ins) == len(outs)
        self.ctx = ctx
        self.nstreams = nstreams
        self.tuning = tuning
        # every system runs with its own Hamiltonian's option overrides (set by autotune), so the whole
        # batch is one fork/join call
        if tuning is not None:
            for h, i in zip(hams, ins):
                _set_all(h, tuning.options(i))
        self.members = list(zip(hams, ins, outs))
        self.graph = None

    def _call(self):
        lib = self.ctx.lib
        n = len(self.members)
        hs = (C.c_void_p * n)(*[m[0].handle.value for m in self.members])
        ins = (C.c_void_p * n)(*[m[1].handle.value for m in self.members])
        outs = (C.c_void_p * n)(*[m[2].handle.value for m in self.members])
        self.ctx.check(lib.inqb_batch_apply(self.ctx.handle, n, hs, ins, outs, self.nstreams))

    def apply(self):
        """Eager batched application (asynchronous on the context's stream)."""
        self._call()

    def capture(self):
        """Record the batched application into a CUDA graph (after one eager warm-up)."""
        self._call()
        self.ctx.synchronize()
        self.ctx.check(self.ctx.lib.inqb_graph_capture_begin(self.ctx.handle))
        try:
            self._call()
        finally:
            g = C.c_void_p()
            code = self.ctx.lib.inqb_graph_capture_end(self.ctx.handle, C.byref(g))
        self.ctx.check(code)
        self.graph = g
        return self

    def launch(self):
        """Replay the captured graph."""
        assert self.graph is not None, "capture() first"
        self.ctx.check(self.ctx.lib.inqb_graph_launch(self.ctx.handle, self.graph))

    def close(self):
        if self.graph is not None:
            self.ctx.lib.inqb_graph_destroy(self.graph)
            self.graph = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
