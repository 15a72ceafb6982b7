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

:func:`autotune` picks, per system shape, the FFT kernel options (specialised TMA
kernel or generic kernel, shared-memory ring depth) by timing them with CUDA events
on the context's stream; :class:`Batch` groups systems by their tuned options.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

from . import _lib
from .core import Context, KSHamiltonian, OrbitalSet

DEFAULT_OPTIONS = {"fft_impl": 0, "fft_stages": 0}


def _apply_options(ctx: Context, opts: dict):
    for k, v in opts.items():
        ctx.set_option(k, v)


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


def autotune(systems, tuning: Tuning | None = None, reps: int = 3,
             candidates=({"fft_impl": 0, "fft_stages": 0}, {"fft_impl": 0, "fft_stages": 2},
                         {"fft_impl": 0, "fft_stages": 4}, {"fft_impl": 1, "fft_stages": 0})) -> Tuning:
    """Time every candidate option set on one representative of each system shape.

    ``systems`` is a sequence of (ham, phi) pairs.  Candidates that a shape cannot use
    (for example a ring too deep for shared memory) are skipped."""
    tuning = tuning or Tuning()
    for ham, phi in systems:
        key = tuning.key(phi)
        if key in tuning.table:
            continue
        ctx = ham.ctx
        out = phi.skeleton()
        best, best_ms = None, float("inf")
        for cand in candidates:
            try:
                _apply_options(ctx, cand)
                ms = _time_apply(ctx, ham, phi, out, reps)
            except _lib.InqbError:
                continue
            finally:
                _apply_options(ctx, DEFAULT_OPTIONS)
            if ms < best_ms:
                best, best_ms = dict(cand), ms
        tuning.table[key] = best or dict(DEFAULT_OPTIONS)
    return tuning


class Batch:
    """Resident systems applied together; see the module docstring."""

    def __init__(self, ctx: Context, hams, ins, outs, nstreams: int = 8, tuning: Tuning | None = None):
        assert len(hams) == len(ins) == len(outs)
        self.ctx = ctx
        self.nstreams = nstreams
        self.tuning = tuning
        # group systems by their kernel options (options are per context, so each group is one call)
        groups: dict = {}
        for h, i, o in zip(hams, ins, outs):
            opts = tuning.options(i) if tuning else dict(DEFAULT_OPTIONS)
            groups.setdefault(tuple(sorted(opts.items())), []).append((h, i, o))
        self.groups = [(dict(k), v) for k, v in groups.items()]
        self.graph = None

    def _call(self):
        lib = self.ctx.lib
        for opts, members in self.groups:
            _apply_options(self.ctx, opts)
            n = len(members)
            hs = (C.c_void_p * n)(*[m[0].handle.value for m in members])
            ins = (C.c_void_p * n)(*[m[1].handle.value for m in members])
            outs = (C.c_void_p * n)(*[m[2].handle.value for m in members])
            self.ctx.check(lib.inqb_batch_apply(self.ctx.handle, n, hs, ins, outs, self.nstreams))
        _apply_options(self.ctx, DEFAULT_OPTIONS)

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
