"""Continuous-batching request loop for H|psi> and short ETRS propagations.

A request carries one system (cell, grid, atoms, potential, orbitals) and asks for either
one H application or ``steps`` ETRS steps.  The server:

* admits a request when a slot is free and its device-memory footprint fits in the budget
  (the free device memory at start-up minus a reserve; the sum of the admitted footprints
  never exceeds it), in arrival order -- requests that arrive while others run are admitted
  as soon as a slot and memory free up;
* gives each slot its own library context (one CUDA stream) and host thread, so the work of
  different requests overlaps on the device, and keeps a request's orbitals and potential
  resident on the device across all its steps; a slot keeps the Hamiltonians (potential and
  projector tables) of the systems it served last, so a returning system skips its setup;
* optionally splits the slots into two classes: "bulk" slots for requests whose footprint is at
  least ``bulk_min_bytes`` and "interactive" slots for the rest.  Each class admits its own
  requests in arrival order (a large request waiting for memory does not hold up small ones);
  interactive contexts run at the device's highest stream priority and bulk contexts size their
  persistent kernels for ``bulk_grid_sms`` SMs, so the kernels of small requests find room on the
  device while a large request runs instead of waiting for each of its passes to drain;
* records every request's latency (completion minus arrival) and result, and reports
  p50 / p99 latency beside throughput.

Results do not depend on what else runs: every kernel is deterministic and requests share no
device state, which ``tests/test_serving.py`` checks by comparing results alone and in a mix.
"""

from __future__ import annotations

import threading
import time
from collections import OrderedDict
from dataclasses import dataclass, field

import numpy as np

from . import core, synthetic
from ._lib import F32, F64


@dataclass
class Payload:
    """Host-side inputs of one system: what a client sends."""
    system: synthetic.System
    potential: np.ndarray          # [npoint] float64
    orbitals: np.ndarray           # [npoint][nst] complex (orthonormal), complex64 or complex128

    @property
    def nbytes(self):
        return self.orbitals.nbytes


@dataclass
class Request:
    rid: int
    kind: str                      # "apply" | "etrs"
    payload: Payload
    steps: int = 1
    dt: float | None = None        # None: 0.05 a.u., or less where the grid needs it (synthetic.taylor_stable_dt)
    arrival: float = 0.0           # seconds after the start of the run
    # filled by the server
    admitted: float = -1.0
    finished: float = -1.0
    result: dict = field(default_factory=dict)
    error: str = ""

    @property
    def latency(self):
        return self.finished - self.arrival

    def footprint(self, precision) -> int:
        """Device bytes the request holds while it runs."""
        n = self.payload.system.npoints
        s = self.payload.system.nst
        cb = 16 if precision == F64 else 8
        # in/out; ETRS: phi, saved half step, the four kept Taylor terms H^n phi of the first exponential
        sets = 2 if self.kind == "apply" else 6
        tables = n * 8 * 4 + self.payload.system.natoms * 4000 * 64   # potential, CSR, projector tables
        return sets * n * s * cb + tables + (64 << 20)


def pinned_empty(shape, dtype):
    """Page-locked host array (host<->device copies run at link speed)."""
    import torch
    tdt = {np.dtype(np.complex64): torch.complex64, np.dtype(np.complex128): torch.complex128,
           np.dtype(np.float64): torch.float64}[np.dtype(dtype)]
    return torch.empty(shape, dtype=tdt, pin_memory=True).numpy()


def make_payload(sysm: synthetic.System, precision=F32, ctx: core.Context | None = None) -> Payload:
    """Generate a system's inputs (on the device, then copied to pinned host memory as a client holds them)."""
    basis, ham, phi = synthetic.build(sysm, precision=precision, ctx=ctx)
    orb = phi.download_into(pinned_empty((sysm.npoints, sysm.nst), phi.dtype))
    return Payload(sysm, sysm.local_potential().reshape(-1), orb)


class Server:
    """``contexts`` and ``execute`` default to one library context per slot and the library
    operators; tests of the admission logic inject stand-ins for both."""

    def __init__(self, device: int = 0, slots: int = 4, precision=F32, reserve_bytes: int = 8 << 30,
                 mixed_compute: int = 0, budget_bytes: int | None = None, contexts=None, execute=None,
                 keep_results: bool = True, cache_per_slot: int = 8, bulk_slots: int = 0,
                 bulk_min_bytes: int = 1 << 30, bulk_grid_sms: int = 0):
        if not 0 <= bulk_slots < slots:
            raise ValueError("bulk_slots must leave at least one interactive slot")
        self.device = device
        self.cache = {}     # slot context -> payload -> (payload, basis, Hamiltonian), least recently used first
        self.cache_per_slot = cache_per_slot
        self.precision = precision
        self.keep_results = keep_results
        self.staging = {}   # slot -> pinned host buffer for results
        if contexts is None:
            contexts = [core.Context(device) for _ in range(slots)]
            for i, c in enumerate(contexts):
                c.set_option("mixed_compute", mixed_compute)
                if bulk_slots and i < bulk_slots:
                    c.set_option("grid_sms", bulk_grid_sms)
                elif bulk_slots:
                    c.set_option("stream_priority", 1)
        self.contexts = list(contexts)
        self.bulk_min_bytes = bulk_min_bytes
        n = len(self.contexts)
        self.free = ({"bulk": list(range(bulk_slots)), "interactive": list(range(bulk_slots, n))}
                     if bulk_slots else {"all": list(range(n))})
        self.slot_class = {i: c for c, idx in self.free.items() for i in idx}
        if budget_bytes is None:
            free, _ = self.contexts[0].mem_info()
            budget_bytes = max(0, free - reserve_bytes)
        self.budget = budget_bytes
        self.execute = execute or self._execute
        self.committed = 0
        self.peak_committed = 0
        self.lock = threading.Condition()

    def _fetch(self, ctx, phi: core.OrbitalSet):
        """Copy a set to the host through the slot's pinned staging buffer."""
        need = phi.basis.size() * phi.nst
        buf = self.staging.get(id(ctx))
        if buf is None or buf.size < need or buf.dtype != phi.dtype:
            buf = pinned_empty((max(need, 1 << 20),), phi.dtype)
            self.staging[id(ctx)] = buf
        view = buf[:need]
        phi.download_into(view)
        if self.keep_results:
            return view.reshape(phi.basis.size(), phi.nst).copy()
        return {"checksum": complex(view[:: max(1, need // 4096)].sum())}

    # ------------------------------------------------------------------ one request on one slot
    def _hamiltonian(self, req: Request, ctx: core.Context):
        """The system's basis and Hamiltonian on this slot: built once per payload and kept (least recently
        used first out, at most ``cache_per_slot`` per slot), so a system that comes back skips the host-side
        sphere construction and the table uploads."""
        cache = self.cache.setdefault(id(ctx), OrderedDict())
        key = id(req.payload)
        hit = cache.get(key)
        if hit is not None and hit[0] is req.payload:
            cache.move_to_end(key)
            return hit[1], hit[2]
        sysm = req.payload.system
        basis = core.RealSpace(core.Cell(sysm.lattice), sizes=sysm.sizes, ctx=ctx)
        ham = core.KSHamiltonian(basis)
        ham.set_scalar_potential(req.payload.potential)
        ham.update_projectors_gaussian(sysm.positions, sysm.radius, sysm.rc, sysm.kb)
        cache[key] = (req.payload, basis, ham)
        while len(cache) > self.cache_per_slot:
            cache.popitem(last=False)
        return basis, ham

    def _execute(self, req: Request, ctx: core.Context):
        t0 = time.perf_counter()
        sysm = req.payload.system
        basis, ham = self._hamiltonian(req, ctx)
        phi = core.OrbitalSet(basis, sysm.nst, precision=self.precision).upload(req.payload.orbitals)
        ctx.synchronize()
        t1 = time.perf_counter()
        if req.kind == "apply":
            out = phi.skeleton()
            ham.apply(phi, out)
            ctx.synchronize()
            t2 = time.perf_counter()
            req.result = {"hphi": self._fetch(ctx, out), "happs": sysm.nst}
        else:
            occ = np.full(sysm.nst, 2.0)
            dt = req.dt if req.dt is not None else min(0.05, synthetic.taylor_stable_dt(sysm))
            dips = []
            happs = 0
            for _ in range(req.steps):
                _, dip, iters = core.etrs(ham, [phi], [occ], dt)
                dips.append(dip)
                happs += (4 + 4 * iters) * sysm.nst   # exponential_2_for_1 + one exponential per SCF pass
            ctx.synchronize()
            t2 = time.perf_counter()
            req.result = {"dipoles": np.array(dips), "phi": self._fetch(ctx, phi), "happs": happs}
        ctx.synchronize()
        req.result["phases_ms"] = ((t1 - t0) * 1e3, (t2 - t1) * 1e3, (time.perf_counter() - t2) * 1e3)

    def _worker(self, slot: int, req: Request, t0: float, fp: int):
        try:
            self.execute(req, self.contexts[slot])
        except Exception as e:  # a failing request is reported, the server goes on
            req.error = f"{type(e).__name__}: {e}"
        finally:
            req.finished = time.perf_counter() - t0
            with self.lock:
                self.committed -= fp
                self.free[self.slot_class[slot]].append(slot)
                self.lock.notify_all()

    def request_class(self, fp: int) -> str:
        if "all" in self.free:
            return "all"
        return "bulk" if fp >= self.bulk_min_bytes else "interactive"

    def _dispatch(self, queue, cls, t0, realtime, threads):
        """Admit one class's requests in arrival order: wait for the arrival time, then for a free slot
        of the class and room in the shared memory budget; run each on its own host thread."""
        for req, fp in queue:
            if realtime:
                wait = req.arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
            with self.lock:
                while not self.free[cls] or self.committed + fp > self.budget:
                    self.lock.wait()
                slot = self.free[cls].pop(0)
                self.committed += fp
                self.peak_committed = max(self.peak_committed, self.committed)
            req.admitted = time.perf_counter() - t0
            th = threading.Thread(target=self._worker, args=(slot, req, t0, fp), daemon=True)
            th.start()
            threads.append(th)

    # ------------------------------------------------------------------ the loop
    def run(self, requests: list[Request], realtime: bool = True) -> dict:
        """Serve ``requests`` (sorted by arrival); returns latency / throughput statistics."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        queues = {c: [] for c in self.free}
        t0 = time.perf_counter()
        for req in reqs:
            fp = req.footprint(self.precision)
            if fp > self.budget:
                req.error = f"rejected: needs {fp} bytes, the budget is {self.budget}"
                req.finished = req.admitted = time.perf_counter() - t0
                continue
            queues[self.request_class(fp)].append((req, fp))
        threads = {c: [] for c in queues}
        dispatchers = [threading.Thread(target=self._dispatch, args=(q, c, t0, realtime, threads[c]), daemon=True)
                       for c, q in queues.items()]
        for d in dispatchers:
            d.start()
        for d in dispatchers:
            d.join()
        for ths in threads.values():
            for th in ths:
                th.join()
        wall = time.perf_counter() - t0
        done = [r for r in reqs if not r.error]
        lat = np.array([r.latency for r in done]) if done else np.zeros(1)
        happs = sum(r.result.get("happs", 0) for r in done)
        def phase_means(rs):
            # queue: arrival to admission; setup, compute and fetch as the executor measured them
            ph = np.array([[(r.admitted - r.arrival) * 1e3] + list(r.result["phases_ms"]) for r in rs
                           if "phases_ms" in r.result]).reshape(-1, 4)
            return {k: float(ph[:, i].mean()) if len(ph) else 0.0
                    for i, k in enumerate(("queue_ms", "setup_ms", "compute_ms", "fetch_ms"))}
        phases = phase_means(done)
        tail_cut = np.percentile(lat, 95) if done else 0.0
        tail = phase_means([r for r in done if r.latency >= tail_cut])
        def pct(rs, q):
            return float(np.percentile([r.latency for r in rs], q) * 1000) if rs else 0.0
        big = max((r.payload.system.npoints * r.payload.system.nst for r in done), default=0)
        large = [r for r in done if r.payload.system.npoints * r.payload.system.nst == big]
        small = [r for r in done if r.payload.system.npoints * r.payload.system.nst != big]
        return {"requests": len(reqs), "completed": len(done), "rejected": len(reqs) - len(done),
                "by_size": {"largest_system": {"n": len(large), "p50_ms": pct(large, 50), "p99_ms": pct(large, 99)},
                            "others": {"n": len(small), "p50_ms": pct(small, 50), "p99_ms": pct(small, 99)}},
                "wall_s": wall, "throughput_req_s": len(done) / wall,
                "state_applications_per_s": happs / wall,
                "p50_ms": float(np.percentile(lat, 50) * 1000), "p99_ms": float(np.percentile(lat, 99) * 1000),
                "max_ms": float(lat.max() * 1000), "mean_phase_ms": phases, "slowest_5pct_phase_ms": tail,
                "peak_committed_bytes": self.peak_committed,
                "budget_bytes": self.budget}

    def close(self):
        self.cache.clear()
        for c in self.contexts:
            if hasattr(c, "close"):
                c.close()


def poisson_requests(payloads: list[Payload], n: int, rate: float, seed: int = 7, etrs_fraction: float = 0.3,
                     etrs_steps: int = 10, large: Payload | None = None, large_fraction: float = 0.1):
    """A Poisson arrival stream over the given payloads (the C5 request mix)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        if large is not None and rng.random() < large_fraction:
            p = large
        else:
            p = payloads[int(rng.integers(len(payloads)))]
        kind = "etrs" if rng.random() < etrs_fraction else "apply"
        out.append(Request(i, kind, p, steps=etrs_steps if kind == "etrs" else 1, arrival=t))
    return out
