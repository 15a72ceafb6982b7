#!/usr/bin/env python
"""Benchmark: Kohn-Sham H|psi> state-applications per second on a B200.

Workload (one "step" = one H application to every orbital of the set):
  C2 -- cubic a = 20.52 bohr, 96^3 grid, 256 orbitals, 64 atoms (2x2x2 diamond
  supercell, jittered), Gaussian V_loc, l = 0,1 KB projectors (sphere 2 bohr),
  seeded synthetic orbitals orthonormalised in FP64.  Every orbital set is
  1.8 GB (FP32) / 3.6 GB (FP64), far larger than the 126 MB L2, so no flush is
  needed between steps.

The headline ``value`` is the mixed form (FP32 FFTs / potential / projector
contraction, FP64 reductions); the plain FP64 form is timed beside it under
``fp64`` with the mixed form's error against it.  ``e2e`` is the same metric
through the C ABI with host buffers: every step copies the orbitals in from
pinned host memory and H|psi> back out (the steps streamed through one
inqb_apply_host_many call; one inqb_apply_host call per step beside it).

``--impl reference`` times the reference algorithm's CPU restatement (the FP64
oracle: pocketFFT over all host threads + numpy/OpenBLAS) on a bounded sample
of the same workload.

Multi-GPU (torchrun): every rank applies H to its own full orbital set (the
operator has no exchange between states), timing is the max over ranks and
``value`` the total over ranks (weak scaling).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "H·psi applications/s (96^3, 256 states) mixed vs FP64; serving p50/p99 latency"
UNIT = "state-applications/s"
FALLBACK_HBM_GBS = 6650.0


def measured_hbm_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profile_traffic(kernel_key):
    """DRAM bytes per launch recorded from an ncu capture (profiles/ncu_traffic.txt: 'key bytes' lines)."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.txt")) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 2 and parts[0] == kernel_key:
                    return float(parts[1])
    except Exception:
        pass
    return None


class ClockSampler:
    """SM clock and throttle-reason samples during the timed region.

    NVML is polled every 2 ms from a background thread (the timed regions last tens of milliseconds,
    shorter than nvidia-smi's sampling period); the device is found by its PCI bus id, so the NVML
    index need not equal the CUDA index.  Without NVML, nvidia-smi is sampled every 200 ms instead."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    PERIOD_S = 0.002

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.nvml = None
        self.samples = []      # (sm MHz, reasons bit mask)
        self.smax = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            p = torch.cuda.get_device_properties(device_index)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            try:
                self.handle = pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
            except Exception:
                self.handle = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM))
            self.nvml = pynvml
        except Exception:
            self.nvml = None

    def _poll(self):
        nv = self.nvml
        while not self._stop.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle))
                self.samples.append((sm, rs))
            except Exception:
                pass
            time.sleep(self.PERIOD_S)

    def __enter__(self):
        if self.nvml is not None:
            import threading
            self._stop = threading.Event()
            self._thread = threading.Thread(target=self._poll, daemon=True)
            self._thread.start()
            return self
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.nvml is not None:
            self._stop.set()
            self._thread.join(timeout=5)
            return
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, smax, reasons = [], self.smax, set()
        if self.nvml is not None:
            nv = self.nvml
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
            for f, rs in self.samples:
                sm.append(f)
                for n in names:
                    if rs & bits[n]:
                        reasons.add(n)
            source = "nvml, 2 ms"
        else:
            for l in getattr(self, "lines", []):
                p = [x.strip() for x in l.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    smax = float(p[2])
                except ValueError:
                    continue
                for n, v in zip(names, p[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
            source = "nvidia-smi, 200 ms"
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": [], "samples": 0, "source": source}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm),
                "source": source}


# ---------------------------------------------------------------- CPU restatement timing


def cpu_sample(sysm, nsample, min_seconds=10.0, max_steps=50):
    """Time the FP64 oracle (reference algorithm restated on the CPU) on nsample states of the workload."""
    import numpy as np
    import oracle as O
    O.set_fft_workers(os.cpu_count() or 1)
    cell = O.Cell(sysm.lattice)
    rs = O.RealSpace(cell, sysm.sizes)
    pa = O.ProjectorAll.pack([O.build_projector(rs, R, sysm.radius, sysm.rc, sysm.kb[a])
                              for a, R in enumerate(sysm.positions)])
    oh = O.Hamiltonian(rs, sysm.local_potential(), pa)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(sysm.sizes + (nsample,)) + 1j * rng.standard_normal(sysm.sizes + (nsample,))
    oh.apply_real(x)  # warm
    t0 = time.perf_counter()
    steps = 0
    while True:
        oh.apply_real(x)
        steps += 1
        el = time.perf_counter() - t0
        if el >= min_seconds or steps >= max_steps:
            break
    return nsample * steps / el, el, steps


def run_reference(args):
    """--impl reference: the CPU restatement, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from inq_b200 import synthetic
    sysm = synthetic.config("c2")
    import numpy as np
    import oracle as O
    nsample = 8
    O.set_fft_workers(os.cpu_count() or 1)
    cell = O.Cell(sysm.lattice)
    rs = O.RealSpace(cell, sysm.sizes)
    pa = O.ProjectorAll.pack([O.build_projector(rs, R, sysm.radius, sysm.rc, sysm.kb[a])
                              for a, R in enumerate(sysm.positions)])
    oh = O.Hamiltonian(rs, sysm.local_potential(), pa)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(sysm.sizes + (nsample,)) + 1j * rng.standard_normal(sysm.sizes + (nsample,))
    for _ in range(args.warmup):
        oh.apply_real(x)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oh.apply_real(x)
    el = time.perf_counter() - t0
    v = nsample * args.steps / el
    cores = os.cpu_count() or 1
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * el / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "c2: H|psi> on 96^3, 64 atoms; sample of 8 of the 256 orbitals per step",
                       "grid": 96, "states_per_step": nsample, "atoms": 64},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{nsample} orbitals of the 96^3 / 64-atom workload per step, FP64"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU arm


def batch_leg(ctx, nsys=64, reps=5):
    """C4: 64 uneven systems (grids 24..72^3, 8..128 states, 2..32 atoms), mixed form; eager fork/join
    over streams and the replayed CUDA graph of the same batch."""
    import time as _t
    import inq_b200 as ib
    import torch
    from inq_b200 import synthetic
    from inq_b200.batch import Batch, autotune
    t0 = _t.perf_counter()
    sy = synthetic.batch_systems(nsys)
    built = [synthetic.build(s, precision=ib.F32, ctx=ctx) for s in sy]
    setup_s = _t.perf_counter() - t0
    hams = [b[1] for b in built]
    ins = [b[2] for b in built]
    outs = [p.skeleton() for p in ins]
    states = sum(s.nst for s in sy)
    stream = torch.cuda.ExternalStream(ctx.stream())

    def timed(fn):
        fn()
        ctx.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    ms_serial = timed(lambda: [h.apply(i, o) for h, i, o in zip(hams, ins, outs)])
    tuning = autotune(list(zip(hams, ins)), reps=2)
    b = Batch(ctx, hams, ins, outs, nstreams=16, tuning=tuning)
    ms_eager = timed(b.apply)
    b.capture()
    ms_graph = timed(b.launch)
    b.close()
    grids = sorted({s.sizes[0] for s in sy})
    return {"workload": f"c4: {nsys} systems, grids {grids}^3, {states} states in total, "
                        f"{min(s.natoms for s in sy)}-{max(s.natoms for s in sy)} atoms, mixed form",
            "state_applications_per_s_graph": states / (ms_graph / 1000.0),
            "state_applications_per_s_eager_streams": states / (ms_eager / 1000.0),
            "state_applications_per_s_one_by_one": states / (ms_serial / 1000.0),
            "ms_per_batch_graph": ms_graph, "ms_per_batch_eager": ms_eager, "ms_per_batch_one_by_one": ms_serial,
            "autotuned_shapes": len(tuning.table), "setup_s": setup_s}


def serving_leg(ctx, rates=(10.0, 50.0, 200.0, 1000.0, 2000.0), nreq=120, slots=5, bulk_slots=1,
                bulk_grid_sms=0):
    """C5: Poisson stream of H|psi> and 10-step ETRS requests over C4-like systems plus 10% at 96^3 / 256
    states, admitted by free device memory; ``slots`` slots (streams), of which ``bulk_slots`` take the
    96^3 requests with their persistent kernels sized for ``bulk_grid_sms`` SMs; p50 / p99 latency
    and throughput."""
    import inq_b200 as ib
    from inq_b200 import serving, synthetic
    pool = [serving.make_payload(s, ib.F32, ctx) for s in synthetic.batch_systems(12, seed=99)]
    large = serving.make_payload(synthetic.config("c2"), ib.F32, ctx)
    out = {"slots": slots, "bulk_slots": bulk_slots, "bulk_grid_sms": bulk_grid_sms}
    srv = serving.Server(slots=slots, precision=ib.F32, keep_results=False, bulk_slots=bulk_slots,
                         bulk_min_bytes=1 << 30, bulk_grid_sms=bulk_grid_sms)
    for rate in rates:
        reqs = serving.poisson_requests(pool, nreq, rate, seed=int(rate), large=large)
        st = srv.run(reqs)
        out[f"{int(rate)}_req_s"] = {k: st[k] for k in ("completed", "rejected", "throughput_req_s",
                                                        "state_applications_per_s", "p50_ms", "p99_ms", "max_ms",
                                                        "by_size", "mean_phase_ms", "slowest_5pct_phase_ms")}
    # sustained capacity: the same mix with every request present at the start (the server is never idle),
    # then the latency at half and at 80 % of that rate, where the queue stays bounded
    st = srv.run(serving.poisson_requests(pool, nreq, 1e9, seed=1, large=large))
    cap = st["throughput_req_s"]
    out["capacity"] = {"throughput_req_s": cap, "state_applications_per_s": st["state_applications_per_s"]}
    for frac in (0.5, 0.8):
        st = srv.run(serving.poisson_requests(pool, nreq, frac * cap, seed=2, large=large))
        out["capacity"][f"at_{int(frac * 100)}pct"] = {"rate_req_s": frac * cap, "p50_ms": st["p50_ms"],
                                                        "p99_ms": st["p99_ms"], "completed": st["completed"]}
    srv.close()
    return out


def setup_leg(ctx, reps=3):
    """Projector setup (ks_hamiltonian::update_projectors) of the 64-atom 96^3 and 128-atom 120^3
    systems: the host construction against the device kernels, and moving every atom by ~0.1 bohr
    (milliseconds per build, wall clock around a synchronised call)."""
    import numpy as np
    import inq_b200 as ib
    from inq_b200 import synthetic
    out = {}
    for name in ("c2", "c3"):
        sysm = synthetic.config(name, nst=1)
        rs = ib.RealSpace(ib.Cell(sysm.lattice), sizes=sysm.sizes, ctx=ctx)
        ham = ib.KSHamiltonian(rs)
        res = {"atoms": len(sysm.positions), "grid": list(sysm.sizes)}
        for key, dev in (("host_ms", False), ("device_ms", True)):
            ham.update_projectors_gaussian(sysm.positions, sysm.radius, sysm.rc, sysm.kb, device=dev)
            ctx.synchronize()
            t0 = time.perf_counter()
            for _ in range(reps):
                ham.update_projectors_gaussian(sysm.positions, sysm.radius, sysm.rc, sysm.kb, device=dev)
            ctx.synchronize()
            res[key] = (time.perf_counter() - t0) * 1e3 / reps
        rng = np.random.default_rng(5)
        moves = [sysm.positions + rng.normal(0.0, 0.1, sysm.positions.shape) for _ in range(reps)]
        ctx.synchronize()
        t0 = time.perf_counter()
        for p in moves:
            ham.move_atoms(p)
        ctx.synchronize()
        res["move_ms"] = (time.perf_counter() - t0) * 1e3 / reps
        res["points"] = ham.projectors_info()[2]
        out[name] = res
    return out


def overlap_leg(ctx, phi32, phi64, time_loop, reps=5):
    """Subspace overlap S = dV phi^H phi of the 96^3 / 256-state set: the mixed form's split-BF16
    tensor-core kernel against the FP64 overlap of the FP64 set, on the FP64 tensor cores and on SIMT
    (tensor roofline: the executed BF16 products, 4 x 8 N flop per computed element of S: the tiles on
    and above the diagonal)."""
    import numpy as np
    import inq_b200 as ib
    N = phi32.basis.size()
    S = phi32.nst
    ref = ib.overlap(phi64)
    got = ib.overlap(phi32)
    ms_tc = time_loop(lambda: ib.overlap(phi32), reps) / reps
    # FP64 overlap of the FP64 set: FP64 tensor cores (mma.sync m8n8k4, the default) and SIMT
    ms_64 = time_loop(lambda: ib.overlap(phi64), 2) / 2
    ctx.set_option("fp64_mma", 0)
    ms_64_simt = time_loop(lambda: ib.overlap(phi64), 1)
    ctx.set_option("fp64_mma", 1)
    # executed FP64 products of the FP64 overlap: 8 N per computed element (64 x 64 tiles on and above
    # the diagonal)
    t64 = (S + 63) // 64
    flop64 = 8.0 * N * min((t64 * (t64 + 1) // 2) * 64 * 64, S * S)
    # executed BF16 products: 4 x 8 N per computed result element; a set with itself is Hermitian, so
    # only the 128 x 128 tiles on and above the diagonal are computed
    t = (S + 127) // 128
    computed = (t * (t + 1) // 2) * 128 * 128 if S >= 128 else S * S
    flop = 4.0 * 8.0 * N * min(computed, S * S)
    peak = float(json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                             "MEASURED_PEAKS.json")))["bf16_tflops"]) \
        if os.path.exists(os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")) else 1590.0
    return {"workload": f"overlap of the c2 set: {N} points, {S} x {S} states",
            "ms_tensor_core_split_bf16": ms_tc, "ms_fp64_tensor_core": ms_64, "ms_fp64_simt": ms_64_simt,
            "fp64_tflops_executed": flop64 / (ms_64 / 1000.0) / 1e12,
            "rel_err_vs_fp64": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
            "max_abs_err_vs_fp64": float(np.max(np.abs(got - ref))),
            "roofline": {"bound": "tensor", "achieved": flop / (ms_tc / 1000.0) / 1e12, "peak": peak,
                         "unit": "TFLOP/s", "frac": flop / (ms_tc / 1000.0) / 1e12 / peak,
                         "flop_per_call": flop}}


def etrs_leg(ctx, steps=200, dt=0.005):
    """C3: real-time propagation at 120^3 / 256 states / 128 atoms after a 0.01 a.u. kick along x (phase
    exp(i 0.01 x)), through the real-time driver (real_time::propagate, propagate.hpp:87-119): every step
    is one ETRS step (etrs.hpp:22-79, FP64 density each step) plus the energy of the step
    (energy.calculate, propagate.hpp:99: one more H application and its reductions) and the dipole;
    plain FP64 and mixed series side by side.

    The time step: the order-4 Taylor exponential (exponential.hpp:21-69) is stable only for
    dt * E_max < 2 sqrt(2), and the grid's kinetic energy reaches E_max = 3/2 (pi n / a)^2 = 325 Ha at
    120^3 / a = 25.6 bohr, so dt must stay below 0.0087 a.u.; at dt = 0.05 the norm grows without bound
    (the reference algorithm does the same).  The leg runs at dt = 0.005."""
    import numpy as np
    import torch
    import inq_b200 as ib
    from inq_b200 import real_time, synthetic
    sysm = synthetic.config("c3")
    basis, ham, phi64 = synthetic.build(sysm, ctx=ctx)
    ib.apply_phase_kick(phi64, [0.01, 0.0, 0.0])
    phi32 = phi64.converted(ib.F32)
    occ = np.full(sysm.nst, 2.0)
    emax = 1.5 * (np.pi * sysm.sizes[0] / sysm.lattice[0][0]) ** 2
    out = {}
    stream = torch.cuda.ExternalStream(ctx.stream())
    series = {}
    for name, phi in (("fp64", phi64), ("mixed", phi32)):
        # one untimed step on a copy: the step's work buffers come from the stream-ordered pool, whose
        # first growth to this size (tens of GB at 120^3 FP64) would otherwise land in the timed steps
        warm = phi.copy()
        real_time.propagate(ham, [warm], [occ], dt, 1)
        del warm
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ctx.synchronize()
        e0.record(stream)
        res = real_time.propagate(ham, [phi], [occ], dt, steps)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        norm = ib.overlap_diagonal(phi).real
        dip = np.array(res.dipole)
        ene = np.array(res.total_energy)
        series[name] = (dip, ene)
        out[name] = {"steps_per_s": steps / (ms / 1000.0), "ms_per_step": ms / steps,
                     "max_norm_drift": float(np.max(np.abs(norm - 1.0))),
                     "energy_first_last_ha": [float(ene[0]), float(ene[-1])],
                     "max_energy_drift_ha": float(np.max(np.abs(ene - ene[0]))),
                     "dipole_every_50_steps": dip[::50].tolist()}
    d64, e64 = series["fp64"]
    d32, e32 = series["mixed"]
    out["max_dipole_diff_mixed_vs_fp64"] = float(np.max(np.abs(d64 - d32)))
    out["max_energy_diff_mixed_vs_fp64_ha"] = float(np.max(np.abs(e64 - e32)))
    out["max_dipole_change_fp64"] = float(np.max(np.abs(d64 - d64[0])))
    out["dt"] = dt
    out["steps"] = steps
    out["dt_stability_bound"] = float(2 * np.sqrt(2) / emax)
    # interacting: the potential rebuilt from every density (Hartree + LDA on the device), FP64
    isteps = 5
    ham.set_interaction(sysm.local_potential())
    p = phi64.copy()
    ham.update_hamiltonian(ib.density([p], [occ]).reshape(-1))
    warm = p.copy()
    ib.etrs(ham, [warm], [occ], dt)
    del warm
    ham.update_hamiltonian(ib.density([p], [occ]).reshape(-1))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    its, dips = [], []
    ctx.synchronize()
    e0.record(stream)
    for _ in range(isteps):
        _, dip, it = ib.etrs(ham, [p], [occ], dt)
        its.append(it)
        dips.append(dip.tolist())
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    ham.clear_interaction()
    out["interacting_fp64"] = {"steps_per_s": isteps / (ms / 1000.0), "ms_per_step": ms / isteps,
                               "scf_iterations": its, "dipole_series": dips,
                               "update": "V = V_ion + V_H (Poisson) + V_xc (LDA) from every density of the step"}
    out["workload"] = (f"c3: 120^3, {sysm.nst} states, {sysm.natoms} atoms, kick 0.01 x, dt {dt} "
                       f"(0.05 exceeds the Taylor-4 stability bound {2 * np.sqrt(2) / emax:.4f}), {steps} steps "
                       f"of ETRS + energy + dipole (real_time.propagate)")
    return out


def run_ours(args):
    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    import inq_b200 as ib
    from inq_b200 import synthetic

    ctx = ib.Context(local)
    sysm = synthetic.config("c2", seed=20240601 + rank)
    basis, ham, phi64 = synthetic.build(sysm, ctx=ctx)
    phi32 = phi64.converted(ib.F32)
    out64 = phi64.skeleton()
    out32 = phi32.skeleton()
    S, N = sysm.nst, sysm.npoints
    stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))

    def barrier():
        ctx.synchronize()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def time_loop(fn, steps):
        barrier()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            fn()
        ev1.record(stream)
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1)
        if dist is not None:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        barrier()
        return ms

    # warm up both forms
    for _ in range(args.warmup):
        ham.apply(phi32, out32)
        ham.apply(phi64, out64)
    ctx.synchronize()

    # timed: mixed form (headline) with clock sampling, then FP64
    launches0 = ctx.launch_count()
    with ClockSampler(local) as clk:
        ms32 = time_loop(lambda: ham.apply(phi32, out32), args.steps)
    launches = ctx.launch_count() - launches0
    ms64 = time_loop(lambda: ham.apply(phi64, out64), args.steps)

    v32 = world * S * args.steps / (ms32 / 1000.0)
    v64 = world * S * args.steps / (ms64 / 1000.0)

    # the other butterfly-arithmetic modes of the mixed form (option mixed_compute; 0 is the default)
    mode_ms = {0: ms32}
    for mode in (1, 2, 3):
        ctx.set_option("mixed_compute", mode)
        for _ in range(2):
            ham.apply(phi32, out32)
        mode_ms[mode] = time_loop(lambda: ham.apply(phi32, out32), args.steps)
    ctx.set_option("mixed_compute", 0)

    # accuracy of the mixed forms against the FP64 form on the full workload
    ham.apply(phi64, out64)
    ctx.synchronize()
    h64 = torch.from_numpy(out64.matrix())
    n64 = torch.linalg.vector_norm(h64)
    e64, _ = ham.eigenvalues(phi64)
    acc = {}
    for mode in (0, 1, 2, 3):
        ctx.set_option("mixed_compute", mode)
        ham.apply(phi32, out32)
        ctx.synchronize()
        h32 = torch.from_numpy(out32.matrix()).to(torch.complex128)
        e32, _ = ham.eigenvalues(phi32)
        acc[mode] = (float(torch.linalg.vector_norm(h32 - h64) / n64), float(np.max(np.abs(e32 - e64))))
        del h32
    ctx.set_option("mixed_compute", 0)
    del h64
    rel_err, eig_err = acc[0]

    # dominant kernels: the batched FFT passes (to_fourier = 3 launches, each reads and writes the set once);
    # timed with single-precision butterflies (the headline mode) and, for reference, double
    f32 = phi32.skeleton(ib.FOURIER_SPACE)
    reps = max(3, args.steps)
    pass_ms = {}
    for mode in (1, 0):
        ctx.set_option("mixed_compute", mode)
        for _ in range(2):
            ctx.check(ctx.lib.inqb_to_fourier(phi32.handle, f32.handle))
        pass_ms[mode] = time_loop(lambda: ctx.check(ctx.lib.inqb_to_fourier(phi32.handle, f32.handle)), reps) / (3 * reps)
    ctx.set_option("mixed_compute", 0)
    alg_bytes = 2.0 * N * S * 8
    peak, peak_kind = measured_hbm_gbs()
    achieved = alg_bytes / (pass_ms[0] / 1000.0) / 1e9
    achieved_d = alg_bytes / (pass_ms[1] / 1000.0) / 1e9
    traffic = profile_traffic("fft2_kernel_f32f32w_c2")
    # whole-operator algorithmic bytes s_c (5N + 3P) per state
    _, _, P = ham.projectors_info()
    b_alg = 8.0 * (5 * N + 3 * P) * S
    h_achieved = b_alg / (ms32 / 1000.0 / args.steps) / 1e9

    # e2e through the C ABI with pinned host buffers (mixed form)
    host_in = torch.empty((N, S), dtype=torch.complex64, pin_memory=True)
    host_in.copy_(torch.from_numpy(phi32.matrix()))
    host_out = torch.empty((N, S), dtype=torch.complex64, pin_memory=True)

    hin_np = host_in.numpy()
    hout_np = host_out.numpy()

    def e2e_step():
        # the public host-buffer call: state blocks stream through the device, copies overlap the operator
        ham.apply_host(hin_np, hout_np)

    e2e_step()
    e2e_steps = max(3, min(args.steps, 10))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    barrier()
    e2e_s = time.perf_counter() - t0
    # the same steps streamed through one call (inqb_apply_host_many): every step still uploads its input
    # set and downloads its result, and consecutive steps' copies overlap
    ham.apply_host_many([hin_np] * 2, [hout_np] * 2)
    barrier()
    t0 = time.perf_counter()
    ham.apply_host_many([hin_np] * e2e_steps, [hout_np] * e2e_steps)
    barrier()
    e2e_many_s = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([e2e_s, e2e_many_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s, e2e_many_s = (float(x) for x in t.tolist())
    e2e_single_v = world * S * e2e_steps / e2e_s
    e2e_v = world * S * e2e_steps / e2e_many_s

    legs = {}
    if world == 1 and not args.skip_legs:
        legs["overlap"] = overlap_leg(ctx, phi32, phi64, time_loop)
        legs["batch"] = batch_leg(ctx)
        legs["setup"] = setup_leg(ctx)
        legs["serving"] = serving_leg(ctx)
        if args.etrs_steps > 0:
            legs["etrs"] = etrs_leg(ctx, args.etrs_steps, args.etrs_dt)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        nsample = 8
        v, el, st = cpu_sample(sysm, nsample)
        cpu = {"value": v, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
               "sample": f"FP64 oracle on {nsample} of the 256 orbitals of the same workload, {st} applications "
                         f"in {el:.1f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": v32, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded C2 construction)",
            "config": {"workload": "c2: H|psi> 96^3 grid, 256 states, 64 atoms, mixed form (FP32, FP64 reductions)",
                       "grid": [96, 96, 96], "states": S, "atoms": sysm.natoms, "sphere_points": P,
                       "l2": "inputs larger than L2 (1.8 GB orbital set), no flush",
                       "parallelism": f"each of {world} rank(s) holds its own 256-state set"},
            "mixed_modes": {str(m): {"value": world * S * args.steps / (mode_ms[m] / 1000.0),
                                     "ms_per_step": mode_ms[m] / args.steps, "rel_err_hpsi_vs_fp64": acc[m][0],
                                     "max_eigenvalue_err_ha": acc[m][1]} for m in (0, 1, 2, 3)},
            "roofline": {"bound": "hbm",
                         "kernel": "fft2_kernel<float,float,96,FWD_STORE,1>: one batched 1-D FFT pass over the set "
                                   "(FP32 data and butterflies, 512-byte rows; the forward passes of the headline "
                                   "step)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": traffic,
                         "alg_bytes_per_launch": alg_bytes, "launch_ms": pass_ms[0],
                         "double_butterfly_pass": {"kernel": "fft2_kernel<float,double,96,FWD_STORE>",
                                                   "achieved": achieved_d, "frac": achieved_d / peak,
                                                   "launch_ms": pass_ms[1]}},
            "e2e": {"value": e2e_v, "unit": UNIT, "h2d_bytes_per_step": N * S * 8, "d2h_bytes_per_step": N * S * 8,
                    "steps": e2e_steps, "how": "pinned host buffers; all steps streamed through one "
                    "inqb_apply_host_many call (state blocks of 64, copies of consecutive steps overlapping)",
                    "one_call_per_step": {"value": e2e_single_v, "how": "one inqb_apply_host call per step"}},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        line.update(legs)
        if "serving" in legs:
            line["serving_p50_ms"] = legs["serving"]["50_req_s"]["p50_ms"]
            line["serving_p99_ms"] = legs["serving"]["50_req_s"]["p99_ms"]
            line["serving_capacity_req_s"] = legs["serving"]["capacity"]["throughput_req_s"]
        if cpu is not None:
            line["cpu_baseline"] = cpu
        # the figures the headline comparison rests on come last, so that a reader of the end of the line
        # (a truncated log) still sees them
        line["operator_roofline"] = {"alg_bytes_per_step": b_alg, "achieved_gbs": h_achieved,
                                     "frac": h_achieved / peak, "formula": "8 B * (5N + 3P) * S"}
        line["accuracy"] = {"rel_err_hpsi_mixed_vs_fp64": rel_err, "max_eigenvalue_err_ha": eig_err,
                            "mixed": "FP32 orbitals, intermediates and butterflies (products by constants and "
                                     "twiddles compensated, mixed_compute 0); FP64 overlaps, Cholesky, density, "
                                     "energy and eigenvalue reductions"}
        line["fp64"] = {"value": v64, "ms_per_step": ms64 / args.steps, "dtype": "f64"}
        line["mixed_ms_per_step"] = ms32 / args.steps
        line["mixed_over_fp64"] = v32 / v64
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_profile_case(args):
    """Small case for ncu captures: the C2 (or, with ``--profile-config c3``, C3) grid and atoms with
    ``--profile-states`` orbitals (C2, 32 states: 226 MB per FP32 set, above L2; 128: 0.9 GB).

    Sequence: FP64 build (3 FFT passes), then ``--steps`` mixed-form and ``--steps`` FP64 applications
    (each: 1 projection + 5 FFT passes + 1 nonlocal apply), then ``--steps`` tensor-core overlaps of the
    FP32 set."""
    import inq_b200 as ib
    from inq_b200 import synthetic
    S = args.profile_states
    sysm = synthetic.config(args.profile_config, nst=S)
    basis, ham, phi64 = synthetic.build(sysm)
    phi32 = phi64.converted(ib.F32)
    out32, out64 = phi32.skeleton(), phi64.skeleton()
    for _ in range(args.steps):
        ham.apply(phi32, out32)
    for _ in range(args.steps):
        ham.apply(phi64, out64)
    for _ in range(args.steps):
        ib.overlap(phi32)
    basis.ctx.synchronize()
    print(json.dumps({"profile_case": f"{args.profile_config} grid, {S} states", "launches": basis.ctx.launch_count()}))


def _kernel_table(prof, label):
    """Device time per kernel (summed over launches) of a torch.profiler capture, as a markdown table."""
    import collections
    tot = collections.defaultdict(lambda: [0, 0.0])
    for e in prof.events():
        if e.device_type.name == "CUDA":
            k = e.name.split("(")[0].replace("void ", "").replace("inqb::", "").replace("v2::", "")[:70]
            tot[k][0] += 1
            tot[k][1] += e.device_time_total / 1000.0
    total = sum(v[1] for v in tot.values())
    lines = [f"== {label}: total device time {total:.2f} ms", "| kernel | launches | ms | share |",
             "|---|---|---|---|"]
    for k, (c, t) in sorted(tot.items(), key=lambda x: -x[1][1]):
        lines.append(f"| `{k}` | {c} | {t:.2f} | {100 * t / total:.1f}% |")
    print("\n".join(lines), flush=True)


def run_breakdown(args):
    """Per-kernel device times (torch.profiler, CUDA activity) of one piece of work, after one untimed
    repetition of it:

    * ``etrs``: one step of real_time.propagate at 120^3 / 128 atoms / 256 orbitals (ETRS, the band
      energy, the dipole), FP64 and mixed form, starting from the kicked orbitals (the propagate call also
      forms the step-0 density and energy);
    * ``batch``: the 64 uneven systems of the batched workload applied one by one (mixed form), with the
      time of each grid size's systems."""
    import collections
    import numpy as np
    import torch
    from torch.profiler import profile, ProfilerActivity
    import inq_b200 as ib
    from inq_b200 import synthetic, real_time
    ctx = ib.Context(0)
    if args.breakdown == "etrs":
        sysm = synthetic.config("c3")
        basis, ham, phi64 = synthetic.build(sysm, ctx=ctx)
        ib.apply_phase_kick(phi64, [0.01, 0.0, 0.0])
        phi32 = phi64.converted(ib.F32)
        occ = np.full(sysm.nst, 2.0)
        for name, phi in (("FP64", phi64), ("mixed", phi32)):
            w = phi.copy()
            real_time.propagate(ham, [w], [occ], args.etrs_dt, 1)
            del w
            p = phi.copy()
            ctx.synchronize()
            with profile(activities=[ProfilerActivity.CUDA]) as prof:
                real_time.propagate(ham, [p], [occ], args.etrs_dt, 1)
                ctx.synchronize()
            _kernel_table(prof, f"one step of real_time.propagate at 120^3 x 256, {name}")
            del p
        return
    sy = synthetic.batch_systems(64)
    built = [synthetic.build(s, precision=ib.F32, ctx=ctx) for s in sy]
    outs = [b[2].skeleton() for b in built]
    stream = torch.cuda.ExternalStream(ctx.stream())
    groups = collections.defaultdict(list)
    for i, s in enumerate(sy):
        groups[s.sizes[0]].append(i)
    for n in sorted(groups):
        idx = groups[n]
        for i in idx:
            built[i][1].apply(built[i][2], outs[i])
        ctx.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(5):
            for i in idx:
                built[i][1].apply(built[i][2], outs[i])
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / 5
        set_bytes = sum(sy[i].nst * n ** 3 * 8 for i in idx)
        print(f"grid {n}^3: {len(idx)} systems, {sum(sy[i].nst for i in idx)} states, FP32 sets {set_bytes / 1e6:.1f} MB,"
              f" {ms:.3f} ms one by one, {11 * set_bytes / ms / 1e6:.0f} GB/s for 11 transits of the set", flush=True)
        per = []
        for i in idx:
            e0.record(stream)
            for _ in range(5):
                built[i][1].apply(built[i][2], outs[i])
            e1.record(stream)
            e1.synchronize()
            ms_i = e0.elapsed_time(e1) / 5
            per.append(f"{sy[i].nst}:{ms_i * 1e3:.0f}us/{11 * sy[i].nst * n ** 3 * 8 / ms_i / 1e6:.0f}")
        print("    states:time/GB/s " + " ".join(per), flush=True)
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        for b, o in zip(built, outs):
            b[1].apply(b[2], o)
        ctx.synchronize()
    _kernel_table(prof, "the 64 uneven systems applied one by one, mixed form")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--skip-legs", action="store_true", help="skip the batched-systems, serving and ETRS legs")
    ap.add_argument("--etrs-steps", type=int, default=200, help="ETRS steps of the 120^3 real-time leg (0: skip)")
    ap.add_argument("--etrs-dt", type=float, default=0.005, help="time step of the 120^3 real-time leg (a.u.)")
    ap.add_argument("--profile-case", action="store_true", help="small workload for ncu captures")
    ap.add_argument("--profile-states", type=int, default=32, help="orbitals of the --profile-case workload")
    ap.add_argument("--profile-config", default="c2", choices=["c2", "c3"],
                    help="grid and atoms of the --profile-case workload (96^3 / 64 atoms or 120^3 / 128 atoms)")
    ap.add_argument("--breakdown", choices=["etrs", "batch"],
                    help="print per-kernel device times of one real-time step or of the batched systems")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.breakdown:
        run_breakdown(args)
    elif args.profile_case:
        run_profile_case(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
