#!/usr/bin/env python3
"""Benchmark: HEOM ADO-updates/s in FP64 on B200; batched & adjoint vs plain.

Workload (one GPU): 8 sites, one Drude-Lorentz bath per site (lambda = 35
cm^-1, invnu = 50 fs, T = 300 K) with one Matsubara term (16 modes), depth 8:
735,471 ADOs of 8 x 8 complex doubles (753 MB per state); RK4 with dt = 0.5
fs.  Synthetic H (seed 22): diagonal U[12100, 12700] cm^-1, off-diagonal
N(0, 50 cm^-1), real-symmetric.  One "step" = one RK4 step of the whole
hierarchy; 1 ADO-update = one ADO advanced through one RK4 step.

  value     device-resident throughput: K steps enqueued on the handle's
            stream, timed with CUDA events on that stream (state is 753 MB,
            larger than L2, so no flush is needed between steps)
  e2e       the same metric through the C ABI with host buffers: upload of
            the initial hierarchy state from pinned host memory
            (heom_set_state), K steps with the top matrix recorded every 10
            steps and copied back to the host (heom_propagate)
  roofline  the stage kernel (every launch in the timed region is one):
            algorithmic bytes per launch = ADOs x 32 N^2 B (read the stage
            input, write the stage output) / average launch duration
  cpu_baseline  the reference's own heom_ode.cl + rk_weighted_add.cl compiled
            for the host (oracle/_ref) with OpenMP over all host cores, RK4
            steps of the same workload
  parity    the GPU state after the same RK4 steps from the same initial
            state against that reference run: the error per result
  batched   256 static-disorder realisations of a 7-site system, depth 6, in
            one ensemble (one graph launch per RK4 step) against the same
            realisations solved one after another; populations of a sample
            of realisations against the oracle
  adjoint   gradients of the time-integrated site-3 population of a 7-site,
            depth-8 system (2000 steps) w.r.t. 7 site energies, 21 couplings,
            lambda and gamma by one adjoint sweep, against central finite
            differences of 60 + 4 forward solves

--impl reference times that CPU implementation as the reference arm.
Multi-GPU (torchrun): every rank propagates its own replica of the hierarchy
(replicas only: the single-hierarchy path has no exchange step), value is the
sum of ADO-updates over ranks / the max over ranks of the device time.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dm-heom_b200"))

METRIC = "HEOM ADO-updates/s FP64 on 1 B200; batched & adjoint vs plain at ≤1e-10 error"
UNIT = "ADO-updates/s"
N_SITES, DEPTH, MATSUBARAS, SEED, DT = 8, 8, 2, 22, 0.5e-15
OBSERVE_EVERY = 10
FALLBACK_HBM = 6650.0
POP_FLOOR = 1e-3  # relative population errors: |dp| / max(|p_ref|, POP_FLOOR)


def synthetic_h(n, seed):
    rng = np.random.default_rng(seed)
    h = np.zeros((n, n))
    diag = rng.uniform(12100.0, 12700.0, size=n)
    iu = np.triu_indices(n, 1)
    h[iu] = rng.normal(0.0, 50.0, size=len(iu[0]))
    h = h + h.T
    h[np.diag_indices(n)] = diag
    return h


def rel_pop_err(got, ref):
    got, ref = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    return float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), POP_FLOOR)))


def workload_config(scheme, depth=DEPTH, ados=735471, sites=N_SITES, matsubaras=MATSUBARAS):
    modes = sites * matsubaras
    pairs = sites * (sites - 1) // 2 + (sites + 1) // 2
    mb = ados * pairs * 32 / 1e6
    return {"workload": f"{sites} sites, 1 Drude-Lorentz bath/site, {matsubaras - 1} Matsubara term(s) "
                        f"({modes} modes), depth {depth}, {ados} ADOs of {sites}x{sites}, RK4 dt=0.5 fs",
            "ados": ados, "states": sites, "modes": modes, "depth": depth, "dt_fs": 0.5,
            "rk4_scheme": scheme,
            "l2": f"inputs larger than L2 ({mb:.0f} MB state), no flush" if mb > 126 else
                  f"state of {mb:.0f} MB fits in L2 (no flush)",
            "seed": SEED}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index, period_ms=100):
        self.index = index
        self.period_ms = period_ms
        self.proc = None
        self.lines = []
        self.thread = None
        self.first = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            if self.first is None:
                self.first = time.perf_counter()
            self.lines.append(line.strip())

    def wait_first(self, timeout=5.0):
        """Block until the sampler has delivered its first sample."""
        t0 = time.perf_counter()
        while self.proc is not None and self.first is None and time.perf_counter() - t0 < timeout:
            time.sleep(0.01)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


def kernel_source_hash():
    """Hash of the stage kernel's sources (the kernel header and its sector tables)."""
    h = hashlib.sha256()
    for rel in ("dm-heom_b200/csrc/heom_kernels.cuh", "dm-heom_b200/csrc/pair_tables.inc"):
        with open(os.path.join(ROOT, rel), "rb") as f:
            h.update(f.read())
    return h.hexdigest()[:16]


def profiled_traffic():
    """Per-launch DRAM bytes of the benchmark stage kernel from the committed ncu
    summary, used only when the summary was taken on this build of the kernel
    (its kernel_source_hash line matches); otherwise None."""
    path = os.path.join(ROOT, "profiles", "heom_dmma_stage_n8_depth8.md")
    traffic, src = None, None
    try:
        for line in open(path):
            ln = line.strip()
            if ln.startswith("traffic_bytes_per_launch"):
                traffic = float(ln.split("=")[1].strip().split()[0])
            if ln.startswith("kernel_source_hash"):
                src = ln.split("=")[1].strip().split()[0]
    except Exception:
        return None, "no profile summary"
    if traffic is None or src != kernel_source_hash():
        return None, "profile summary taken on another build of the kernel"
    return traffic, "ncu dram__bytes_read.sum + dram__bytes_write.sum of this build (profiles/heom_dmma_stage_n8_depth8.md)"


def cpu_reference_sample(steps_cap=1):
    """Time the reference's own kernels (compiled for the host) on the bench
    workload: RK4 steps of the full hierarchy with all host threads.  Returns
    the baseline record and the state after 1 + steps_cap steps from the
    initial state (one untimed warm-up step, then the timed ones)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import heom_oracle as ho
    prob = ho.build_problem(ho.drude_system(N_SITES, DEPTH, MATSUBARAS, seed=SEED))
    y = prob.initial_state()
    threads = os.cpu_count() or 1
    kind = "reference" if ho.ref_lib(fast=True) is not None else "port"
    step = (lambda v: ho.ref_rk4_step(prob, DT, v, threads, fast=True)) if kind == "reference" else \
        (lambda v: ho.rk4_step(prob, DT, v, threads))
    y = step(y)  # warm-up (page in, thread pool)
    t0 = time.perf_counter()
    for _ in range(steps_cap):
        y = step(y)
    secs = time.perf_counter() - t0
    value = prob.graph.nodes * steps_cap / secs
    rec = {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
           "sample": f"{steps_cap} RK4 step(s) of the full 735471-ADO hierarchy "
                     f"({'heom_ode.cl + rk_weighted_add.cl compiled for the host with -O3 -march=x86-64-v3' if kind == 'reference' else 'oracle C port'}, "
                     f"OpenMP over {threads} threads), {secs:.2f} s",
           "opencl_cpu": opencl_cpu_note()}
    return rec, y, 1 + steps_cap


def opencl_cpu_note():
    """Whether this box offers a CPU OpenCL device (an installable client
    driver other than the GPU vendor's); the reference's own OpenCL path is
    timed only through its kernels compiled for the host."""
    import glob
    icds = sorted(os.path.basename(p) for p in glob.glob("/etc/OpenCL/vendors/*.icd"))
    cpu = [i for i in icds if "nvidia" not in i.lower()]
    if not cpu:
        return "OpenCL CPU device unavailable on this box" + (f" (ICDs: {', '.join(icds)})" if icds else " (no ICD)")
    return f"CPU OpenCL ICDs present but not timed: {', '.join(cpu)}"


def run_reference_arm(args, rank):
    if rank != 0:
        return
    # each step is one full-hierarchy RK4 step of the reference kernels on the
    # host; the number of timed steps is capped so the run ends in minutes
    per_step_cap = max(1, min(args.steps, 6))
    base, _, _ = cpu_reference_sample(steps_cap=per_step_cap)
    line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": per_step_cap, "warmup": 1,
            "ms_per_step": 735471 / base["value"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config("classical RK4 (rk_weighted_add)"),
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": f"requested --steps {args.steps}; timed {per_step_cap} full-hierarchy steps on the host"}
    print(json.dumps(line), flush=True)


def run_e2e(H, y0, args, world, dist, nodes, barrier):
    """Same metric through the C ABI with host buffers: full state upload from
    pinned host memory, then heom_propagate with the top matrix copied back."""
    import torch
    barrier()
    e2e_steps = args.steps - args.steps % OBSERVE_EVERY or OBSERVE_EVERY
    t0 = time.perf_counter()
    H.set_state(y0.numpy())
    tops = H.propagate(DT, e2e_steps, OBSERVE_EVERY)
    e2e_secs = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([e2e_secs], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_secs = float(t.item())
    n = H.states
    trace = float(np.sum([tops[-1][(n + 1) * 2 * i] for i in range(n)]))
    return {"value": world * nodes * e2e_steps / e2e_secs, "unit": UNIT,
            "h2d_bytes_per_step": H.state_len * 8 / e2e_steps,
            "d2h_bytes_per_step": tops.size * 8 / e2e_steps,
            "note": f"{e2e_steps} steps: full state upload from pinned host memory + top matrix "
                    f"every {OBSERVE_EVERY} steps copied back; final trace {trace:.15f}"}


def plain_parity(H, y0, ref_state, ref_steps):
    """The GPU state after ref_steps RK4 steps from y0 against the reference
    kernels' state after the same steps (FP64 both)."""
    n = H.states
    H.set_state(y0)
    H.rk4_steps(DT, ref_steps)
    got = H.get_state()
    idx = [(n + 1) * 2 * i for i in range(n)]
    return {"steps": ref_steps,
            "against": "the reference kernels (heom_ode.cl + rk_weighted_add.cl, FP64) from the same initial state",
            "max_rel_pop_err": rel_pop_err(got[idx], ref_state[idx]),
            "max_rel_state_err": float(np.max(np.abs(got - ref_state)) / np.max(np.abs(ref_state))),
            "pop_floor": POP_FLOOR}


# --------------------------------------------------------------------------
# batched workloads
# --------------------------------------------------------------------------

ENS_SITES, ENS_DEPTH, ENS_COUNT, ENS_SEED, ENS_DT = 7, 6, 256, 33, 1e-15
UNEVEN_COUNT, UNEVEN_SEED = 64, 5


def ensemble_systems(count):
    """Static-disorder ensemble: 7 sites, 1 Drude-Lorentz bath per site, no
    Matsubara term (M = 1), depth 6 (1716 ADOs); realisation k adds N(0, 100
    cm^-1) to every site energy of the seeded H."""
    import heom_b200 as hb
    base = synthetic_h(ENS_SITES, ENS_SEED)
    rng = np.random.default_rng(ENS_SEED + 1)
    out = []
    for _ in range(count):
        h = base.copy()
        h[np.diag_indices(ENS_SITES)] += rng.normal(0.0, 100.0, size=ENS_SITES)
        out.append(hb.System(h, [35.0] * ENS_SITES, [50.0] * ENS_SITES, [0.0] * ENS_SITES, 1, 300.0, ENS_DEPTH))
    return out


def uneven_systems(count):
    """Uneven batch: sites uniform in {4..12}, depth uniform in {4..8}, 0 or 1
    Matsubara term (M = 1 or 2), H drawn as for the plain workload."""
    import heom_b200 as hb
    rng = np.random.default_rng(UNEVEN_SEED)
    out = []
    for k in range(count):
        n = int(rng.integers(4, 13))
        d = int(rng.integers(4, 9))
        m = int(rng.integers(1, 3))
        h = synthetic_h(n, UNEVEN_SEED * 1000 + k)
        out.append(hb.System(h, [35.0] * n, [50.0] * n, [0.0] * n, m, 300.0, d))
    return out


def oracle_populations(system, steps, dt):
    """Site populations after `steps` RK4 steps from rho0 = |0><0| by the oracle."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import heom_oracle as ho
    n = system.sites
    h = (system.h[0::2] + 1j * system.h[1::2]).reshape(n, n)
    prob = ho.build_problem(ho.make_system(h.real if not np.any(h.imag) else h, [35.0] * n, [50.0] * n,
                                           [0.0] * n, system.matsubaras, 300.0, system.depth))
    _, pops = ho.propagate(prob, dt, steps, steps)
    return pops[-1]


def batched_measure(workload, count, steps, warmup, seq_steps, seq_sample, parity_sample, parity_steps,
                    world=1, rank=0, local_rank=0, dist=None):
    """Ensemble throughput (one graph launch per RK4 step over all classes),
    the same instances solved one after another, the e2e path and the
    populations of a sample of instances against the oracle."""
    import torch
    import heom_b200 as hb
    from math import comb
    systems = ensemble_systems(count) if workload == "ensemble" else uneven_systems(count)
    t_setup = time.perf_counter()
    sizes = [comb(s.sites * s.matsubaras + s.depth, s.depth) * (s.sites * (s.sites - 1) // 2 + (s.sites + 1) // 2) * 32
             for s in systems]
    mine = hb.shard_instances(sizes, world, rank)
    tables = [hb.build_tables(systems[k]) for k in mine]
    footprint = hb.Ensemble.footprint(tables)
    E = hb.Ensemble(tables, device=local_rank)
    nodes = [int(t["matrices"]) for t in tables]
    states = [int(t["states"]) for t in tables]
    total_nodes = sum(nodes)

    def seed_tops():
        E.clear()
        for q, n in enumerate(states):
            top = np.zeros(n * n * 2)
            top[0] = 1.0
            E.set_top(q, top)

    seed_tops()
    stage_us = E.autotune()
    setup_s = time.perf_counter() - t_setup
    stream = torch.cuda.ExternalStream(E.stream(), device=local_rank)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    E.rk4_steps(ENS_DT, max(warmup, 3))
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local_rank)
    barrier()
    launches0 = E.kernel_launches()
    clocks.start()
    start.record(stream)
    E.rk4_steps(ENS_DT, steps)
    stop.record(stream)
    stop.synchronize()
    clk = clocks.stop()
    launches = E.kernel_launches() - launches0
    secs_local = start.elapsed_time(stop) / 1e3
    job_ados, job_secs = hb.reduce_throughput(dist, total_nodes * steps, secs_local, "cuda")
    value = job_ados / job_secs

    # e2e through the C ABI: initial tops from the host, propagate with every
    # observation copied back
    e2e_steps = steps - steps % OBSERVE_EVERY or OBSERVE_EVERY
    barrier()
    t0 = time.perf_counter()
    seed_tops()
    tops = E.propagate(ENS_DT, e2e_steps, OBSERVE_EVERY)
    e2e_secs = time.perf_counter() - t0
    traces = [float(np.sum(E.populations(tops[q], q)[-1])) for q in range(len(tables))]
    e2e = {"value": total_nodes * e2e_steps / e2e_secs, "unit": UNIT,
           "h2d_bytes_per_step": sum(n * n * 16 for n in states) / e2e_steps,
           "d2h_bytes_per_step": sum(t.size for t in tops) * 8 / e2e_steps,
           "note": f"{e2e_steps} steps: every hierarchy cleared and its initial top from the host "
                   f"(heom_ensemble_clear + heom_ensemble_set_top), heom_ensemble_propagate with all tops "
                   f"copied back every {OBSERVE_EVERY} steps; trace of every instance within "
                   f"{max(abs(t - 1.0) for t in traces):.1e} of 1"}

    # populations of a sample of instances against the oracle
    seed_tops()
    ptops = E.propagate(ENS_DT, parity_steps, parity_steps)
    sample = mine[:: max(1, len(mine) // parity_sample)][:parity_sample]
    perr = 0.0
    for k in sample:
        q = mine.index(k)
        perr = max(perr, rel_pop_err(E.populations(ptops[q], q)[-1], oracle_populations(systems[k], parity_steps,
                                                                                          ENS_DT)))
    mean_pops = np.mean([E.populations(ptops[q], q)[-1][:3] for q in range(len(mine))
                         if states[q] == states[0]], axis=0)

    # sequential plain solves of the same instances (one handle each, graphs)
    seq_sample_k = mine if workload == "uneven" else mine[:seq_sample]
    seq_ms = []
    for k in seq_sample_k:
        with hb.Heom(**tables[mine.index(k)], device=local_rank) as H:
            top = np.zeros(int(tables[mine.index(k)]["states"]) ** 2 * 2)
            top[0] = 1.0
            H.set_top(top)
            H.rk4_steps(ENS_DT, 3)
            st = torch.cuda.ExternalStream(H.stream(), device=local_rank)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(st)
            H.rk4_steps_async(ENS_DT, seq_steps)
            b.record(st)
            H.synchronize()
            seq_ms.append(a.elapsed_time(b) / seq_steps)
    seq_step_ms = (float(np.mean(seq_ms)) * len(mine) if workload == "ensemble" else float(np.sum(seq_ms)))
    seq_value = total_nodes / (seq_step_ms / 1e3)
    classes = E.classes()
    E.close()
    if workload == "ensemble":
        desc = (f"{count} static-disorder realisations of 7 sites (site energies + N(0,100 cm^-1)), "
                f"1 Drude-Lorentz bath/site, no Matsubara term, depth 6 (1716 ADOs each), RK4 dt=1 fs")
    else:
        desc = (f"{count} instances, sites U{{4..12}}, depth U{{4..8}}, 0 or 1 Matsubara term, "
                f"RK4 dt=1 fs (seed {UNEVEN_SEED})")
    return {"workload": desc, "instances": count, "ados": total_nodes * world, "classes": classes,
            "device_footprint_gb": footprint / 1e9, "steps": steps, "value": value, "unit": UNIT,
            "ms_per_step": job_secs * 1e3 / steps, "gpu_launches": int(launches), "clocks": clk,
            "l2": "state larger than L2 (no flush)" if total_nodes * 800 > 126e6 else
                  "state fits in L2 (no flush; L2-resident by design)",
            "autotuned_stage_us": stage_us, "setup_s": setup_s,
            "sequential_value": seq_value,
            "sequential_note": (f"each instance alone through heom_rk4_steps (graph-captured), "
                                f"{seq_steps} steps timed per instance on {len(seq_sample_k)} of {len(mine)} "
                                f"instances{', scaled to all' if len(seq_sample_k) < len(mine) else ''}"),
            "speedup_vs_sequential": value / seq_value / world,
            "e2e": e2e,
            "parity": {"instances_checked": len(sample), "steps": parity_steps,
                       "against": "the oracle (C restatement of heom_ode.cl, FP64), each instance alone",
                       "max_rel_pop_err": perr, "pop_floor": POP_FLOOR},
            "ensemble_mean_populations": [float(v) for v in mean_pops]}


def run_batched(args, world, rank, local_rank):
    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    count = args.instances or (ENS_COUNT if args.workload == "ensemble" else UNEVEN_COUNT)
    r = batched_measure(args.workload, count, args.steps, args.warmup, args.seq_steps, args.seq_sample,
                        args.parity_sample, args.parity_steps, world, rank, local_rank, dist)
    if rank == 0:
        line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded H, Drude-Lorentz baths)",
                "config": {"workload": r["workload"], "instances": count, "ados": r["ados"],
                           "classes": r["classes"], "device_footprint_gb": r["device_footprint_gb"],
                           "l2": r["l2"],
                           "parallelism": f"instances sharded over {world} ranks" if world > 1 else "single"},
                "e2e": r["e2e"], "gpu_launches": r["gpu_launches"], "clocks": r["clocks"],
                "batched": {k: r[k] for k in ("autotuned_stage_us", "setup_s", "sequential_value",
                                              "sequential_note", "speedup_vs_sequential", "parity",
                                              "ensemble_mean_populations")}}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


ADJ_SITES, ADJ_DEPTH, ADJ_SEED, ADJ_DT_FS, ADJ_STEPS = 7, 8, 44, 1.0, 2000


def adjoint_measure(steps, warmup, local_rank):
    """Gradients of the time-integrated site-3 population (trapezoid rule)
    w.r.t. 7 site energies, 21 couplings, lambda and gamma: one adjoint sweep
    against central finite differences (h = 1e-4 cm^-1; gamma relative 1e-5)
    of the same forward solver, both timed on the host around blocking calls."""
    import torch
    import heom_b200 as hb
    n = ADJ_SITES
    h = synthetic_h(n, ADJ_SEED)
    lam, inv = 35.0, 50.0
    system = hb.System(h, [lam] * n, [inv] * n, [0.0] * n, 1, 300.0, ADJ_DEPTH)
    rho0 = np.zeros((n, n), complex)
    rho0[0, 0] = 1.0
    obs = np.zeros((n, n), complex)
    obs[2, 2] = 1.0
    w = hb.trapezoid_weights(steps, ADJ_DT_FS)
    dt = ADJ_DT_FS * 1e-15
    A = hb.Adjoint(system, device=local_rank)
    for _ in range(max(warmup, 1)):  # also sizes the checkpoint buffers outside the timed call
        A.gradient(rho0, obs, w, dt, steps)
    clocks = ClockSampler(local_rank)
    clocks.start()
    torch.cuda.synchronize()
    launches0 = A.kernel_launches()
    t0 = time.perf_counter()
    out = A.gradient(rho0, obs, w, dt, steps)
    t_adj = time.perf_counter() - t0
    launches = A.kernel_launches() - launches0
    clk = clocks.stop()
    A.close()

    # finite differences: 2 forward solves per parameter through heom_propagate
    top0 = rho0.reshape(-1).view(np.float64).copy()
    idx = 2 * (2 * n + 2)

    def solve(hh, ll=lam, ii=inv):
        sysd = hb.System(hh, [ll] * n, [ii] * n, [0.0] * n, 1, 300.0, ADJ_DEPTH)
        with hb.from_system(sysd, scheme="product", device=local_rank) as H:
            H.set_top(top0)
            torch.cuda.synchronize()
            t = time.perf_counter()
            tops = H.propagate(dt, steps, 1)
            el = time.perf_counter() - t
        return float(np.dot(w, tops[:, idx])), el

    hstep = 1e-4
    params = [(a, a) for a in range(n)] + [(a, b) for a in range(n) for b in range(a + 1, n)]
    fd, ad, t_fd = [], [], 0.0
    for (a, b) in params:
        e = np.zeros((n, n))
        e[a, b] = e[b, a] = 1.0
        fp, tp = solve(h + hstep * e)
        fm, tm = solve(h - hstep * e)
        t_fd += tp + tm
        fd.append((fp - fm) / (2 * hstep))
        g = out["h"].real
        ad.append(g[a, b] + (g[b, a] if a != b else 0.0))
    fp, tp = solve(h, lam + hstep)
    fm, tm = solve(h, lam - hstep)
    t_fd += tp + tm
    fd.append((fp - fm) / (2 * hstep))
    ad.append(out["lambda"])
    gm = 1.0 / inv
    dg = 1e-5 * gm
    fp, tp = solve(h, lam, 1.0 / (gm + dg))
    fm, tm = solve(h, lam, 1.0 / (gm - dg))
    t_fd += tp + tm
    fd.append((fp - fm) / (2 * dg))
    ad.append(out["gamma"])
    fd, ad = np.array(fd), np.array(ad)
    rel = np.abs(ad - fd) / np.maximum(np.abs(fd), 1e-3 * np.max(np.abs(fd[:-2])))
    return {"workload": f"adjoint: 7 sites, 1 Drude-Lorentz bath/site, no Matsubara term, depth 8 "
                        f"(6435 ADOs), RK4 dt=1 fs, {steps} steps, loss = trapezoid integral of the "
                        f"site-3 population; gradients w.r.t. 7 site energies, 21 couplings, lambda, gamma",
            "ados": 6435, "steps": steps, "seconds": t_adj, "value": 6435 * steps / t_adj, "unit": UNIT,
            "value_note": "ADOs x steps / seconds of one heom_adjoint_gradient call "
                          "(forward sweep + checkpointed backward sweep, host I/O included)",
            "loss": out["loss"], "gpu_launches": int(launches), "clocks": clk,
            "fd_seconds": t_fd, "fd_solves": 2 * len(params) + 4, "speedup_vs_fd": t_fd / t_adj,
            "max_rel_diff_vs_fd": float(np.max(rel)),
            "fd_note": "central differences carry an O(h^2) truncation error; the FP64 reference "
                       "gradient check (oracle tangents) is in tests/test_gpu_adjoint.py",
            "grad_site_energies": ad[:n].tolist(), "grad_lambda": out["lambda"], "grad_gamma": out["gamma"]}


def run_adjoint(args, rank, local_rank):
    import torch
    if rank != 0:
        return
    torch.cuda.set_device(local_rank)
    r = adjoint_measure(args.steps, args.warmup, local_rank)
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": 1, "steps": r["steps"],
            "warmup": args.warmup, "ms_per_step": r["seconds"] * 1e3 / r["steps"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded H, Drude-Lorentz baths)",
            "config": {"workload": r["workload"], "ados": r["ados"], "seed": ADJ_SEED, "parallelism": "single"},
            "gpu_launches": r["gpu_launches"], "clocks": r["clocks"],
            "adjoint": {k: r[k] for k in ("seconds", "loss", "value_note", "fd_seconds", "fd_solves",
                                          "speedup_vs_fd", "max_rel_diff_vs_fd", "grad_site_energies",
                                          "grad_lambda", "grad_gamma")}}
    print(json.dumps(line), flush=True)


def run_uneven_adjoint(args, rank, local_rank):
    """Gradients of every instance's time-integrated site-0 population w.r.t.
    its site energies for the uneven batch, by the library's ensemble adjoint
    (heom_ensemble_adjoint_*: class grouping, packing within the memory
    budget and recursive checkpointing of instances that do not fit), against
    central differences of the site energies on a sample of instances."""
    import torch
    import heom_b200 as hb
    from math import comb
    if rank != 0:
        return
    torch.cuda.set_device(local_rank)
    count = args.instances or UNEVEN_COUNT
    systems = uneven_systems(count)
    steps, dt = args.steps, 1e-15
    w = hb.trapezoid_weights(steps, 1.0)
    rho0, obs = [], []
    for s in systems:
        r = np.zeros((s.sites, s.sites), complex)
        r[0, 0] = 1.0
        rho0.append(r)
        obs.append(r)
    E = hb.EnsembleAdjoint(systems, device=local_rank)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = E.gradient(rho0, obs, w, dt, steps, outputs=("h",))  # site energies: the diagonal of dJ/dH
    t_adj = time.perf_counter() - t0
    groups = E.groups()
    launches = E.kernel_launches()
    E.close()
    grads = [np.diag(g.real).copy() for g in out["h"]]

    def ados(k):
        return comb(systems[k].sites * systems[k].matsubaras + systems[k].depth, systems[k].depth)

    small = [k for k in range(count) if ados(k) <= 1_000_000]
    sample = small[:: max(1, len(small) // 6)][:6]
    t_fd_sample, fd_err, fd_sites = 0.0, 0.0, 0
    for k in sample:
        sysd = systems[k]
        n = sysd.sites
        h = sysd.h[0::2].reshape(n, n).copy()
        top = np.zeros(n * n * 2)
        top[0] = 1.0

        def solve(hh):
            s2 = hb.System(hh, [35.0] * n, [50.0] * n, [0.0] * n, sysd.matsubaras, 300.0, sysd.depth)
            with hb.from_system(s2, device=local_rank) as H:
                H.set_top(top)
                torch.cuda.synchronize()
                t = time.perf_counter()
                tops = H.propagate(dt, steps, 1)
                el = time.perf_counter() - t
            return float(np.dot(w, tops[:, 0])), el

        for a in range(min(n, 2)):  # two sites per sampled instance
            e = np.zeros((n, n))
            e[a, a] = 1e-4
            fp, tp = solve(h + e)
            fm, tm = solve(h - e)
            t_fd_sample += tp + tm
            fd = (fp - fm) / 2e-4
            fd_err = max(fd_err, abs(grads[k][a] - fd) / max(abs(fd), 1e-12))
            fd_sites += 1
    sample_nodes = sum(ados(k) for k in sample) * 2  # two sites each
    per_node_s = t_fd_sample / max(1, sample_nodes)
    fd_total = sum(per_node_s * ados(k) * systems[k].sites for k in range(count))
    n_groups = len(set(g for g, _ in groups))
    line = {"metric": METRIC, "value": sum(ados(k) for k in range(count)) * steps / max(t_adj, 1e-12),
            "unit": UNIT, "n_gpus": 1, "steps": steps, "warmup": 0, "ms_per_step": t_adj * 1e3 / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded H, Drude-Lorentz baths)",
            "config": {"workload": f"adjoint of the uneven batch ({count} instances, seed {UNEVEN_SEED}): gradient of "
                                   f"each instance's time-integrated site-0 population w.r.t. its site energies, "
                                   f"{steps} steps of 1 fs, heom_ensemble_adjoint_gradient",
                       "instances": count, "groups": n_groups, "parallelism": "single"},
            "gpu_launches": int(launches),
            "uneven_adjoint": {"seconds": t_adj, "fd_seconds_estimate": fd_total,
                               "speedup_vs_fd": fd_total / max(t_adj, 1e-12),
                               "fd_note": f"central differences of {fd_sites} site energies on {len(sample)} "
                                          f"instances timed ({t_fd_sample:.2f} s) and scaled by ADOs to every "
                                          f"site energy of the batch",
                               "max_rel_diff_vs_fd": fd_err,
                               "recursive": [{"instance": k, "slots": sl} for k, (g, sl) in enumerate(groups) if sl],
                               "value_note": "includes the creation of every group's batch adjoint"}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--scheme", default="product", choices=["product", "horner", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="plain workload: skip the batched sub-object")
    ap.add_argument("--no-adjoint", action="store_true", help="plain workload: skip the adjoint sub-object")
    ap.add_argument("--depth", type=int, default=DEPTH,
                    help="hierarchy depth (8 = the benchmark workload; smaller for profiling captures)")
    ap.add_argument("--sites", type=int, default=N_SITES, help="plain workload: states (8 = the benchmark)")
    ap.add_argument("--matsubaras", type=int, default=MATSUBARAS,
                    help="plain workload: modes per bath (2 = the benchmark's one Matsubara term)")
    ap.add_argument("--workload", default="plain",
                    choices=["plain", "ensemble", "uneven", "adjoint", "uneven-adjoint"],
                    help="plain: one 735471-ADO hierarchy (with the batched and adjoint sub-objects); "
                         "ensemble: 256 disorder realisations (7 sites, depth 6); uneven: 64 instances of "
                         "uneven sizes; adjoint, uneven-adjoint: gradients")
    ap.add_argument("--instances", type=int, default=0, help="instance count of a batched workload")
    ap.add_argument("--seq-steps", type=int, default=100, help="steps per instance of the sequential timing")
    ap.add_argument("--seq-sample", type=int, default=16, help="instances timed alone (ensemble workload)")
    ap.add_argument("--parity-sample", type=int, default=8, help="instances checked against the oracle")
    ap.add_argument("--parity-steps", type=int, default=200, help="steps of the batched parity check")
    ap.add_argument("--batched-steps", type=int, default=500, help="timed steps of the batched sub-object")
    ap.add_argument("--adjoint-steps", type=int, default=ADJ_STEPS, help="steps of the adjoint sub-object")
    ap.add_argument("--clock-load-s", type=float, default=0.5,
                    help="seconds of untimed steps the clock sampler sees before the timed region (0: none)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    if args.workload == "adjoint":
        run_adjoint(args, rank, local_rank)
        return
    if args.workload == "uneven-adjoint":
        run_uneven_adjoint(args, rank, local_rank)
        return
    if args.workload != "plain":
        run_batched(args, world, rank, local_rank)
        return

    import torch
    import heom_b200 as hb

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    ns, nm = args.sites, args.matsubaras
    benchmark_case = (ns, nm, args.depth) == (N_SITES, MATSUBARAS, DEPTH)
    h = synthetic_h(ns, SEED)
    system = hb.System(h, [35.0] * ns, [50.0] * ns, [0.0] * ns, nm, 300.0, args.depth)
    H = hb.from_system(system, device=local_rank, scheme=args.scheme)
    nodes = H.matrices
    y0 = torch.zeros(H.state_len, dtype=torch.float64, pin_memory=True)
    y0[0] = 1.0
    H.set_state(y0.numpy())
    stream = torch.cuda.ExternalStream(H.stream(), device=local_rank)

    # warm-up
    H.rk4_steps(DT, max(args.warmup, 0))
    w0 = time.perf_counter()
    H.rk4_steps(DT, 5)  # untimed: sizes the load phase of the clock sampling below
    warm_step_s = (time.perf_counter() - w0) / 5

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    # clocks under load: the sampler (100 ms) runs through an untimed load
    # phase of about half a second that leads straight into the timed region,
    # so that a short timed region still has samples of the loaded GPU around it
    clocks = ClockSampler(local_rank)
    clocks.start()
    clocks.wait_first()
    if args.clock_load_s > 0:
        H.rk4_steps_async(DT, max(1, min(1000, int(args.clock_load_s / max(warm_step_s, 1e-5)))))
    barrier()
    launches0 = H.kernel_launches()
    with torch.cuda.stream(stream):
        start.record(stream)
        H.rk4_steps_async(DT, args.steps)
        stop.record(stream)
    H.synchronize()
    clk = clocks.stop()
    barrier()
    launches = H.kernel_launches() - launches0
    ms = start.elapsed_time(stop)
    if dist is not None:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    secs = ms / 1e3
    value = world * nodes * args.steps / secs
    per_launch_s = secs / launches if args.scheme != "reference" else None

    # e2e through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(H, y0, args, world, dist, nodes, barrier)

    peak, peak_kind = measured_hbm_peak()
    roofline = None
    if per_launch_s:
        alg_bytes = nodes * 32 * ns * ns
        achieved = alg_bytes / per_launch_s / 1e9
        traffic, traffic_src = profiled_traffic() if benchmark_case else (None, "not the benchmark workload")
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_src,
                    "peak_source": f"{peak_kind} hbm_gbs",
                    "kernel": "heom_dmma_stage" if ns <= 8 else "heom_pair_stage",
                    "kernel_source_hash": kernel_source_hash(),
                    "alg_bytes_per_launch": alg_bytes, "avg_launch_us": per_launch_s * 1e6}

    line = None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded H, Drude-Lorentz baths)",
                "config": dict(workload_config(args.scheme, args.depth, nodes, ns, nm),
                               parallelism=f"replicas{world}" if world > 1 else "single"),
                "e2e": e2e,
                "gpu_launches": int(launches), "roofline": roofline, "clocks": clk,
                "derivative_evals_per_s": 4 * value}
        if world == 1 and not args.no_cpu_baseline and benchmark_case:
            base, ref_state, ref_steps = cpu_reference_sample(steps_cap=3)
            line["cpu_baseline"] = base
            line["parity"] = plain_parity(H, y0.numpy(), ref_state, ref_steps)
    H.close()

    if rank == 0 and world == 1:
        if not args.no_batched:
            b = batched_measure("ensemble", ENS_COUNT, args.batched_steps, args.warmup, args.seq_steps,
                                args.seq_sample, args.parity_sample, args.parity_steps, local_rank=local_rank)
            line["batched"] = b
        if not args.no_adjoint:
            line["adjoint"] = adjoint_measure(args.adjoint_steps, 1, local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
