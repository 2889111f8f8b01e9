#!/usr/bin/env python
"""Benchmark of the FibreNet step loop on B200: bead-steps/s.

Default workload: the tensile test (1,000,000 beads = 20,000 fibres x 50,
finite box 1000x1000x20 with x and z walls and periodic y, HR_FL springs with
E = 1e3 and lognormal failure stress, HR angles, LJ contacts with cut-off
2.5, clamps at x < 2 and x > 998, dt = 0.0005), generated from a fixed seed
because the reference ships no models.  One bench step is one time step of
RunSimulationLoop over all beads; the contact list is rebuilt at step 0 of
every call and every 8 steps, as in the reference.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

The timed region is fn_step(K) from one saved state, repeated (the state
restored between repetitions, outside the events) until about a second of
device time has been measured; the line reports the median repetition.
At N = 1 the line also carries the other parts of the task's metric as
sub-objects: the batched ensemble against the same networks one by one, the
adjoint sweep against the forward pass, the dense mat and the small
network.

--impl reference times the reference's own kernels (FibreNet/kernel.cl compiled
as C, oracle/_ref) on the host cores for the same workload, the same K and W.
With N > 1 (torchrun) every rank runs an independent replica: the path is one
network and does not shard ("replicas only"); value = all ranks' bead-steps
over the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "bead-steps/s (tensile network, 1 B200 per replica)"
UNIT = "bead-steps/s"
WORKLOAD = "tensile_1M"
OUTPUT_FREQ = 100  # the tensile test records reaction force / broken springs every 100 steps
REBUILD_KERNELS = 6  # k_cells, two scan kernels, k_scatter, k_cell_sort, the list build


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--fibres", type=int, default=None,
                   help="fibre count (default 20,000 tensile / 40,000 dense)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the ensemble / adjoint / dense / small-network sub-results")
    p.add_argument("--min-ms", type=float, default=1000.0,
                   help="device time the repeated timed region covers at least")
    p.add_argument("--cpu-seconds", type=float, default=20.0)
    p.add_argument("--workload", choices=["tensile", "dense", "ensemble", "adjoint", "plain"],
                   default="tensile",
                   help="tensile: the 1M-bead network (default, the headline); dense: the 4M-bead "
                        "periodic 3D mat with penalty + soft-repulsion contacts; ensemble: 256 "
                        "independent networks batched in one context vs run one by one; adjoint: "
                        "64 networks, reaction-curve loss, forward + backward sweep vs forward; plain: "
                        "the 10k-bead network of the reference's CPU-runnable case, us per step "
                        "with the steps replayed as CUDA graphs")
    p.add_argument("--networks", type=int, default=None)
    p.add_argument("--adam-iters", type=int, default=0,
                   help="adjoint workload: stiffness-recovery iterations after the timing")
    a = p.parse_args()
    if a.fibres is None:
        a.fibres = 40000 if a.workload == "dense" else 20000
    if a.networks is None:
        a.networks = 64 if a.workload == "adjoint" else 256
    return a


def tensile_model(fibres: int = 20000):
    """The tensile network, placed by the numpy generator (no native code), so
    that both arms of the bench build the same model without loading the
    library under test."""
    from fibrenet_b200 import generate as g
    s = (fibres / 20000.0) ** 0.5
    box = (1000.0 * s, 1000.0 * s, 20.0)
    return g.tensile_network(seed=1, fibres=fibres, beads=50, box=box, clamp_lo=2.0,
                             clamp_hi=box[0] - 2.0, placement="host")


def dense_model(fibres: int = 40000):
    from fibrenet_b200 import generate as g
    s = (fibres / 40000.0) ** (1.0 / 3.0)
    return g.dense_mat(seed=2, fibres=fibres, beads=100, box=(200.0 * s,) * 3)


def workload(args):
    from fibrenet_b200 import generate as g
    if args.workload == "plain":
        return g.plain_network(seed=0)
    if args.workload == "dense":
        return dense_model(args.fibres)
    return tensile_model(args.fibres)


def metric_for(args):
    if args.workload == "plain":
        return "bead-steps/s (10k-bead network, steps as CUDA graphs)"
    if args.workload == "dense":
        return "bead-steps/s (dense 3D mat, 1 B200 per replica)"
    return METRIC


def l2_note(m) -> str:
    """The timing rule this workload meets: a step's device working set (the
    layout's 239 B per bead in the chain form) against the 126 MB L2."""
    if 239 * m.n_beads > 126e6:
        return "working set above 126 MB L2 (inputs larger than L2, no flush)"
    return "working set within 126 MB L2 (a small network: L2-resident, not judged against HBM)"


def config_dict(m, args, extra=None, workload_name=None):
    wl = workload_name or args.workload
    if wl == "plain":
        d = {"workload": "plain_10k", "beads": m.n_beads, "fibres": 200, "beads_per_fibre": 50,
             "box": list(m.settings.box), "contacts": "penalty k 50", "dt": m.settings.dt,
             "grid_update_freq": m.settings.grid_update_freq}
    elif wl == "dense":
        fib = m.n_beads // 100
        d = {"workload": "dense_4M" if fib == 40000 else f"dense_{m.n_beads}", "beads": m.n_beads,
             "springs": m.n_springs, "angles": m.n_angles, "fibres": fib, "beads_per_fibre": 100,
             "box": list(m.settings.box), "bc": "periodic x,y,z",
             "contacts": "penalty k 100 on overlap + soft harmonic k 10 below 1.2 (pair kind hsr)",
             "dt": m.settings.dt, "grid_update_freq": m.settings.grid_update_freq,
             "cell": m.settings.box_unit_cell, "seed": 2, "l2": l2_note(m)}
    else:
        fib = m.n_beads // 50
        d = {"workload": WORKLOAD if fib == 20000 else f"tensile_{m.n_beads}",
             "beads": m.n_beads, "springs": m.n_springs, "angles": m.n_angles,
             "fibres": fib, "beads_per_fibre": 50, "box": list(m.settings.box),
             "bc": "finite x,z / periodic y", "contacts": "LJ eps 1 sigma 1 cut 2.5",
             "dt": m.settings.dt, "grid_update_freq": m.settings.grid_update_freq,
             "cell": m.settings.box_unit_cell, "seed": 1, "placement": "numpy generator, min separation 1.0",
             "l2": l2_note(m)}
    if args is not None:
        d["parallelism"] = f"replicas{args.gpus}" if args.gpus > 1 else "single"
    if extra:
        d.update(extra)
    return d


# --------------------------------------------------------------------------
# clocks during the timed region


class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.path = None

    def start(self):
        import tempfile
        try:
            fd, self.path = tempfile.mkstemp(prefix=f"fn_clocks{self.idx}_", suffix=".csv")
            self.f = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            if self.path:
                self.f.close()
                os.remove(self.path)
        return self

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.remove(self.path)
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# --------------------------------------------------------------------------


def peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def algorithmic_bytes(m, half_pairs: float) -> float:
    """Algorithmic bytes of one step: per bead 4 state arrays
    x 16 B read + written and 16 B of constants, per spring 16 B (+9 B HR_FL),
    per angle 20 B, list offsets 4 B per bead, 4 B per half-list pair."""
    import numpy as np
    n_fl = int((np.asarray(m.s_type) == 1).sum())
    return (m.n_beads * (4 * 16 * 2 + 16) + m.n_springs * 16 + n_fl * 9 + m.n_angles * 20
            + (m.n_beads + 1) * 4 + half_pairs * 4)


def layout_bytes(m, half_pairs: float, chain: bool = True) -> float:
    """Bytes the step kernel's own layout moves at minimum (FP64 positions).
    Chain form: position and image (double4) and force and velocity_old
    (float4) read and written, 26 B of bond records, the list length and the
    list entries per bead.  Otherwise the incidence layout."""
    n, ns, na = m.n_beads, m.n_springs, m.n_angles
    if chain:
        return n * (2 * 32 + 2 * 16) * 2 + n * 26 + n * 4 + 2 * half_pairs * 4
    state = n * (2 * 32 + 2 * 32 + 2 * 16 + 2 * 16)  # pos, img double4 r/w; v_old, F float4 r/w
    bonds = ns * (8 + 16 + 2) + na * (16 + 8 + 8 + 1)
    incid = (n + 1) * 8 + 2 * ns * 4 + 3 * na * 4
    lists = n * 4 + 2 * half_pairs * 4
    return state + bonds + incid + lists


def traffic_from_profiles():
    path = os.path.join(ROOT, "profiles", "k_step_tensile_traffic.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_bead_step:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def traffic_bytes(m):
    """DRAM bytes of one step launch (ncu capture of the tensile network),
    for the 1M-bead tensile workload only; null for other networks."""
    per = traffic_from_profiles()
    if per is None or m.n_beads != 1_000_000 or int(m.meta.get("beads", 0)) != 50 or m.n_types != 3:
        return None
    return per * m.n_beads


def rebuilds_per_call(K: int, freq: int) -> int:
    """Contact rebuilds of one fn_step(K) call: at step 0 and every freq steps
    (the counter restarts with every call, SimulationManager.cpp:152)."""
    return -(-K // freq)


def cpu_reference_rate(model, seconds: float, threads: int | None = None, steps_cap: int = 10**9,
                       warmup: int = 1, chunk: int = 8):
    """Reference kernels (oracle/_ref) on the host cores; a time-bounded
    sample of whole steps in calls of `chunk` steps.  Returns (bead-steps/s,
    steps, threads, kind)."""
    threads = threads or len(os.sched_getaffinity(0))
    os.environ.setdefault("OMP_PROC_BIND", "true")
    os.environ.setdefault("OMP_PLACES", "cores")
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    m = model.fp32_representable()
    if m.settings.bc_type == 1:
        # the reference has one global boundary type; walls on every axis is
        # the closest it can express to the finite-x / periodic-y box
        m.settings.periodic_mask = -1
    import numpy as np
    hsr = np.asarray(m.pair_kind) == 4
    if hsr.any():
        # the reference holds one pair kind per type pair: its closest form of
        # penalty + soft repulsion is the penalty (hs) alone, same lists
        m.pair_kind = np.where(hsr, 2, m.pair_kind).astype(np.int32)
    kind = "reference"
    if po.ref_available():
        sim = po.RefSim(m, threads=threads)
    else:
        kind = "port"
        threads = 1
        sim = po.OracleSim(m, po.MODE_REF)
    if warmup > 0:
        sim.run(warmup)
    done = 0
    t0 = time.perf_counter()
    while done < steps_cap:
        k = min(chunk, steps_cap - done)
        sim.run(k)
        done += k
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    return m.n_beads * done / dt, done, threads, kind


def ref_note(args) -> dict:
    """What the reference's kernels run instead where they cannot express the
    workload exactly."""
    if args.workload == "tensile":
        return {"boundary_in_reference": "walls on all axes"}
    if args.workload == "dense":
        return {"contacts_in_reference": "hs penalty k 100 only (one pair kind per type pair in the reference)"}
    return {}


def run_reference_arm(args):
    """The reference's own kernels (oracle/_ref, OpenMP on every host core the
    process may use) for the same workload: W untimed steps, then exactly K
    timed steps in one RunSimulationLoop call, as our arm's fn_step(K)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    m = workload(args)
    K, W = args.steps, args.warmup
    rate, done, threads, kind = cpu_reference_rate(m, float("inf"), steps_cap=K, warmup=W, chunk=K)
    line = {"metric": metric_for(args), "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": done,
            "warmup": W, "ms_per_step": 1e3 * m.n_beads / rate,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator)", "impl": "reference",
            "config": config_dict(m, args, ref_note(args)),
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"{done} whole steps of the full {m.n_beads}-bead network in one "
                                       f"call after {W} warm-up steps"},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# our arm


def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local, dist


def dist_close(dist):
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def time_reps(sim, K: int, min_ms: float, dist=None, max_reps: int = 2000):
    """fn_step(K) from one saved state, timed with CUDA events on the
    context's stream and repeated (the state restored between repetitions,
    outside the events) until min_ms of device time; every rank runs the
    same number of repetitions.  Returns the per-repetition times (ms); the
    state is left as it was before."""
    from fibrenet_b200.ranks import slowest
    sim.save_state()
    first = sim.step_timed(K)
    reps = int(min(max_reps, max(3, math.ceil(min_ms / max(first, 1e-3)))))
    reps = int(slowest(reps, dist, "cuda"))
    times = []
    for _ in range(reps):
        sim.restore_state()
        times.append(sim.step_timed(K))
    sim.restore_state()
    return times


def run_e2e(args, m, local, dist, world, nb, barrier, block=0, shape=None):
    """Same metric through the public API with host buffers: model upload from
    pinned host arrays, RunSimulationLoop in output_freq chunks with the
    recorded observables read back after each chunk, final state download."""
    import torch

    from fibrenet_b200.native import Simulation

    e2e_steps = args.steps
    mm = m.normalised()
    names = ["pos", "img", "vel", "vel_old", "force", "radius", "mass", "type", "tag", "loc_id",
             "s_type", "s_p1", "s_p2", "s_rest", "s_k", "s_c1", "s_c2", "a_type", "a_b1", "a_b2",
             "a_b3", "a_s1", "a_s2", "a_theta0", "a_k"]
    keep = []
    for name in names:
        t = torch.from_numpy(getattr(mm, name)).pin_memory()
        keep.append(t)
        setattr(mm, name, t.numpy())
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    w0 = time.perf_counter()
    sim2 = Simulation(mm, device=local, list_capacity=64, cell_capacity=64, reorder=True,
                      block_size=block)
    if shape is not None and shape[1] != 0:
        sim2.set_kernel_shape(*shape)  # the tuned shape, when it stages contacts
    w1 = time.perf_counter()
    done = 0
    obs_bytes = 0
    while done < e2e_steps:
        k = min(OUTPUT_FREQ, e2e_steps - done)
        sim2.step(k)
        sim2.observe(0, reaction_type=2 if m.n_types > 2 else -1)
        obs_bytes += 5 * 8
        done += k
    w2 = time.perf_counter()
    final = sim2.get("pos")
    sim2.sync()
    e1.record()
    torch.cuda.synchronize()
    w3 = time.perf_counter()
    e2e_ms = max(e0.elapsed_time(e1), 1e3 * (w3 - w0))
    from fibrenet_b200.ranks import slowest
    e2e_ms = slowest(e2e_ms, dist, "cuda")
    h2d = sum(getattr(mm, k).nbytes for k in names)
    d2h = obs_bytes + final.nbytes
    e2e_value = world * nb * e2e_steps / (e2e_ms / 1e3)
    sim2.close()
    return {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d / e2e_steps,
            "d2h_bytes_per_step": d2h / e2e_steps,
            "what": "Simulation(model from pinned host arrays) + step() in chunks of "
                    f"{OUTPUT_FREQ} with observe() after each + final get('pos')",
            "split_ms": {"upload": 1e3 * (w1 - w0), "steps_and_observe": 1e3 * (w2 - w1),
                         "download": 1e3 * (w3 - w2)}}


def headline(args, m, world, rank, local, dist, e2e=True, cpu=True, label=None):
    """One network's bead-steps/s line (tensile or dense): autotuned block
    size, repeated timed region, kernel split, end-to-end leg, CPU baseline."""
    import torch

    from fibrenet_b200.native import Simulation
    from fibrenet_b200.ranks import job_rate, slowest

    K = args.steps
    sim = Simulation(m, device=local, list_capacity=64, cell_capacity=64, reorder=True)
    nb = m.n_beads
    sim.step(max(args.warmup, 3))
    block = sim.autotune(16)  # block size of the step kernel; the state is restored
    sim.step(8)
    sim.sync()
    sim.rebuild()
    cnt, _ = sim.lists()
    half_pairs = float(cnt.sum()) / 2.0

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- timed region: device-resident state, fn_step(K) repeated from one state
    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    times = time_reps(sim, K, args.min_ms, dist)
    clk = clocks.stop()
    barrier()
    med = statistics.median(times)
    value = job_rate(nb * K, med, dist, "cuda")
    med = slowest(med, dist, "cuda")
    # kernel split over one repetition (events around every launch)
    sim.restore_state()
    sim.enable_timing(True)
    sim.step(K)
    kt = sim.kernel_time()
    sim.enable_timing(False)
    sim.restore_state()
    stats = sim.stats()
    freq = m.settings.grid_update_freq
    rb = rebuilds_per_call(K, freq)
    launches_per_call = 1 + K + rb * REBUILD_KERNELS

    out = {"value": value, "ms_per_step": med / K, "steps": K, "reps": len(times),
           "timed_steps_total": K * len(times), "rep_ms": {"median": statistics.median(times),
                                                            "min": min(times), "max": max(times)},
           "rebuilds_per_step": rb / K, "block": block, "half_pairs": half_pairs, "stats": stats,
           "kt": kt, "clocks": clk, "gpu_launches": launches_per_call * len(times),
           "launches_per_call": launches_per_call}
    peak, peak_kind = peaks()
    alg = algorithmic_bytes(m, half_pairs)
    step_ms = kt["step_ms"]
    achieved = alg / (step_ms / 1e3) / 1e9 if step_ms > 0 else None
    out["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                       "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
                       "kernel": "step kernel (force + kick + drift, one launch per step)",
                       "algorithmic_bytes_per_launch": alg,
                       "layout_bytes_per_launch": layout_bytes(m, half_pairs, stats["bond_path"] == 2),
                       "step_kernel_ms": step_ms, "rebuild_ms": kt["rebuild_ms"],
                       "whole_step_frac": alg / (med / K / 1e3) / 1e9 / peak,
                       "traffic": traffic_bytes(m),
                       "traffic_source": "profiles/k_step_tensile_traffic.txt (ncu dram__bytes_read.sum + "
                                         "dram__bytes_write.sum of one step launch on this network)"}
    sim.close()

    if e2e and not args.no_e2e:
        # three end-to-end runs, the median reported: host-side allocation
        # and page-mapping times on these shared machines vary from run to run
        shape = (stats["block_size"], stats["items_per_thread"])
        runs = [run_e2e(args, m, local, dist, world, nb, barrier, block, shape) for _ in range(3)]
        order = sorted(range(3), key=lambda i: runs[i]["value"])
        e2e_line = dict(runs[order[1]])
        e2e_line["runs"] = [r["value"] for r in runs]
        e2e_line["what"] = runs[0]["what"] + " (median of 3 runs)"
        out["e2e"] = e2e_line
    if cpu and rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, done_cpu, threads, kind = cpu_reference_rate(m, args.cpu_seconds)
        out["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
                               "sample": f"{done_cpu} whole steps of the same {nb}-bead network on "
                                         f"the host in calls of 8 (reference kernels as C, OpenMP"
                                         f"{''.join(', ' + v for v in ref_note(args).values())})"}
    return out


def ensemble_result(args, local, dist, world, rank, steps: int = 100, networks: int = 256):
    """Batched ensemble: the networks in one context (one launch per kernel
    for all of them, steps replayed as CUDA graphs, tuned block size) against
    the same networks each in its own context, run one after the other."""
    from fibrenet_b200 import generate as g
    from fibrenet_b200.native import Simulation
    from fibrenet_b200.ranks import job_rate, partition_networks, slowest
    all_ms = g.ensemble_networks(seed=3, n_networks=networks)
    mine = partition_networks([m.n_beads for m in all_ms], world)[rank]
    ms = [all_ms[i] for i in mine]
    nb = sum(m.n_beads for m in ms)
    nb_all = sum(m.n_beads for m in all_ms)
    K = steps
    batched = Simulation(ms, device=local, list_capacity=32, reorder=True, use_graphs=True)
    batched.step(max(args.warmup, 3))
    block = batched.autotune(16)
    batched.step(8)
    batched.sync()
    clocks = ClockSampler(local).start()
    t_batched = statistics.median(time_reps(batched, K, 300.0, dist, max_reps=20))
    batched.enable_timing(True)
    batched.step(16)
    kt = batched.kernel_time()
    batched.close()
    t_single = 0.0
    for m in ms:
        one = Simulation(m, device=local, list_capacity=32, reorder=True, use_graphs=True)
        one.step(max(args.warmup, 3))
        one.sync()
        one.step_timed(K)  # graphs of this call length captured
        t_single += one.step_timed(K)
        one.close()
    clk = clocks.stop()
    v_b = job_rate(nb * K, t_batched, dist, "cuda")
    v_s = job_rate(nb * K, t_single, dist, "cuda")
    t_batched = slowest(t_batched, dist, "cuda")
    return {"workload": f"ensemble_{len(all_ms)}", "networks": len(all_ms), "beads": nb_all,
            "steps": K, "fibres_per_network": "U[50, 2000] x 50 beads", "graphs": True,
            "block_size": block, "batched_bead_steps_per_s": v_b, "one_by_one_bead_steps_per_s": v_s,
            "batched_over_one_by_one": v_b / v_s, "batched_ms_per_step": t_batched / K,
            "one_by_one_ms_per_step": t_single / K, "step_kernel_ms": kt["step_ms"],
            "rebuild_ms": kt["rebuild_ms"], "clocks": clk,
            "timing": "fn_step(K) with CUDA events on the context stream; batched: median of "
                      "repetitions from one state; one by one: sum over the networks of one "
                      "timed call each after a call of the same length"}


def adjoint_result(args, local, dist, world, rank, networks: int = 64, steps: int = 2000):
    """Stiffness fitting: 64 tensile networks in one context, loss = squared
    error of the x reaction curve (sampled every 20 steps) against a target
    run with lognormal(0, 0.2)-perturbed stiffnesses.  Times the plain
    forward, the recorded forward (checkpoints every 100 steps) and the
    backward sweep (segment replay + adjoint), each with CUDA events."""
    import numpy as np
    import torch

    from fibrenet_b200 import generate as g
    from fibrenet_b200.fitting import ReactionCurve
    from fibrenet_b200.ranks import partition_networks, slowest, total
    every, ckpt = 20, 100
    steps = max(ckpt, (steps // ckpt) * ckpt)
    nsamples = steps // every
    all_ms = g.fitting_networks(seed=4, n_networks=networks)
    mine = partition_networks([m.n_beads for m in all_ms], world)[rank]
    ms = [all_ms[i] for i in mine]
    nb = sum(m.n_beads for m in ms)
    CR = 2
    target_ms = g.perturbed_stiffness(ms, seed=5)
    tgt = ReactionCurve(target_ms, nsamples, every, ckpt, CR, device=local, use_graphs=True)
    target = tgt.run(tgt.params["spring_k"], tgt.params["spring_rest"], tgt.params["angle_k"])
    tgt.close()
    curve = ReactionCurve(ms, nsamples, every, ckpt, CR, device=local, use_graphs=True)
    k0, r0, a0 = curve.params["spring_k"], curve.params["spring_rest"], curve.params["angle_k"]

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def timed(fn):
        e0, e1 = ev(), ev()
        torch.cuda.synchronize()
        e0.record()
        out = fn()
        curve.sim.sync()
        e1.record()
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1)

    # warm-up: graphs, replay buffers
    R = curve.run(k0, r0, a0)
    curve.sim.adjoint_backward(np.zeros_like(R))
    obs = torch.zeros(5, dtype=torch.float64, device=f"cuda:{local}")

    def plain():
        curve._load(k0, r0, a0, None)
        curve.sim.sync()
        e0, e1 = ev(), ev()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(nsamples):
            curve.sim.step(every)
            curve.sim.observe_noalloc(obs.data_ptr(), 0, CR)
        curve.sim.sync()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    clocks = ClockSampler(local).start()
    t_plain = plain()
    curve._load(k0, r0, a0, None)
    R, t_fwd = timed(lambda: curve.sim.adjoint_forward(nsamples, every, ckpt, CR))
    dR = np.zeros_like(R)
    dR[..., 0] = 2.0 * (R[..., 0] - target[..., 0])
    grads, t_bwd = timed(lambda: curve.sim.adjoint_backward(dR))
    clk = clocks.stop()
    loss0 = float(((R[..., 0] - target[..., 0]) ** 2).sum())
    fit = None
    if args.adam_iters > 0:
        logk = torch.tensor(np.log(k0), requires_grad=True)
        opt = torch.optim.Adam([logk], lr=0.02)
        rest_t, ka_t = torch.tensor(r0), torch.tensor(a0)
        tgt_t = torch.tensor(target[..., 0])
        hist = []
        for _ in range(args.adam_iters):
            opt.zero_grad()
            Rt = curve(torch.exp(logk), rest_t, ka_t)
            loss = ((Rt[..., 0] - tgt_t) ** 2).sum()
            loss.backward()
            opt.step()
            hist.append(float(loss.detach()))
        true_k = np.concatenate([np.asarray(t.s_k, np.float64) for t in target_ms])
        k_fit = np.exp(logk.detach().numpy())
        fit = {"iterations": args.adam_iters, "loss_first": hist[0], "loss_last": hist[-1],
               "median_rel_err_k_start": float(np.median(np.abs(k0 / true_k - 1))),
               "median_rel_err_k_fit": float(np.median(np.abs(k_fit / true_k - 1)))}
    curve.close()
    # networks are independent: the loss and the bead count add up over the
    # ranks, times are the slowest rank's, gradient norms combine as squares
    t_plain, t_fwd, t_bwd = (slowest(t, dist, "cuda") for t in (t_plain, t_fwd, t_bwd))
    loss0 = total(loss0, dist, "cuda")
    nb_all = int(total(nb, dist, "cuda"))
    gnorm = {k: float(np.sqrt(total(float(np.sum(np.asarray(v) ** 2)), dist, "cuda")))
             for k, v in grads.items()}
    if fit is not None:
        fit["loss_first"] = total(fit["loss_first"], dist, "cuda")
        fit["loss_last"] = total(fit["loss_last"], dist, "cuda")
    return {"workload": f"fit_{len(all_ms)}", "networks": len(all_ms), "beads": nb_all,
            "steps": steps, "every": every, "checkpoint_every": ckpt,
            "adjoint_over_forward": t_bwd / t_plain, "forward_ms": t_plain,
            "recorded_forward_ms": t_fwd, "backward_ms": t_bwd,
            "forward_bead_steps_per_s": nb_all * steps / (t_plain / 1e3),
            "backward_over_recorded_forward": t_bwd / t_fwd, "loss": loss0, "grad_norm": gnorm,
            "loss_def": "sum (R_x - R*_x)^2", "fit": fit, "clocks": clk,
            "params": {"spring_k": len(k0), "spring_rest": len(r0), "angle_k": len(a0)}}


def plain_result(args, local, dist, steps: int = 2000):
    """The small network (200 fibres x 50 beads, penalty contacts): its working
    set sits in L2, so the step is launch- and latency-bound; steps run as
    CUDA graphs, timed with CUDA events on the context stream."""
    from fibrenet_b200 import generate as g
    from fibrenet_b200.native import Simulation
    from fibrenet_b200.ranks import job_rate, slowest
    m = g.plain_network(seed=0)
    sim = Simulation(m, device=local, list_capacity=64, reorder=True, use_graphs=True)
    sim.step(max(args.warmup, 3))
    block = sim.autotune(64)  # 10k beads fill few SMs at the default block size
    sim.step(8)
    sim.sync()
    clocks = ClockSampler(local).start()
    times = time_reps(sim, steps, 300.0, dist, max_reps=10)
    clk = clocks.stop()
    med = statistics.median(times)
    sim.enable_timing(True)
    sim.step(min(steps, 400))
    kt = sim.kernel_time()
    sim.close()
    value = job_rate(m.n_beads * steps, med, dist, "cuda")
    med = slowest(med, dist, "cuda")
    return {"workload": "plain_10k", "beads": m.n_beads, "steps": steps, "value": value,
            "us_per_step": 1e3 * med / steps, "graphs": True, "block_size": block,
            "step_kernel_us": 1e3 * kt["step_ms"], "rebuild_us": 1e3 * kt["rebuild_ms"],
            "clocks": clk, "l2": "working set in L2 (launch- and latency-bound)"}


def dense_result(args, local, dist, world, rank):
    m = dense_model(40000)
    r = headline(args, m, world, rank, local, dist, e2e=False, cpu=False)
    return {"workload": "dense_4M", "beads": m.n_beads, "value": r["value"],
            "ms_per_step": r["ms_per_step"], "steps": r["steps"], "reps": r["reps"],
            "block_size": r["block"], "step_kernel_ms": r["kt"]["step_ms"],
            "rebuild_ms": r["kt"]["rebuild_ms"], "roofline_frac": r["roofline"]["frac"],
            "half_list_pairs": r["half_pairs"], "clocks": r["clocks"],
            "overflow": {"cell": r["stats"]["cell_overflow"], "list": r["stats"]["list_overflow"]}}


def run_ours(args):
    world, rank, local, dist = dist_setup()
    m = workload(args)
    r = headline(args, m, world, rank, local, dist)
    extras = {}
    if world == 1 and not args.no_extras and args.workload == "tensile":
        extras["ensemble"] = ensemble_result(args, local, dist, world, rank)
        extras["adjoint"] = adjoint_result(args, local, dist, world, rank)
        extras["dense"] = dense_result(args, local, dist, world, rank)
        extras["plain"] = plain_result(args, local, dist)
    if rank == 0:
        line = {
            "metric": metric_for(args), "value": r["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": r["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator; reference ships no models)",
            "config": config_dict(m, args, {"half_list_pairs": r["half_pairs"], "block_size": r["block"],
                                            "items_per_thread": r["stats"]["items_per_thread"],
                                            "list_build": ("beads", "bricks", "groups")[r["stats"]["list_build"]],
                                            "storage": "positions f64, velocities/forces f32",
                                            "timed_region": f"fn_step({args.steps}) from one saved state, "
                                                            f"{r['reps']} repetitions, median"}),
            "reps": r["reps"], "timed_steps_total": r["timed_steps_total"], "rep_ms": r["rep_ms"],
            "rebuilds_per_step": r["rebuilds_per_step"],
            "roofline": r["roofline"], "cpu_baseline": r.get("cpu_baseline"), "e2e": r.get("e2e"),
            "gpu_launches": r["gpu_launches"], "launches_per_call": r["launches_per_call"],
            "clocks": r["clocks"],
            "overflow": {"cell": r["stats"]["cell_overflow"], "list": r["stats"]["list_overflow"]},
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    dist_close(dist)


def run_single_workload(args):
    """--workload ensemble | adjoint | plain: that sub-result alone as the line."""
    world, rank, local, dist = dist_setup()
    if args.workload == "ensemble":
        r = ensemble_result(args, local, dist, world, rank, steps=args.steps, networks=args.networks)
        line = {"metric": "bead-steps/s (256-network ensemble, batched in one launch per kernel)",
                "value": r["batched_bead_steps_per_s"], "unit": UNIT, "n_gpus": world, "steps": r["steps"],
                "warmup": max(args.warmup, 3), "ms_per_step": r["batched_ms_per_step"],
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded generator)",
                "config": {"workload": r["workload"], "networks": r["networks"], "beads": r["beads"],
                           "parallelism": f"networks split over {world} rank(s) by bead count"}}
    elif args.workload == "adjoint":
        r = adjoint_result(args, local, dist, world, rank, networks=args.networks, steps=max(args.steps, 100))
        line = {"metric": "adjoint/forward time (64-network tensile fit)",
                "value": r["adjoint_over_forward"], "unit": "ratio", "n_gpus": world, "steps": r["steps"],
                "warmup": 1, "ms_per_step": r["backward_ms"] / r["steps"], "higher_is_better": False,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64 forces / f32 state / f64 gradient sums",
                "data": "synthetic (seeded generator; target from lognormal(0, 0.2) stiffness factors)",
                "config": {"workload": r["workload"], "networks": r["networks"], "beads": r["beads"],
                           "parallelism": f"networks split over {world} rank(s) by bead count"}}
    else:
        r = plain_result(args, local, dist, steps=args.steps)
        line = {"metric": "bead-steps/s (10k-bead network, steps as CUDA graphs)", "value": r["value"],
                "unit": UNIT, "n_gpus": world, "steps": r["steps"], "warmup": max(args.warmup, 3),
                "ms_per_step": r["us_per_step"] / 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
                "config": {"workload": "plain_10k", "beads": r["beads"]}}
    line["result"] = r
    dist_close(dist)
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.workload in ("ensemble", "adjoint", "plain"):
        run_single_workload(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
