#!/usr/bin/env python
"""Benchmark of the Grains3D DEM time step on B200 (pacific_b200).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision mixed|fp64]
                    [--workload polydisperse_200k|drum_100k|settling_1k|adjoint_4k] [--impl reference]

One bench step = one chunk of `--chunk` DEM time steps (default 1000) of the
workload, replayed from CUDA graphs on resident device state; the default
--steps 20 therefore times the whole 20,000-step run from the initial state
(after W warm-up chunks and a reset).  L2 is flushed (a 256 MiB write)
between timed chunks.  `value` is particle-steps/s of the
whole job (all ranks); `e2e` is the same metric through the C ABI with host
buffers in pinned memory: update of the kinematic state, the chunk, download
of the state.

Config 1 starts from a sparse lattice (mean coordination ~0.1 over its 20,000
steps), so the line also carries a `settled` leg: the bed settled on the
device (70,000 steps), saved as a reference reload file and read back, then
10 x 1,000 steps timed in mixed precision and in FP64 from that state (mean
coordination ~5), with its per-phase times, roofline and contact-force error.

With --gpus N (launched by torchrun) every rank runs an independent replica
(the single system is not partitioned across GPUs): weak scaling.
`--impl reference` times the reference's CPU implementation of the step
(oracle/_ref when it was built from the reference sources, otherwise the
oracle restatement) on the host cores, rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic HBM bytes per particle of one launch of each step kernel: every
# array the kernel must touch, once (z = contacts per particle incl. walls,
# the list entries of the force evaluation; R4 = 16 B in mixed precision, 32 B
# in FP64; a contact-memory entry is 44 B / 80 B; a pair's two list entries and
# its work item count once per particle on average):
#  contacts_kernel: own position+radius (32), meta (16) and cell key (4), the
#   9 cell-row ranges (72), list length (4) in/out; z list entries (4 z) and
#   z/2 work items (8 z/2) out.  Neighbour positions are re-read from L1/L2
#   and not counted.
#  pairs_kernel: own xr, meta, md, upload index (32 + 16 + 32 + 4), v, w
#   (2 R4), the list (4 z) and the work items (8 z/2) in; the owner's z/2
#   memory entries in and out; the results of the z entries (2 R4 each) out.
#  sums_kernel: md, meta, upload index, list length (32 + 16 + 4 + 4), the list
#   (4 z) and the z results (2 R4 each) in; F, T (2 R4), coordination and
#   memory count (8) out, the memory row packed (z/2 entries in place).
#  kick_move_kernel: xr, q, meta, md (32 + 32 + 16 + 32), v, w, wbf, inertia,
#   F, T (6 R4) in; xr, q (64), v, w, wbf (3 R4), cell key and count (8) out.
#   Bodies that are not spheres also carry their rotation matrix (72 B in and out).
def kernel_bytes(kernel, precision, z, basis=False):
    r4 = 16 if precision == "mixed" else 32
    entry = 44 if precision == "mixed" else 80
    if kernel == "contacts":
        return 32 + 16 + 4 + 72 + 4 + 4 * z + 8 * z / 2.0
    if kernel == "pairs":
        return 84 + 2 * r4 + 4 * z + 8 * z / 2.0 + 2 * (z / 2.0) * entry + 2 * r4 * z
    kick = (32 + 32 + 16 + 32 + 6 * r4) + (64 + 3 * r4 + 8) + (144 if basis else 0)
    sums = 56 + 4 * z + 2 * r4 * z + 2 * r4 + 8 + (z / 2.0) * entry
    if kernel == "sums":
        return sums
    if kernel == "sums_kick":  # the sums with the kick: the torsor stays in registers
        return sums - 2 * r4 + kick - 2 * r4
    return kick


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--chunk", type=int, default=1000)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--workload", default="polydisperse_200k")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--ref-dem-steps", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--adjoint", action="store_true", help="time the adjoint workload (4,096 spheres)")
    ap.add_argument("--no-io", action="store_true", help="skip the reload / RawData file writers")
    ap.add_argument("--settle-steps", type=int, default=None,
                    help="DEM steps that settle the bed before the settled leg (0: no settled leg; default "
                         "70,000 for polydisperse_200k, 100,000 for drum_100k, none otherwise)")
    ap.add_argument("--settled-chunks", type=int, default=10, help="timed chunks of the settled leg")
    ap.add_argument("--settled-state", default=None,
                    help="hybrid-binary reload file of the settled bed: read when it exists (it must come from "
                         "the same workload and --settle-steps), else written after settling")
    return ap.parse_args()


def scenario(name):
    from pacific_b200 import scenarios as S
    return {"polydisperse_200k": S.polydisperse_200k, "settling_1k": S.settling_1k,
            "adjoint_4k": S.adjoint_4k, "drum_100k": S.drum, "ensemble_512": S.ensemble_512}[name]()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(kernel, workload, precision):
    """dram bytes per launch of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "%s_%s_%s.md" % (kernel, workload, precision))
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""
    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.stop = threading.Event()
        self.t = threading.Thread(target=self.run, daemon=True)

    def run(self):
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.t.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 2 + k and "Active" in r[2 + k]
                          and "Not" not in r[2 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def quantize_radii(sc, n_classes=64):
    """The reference builds one particle class per distinct sphere; radii are
    rounded to n_classes values (spacing 6 um for U[0.8, 1.2] mm) so that its
    set-up stays tractable at 200k particles."""
    from pacific_b200 import scenarios as S
    r = sc.particles["radius"]
    lo, hi = float(r.min()), float(r.max())
    if hi <= lo or any(sc.shapes[k][0] != S.SPHERE for k in set(np.asarray(sc.particles["shape"]).tolist())):
        return sc
    sc.meta["radius_classes"] = n_classes
    q = lo + np.round((r - lo) / (hi - lo) * (n_classes - 1)) / (n_classes - 1) * (hi - lo)
    sc.particles["radius"] = q
    sc.particles["mass"], sc.particles["inertia"] = S.sphere_mass_inertia(q, 2500.0)
    return sc


def one_system(sc, k):
    """System k of a multi-system scenario as a scenario of its own."""
    from pacific_b200 import scenarios as S
    sel = np.asarray(sc.particles["system"]) == k
    p = {key: (None if v is None else np.asarray(v)[sel]) for key, v in sc.particles.items()}
    p["system"] = np.zeros(int(sel.sum()), np.int32)
    meta = {key: v for key, v in sc.meta.items() if key != "sizes"}
    meta["sample_system"] = (k, len(sc.domains))
    return S.Scenario(sc.name, sc.shapes, [sc.domains[k]], [sc.laws[k]], [sc.obstacles[k]], p, sc.dt, sc.n_steps,
                      meta=meta)


def sample_note(sc):
    """What the CPU sample left out of the workload."""
    note = ""
    if "sample_system" in sc.meta:
        k, n = sc.meta["sample_system"]
        note += ", its largest system (%d of %d, %d particles) alone: the reference holds one system" % (k, n, sc.n)
    if "radius_classes" in sc.meta:
        note += ", sphere radii rounded to 64 classes (one reference particle class each)"
    return note


def cpu_context(sc):
    """A context of the CPU implementation: the reference built from its own
    sources (oracle/_ref) when present, else the oracle restatement.  The
    reference runs one system: of a multi-system workload it runs the largest."""
    from pacific_b200.abi import FP64, GrainsLib, Simulation
    from pacific_b200 import scenarios as S
    ref = os.path.join(ROOT, "oracle", "_ref", "libgrains_ref.so")
    if os.path.exists(ref):
        lib, kind = GrainsLib(ref, "grains_ref_"), "reference"
        if len(sc.domains) > 1:
            sizes = np.bincount(np.asarray(sc.particles["system"]), minlength=len(sc.domains))
            sc = one_system(sc, int(np.argmax(sizes)))
        sc = quantize_radii(sc)
    else:
        path = os.path.join(ROOT, "oracle", "_build", "libgrains_oracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-s"], check=True)
        lib, kind = GrainsLib(path, "grains_oracle_"), "port"
    sim = Simulation(lib, FP64, max_particles=sc.n, n_systems=len(sc.domains))
    S.apply(sim, sc)
    sim.initialize_leapfrog(0.0, sc.dt)
    return sim, kind, sc


def cpu_baseline(sc, steps, keep=False):
    """Times `steps` DEM steps of the CPU implementation (serial, one core)
    from the initial state of the same workload."""
    sim, kind, sc = cpu_context(sc)
    t0 = time.perf_counter()
    sim.step(steps, 0.0, sc.dt)
    el = time.perf_counter() - t0
    sample = "%s, %d DEM steps after the leapfrog start, serial" % (sc.name, steps) + sample_note(sc)
    res = {"value": sc.n * steps / el, "unit": "particle-steps/s", "cores": 1, "kind": kind, "sample": sample}
    if keep:
        return res, sim
    sim.close()
    return res


def io_measure(lib, sim, t, cpu=None, reps=3):
    """Output files of the reference's formats from the device state (the end
    of the timed run): the particle file of a reload (text and hybrid binary),
    read back, and one RawData output (text and binary); host wall time per
    call, files in a temporary directory.  `cpu`: (context, kind) of the CPU
    implementation, whose writers are timed once on its own state."""
    import tempfile
    from pacific_b200.abi import read_reload_particles
    out = {}

    def timed(fn, n_reps):
        ts, nb = [], 0
        for _ in range(n_reps):
            t0 = time.perf_counter()
            nb = fn()
            ts.append(time.perf_counter() - t0)
        return float(np.median(ts)), int(nb)

    def entry(s, nb, n):
        return {"ms": s * 1e3, "bytes": nb, "GB_per_s": nb / s / 1e9, "particles_per_s": n / s}

    with tempfile.TemporaryDirectory(prefix="gg_bench_io") as d:
        for binary in (False, True):
            key = "hybrid" if binary else "text"
            path = os.path.join(d, "save_" + key)
            s, nb = timed(lambda: sim.write_reload_particles(path, binary), reps)
            out["reload_write_" + key] = entry(s, nb, sim.n)
            s, nb = timed(lambda: (read_reload_particles(lib, path, binary), os.path.getsize(path))[1], reps)
            out["reload_read_" + key] = entry(s, nb, sim.n)
            rkey = "binary" if binary else "text"
            root = os.path.join(d, "raw_" + rkey)
            s, nb = timed(lambda: sim.write_rawdata(root, t, binary=binary, truncate=True), reps)
            out["rawdata_write_" + rkey] = entry(s, nb, sim.n)
        if cpu is not None:
            csim, kind = cpu
            base = {}
            for name, fn in [("reload_write_text", lambda: csim.write_reload_particles(os.path.join(d, "c.txt"))),
                             ("rawdata_write_text", lambda: csim.write_rawdata(os.path.join(d, "craw"), t,
                                                                               truncate=True))]:
                s, nb = timed(fn, 1)
                base[name] = entry(s, nb if nb else sum(os.path.getsize(os.path.join(d, f)) for f in os.listdir(d)
                                                        if f.startswith("craw")), csim.n)
            base["kind"] = kind
            base["cores"] = 1
            base["sample"] = "the CPU implementation's writers, serial, on its own state of the same workload"
            out["cpu_baseline"] = base
    return out


def run_reference(args, rank, world):
    """The reference arm: the CPU implementation on the host cores, rank 0 only.
    One bench step = `--ref-dem-steps` DEM steps of the workload."""
    if rank != 0:
        return
    sc = scenario(args.workload)
    sim, kind, sc = cpu_context(sc)
    t = 0.0
    for _ in range(args.warmup):
        t = sim.step(args.ref_dem_steps, t, sc.dt)
    per = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        t = sim.step(args.ref_dem_steps, t, sc.dt)
        per.append(time.perf_counter() - t0)
    total = sum(per)
    v = sc.n * args.ref_dem_steps * args.steps / total
    sample = "%s, %d DEM steps per bench step from the initial state, serial" % (sc.name, args.ref_dem_steps)
    sample += sample_note(sc)
    line = {"metric": "particle-steps/s", "value": v, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "impl": "reference", "dtype": "f64", "data": "synthetic",
            "scaling": "weak", "vs_baseline": None,
            "config": {"workload": sc.name, "particles": sc.n, "dem_steps_per_step": args.ref_dem_steps,
                       "precision": "fp64"},
            "cpu_baseline": {"value": v, "unit": "particle-steps/s", "cores": 1, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def nvtx(name):
    """An NVTX range around a leg of the bench, so that a profiler can be
    limited to it (ncu --nvtx --nvtx-include "<name>/")."""
    import torch
    return torch.cuda.nvtx.range(name)


def contact_force_error(lib, sc, state, mem, device, where):
    """Per-contact relative error of the mixed-precision contact forces against
    the plain FP64 path on identical states and contact memories: max and 99th
    percentile of |f_mixed - f_fp64| / max(|f_fp64|, weight) over the
    particle-particle contacts of every system."""
    from pacific_b200 import scenarios as S
    from pacific_b200.abi import FP64, MIXED, Simulation
    p = dict(sc.particles)
    for k in ["position", "quaternion", "velocity", "omega"]:
        p[k] = state[k]
    if sc.particles.get("basis") is not None:
        p["basis"] = state["basis"]
    sc2 = S.Scenario(sc.name, sc.shapes, sc.domains, sc.laws, sc.obstacles, p, sc.dt, sc.n_steps, meta=sc.meta)
    res = {}
    for name, prec in [("fp64", FP64), ("mixed", MIXED)]:
        s = Simulation(lib, prec, max_particles=sc.n, n_systems=len(sc.domains), device=device)
        S.apply(s, sc2)
        s.upload_contact_memory(mem)
        s.compute_forces(0.0, sc.dt)
        per = [s.contact_forces(k) for k in range(len(sc.domains))]
        res[name] = (np.concatenate([q[0] for q in per]), np.concatenate([q[1] for q in per]))
        s.close()
    (p64, f64_), (pm, fm) = res["fp64"], res["mixed"]
    if len(p64) == 0 or not np.array_equal(p64, pm):
        return {"n_contacts": int(len(p64)), "pairs_equal": bool(np.array_equal(p64, pm))}
    w = float(np.min(sc.particles["mass"])) * 9.81
    rel = np.linalg.norm(fm - f64_, axis=1) / np.maximum(np.linalg.norm(f64_, axis=1), w)
    return {"max": float(rel.max()), "p99": float(np.quantile(rel, 0.99)), "median": float(np.median(rel)),
            "n_contacts": int(len(rel)), "systems": len(sc.domains), "pairs_equal": True, "floor": "particle weight",
            "state": where + ", same state and contact memory in both precisions"}


def profile_run(sim, sc, n_steps, t):
    """Per-phase device times (ms per DEM step) of n_steps uncaptured steps and
    the dominant kernel of the step with its algorithmic bytes."""
    tp, prof = sim.profile_kernels(n_steps, t, sc.dt)
    return tp, {k: v[0] / n_steps for k, v in prof.items()}, {k: v for k, v in prof.items()}


def roofline(prof_tot, sc, precision, z, peak, peak_kind, traffic_of):
    from pacific_b200 import scenarios as S
    dom = max([k for k in ["contacts", "pairs", "sums", "sums_kick", "kick_move"] if k in prof_tot],
              key=lambda k: prof_tot[k][0])
    k_ms, k_n = prof_tot[dom]
    basis = any(sc.shapes[k][0] != S.SPHERE for k in set(np.asarray(sc.particles["shape"]).tolist()))
    alg = sc.n * kernel_bytes(dom, precision, z, basis)
    achieved = alg / (k_ms / k_n / 1e3) / 1e9
    # with convex bodies the pair phase also holds the GJK kernels (their runs
    # are bound by divergence and FP64 latency, not by these bytes)
    kernel = "pair phase: gjk_count, gjk_place, gjk_kernel, pairs_kernel" if basis and dom == "pairs" else dom + "_kernel"
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic_of(dom), "kernel": kernel, "peak_source": peak_kind,
            "algorithmic_bytes_per_launch": alg, "mean_coordination": z, "launch_ms": k_ms / k_n}


def mean_coordination(sim, sc, t):
    sim.reset_stats()
    sim.compute_forces(t, sc.dt)
    st = sim.stats()
    return (2.0 * st["n_contacts"] + st["n_obstacle_contacts"]) / sc.n


def settled_leg(args, lib, sc, local, flush, peak, peak_kind):
    """The 200k bed settled on the device: `settle_steps` DEM steps from the
    initial state, saved as a reference reload file (hybrid binary) and read
    back; then `settled_chunks` x chunk steps timed in mixed precision and in
    FP64 from that same state (after the same warm-up), the per-phase times,
    the roofline of the dominant kernel and the contact-force error there."""
    import tempfile
    import torch
    from pacific_b200 import scenarios as S
    from pacific_b200.abi import FP64, MIXED, Simulation, read_reload_particles
    t = args.settle_steps * sc.dt
    n_obs = len(sc.obstacles[0]) if len(sc.domains) == 1 else 0
    poses = None
    if args.settled_state and os.path.exists(args.settled_state):
        r = read_reload_particles(lib, args.settled_state, True)
        z_settled, nbytes, w_s = None, os.path.getsize(args.settled_state), None
        if n_obs:
            poses = np.load(args.settled_state + ".obstacles.npy")
    else:
        sim = Simulation(lib, MIXED, max_particles=sc.n, device=local)
        S.apply(sim, sc)
        sim.initialize_leapfrog(0.0, sc.dt)
        t, done = 0.0, 0
        with nvtx("settling"):
            while done < args.settle_steps:
                k = min(5000, args.settle_steps - done)
                t = sim.step(k, t, sc.dt)
                done += k
            sim.synchronize()
        z_settled = mean_coordination(sim, sc, t)
        if n_obs:
            # the particle file holds no obstacles: their poses after the
            # settling (rotating drum) go with it
            poses = sim.obstacles(0, n_obs)
            if args.settled_state:
                np.save(args.settled_state + ".obstacles.npy", poses)
        with tempfile.TemporaryDirectory(prefix="gg_settled") as d:
            path = args.settled_state or os.path.join(d, "settled_Particles.bin")
            t0 = time.perf_counter()
            nbytes = sim.write_reload_particles(path, binary=True)
            w_s = time.perf_counter() - t0
            r = read_reload_particles(lib, path, True)
        sim.close()
    p = dict(sc.particles)
    order = np.argsort(r["id"])
    for k in ["position", "quaternion", "velocity", "omega"] + (["basis"] if p.get("basis") is not None else []):
        p[k] = np.ascontiguousarray(r[k][order])
    obstacles = sc.obstacles
    if poses is not None:
        obstacles = [[dict(o, transform=[float(x) for x in poses[i]]) for i, o in enumerate(sc.obstacles[0])]]
    sc2 = S.Scenario(sc.name, sc.shapes, sc.domains, sc.laws, obstacles, p, sc.dt, sc.n_steps, meta=sc.meta)
    mem = r["memory"]
    out = {"settle_steps": args.settle_steps, "mean_coordination_after_settling": z_settled,
           "reload_file": {"bytes": int(nbytes), "write_ms": None if w_s is None else w_s * 1e3,
                           "format": "hybrid binary", "read_from_settled_state": w_s is None}}

    def run(prec):
        s = Simulation(lib, prec, max_particles=sc.n, device=local)
        S.apply(s, sc2)
        s.upload_contact_memory(mem)
        s.initialize_leapfrog(t, sc.dt)
        stream = torch.cuda.ExternalStream(s.stream_handle(), device=local)
        tt = t
        for _ in range(args.warmup):
            tt = s.step(args.chunk, tt, sc.dt)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.settled_chunks)]
        torch.cuda.synchronize()
        with nvtx("settled_%s_timed" % ("fp64" if prec == FP64 else "mixed")):
            for k in range(args.settled_chunks):
                with torch.cuda.stream(stream):
                    flush.fill_(k & 0xFF)
                    ev[k][0].record(stream)
                tt = s.step(args.chunk, tt, sc.dt)
                ev[k][1].record(stream)
            torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in ev)
        return s, tt, ms
    sm, tm, ms_m = run(MIXED)
    z = mean_coordination(sm, sc, tm)
    gst = sm.stats()  # of that one force evaluation
    with nvtx("settled_kernels"):
        _, per_step, tot = profile_run(sm, sc, 500, tm)
    sm.close()
    s64, _, ms_64 = run(FP64)
    s64.close()
    steps = args.settled_chunks * args.chunk
    v_m, v_64 = sc.n * steps / (ms_m / 1e3), sc.n * steps / (ms_64 / 1e3)
    out.update({"value": v_m, "unit": "particle-steps/s", "ms_per_dem_step": ms_m / steps,
                "timed_dem_steps": steps, "mean_coordination": z,
                "fp64": {"value": v_64, "ms_per_dem_step": ms_64 / steps, "mixed_over_fp64": v_m / v_64},
                "kernels_ms_per_dem_step": per_step,
                "roofline": roofline(tot, sc, "mixed", z, peak, peak_kind,
                                     lambda k: profiled_traffic(k, sc.name + "_settled", "mixed")),
                "contact_force_error": contact_force_error(lib, sc, sc2.particles, mem, local,
                                                           "the settled bed read back from its reload file")})
    if gst["n_gjk_calls"]:
        # GJK calls and iterations of one force evaluation (the running
        # statistics of AppCollision::addToContactsFeatures, AppCollision.cpp:160-187)
        out["gjk"] = {"calls_per_dem_step": gst["n_gjk_calls"],
                      "mean_iterations": gst["n_gjk_iterations"] / gst["n_gjk_calls"],
                      "pairs_per_s": gst["n_gjk_calls"] / (ms_m / 1e3 / steps)}
    return out


def run_adjoint(args, rank, world, local):
    """The adjoint workload (4,096 spheres, 2,000 steps, a checkpoint every 100
    force evaluations): device time of a differentiable forward run plus its
    adjoint, in both precisions.  (Gradient accuracy against the FP64
    dual-number oracle: tests/test_adjoint_gpu.py and
    tests/measure_adjoint_accuracy.py.)"""
    import torch
    import pacific_b200
    from pacific_b200 import scenarios as S
    from pacific_b200.abi import FP64, MIXED, Adjoint, Simulation
    torch.cuda.set_device(local)
    lib = pacific_b200.load_library()
    sc = S.adjoint_4k()
    n, steps, every = sc.n, sc.n_steps, 100

    def loss_grads(final):
        m = sc.particles["mass"]
        inertia = np.asarray(sc.particles["inertia"])[:, 0]
        v, w = final["velocity"], final["omega"]
        zc = final["position"][:, 2].mean()
        ke = np.mean(0.5 * m * (v * v).sum(1) + 0.5 * inertia * (w * w).sum(1))
        z0, k0 = 0.9 * zc, 0.5 * ke
        gx = np.zeros_like(v)
        gx[:, 2] = 2.0 * (zc - z0) / n
        return (gx, 2.0 * (ke - k0) * (m[:, None] * v) / n, 2.0 * (ke - k0) * (inertia[:, None] * w) / n)

    out = {}
    for name, prec in [("mixed", MIXED), ("fp64", FP64)]:
        sim = Simulation(lib, prec, max_particles=n, device=local)
        S.apply(sim, sc)
        adj = Adjoint(sim, every)
        stream = torch.cuda.ExternalStream(sim.stream_handle(), device=local)
        for _ in range(args.warmup):
            adj.backward(*loss_grads(adj.forward(steps, sc.dt)))
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        fwd = bwd = 0.0
        for _ in range(args.steps):
            e[0].record(stream)
            fin = adj.forward(steps, sc.dt)
            e[1].record(stream)
            adj.backward(*loss_grads(fin))
            e[2].record(stream)
            torch.cuda.synchronize()
            fwd += e[0].elapsed_time(e[1])
            bwd += e[1].elapsed_time(e[2])
        out[name] = {"forward_ms": fwd / args.steps, "backward_ms": bwd / args.steps,
                     "value": n * steps * args.steps / ((fwd + bwd) / 1e3), "contacts": adj.signature()[1]}
        adj.close()
        sim.close()
    line = {"metric": "particle-steps/s (differentiable forward + adjoint)", "value": out["mixed"]["value"],
            "unit": "particle-steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": out["mixed"]["forward_ms"] + out["mixed"]["backward_ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "adjoint_4k", "particles": n, "dem_steps": steps, "checkpoint_every": every,
                       "loss": "(z_com - 0.9 z_com0)^2 + (KE - 0.5 KE0)^2"},
            "mixed": out["mixed"], "fp64": out["fp64"]}
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.adjoint:
        return run_adjoint(args, rank, world, local)

    import torch
    import torch.distributed as dist
    if world > 1:
        import datetime
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    import pacific_b200
    from pacific_b200 import scenarios as S
    from pacific_b200.abi import FP64, MIXED, Simulation

    lib = pacific_b200.load_library()
    prec = MIXED if args.precision == "mixed" else FP64
    sc = scenario(args.workload)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda:%d" % local)

    def timed_run(precision, sample_clocks):
        """W warm-up chunks, then K timed chunks from the initial state (the
        whole 20,000-step run by default); device time in ms over the K chunks."""
        sim = Simulation(lib, precision, max_particles=sc.n, n_systems=len(sc.domains), device=local)
        S.apply(sim, sc)
        sim.initialize_leapfrog(0.0, sc.dt)
        stream = torch.cuda.ExternalStream(sim.stream_handle(), device=local)
        t = 0.0
        for _ in range(args.warmup):
            t = sim.step(args.chunk, t, sc.dt)
        sim.synchronize()
        sim.update(sc.particles)
        sim.reset_stats()
        sim.initialize_leapfrog(0.0, sc.dt)
        t = 0.0
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        clk = ClockSampler(local) if sample_clocks else None
        if clk:
            clk.__enter__()
        with nvtx("%s_timed" % ("fp64" if precision == FP64 else "mixed")):
            for k in range(args.steps):
                with torch.cuda.stream(stream):
                    flush.fill_(k & 0xFF)          # L2 flush between timed chunks (untimed)
                    ev[k][0].record(stream)
                t = sim.step(args.chunk, t, sc.dt)
                ev[k][1].record(stream)
            torch.cuda.synchronize()
        sim.synchronize()
        if clk:
            clk.__exit__()
        return sim, stream, t, sum(a.elapsed_time(b) for a, b in ev), clk

    sim, stream, t, ms, clk = timed_run(prec, True)
    st_end, mem_end = sim.download(), sim.contact_memory()   # state at the end of the timed run
    if world > 1:
        tt = torch.tensor([ms], device="cuda:%d" % local, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
        dist.barrier()
    st = sim.stats()
    total_particles = sc.n * world
    value = total_particles * args.chunk * args.steps / (ms / 1e3)

    # kernel timing over the same run: from the initial state again, the whole
    # window of K chunks uncaptured with CUDA events around each phase on the
    # library's stream; the mean coordination is sampled once per chunk
    sim.update(sc.particles)
    sim.initialize_leapfrog(0.0, sc.dt)
    tp = 0.0
    prof_tot = {}
    zs = []
    for k in range(args.steps):
        with nvtx("kernels"):
            tp, _, prof = profile_run(sim, sc, args.chunk, tp)
        for name, (ms_k, n_k) in prof.items():
            a0, b0 = prof_tot.get(name, (0.0, 0))
            prof_tot[name] = (a0 + ms_k, b0 + n_k)
        zs.append(mean_coordination(sim, sc, tp))
    z = float(np.mean(zs))
    peak, peak_kind = measured_peaks()
    n_prof = args.chunk * args.steps

    # end to end through the C ABI with host buffers in pinned memory, over
    # the same window of K chunks from the initial state: every chunk updates
    # the kinematic state from the host, steps, and downloads the state and
    # the coordination numbers
    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype, pin_memory=True).numpy()
    host = {"position": pinned((sc.n, 3), torch.float64), "quaternion": pinned((sc.n, 4), torch.float64),
            "velocity": pinned((sc.n, 3), torch.float64), "omega": pinned((sc.n, 3), torch.float64),
            "coordination": pinned((sc.n,), torch.int32)}
    sim.update(sc.particles)
    sim.initialize_leapfrog(0.0, sc.dt)
    t = 0.0
    sim.download(out=host)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(args.steps):
        sim.update(host)
        t = sim.step(args.chunk, t, sc.dt)
        sim.download(out=host)
    e2e_s = (time.perf_counter() - t0) / args.steps
    h2d = sum(host[kk].nbytes for kk in ["position", "quaternion", "velocity", "omega"])
    d2h = sum(v.nbytes for v in host.values())
    e2e_value = total_particles * args.chunk / e2e_s
    gather_every = sim.tuning()["gather_every"]
    launches = sim.launches_per_step() * args.chunk * args.steps + (args.chunk * args.steps) // gather_every

    line = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if args.precision == "mixed" else "f64",
        "data": "synthetic",
        "config": {"workload": sc.name, "particles_per_gpu": sc.n, "precision": args.precision,
                   "dem_steps_per_step": args.chunk, "dt": sc.dt,
                   "parallelism": "replicas" if world > 1 else "1gpu",
                   "l2": "flushed (256 MiB write) between timed steps"},
        "gpu_launches": int(launches),
        "roofline": roofline(prof_tot, sc, args.precision, z, peak, peak_kind,
                             lambda k: profiled_traffic(k, sc.name, args.precision)),
        "e2e": {"value": e2e_value, "unit": "particle-steps/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "host_buffers": "pinned", "over_device": e2e_value / value},
        "kernels_ms_per_dem_step": {k: v[0] / n_prof for k, v in prof_tot.items()},
        "kernel_timing": "uncaptured re-run of the timed window with CUDA events around each phase",
        "status": st["status"],
        "clocks": clk.summary(),
    }
    if prec == MIXED and not args.no_fp64:
        # the plain FP64 path on the same run, and the mixed-precision contact
        # force error against it on identical states (the end of the run)
        sim64, _, _, ms64, _ = timed_run(FP64, False)
        if world > 1:
            tt = torch.tensor([ms64], device="cuda:%d" % local, dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms64 = float(tt.item())
        sim64.close()
        v64 = total_particles * args.chunk * args.steps / (ms64 / 1e3)
        line["fp64"] = {"value": v64, "unit": "particle-steps/s", "ms_per_step": ms64 / args.steps,
                        "mixed_over_fp64": value / v64}
        line["contact_force_error"] = contact_force_error(lib, sc, st_end, mem_end, local, "end of the timed run")
    if args.settle_steps is None:
        args.settle_steps = {"polydisperse_200k": 70000, "drum_100k": 100000}.get(sc.name, 0)
    if world == 1 and prec == MIXED and args.settle_steps > 0 and not args.no_fp64:
        line["settled"] = settled_leg(args, lib, sc, local, flush, peak, peak_kind)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"], cpu_sim = cpu_baseline(scenario(args.workload), args.cpu_steps, keep=True)
        cpu = (cpu_sim, line["cpu_baseline"]["kind"])
    if rank == 0 and not args.no_io:
        line["io"] = io_measure(lib, sim, t, cpu)
    if cpu is not None:
        cpu[0].close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    sim.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
