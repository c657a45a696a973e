"""Benchmark: ESP particle-steps/s on the mixed batch of 256 rock-salt systems.

One step = one request round for every system of the batch: neighbour
list build (cell list, r_list = r_c + 0.4), one evaluation, then 10
velocity-Verlet NVE steps at dt = 0.002, each with a full ESP evaluation
(mesh + pair), the 10 steps replayed from a CUDA graph. A step therefore
advances sum(N) particles by 10 MD steps (particle-steps = 10 sum N).

Reported beside the batched number: the plain path (the same systems, one
system per launch sequence), the end-to-end number through the C ABI with
pinned host buffers copied in and results copied out every step (on a
copy stream, overlapping the neighbouring steps' compute), the
roofline of the dominant kernel (CUDA events on the launching stream), the
CPU baseline (the FP64 oracle port on the host cores), and the served
stream: Poisson arrivals of mixed rock-salt / water requests through the
continuous-batching server at several rates, with p50/p99 latency and
throughput per rate.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                       [--no-serve] [--serve-requests R] [--serve-rates a,b,c]
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s at <=1e-5 rel RMS force err, batched vs plain; p50/p99 latency"
UNIT = "particle-steps/s"
N_SYS = 256
SEED = 1004
RCUT = 3.0
SKIN = 0.4
CAP = 256
DT = 0.002
MD_STEPS = 10
# kernels per launch group (used to count launches in the timed region)
# bin, scan, scatter, tile_sort, spread, interp, pair, add_forces (the pair
# term runs on a second stream into its own array), finalize; plus the FFT
# passes: 3 whole-plane/slab kernels (fft_mode 0) or 5 per-line kernels
K_EVAL_BASE = 9
K_FFT = {0: 3, 1: 5}
K_NLIST = 5      # cell_bin, scan, scatter, cell_sort, nlist
K_NVE = 2


def _env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def max_over_ranks(ms: float, world: int, device=None) -> float:
    """The slowest rank's time: every rank calls this with its own device-timed
    milliseconds (an all-reduce MAX; ranks run independent replicas, so this is
    the only collective of the data path)."""
    if world <= 1:
        return float(ms)
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _systems(rank: int, count: int = N_SYS):
    """The first `count` systems of the rank's 256-system batch."""
    from esp_hoomd_b200 import systems
    rng = np.random.default_rng(SEED + 7919 * rank)
    evens = np.arange(8, 41, 2)
    ns = rng.choice(evens, size=N_SYS)[:count]
    return [systems.rocksalt(int(n), seed=SEED * 100000 + rank * N_SYS + i) for i, n in enumerate(ns)]


def _smooth235(n: int) -> int:
    """Smallest 2/3/5-smooth integer >= n."""
    m = max(int(n), 1)
    while True:
        k = m
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1:
            return m
        m += 1


def workload_config(count: int, world: int) -> dict:
    """The workload's description, the same in both arms: rank 0's batch
    (the first `count` systems), its particle and mesh-point totals from the
    mesh rule (h = pi r_c / 18.5 for the 1e-5 target)."""
    rng = np.random.default_rng(SEED)
    ns = [int(n) for n in rng.choice(np.arange(8, 41, 2), size=N_SYS)[:count]]
    h = math.pi * RCUT / 18.5
    M = sum(_smooth235(max(8, math.ceil(n / h))) ** 3 for n in ns)
    return {"workload": "batched%d: %d rock-salt systems n^3, n even ~U{8..40} (seed %d), 1 nlist + 1 eval + "
                        "10 NVE steps per system per step" % (count, count, SEED),
            "systems_per_gpu": count, "particles_per_gpu": sum(n ** 3 for n in ns), "order": 8, "rcut": RCUT,
            "skin": SKIN, "mesh_rule": "smallest 2/3/5-smooth >= L/h, h = pi r_c / 18.5 (1e-5 target)",
            "mesh_points_per_gpu": int(M), "dt": DT,
            "l2": "inputs larger than L2 (neighbour rows: 4 B x ~164 entries per particle)",
            "parallelism": "replicas over systems (dp%d)" % world}


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def _peak_gbs():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def _traffic_from_profiles(kernel: str):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.txt")
    try:
        with open(p) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 2 and parts[0] == kernel:
                    return float(parts[1])
    except OSError:
        pass
    return None


# ----------------------------------------------------------------------------- CPU baseline
def cpu_sample(count: int, rank: int = 0):
    """The first `count` systems of the rank's batch (the same systems the
    GPU step runs), with the C oracle's parameters (same mesh rule)."""
    from oracle import esp_port as EP
    sl = _systems(rank, min(count, N_SYS))
    return sl, EP.plan(sl, RCUT)


def cpu_baseline(sl, prm, threads: int, cache=None):
    """One GPU-step's work on the CPU: for every system of the sample a
    neighbour list, one evaluation and 10 NVE steps, FP64, in the compiled
    restatement of the pipeline (oracle/esp_oracle.c), one system per
    OpenMP thread. Returns (particle-steps, seconds)."""
    from oracle import esp_port as EP
    t0 = time.perf_counter()
    EP.run_batch(sl, prm, RCUT + SKIN, MD_STEPS, DT, threads=threads, influence_cache=cache)
    return MD_STEPS * sum(s.N for s in sl), time.perf_counter() - t0


def run_reference(args):
    """The reference's CPU path is stubs (src/ESPForceCompute.cc:236-248) and
    the plugin cannot be built without HOOMD; this arm times the FP64 C
    restatement of the same path on all host threads, each step one bounded
    sample of the batched workload."""
    from oracle import esp_port as EP
    rank, world, _ = _env_rank()
    if rank != 0:
        return
    threads = EP.max_threads()
    sl, prm = cpu_sample(max(4, 2 * threads))
    cache = EP.influence_tables(prm)  # built outside the timed steps
    for _ in range(args.warmup):
        cpu_baseline(sl[:1], prm[:1], threads, cache)
    times, n_ps = [], 0
    for _ in range(args.steps):
        n_ps, wall = cpu_baseline(sl, prm, threads, cache)
        times.append(wall)
    t = sum(times) / len(times)
    value = n_ps / t
    sample = ("FP64 C restatement (oracle/esp_oracle.c): nlist + 1 evaluation + 10 NVE steps of the first %d "
              "systems of the batched256 workload (%d particles) per step, %d OpenMP threads"
              % (len(sl), sum(s.N for s in sl), threads))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args.systems, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- checker and comparison legs
def accuracy_leg(b, sl, pos_h, q, nlist, dev):
    """The metric's accuracy bar, measured on the timed workload: one
    evaluation of the timed plan (same Batch, same shared split) at the
    batch's initial positions, and the forces and energies of its smallest,
    a middle (n = 24) and its largest member against FP64 Ewald (the
    oracle's workload-size sum, run as the checker after the timed regions)."""
    import torch
    from oracle.ewald_torch import ewald_torch
    tot = pos_h.shape[0]
    pos = torch.tensor(pos_h, device=dev)
    if nlist is not None:
        b.build_nlist(pos, RCUT + SKIN, CAP, *nlist)
    else:
        b.build_pairlist(pos, RCUT + SKIN, CAP)
    force = torch.zeros((tot, 4), device=dev)
    energy = torch.zeros(len(sl), dtype=torch.float64, device=dev)
    b.compute(pos, q, force, energy, None, nlist=nlist)
    torch.cuda.synchronize(dev)
    f = force.double().cpu().numpy()
    e = energy.cpu().numpy()
    ns = [round(s.N ** (1.0 / 3.0)) for s in sl]
    off = np.concatenate([[0], np.cumsum([s.N for s in sl])])
    picks = sorted({ns.index(min(ns)), ns.index(max(ns))} | ({ns.index(24)} if 24 in ns else set()))
    rows = []
    for i in picks:
        p = pos_h[off[i]:off[i + 1], :3].astype(np.float64)
        E0, F0, _ = ewald_torch(p, sl[i].q, sl[i].box, device=dev)
        fi = f[off[i]:off[i + 1], :3]
        rows.append({"system": int(i), "n": int(ns[i]), "N": int(sl[i].N),
                     "mesh": b.info(i)["nx"], "force_rel_rms": float(np.sqrt(((fi - F0) ** 2).sum() / (F0 ** 2).sum())),
                     "energy_rel": float(abs(e[i] - E0) / abs(E0))})
    return {"reference": "FP64 Ewald (oracle/ewald_torch.py, truncation ~1e-11), same positions",
            "split_c": b.info(0)["c_split"], "systems": rows,
            "force_rel_rms": max(r["force_rel_rms"] for r in rows),
            "energy_rel": max(r["energy_rel"] for r in rows)}


def cufft_leg(b, nsys, dev, reps=5):
    """cuFFT (through torch.fft) on the batch's meshes, timed only as a
    comparison with the hand-written passes: per mesh size class one batched
    R2C, the influence multiply, one batched C2R -- the FFT stage's work."""
    import torch
    from collections import Counter
    sizes = Counter((b.info(i)["nx"], b.info(i)["ny"], b.info(i)["nz"]) for i in range(nsys))
    bufs = []
    for (nx, ny, nz), c in sorted(sizes.items()):
        x = torch.randn((c, nz, ny, nx), device=dev)
        g = torch.rand((nz, ny, nx // 2 + 1), device=dev)
        bufs.append((x, g, (nz, ny, nx)))

    def run():
        for x, g, s in bufs:
            y = torch.fft.rfftn(x, dim=(1, 2, 3))
            y *= g
            torch.fft.irfftn(y, s=s, dim=(1, 2, 3), out=x)

    for _ in range(3):
        run()
    torch.cuda.synchronize(dev)
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st.record()
    for _ in range(reps):
        run()
    en.record()
    torch.cuda.synchronize(dev)
    return {"cufft_ms": st.elapsed_time(en) / reps, "size_classes": len(bufs),
            "desc": "torch.fft (cuFFT) batched rfftn + multiply + irfftn per mesh size class, FP32"}


# ----------------------------------------------------------------------------- serving
SERVE_BUDGET = 64 << 30
SERVE_STEPS = 10


def _serve_pool(seed: int):
    """Request templates: every rock-salt size n = 8, 10, ..., 64 (r_c 3.0,
    skin 0.4) and 16 water boxes of 1,000-32,768 molecules (r_c 0.9 nm, skin
    0.1), as page-locked host inputs."""
    import torch
    from esp_hoomd_b200 import systems
    rng = np.random.default_rng(seed)
    pool = {"rocksalt": [], "water": []}

    def pinned(s):
        p4 = np.zeros((s.N, 4), np.float32)
        p4[:, :3] = s.pos
        v4 = np.zeros((s.N, 4), np.float32)
        v4[:, :3] = s.vel
        v4[:, 3] = s.mass
        t = [torch.from_numpy(a).pin_memory() for a in (p4, v4, s.q.astype(np.float32))]
        out = torch.empty((s.N, 4), dtype=torch.float32).pin_memory()
        return {"N": s.N, "box": s.box, "pos4": t[0], "vel4": t[1], "q": t[2], "out_pos4": out}

    for n in range(8, 65, 2):
        d = pinned(systems.rocksalt(n, seed=int(rng.integers(1 << 30))))
        d.update(rcut=3.0, skin=0.4)
        pool["rocksalt"].append(d)
    for m in np.sort(rng.integers(1000, 32769, size=16)):
        d = pinned(systems.water(int(m), seed=int(rng.integers(1 << 30))))
        # rigid three-site molecules (SETTLE / RATTLE in the NVE steps)
        d.update(rcut=0.9, skin=0.1, rigid=(0.1, 2 * 0.1 * math.sin(math.radians(109.47 / 2))))
        pool["water"].append(d)
    return pool


def run_serving(args, pool):
    """Poisson streams of requests (50/50 rock-salt / water, each one
    neighbour list + 1 evaluation + 10 NVE steps) through the server at
    several arrival rates; latency = completion - arrival per request."""
    import torch
    from esp_hoomd_b200 import native
    srv = native.Server(native.make_params(order=8, target_error=1e-5), hbm_budget=SERVE_BUDGET,
                        max_systems=1024, max_particles=262144)
    rng = np.random.default_rng(SEED + 5)
    n_warm = len(pool["rocksalt"]) + len(pool["water"])
    energies = torch.zeros(n_warm + args.serve_requests * len(args.serve_rates), dtype=torch.float64).pin_memory()
    slot = [0]

    def submit(d, arrival):
        i = slot[0]
        slot[0] += 1
        return srv.submit(d["pos4"], d["q"], d["box"], d["rcut"], vel4=d["vel4"], nsteps=SERVE_STEPS, dt=DT,
                          skin=d["skin"], arrival=arrival, out_pos4=d["out_pos4"], out_energy=energies[i:i + 1],
                          rigid_water=d.get("rigid"))

    # warm-up: every template once (kernels, parameter sets, influence tables)
    warm = [submit(d, 0.0) for kind in ("rocksalt", "water") for d in pool[kind]]
    srv.start()
    srv.wait_all(600)
    base = max(srv.status(i)["t_done"] for i in warm) + 0.05
    out = []
    for rate in args.serve_rates:
        # rate 0: every request arrives at once (a saturating burst: the
        # server's own throughput, the queue never empties)
        gaps = rng.exponential(1.0 / rate, size=args.serve_requests) if rate > 0 else np.zeros(args.serve_requests)
        arr = base + np.cumsum(gaps)
        kinds = rng.random(args.serve_requests) < 0.5
        ids, nsum = [], 0
        for a, is_rs in zip(arr, kinds):
            tmpl = pool["rocksalt" if is_rs else "water"]
            d = tmpl[int(rng.integers(len(tmpl)))]
            nsum += d["N"]
            ids.append(submit(d, float(a)))
        srv.wait_all(1800)
        st = [srv.status(i) for i in ids]
        ok = [s for s in st if s["state"] == 2]
        lat = np.array([s["t_done"] - s["t_arrival"] for s in ok]) * 1e3
        span = max(s["t_done"] for s in ok) - arr[0]
        out.append({"rate_per_s": rate if rate > 0 else "burst", "requests": len(ids), "completed": len(ok),
                    "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                    "mean_ms": float(lat.mean()), "throughput": nsum * SERVE_STEPS / span,
                    "requests_per_s": len(ok) / span})
        base = max(s["t_done"] for s in ok) + 0.05
    stats = srv.stats()
    srv.close()
    return out, stats


# ----------------------------------------------------------------------------- scale-up
def run_c1(args):
    """The CPU-runnable plain case, timed: N = 1,000 rock-salt ions (10^3
    lattice, L = 10, seed 1000), mesh 32^3, support 8, r_c 3.0, FP64 mode,
    Lennard-Jones core repulsion (eps 1, sigma 0.9, r_cut 2.5); a step = one
    evaluation + 100 NVE steps at dt 0.002 with the neighbour list (r_c + 0.4)
    rebuilt every 10 steps (10 steps per esp_batch_md_run_f64 call, replayed
    from a captured graph). One small system: launch-bound by nature."""
    import torch
    from esp_hoomd_b200 import native, systems
    dev = torch.device("cuda", 0)
    s = systems.rocksalt(10, seed=1000)
    N = s.N
    b = native.Batch(native.make_params(order=8, rcut=RCUT, mesh=(32, 32, 32), precision=1), [N], [s.box])
    b32 = native.Batch(native.make_params(order=8, rcut=RCUT, mesh=(32, 32, 32)), [N], [s.box])  # list builder
    p4 = np.zeros((N, 4))
    p4[:, :3] = s.pos
    v4 = np.zeros((N, 4))
    v4[:, :3] = s.vel
    v4[:, 3] = 1.0
    pos0 = torch.tensor(p4, dtype=torch.float64, device=dev)
    vel0 = torch.tensor(v4, dtype=torch.float64, device=dev)
    pos, vel = pos0.clone(), vel0.clone()
    q = torch.tensor(s.q, dtype=torch.float64, device=dev)
    force = torch.zeros((N, 4), dtype=torch.float64, device=dev)
    e_esp = torch.zeros(1, dtype=torch.float64, device=dev)
    e_lj = torch.zeros(1, dtype=torch.float64, device=dev)
    head = torch.zeros(N, dtype=torch.int32, device=dev)
    nn = torch.zeros_like(head)
    nl = torch.zeros(N * CAP, dtype=torch.int32, device=dev)
    nlist = (head, nn, nl)

    def evaluate():
        e_lj.zero_()
        b.compute_f64(pos, q, force, e_esp, nlist=nlist)
        b.lj(pos, nlist, 1.0, 0.9, 2.5, force, e_lj)

    def step():
        pos.copy_(pos0)
        vel.copy_(vel0)
        b32.build_nlist(pos.float(), RCUT + SKIN, CAP, head, nn, nl)
        evaluate()
        e_esp.add_(e_lj)  # md_run_f64 carries ESP + LJ in one energy
        for k in range(10):
            if k:
                b32.build_nlist(pos.float(), RCUT + SKIN, CAP, head, nn, nl)
            # 10 velocity-Verlet steps (ESP + LJ) replayed from a captured graph
            b.md_run_f64(pos, vel, q, force, e_esp, None, nlist, 10, DT, lj=(1.0, 0.9, 2.5))

    for _ in range(max(3, args.warmup)):
        step()
    b32.nlist_check()
    torch.cuda.synchronize()
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(0) as clk:
        st.record()
        for _ in range(args.steps):
            step()
        en.record()
        torch.cuda.synchronize()
    ms = st.elapsed_time(en) / args.steps
    line = {"metric": "particle-steps/s (C1: FP64 ESP + LJ, N = 1,000, 100 NVE steps per step)",
            "value": N * 100 / (ms * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "c1: rock-salt 10^3 (N = 1,000), L = 10, seed 1000, mesh 32^3, order 8, r_c 3.0, "
                                   "LJ eps 1 sigma 0.9 r_cut 2.5, 1 eval + 100 NVE steps (dt 0.002), list r_c + 0.4 "
                                   "rebuilt every 10 steps"},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def water_rows(spec: str) -> set:
    """--water-rows "1e-5:f64,1e-3:f32" -> {(1e-5, "f64"), (1e-3, "f32")}; "" -> all rows."""
    out = set()
    for r in spec.split(","):
        if not r.strip():
            continue
        t, p = r.split(":")
        if p not in ("f32", "f64"):
            raise ValueError("water row precision must be f32 or f64: " + r)
        out.add((float(t), p))
    return out


def run_water(args):
    """The water-like accuracy sweep (32,768 rigid three-site molecules,
    98,304 charges, no exclusions, r_c 0.9 nm): for each target (1e-3, 1e-5,
    1e-7 with supports 6, 8, 10) the planner's mesh, one evaluation timed
    in FP32 (library pair list) and in FP64 (list from the FP32 builder),
    and its force and energy error against FP64 Ewald (oracle/ewald_torch.py
    as the checker, outside the timed region). A step = one evaluation."""
    import torch
    from esp_hoomd_b200 import native, systems
    from esp_hoomd_b200._lib import ESP_ALL
    from oracle.ewald_torch import ewald_torch
    dev = torch.device("cuda", 0)
    w = systems.water(32768, seed=1003)
    N = w.N
    posd = w.pos.astype(np.float32).astype(np.float64)
    E0, F0, _ = ewald_torch(posd, w.q, w.box, device=dev)
    p4 = np.zeros((N, 4))
    p4[:, :3] = posd
    rows = []
    only = water_rows(args.water_rows)
    for target, order in ((1e-3, 6), (1e-5, 8), (1e-7, 10)):
        for prec in (0, 1):
            if only and (target, ("f32", "f64")[prec]) not in only:
                continue
            params = native.make_params(order=order, rcut=0.9, target_error=target, precision=prec)
            b = native.Batch(params, [N], [w.box])
            if prec == 0:
                pos = torch.tensor(p4, dtype=torch.float32, device=dev)
                q = torch.tensor(w.q.astype(np.float32), device=dev)
                force = torch.zeros((N, 4), device=dev)
                b.build_pairlist(pos, 0.9, 1024)

                def ev():
                    b.compute(pos, q, force, energy, None, nlist=None, flags=ESP_ALL)
            else:
                b32 = native.Batch(native.make_params(order=order, rcut=0.9, target_error=target), [N], [w.box])
                pos = torch.tensor(p4, dtype=torch.float64, device=dev)
                q = torch.tensor(w.q, dtype=torch.float64, device=dev)
                force = torch.zeros((N, 4), dtype=torch.float64, device=dev)
                head = torch.zeros(N, dtype=torch.int32, device=dev)
                nn = torch.zeros_like(head)
                nl = torch.zeros(N * 1024, dtype=torch.int32, device=dev)
                b32.build_nlist(pos.float(), 0.9, 1024, head, nn, nl)
                b32.nlist_check()

                def ev():
                    b.compute_f64(pos, q, force, energy, None, nlist=(head, nn, nl))
            energy = torch.zeros(1, dtype=torch.float64, device=dev)
            # warm-up: at least W evaluations and half a second (clocks settle)
            t0, k = time.perf_counter(), 0
            while k < max(3, args.warmup) or time.perf_counter() - t0 < 0.5:
                ev()
                torch.cuda.synchronize()
                k += 1
            st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            st.record()
            for _ in range(args.steps):
                ev()
            en.record()
            torch.cuda.synchronize()
            ms = st.elapsed_time(en) / args.steps
            stages = None
            if prec == 0:
                # per-stage times of two more evaluations (stage timer; the pair term not forked)
                b.set_timing(True)
                for _ in range(2):
                    ev()
                stages = {k: v[0] / v[1] for k, v in b.stage_times().items() if v[1] > 0}
                b.set_timing(False)
            f = force.double().cpu().numpy()[:, :3]
            err = float(np.sqrt(((f - F0) ** 2).sum() / (F0 ** 2).sum()))
            inf = b.info(0)
            rows.append({"target": target, "order": order, "precision": "f64" if prec else "f32",
                         "mesh": [inf["nx"], inf["ny"], inf["nz"]], "ms_per_eval": ms,
                         "particle_evals_per_s": N / (ms * 1e-3), "force_rel_rms": err,
                         "energy_rel": abs(energy.item() - E0) / abs(E0), "stage_ms": stages})
            del b
    head_row = next((r for r in rows if r["target"] == 1e-5 and r["precision"] == "f32"), rows[0])
    line = {"metric": "particle-evals/s and error vs FP64 Ewald (C3: water accuracy sweep)",
            "value": head_row["particle_evals_per_s"], "unit": "particle-evals/s", "n_gpus": 1, "steps": args.steps,
            "warmup": max(3, args.warmup), "higher_is_better": True, "dtype": head_row["precision"],
            "data": "synthetic",
            "config": {"workload": "c3: 32,768 rigid three-site molecules (98,304 charges), seed 1003, r_c 0.9 nm, "
                                   "no exclusions; value = the 1e-5 FP32 row (else the first row run)"},
            "rows": rows}
    print(json.dumps(line), flush=True)


def run_scaleup(args):
    """The plain one-system path at the scale-up size: 10^6 rock-salt ions
    (100^3 lattice, L = 100, mesh 200^3, support 8, r_c 3.0, 1e-5 target).
    A step = neighbour list + one evaluation + 10 NVE steps (CUDA graph), as
    in the batched workload. Reports every stage's live CUDA-event time and
    its fraction of the measured HBM peak for its algorithmic bytes."""
    import torch
    from esp_hoomd_b200 import native, systems
    from esp_hoomd_b200._lib import ESP_ALL
    dev = torch.device("cuda", 0)
    s = systems.rocksalt(100, seed=1001)
    N = s.N
    b = native.Batch(native.make_params(order=8, rcut=RCUT, target_error=1e-5), [N], [s.box])
    p4 = np.zeros((N, 4), np.float32)
    p4[:, :3] = s.pos
    v4 = np.zeros((N, 4), np.float32)
    v4[:, :3] = s.vel
    v4[:, 3] = 1.0
    pos = torch.tensor(p4, device=dev)
    vel = torch.tensor(v4, device=dev)
    q = torch.tensor(s.q.astype(np.float32), device=dev)
    head = torch.zeros(N, dtype=torch.int32, device=dev)
    nn = torch.zeros_like(head)
    nl = torch.zeros(N * CAP, dtype=torch.int32, device=dev)
    force = torch.zeros((N, 4), device=dev)
    energy = torch.zeros(1, dtype=torch.float64, device=dev)
    virial = torch.zeros(6, dtype=torch.float64, device=dev)

    def request(use_graph=True):
        if args.hoomd_list:
            b.build_nlist(pos, RCUT + SKIN, CAP, head, nn, nl)
            nlist = (head, nn, nl)
        else:
            b.build_pairlist(pos, RCUT + SKIN, CAP)
            nlist = None
        b.compute(pos, q, force, energy, virial, nlist=nlist, flags=ESP_ALL)
        b.md_run(pos, vel, q, force, energy, None, nlist, MD_STEPS, DT, use_graph=use_graph)

    for _ in range(max(3, args.warmup)):
        request()
    torch.cuda.synchronize()
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(0) as clk:
        st.record()
        for _ in range(args.steps):
            request()
        en.record()
        torch.cuda.synchronize()
    ms = st.elapsed_time(en) / args.steps
    b.set_timing(True)
    for _ in range(2):
        request(use_graph=False)
    stt = b.stage_times()
    b.set_timing(False)
    inf = b.info(0)
    M = inf["nx"] * inf["ny"] * inf["nz"]
    if not args.hoomd_list:
        b.pairlist_check()
        b.build_nlist(pos, RCUT + SKIN, CAP, head, nn, nl)  # neighbour counts for the byte model
    mean_nn = float(nn.double().mean().item())
    # single evaluations in both precisions (the configuration's FP64 and FP32
    # modes), same mesh and target: FP32 over the library's pair list, FP64
    # over the HOOMD-layout list just built
    def eval_ms(fn, reps=5):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    b.build_pairlist(pos, RCUT + SKIN, CAP)
    f32_ms = eval_ms(lambda: b.compute(pos, q, force, energy, virial, nlist=None, flags=ESP_ALL))
    b64 = native.Batch(native.make_params(order=8, rcut=RCUT, target_error=1e-5, precision=1), [N], [s.box])
    pos64 = pos.double()
    q64 = q.double()
    force64 = torch.zeros((N, 4), dtype=torch.float64, device=dev)
    f64_ms = eval_ms(lambda: b64.compute_f64(pos64, q64, force64, energy, virial, nlist=(head, nn, nl)))
    del b64, pos64, q64, force64
    alg = {"pair": 4.0 * N * mean_nn + 32.0 * N, "spread": 20.0 * N + 4.0 * M, "interp": 36.0 * N + 4.0 * M,
           "fft": 5 * 2 * 8.0 * M / 2, "sort": 40.0 * N, "bin": 40.0 * N, "nlist": 16.0 * N + 4.0 * N * mean_nn,
           "nve": 48.0 * N}
    peak, peak_kind = _peak_gbs()
    stages = {}
    for k, (tot_ms, cnt) in stt.items():
        if cnt == 0:
            continue
        t = tot_ms / cnt
        gbs = alg[k] / (t * 1e-3) / 1e9
        stages[k] = {"ms_per_launch": t, "algorithmic_bytes": alg[k], "achieved_gbs": gbs, "frac_hbm": gbs / peak}
    line = {"metric": "particle-steps/s (plain path, one 10^6-particle system)", "value": N * MD_STEPS / (ms * 1e-3),
            "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "scaleup: rock-salt 100^3 (N = 1,000,000), L = 100, seed 1001, "
                                   "1 nlist + 1 eval + 10 NVE steps per step",
                       "mesh": [inf["nx"], inf["ny"], inf["nz"]], "order": 8, "rcut": RCUT,
                       "mean_neighbours": mean_nn},
            "peak_gbs": peak, "peak_kind": peak_kind, "stages": stages, "clocks": clk.summary(),
            "single_eval_ms": {"f32": f32_ms, "f64": f64_ms}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- GPU arm
def run_ours(args):
    import torch
    import torch.distributed as dist
    from esp_hoomd_b200 import native
    from esp_hoomd_b200._lib import ESP_ALL

    rank, world, local = _env_rank()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", rank=rank, world_size=world,
                                timeout=__import__("datetime").timedelta(seconds=600))
    sl = _systems(rank, args.systems)
    N = np.array([s.N for s in sl])
    tot = int(N.sum())
    params = native.make_params(order=8, rcut=RCUT, target_error=1e-5)
    b = native.Batch(params, N, [s.box for s in sl])
    pos_h = np.zeros((tot, 4), np.float32)
    pos_h[:, :3] = np.concatenate([s.pos for s in sl])
    vel_h = np.zeros((tot, 4), np.float32)
    vel_h[:, :3] = np.concatenate([s.vel for s in sl])
    vel_h[:, 3] = 1.0
    q_h = np.concatenate([s.q for s in sl]).astype(np.float32)
    pos0 = torch.tensor(pos_h, device=dev)
    vel0 = torch.tensor(vel_h, device=dev)
    q = torch.tensor(q_h, device=dev)
    pos = pos0.clone()
    vel = vel0.clone()
    head = torch.zeros(tot, dtype=torch.int32, device=dev)
    nn = torch.zeros_like(head)
    nl = torch.zeros(tot * CAP, dtype=torch.int32, device=dev)
    force = torch.zeros((tot, 4), dtype=torch.float32, device=dev)
    energy = torch.zeros(N.size, dtype=torch.float64, device=dev)
    virial = torch.zeros(6 * N.size, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def request(bb, p, v, use_graph=True, qq=q, e=energy):
        # the first evaluation reports energy and virial; the NVE steps need
        # forces and energies only. Default: the library's pair list (rows in
        # cell order); --hoomd-list: HOOMD-layout rows built by the harness
        if args.hoomd_list:
            bb.build_nlist(p, RCUT + SKIN, CAP, head, nn, nl)
            nlist = (head, nn, nl)
        else:
            bb.build_pairlist(p, RCUT + SKIN, CAP)
            nlist = None
        bb.compute(p, qq, force, e, virial, nlist=nlist, flags=ESP_ALL)
        bb.md_run(p, v, qq, force, e, None, nlist, MD_STEPS, DT, use_graph=use_graph)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    tuned = None
    if not args.no_tune:
        # the autotuner picks pair lanes (HOOMD-list kernel), tile edge and FFT pass form on this batch
        if args.hoomd_list:
            b.build_nlist(pos, RCUT + SKIN, CAP, head, nn, nl)
            tuned = b.autotune(pos, q, nlist=(head, nn, nl), reps=2)
        else:
            b.build_pairlist(pos, RCUT + SKIN, CAP)
            tuned = b.autotune(pos, q, nlist=None, reps=2)
        pos.copy_(pos0)
    for _ in range(max(3, args.warmup)):
        request(b, pos, vel)
    barrier()
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        st.record(stream)
        for _ in range(args.steps):
            request(b, pos, vel)
        en.record(stream)
        barrier()
    ms = st.elapsed_time(en) / args.steps
    ms_max = max_over_ranks(ms, world, dev)
    value = world * tot * MD_STEPS / (ms_max * 1e-3)

    # -- stage timing (live CUDA events on the launching stream, same workload, no graph)
    b.set_timing(True)
    for _ in range(2):
        request(b, pos, vel, use_graph=False)
    stt = b.stage_times()
    b.set_timing(False)
    stage_ms = {k: v[0] / max(v[1], 1) for k, v in stt.items() if v[1] > 0}
    stage_total = {k: v[0] for k, v in stt.items() if v[1] > 0}
    dom = max(stage_total, key=stage_total.get)
    if not args.hoomd_list:
        b.pairlist_check()  # no row of the timed steps overflowed
        b.build_nlist(pos, RCUT + SKIN, CAP, head, nn, nl)  # neighbour counts for the byte model
    mean_nn = float(nn.double().mean().item())
    M = sum(b.info(i)["nx"] * b.info(i)["ny"] * b.info(i)["nz"] for i in range(N.size))
    # algorithmic bytes per launch of each stage (FP32 storage)
    # pair: index stream (4 B per entry) + positions in + forces out
    alg = {"pair": 4.0 * tot * mean_nn + 16.0 * tot + 16.0 * tot,
           "spread": 20.0 * tot + 4.0 * M,
           "interp": 20.0 * tot + 4.0 * M + 16.0 * tot,
           "fft": 5 * 2 * 8.0 * M / 2,
           "sort": 40.0 * tot,
           "bin": 40.0 * tot,
           "nlist": 16.0 * tot + 4.0 * tot * mean_nn,
           "nve": 48.0 * tot}
    kname = {"pair": "k_pair", "spread": "k_spread", "interp": "k_interp", "fft": "k_fft", "nlist": "k_nlist",
             "sort": "k_tile_sort", "bin": "k_bin", "nve": "k_nve"}
    peak, peak_kind = _peak_gbs()
    ach = alg[dom] / (stage_ms[dom] * 1e-3) / 1e9
    roof = {"kernel": kname.get(dom, dom), "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
            "frac": ach / peak, "peak_kind": peak_kind, "traffic": _traffic_from_profiles(kname.get(dom, dom)),
            "stage_ms_per_launch": stage_ms,
            "algorithmic_bytes_per_launch": alg[dom]}

    # -- plain path: one system per launch sequence (separate contexts, no graph)
    plain_value = None
    if rank == 0 and not args.no_plain:
        ctxs = [native.Batch(params, [int(n)], [s.box]) for n, s in zip(N, sl)]
        offs = np.concatenate([[0], np.cumsum(N)])
        pos_p = pos0.clone()
        vel_p = vel0.clone()
        views = [(pos_p[offs[i]:offs[i + 1]], vel_p[offs[i]:offs[i + 1]], q[offs[i]:offs[i + 1]],
                  head[offs[i]:offs[i + 1]], nn[offs[i]:offs[i + 1]], nl[offs[i] * CAP:offs[i + 1] * CAP],
                  force[offs[i]:offs[i + 1]], energy[i:i + 1], virial[6 * i:6 * i + 6]) for i in range(N.size)]

        def plain_round():
            for c, (p, v, qq, h, n_, l_, f, e, w) in zip(ctxs, views):
                if args.hoomd_list:
                    c.build_nlist(p, RCUT + SKIN, CAP, h, n_, l_)
                    nlist = (h, n_, l_)
                else:
                    c.build_pairlist(p, RCUT + SKIN, CAP)
                    nlist = None
                c.compute(p, qq, f, e, w, nlist=nlist, flags=ESP_ALL)
                c.md_run(p, v, qq, f, e, None, nlist, MD_STEPS, DT, use_graph=False)

        plain_round()
        torch.cuda.synchronize(dev)
        st.record(stream)
        for _ in range(args.plain_steps):
            plain_round()
        en.record(stream)
        torch.cuda.synchronize(dev)
        plain_ms = st.elapsed_time(en) / args.plain_steps
        plain_value = tot * MD_STEPS / (plain_ms * 1e-3)
        del ctxs

    # -- end to end through the public API with host buffers
    pin_pos = torch.from_numpy(pos_h).pin_memory()
    pin_vel = torch.from_numpy(vel_h).pin_memory()
    pin_q = torch.from_numpy(q_h).pin_memory()
    out_pos = torch.empty_like(pin_pos).pin_memory()
    out_vel = torch.empty_like(pin_vel).pin_memory()
    out_e = torch.empty(N.size, dtype=torch.float64).pin_memory()
    h2d = pin_pos.numel() * 4 + pin_vel.numel() * 4 + pin_q.numel() * 4
    d2h = out_pos.numel() * 4 + out_vel.numel() * 4 + out_e.numel() * 8

    # two device buffer sets: step k+1's uploads and step k-1's downloads run
    # on a copy stream while step k computes (the neighbour list and force
    # scratch are shared; the compute stream orders their reuse)
    sets = [(pos, vel, q, energy),
            (torch.empty_like(pos), torch.empty_like(vel), torch.empty_like(q), torch.empty_like(energy))]
    copy = torch.cuda.Stream(dev)

    def upload(k):
        p, v, qq, _ = sets[k % 2]
        with torch.cuda.stream(copy):
            p.copy_(pin_pos, non_blocking=True)
            v.copy_(pin_vel, non_blocking=True)
            qq.copy_(pin_q, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(copy)
        return ev

    def e2e_run(n):
        copy.wait_stream(stream)
        up = {0: upload(0)}
        for k in range(n):
            p, v, qq, e = sets[k % 2]
            if k + 1 < n:
                up[k + 1] = upload(k + 1)
            stream.wait_event(up.pop(k))
            request(b, p, v, qq=qq, e=e)
            done = torch.cuda.Event()
            done.record(stream)
            copy.wait_event(done)
            with torch.cuda.stream(copy):
                out_pos.copy_(p, non_blocking=True)
                out_vel.copy_(v, non_blocking=True)
                out_e.copy_(e, non_blocking=True)
        stream.wait_stream(copy)

    e2e_run(2)
    barrier()
    st.record(stream)
    e2e_run(args.steps)
    en.record(stream)
    barrier()
    e2e_ms = max_over_ranks(st.elapsed_time(en) / args.steps, world, dev)
    e2e_value = world * tot * MD_STEPS / (e2e_ms * 1e-3)

    k_eval = K_EVAL_BASE + K_FFT[tuned["fft_mode"] if tuned else 0]
    if rank == 0:
        cores = os.cpu_count() or 1
        cfg = workload_config(int(N.size), world)
        if cfg["particles_per_gpu"] != tot or cfg["mesh_points_per_gpu"] != int(M):
            cfg["note"] = "the planned batch differs from this description (see measured)"
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": max(3, args.warmup), "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": cfg,
                "measured": {"mean_neighbours": mean_nn, "mesh_points": int(M), "particles": tot,
                             "neighbour_rows_gb": tot * mean_nn * 4 / 1e9},
                "plain": {"value": plain_value, "unit": UNIT,
                          "desc": "same systems, one system per launch sequence, no graph"},
                "batched_over_plain": (value / world / plain_value) if plain_value else None,
                "roofline": roof,
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h),
                        "desc": "pinned host pos/vel/charge in, pos/vel/energy out, every step; two device "
                                "buffer sets, step k+1 uploads and step k-1 downloads on a copy stream "
                                "during step k"},
                "autotune": tuned,
                "gpu_launches": int(args.steps * (K_NLIST + k_eval +
                                                  MD_STEPS * (k_eval + K_NVE))),
                "pair_list": "HOOMD-layout rows" if args.hoomd_list else "the library's pair list (rows in cell order)",
                "clocks": clk.summary()}
        line["fft"] = {"ours_ms": stage_ms.get("fft")}
        try:
            line["fft"].update(cufft_leg(b, N.size, dev))
        except Exception as ex:  # a comparison only
            line["fft"]["error"] = "%s: %s" % (type(ex).__name__, ex)
        if not args.no_accuracy:
            try:
                line["accuracy"] = accuracy_leg(b, sl, pos_h, q, (head, nn, nl) if args.hoomd_list else None, dev)
            except Exception as ex:  # reported in the line, the timed figures stand
                line["accuracy"] = {"error": "%s: %s" % (type(ex).__name__, ex)}
        if not args.no_cpu:
            from oracle import esp_port as EP
            threads = EP.max_threads()
            csl, cprm = cpu_sample(max(4, 2 * threads), rank)
            cache = EP.influence_tables(cprm)
            n_ps, wall = cpu_baseline(csl, cprm, threads, cache)
            line["cpu_baseline"] = {
                "value": n_ps / wall, "unit": UNIT, "cores": threads, "kind": "port",
                "sample": "FP64 C restatement (oracle/esp_oracle.c): nlist + 1 evaluation + 10 NVE steps of the "
                          "first %d systems of this batch (%d particles), %d OpenMP threads"
                          % (len(csl), sum(s.N for s in csl), threads)}
        if not args.no_serve:
            b.close()
            torch.cuda.empty_cache()
            try:
                rates, sst = run_serving(args, _serve_pool(SEED + 6))
            except Exception as ex:  # the timed figures above stand; report the failure in the line
                rates, sst = None, None
                line["serving"] = {"error": "%s: %s" % (type(ex).__name__, ex)}
        if not args.no_serve and rates:
            mid = rates[0]
            sat = max(rates, key=lambda r: r["throughput"])
            line["serving"] = {
                "workload": "Poisson arrivals, 50/50 rock-salt n even ~U{8..64} (r_c 3.0) / rigid water 1,000-32,768 "
                            "molecules (r_c 0.9 nm, SETTLE); each request = nlist + 1 evaluation + 10 NVE steps; "
                            "64 GB HBM budget; latency = completion - arrival (host clock)",
                "unit": UNIT, "rates": rates, "p50_ms": mid["p50_ms"], "p99_ms": mid["p99_ms"],
                "at_rate_per_s": mid["rate_per_s"],
                "saturated_throughput": sat["throughput"],
                "saturated_over_batched": sat["throughput"] / value if value else None,
                "server": {k: sst[k] for k in ("rounds", "max_active", "peak_bytes", "arena_bytes",
                                               "influence_builds", "influence_hits", "failed")}}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--plain-steps", type=int, default=1)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the FP64 Ewald check of the timed plan")
    ap.add_argument("--systems", type=int, default=N_SYS,
                    help="evaluate only the first S systems of the batch (small cases for profiling)")
    ap.add_argument("--workload", default="batched256", choices=["batched256", "scaleup", "c1", "water"],
                    help="second measurements: scaleup (the plain path on one 10^6-particle system), c1 (FP64 "
                         "plain case with LJ, 100 NVE steps), water (the C3 accuracy sweep)")
    ap.add_argument("--water-rows", default="",
                    help="water sweep rows to run, comma-separated target:precision (e.g. 1e-5:f64); default all")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (default plan)")
    ap.add_argument("--hoomd-list", action="store_true",
                    help="short-range term over HOOMD-layout neighbour rows built by the harness instead of the "
                         "library's pair list (rows in cell order, the default)")
    ap.add_argument("--serve-requests", type=int, default=10000, help="requests per arrival rate")
    ap.add_argument("--serve-rates", type=lambda v: [float(x) for x in v.split(",")], default=[200.0, 800.0, 0.0],
                    help="comma-separated arrival rates (requests/s); 0 = all requests at once (saturation)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "scaleup":
        run_scaleup(args)
    elif args.workload == "c1":
        run_c1(args)
    elif args.workload == "water":
        run_water(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
