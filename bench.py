"""Benchmark of the trajectory-method CCS hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config NAME]
    python bench.py --impl reference ...   # the reference's own CPU implementation

One step = one pass of the trajectory loop over the workload's trajectories:
by default the charged 1231-atom globule with the 3-site N2 probe, 3e5
trajectories (the configuration the headline metric is quoted on).  Other
workloads (`--config`): c60_he (60-atom cage, He), shell_he / shell_n2 (5e5-atom
shell), batch_he (256 ions in one batched call), field_n2 / field_co2
(20,000-atom globule, plain FP32 and the learned field side by side).  Prints
one JSON line.

value      trajectories/s with the random inputs resident in HBM (ccs_run_device),
           whole job over all ranks (each rank its own trajectories: weak scaling)
e2e        the same metric through the public host API (mh_predraw on the host,
           ccs_run with pinned host buffers: H2D of the inputs and D2H of the
           per-trajectory results inside the timed region, then the reduction)
roofline   FP32-pipe roofline of the trajectory kernels: algorithmic flops (the
           reference's target-atom visits per trajectory x flops per visit) over
           the device time, against the device's measured FP32 FMA peak
cpu_baseline  the reference binary (oracle/_ref/massccs[_v4], the highest ISA
           level the host runs) on this host's cores, on a bounded sample of the
           same workload (>= 3e4 trajectories), with the thread count (physical
           cores or all logical CPUs) that runs it fastest
accuracy   the metric's condition: the FP32 CCS against the engine's FP64
           mode on the same initial conditions (all of the step's trajectories
           by default; paired relative difference and its standard error)
"""
import argparse
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "trajectories/s on 1 B200 at <=0.5% CCS err vs FP64: plain FP32 vs surrogate vs CPU"
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
REF_SAMPLE = 30000  # fewest trajectories per timed reference sample


def ref_sample_size(rs, total, cap=None):
    """Trajectories per timed reference sample: at least REF_SAMPLE and about
    10 s of CPU work, at most the workload's own count (and, for the large
    assembly, the subset size its configuration states)."""
    n = min(total, max(REF_SAMPLE, rs["probe_rate"] * 10.0))
    if cap:
        n = min(n, cap)
    return int(n // 10 * 10)

# flops per target-atom visit of one probe site (fixed constants of the work
# model): LJ + induced dipole 45, LJ + Coulomb 25, Coulomb + induced dipole 40,
# LJ only 20
FLOPS_PER_VISIT = {("He", 4): 45.0, ("N2", 6): (25.0 + 25.0 + 40.0) / 3.0}

CONFIGS = {
    "globule_n2": dict(gen="globule_n2", ntraj=300000, nprobe=30000, niter=10, gas="N2", ft=6,
                       desc="1231-atom globule (Rg 11.5 A, +4 e), N2 3-site, force type 6, 3e5 trajectories"),
    "c60_he": dict(gen="c60_he", ntraj=300000, nprobe=30000, niter=10, gas="He", ft=4,
                   desc="60-atom C60 cage (C-C 1.40 A, neutral, uff.ff), He, force type 4, 3e5 trajectories"),
    "batch_he": dict(gen="batch", gas="He", ft=4,
                     desc="batched ions: globules of 500-50000 atoms (log-uniform), net charge 0-30 e, He, "
                          "force type 4; one ccs_run_batch call per step"),
    "shell_he": dict(gen="shell", gas="He", ft=4, ntraj=1000000, nprobe=100000, niter=10, ref_max=10000,
                     desc="large assembly: 5e5-atom spherical shell (r 100-130 A, +40 e), He, force type 4, "
                          "1e6 trajectories; the reference timed on a 1e4-trajectory subset"),
    "shell_n2": dict(gen="shell", gas="N2", ft=6, ntraj=100000, nprobe=10000, niter=10, ref_max=2000,
                     desc="large assembly: 5e5-atom spherical shell (r 100-130 A, +40 e), N2 3-site, force type 6, "
                          "1e5 trajectories per step; the reference timed on a 2e3-trajectory subset"),
    "field_n2": dict(gen="field_globule", gas="N2", ft=6, ntraj=100000, nprobe=100000, niter=10,
                     desc="learned field: 20,000-atom globule (+12 e), N2 3-site, force type 6; "
                          "plain FP32 and the learned field on the same trajectories"),
    "field_co2": dict(gen="field_globule", gas="CO2", ft=6, ntraj=100000, nprobe=100000, niter=10,
                      desc="learned field: 20,000-atom globule (+12 e), CO2 3-site, force type 6; "
                           "plain FP32 and the learned field on the same trajectories"),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_workload(name, d):
    from massccs_b200 import synth
    c = CONFIGS[name]
    gen = getattr(synth, c["gen"])
    if c["gen"] in ("field_globule", "shell"):
        return gen(d, gas=c["gas"], nprobe=c["nprobe"], niter=c["niter"])
    return gen(d, nprobe=c["nprobe"], niter=c["niter"])


class ClockSampler:
    """nvidia-smi clock and throttle samples while the timed region runs."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi") is None:
            return self
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def host_cpu():
    """CPU model, logical CPUs, physical cores and the AVX-512 subset the
    x86-64-v4 build needs (from /proc/cpuinfo)."""
    model, flags, cores, logical = None, set(), set(), 0
    phys = None
    try:
        for line in open("/proc/cpuinfo"):
            k, _, v = line.partition(":")
            k, v = k.strip(), v.strip()
            if k == "processor":
                logical += 1
            elif k == "model name" and model is None:
                model = v
            elif k == "flags" and not flags:
                flags = set(v.split())
            elif k == "physical id":
                phys = v
            elif k == "core id":
                cores.add((phys, v))
    except OSError:
        pass
    logical = logical or (os.cpu_count() or 1)
    v4 = {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= flags
    return {"model": model, "logical_cpus": logical, "physical_cores": len(cores) or logical, "avx512": v4}


def ref_binary(cpu):
    """The reference binary at the highest ISA level this host supports."""
    v4 = os.path.join(REF_DIR, "massccs_v4")
    v3 = os.path.join(REF_DIR, "massccs")
    if cpu["avx512"] and os.path.exists(v4):
        return v4, "x86-64-v4"
    return (v3, "x86-64-v3") if os.path.exists(v3) else (None, None)


def ref_sample_run(binary, json_path, nprobe, niter, threads):
    """Run the reference binary on a sample; returns (trajectories, CCS time s, ccs)."""
    d = os.path.dirname(json_path)
    cfg = json.load(open(json_path))
    cfg.update({"numberProbe": nprobe, "nIter": niter, "nthreads": threads})
    p = os.path.join(d, "input_ref.json")
    json.dump(cfg, open(p, "w"))
    out = subprocess.run([binary, "input_ref.json"], cwd=d, capture_output=True, text=True, timeout=1800)
    m = re.search(r"CCS time: (\S+) s", out.stdout)
    c = re.search(r"average value of CCS = (\S+)", out.stdout)
    if out.returncode != 0 or not m:
        raise RuntimeError("reference run failed: " + out.stderr[-400:])
    return nprobe * niter, float(m.group(1)), float(c.group(1)) if c else None


def ref_setup(json_path, probe_n=2000):
    """Binary, thread count and sample shape of the timed reference runs: the
    faster of all physical cores and all logical CPUs on a probe sample of
    2000 trajectories (the reference's results do not depend on it)."""
    cpu = host_cpu()
    binary, isa = ref_binary(cpu)
    if binary is None:
        return None
    best = None
    for threads in sorted({cpu["physical_cores"], cpu["logical_cpus"]}):
        n0, t0, _ = ref_sample_run(binary, json_path, max(1, probe_n // 10), 10, threads)
        rate = n0 / max(t0, 1e-3)
        if best is None or rate > best[1]:
            best = (threads, rate)
    return {"binary": binary, "isa": isa, "threads": best[0], "probe_rate": best[1], "cpu": cpu}


def ref_describe(rs, n, nprobe, niter, extra=""):
    c = rs["cpu"]
    return (f"{n} trajectories ({nprobe} x {niter}) of the workload, reference binary "
            f"{os.path.basename(rs['binary'])} ({rs['isa']}, -O3 -ffast-math, OpenMP), nthreads {rs['threads']} "
            f"on {c['model']} ({c['physical_cores']} physical cores, {c['logical_cpus']} logical CPUs){extra}")


def cpu_baseline(json_path, config):
    """The reference binary on this host's cores, on a bounded sample of the
    workload (REF_SAMPLE trajectories), plus the reference's visit count per
    trajectory (from the oracle, on a smaller sample) for the roofline's
    algorithmic work."""
    out = {"value": None, "unit": "trajectories/s", "cores": None, "kind": "reference", "sample": None}
    visits = None
    cap = CONFIGS[config].get("ref_max")
    rs = ref_setup(json_path, probe_n=min(2000, cap // 5) if cap else 2000)
    if rs:
        niter = 10
        nprobe = ref_sample_size(rs, CONFIGS[config].get("ntraj", REF_SAMPLE), CONFIGS[config].get("ref_max")) // niter
        n, t, _ = ref_sample_run(rs["binary"], json_path, nprobe, niter, rs["threads"])
        out.update(value=n / t, cores=rs["threads"], isa=rs["isa"], cpu=rs["cpu"],
                   sample=ref_describe(rs, n, nprobe, niter, f"; CCS time {t:.2f} s"))
    try:
        from oracle import pyoracle
        sys_ = pyoracle.OracleSystem(json_path)
        m = 400
        res = sys_.run(sys_.predraw(m), nthreads=os.cpu_count() or 1)
        visits = float(res["visits"].mean())
    except Exception as e:  # the roofline then reports the engine's own count only
        log("oracle visit count unavailable:", e)
    return out, visits


def cpu_baseline_batch(paths, natoms, per_ion=8000, nsample=8):
    """The reference binary over the batched-ion workload: nsample ions spread
    evenly over the sorted sizes, per_ion trajectories each; every ion of the
    batch has the same trajectory count, so the batch rate is the harmonic
    mean of the sampled ions' rates."""
    import numpy as np
    out = {"value": None, "unit": "trajectories/s", "cores": None, "kind": "reference", "sample": None}
    order = np.argsort(natoms)
    pick = [int(order[k]) for k in np.linspace(0, len(order) - 1, nsample).round().astype(int)]
    rs = ref_setup(paths[pick[len(pick) // 2]], probe_n=200)
    if not rs:
        return out
    inv, secs = [], 0.0
    for i in pick:
        n, t, _ = ref_sample_run(rs["binary"], paths[i], per_ion // 10, 10, rs["threads"])
        inv.append(t / n)
        secs += t
    out.update(value=1.0 / float(np.mean(inv)), cores=rs["threads"], isa=rs["isa"], cpu=rs["cpu"],
               sample=ref_describe(rs, per_ion * len(pick), per_ion // 10, 10,
                                   f" per ion, {len(pick)} ions of {min(natoms[i] for i in pick)}-"
                                   f"{max(natoms[i] for i in pick)} atoms spread over the sorted sizes; "
                                   f"harmonic mean of the ions' rates; CCS time {secs:.1f} s"))
    return out


def fp64_check(S, eng, rnd, status, omc, m, device):
    """The metric's accuracy condition: the first m trajectories of the last
    end-to-end step rerun in the engine's FP64 mode on the same initial
    conditions; CCS estimate = mean dOmega over free + scatter (the reference's
    estimator), paired difference and its standard error."""
    import numpy as np
    m = min(m, rnd.shape[1])
    e64 = S.engine(device=device, precision=1)
    r64 = e64.run(np.ascontiguousarray(rnd[:, :m]), want_steps=False, want_visits=False)
    e64.close()
    bmax = S.info["bmax"]
    a = np.pi * np.where(r64["status"] == 1, r64["one_minus_cos"], 0.0) * bmax ** 2
    b = np.pi * np.where(status[:m] == 1, omc[:m], 0.0) * bmax ** 2
    ok = (r64["status"] <= 1) & (status[:m] <= 1)
    ref = float(a[ok].mean())
    d = (b - a)[ok]
    return {"vs": "FP64 engine mode on the same initial conditions (paired)", "trajectories": int(m),
            "ccs_fp64_A2": ref, "ccs_fp32_A2": float(b[ok].mean()), "rel_diff": float(d.mean() / ref),
            "rel_se": float(d.std(ddof=1) / np.sqrt(len(d)) / ref),
            "status_agreement": float((r64["status"] == status[:m]).mean())}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    cfg = CONFIGS[args.config]
    line = {"metric": METRIC, "impl": "reference", "unit": "trajectories/s", "higher_is_better": True,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "dtype": "f64",
            "data": "synthetic", "config": {"workload": args.config, "description": cfg["desc"]}}
    if not os.path.exists(os.path.join(REF_DIR, "massccs")):
        line["unavailable"] = "reference binary oracle/_ref/massccs not built (make -C oracle ref)"
        print(json.dumps(line), flush=True)
        return
    d = tempfile.mkdtemp(prefix="bench_ref_")
    json_path = make_workload(args.config, d)
    cap = cfg.get("ref_max")
    rs = ref_setup(json_path, probe_n=min(2000, cap // 5) if cap else 2000)
    niter = 10
    nprobe = ref_sample_size(rs, cfg.get("ntraj", REF_SAMPLE), cfg.get("ref_max")) // niter  # >= 3e4 per step
    for _ in range(args.warmup):  # warm-up steps at a tenth of the size
        ref_sample_run(rs["binary"], json_path, nprobe // 10, niter, rs["threads"])
    times, n = [], 0
    for _ in range(args.steps):
        k, t, _ = ref_sample_run(rs["binary"], json_path, nprobe, niter, rs["threads"])
        times.append(t)
        n = k
    total = sum(times)
    value = n * len(times) / total
    line.update(value=value, ms_per_step=1e3 * total / len(times),
                cpu_baseline={"value": value, "unit": "trajectories/s", "cores": rs["threads"], "kind": "reference",
                              "isa": rs["isa"], "cpu": rs["cpu"],
                              "sample": ref_describe(rs, n, nprobe, niter, " per step; the reference's CCS time")},
                e2e={"value": value, "unit": "trajectories/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
    shutil.rmtree(d, ignore_errors=True)
    print(json.dumps(line), flush=True)


def run_batch_bench(args, rank, world, local):
    """batch_he: every step runs all ions through one ccs_run_batch call (host
    buffers in and out: the call a user makes), against one ccs_run per ion."""
    import numpy as np
    import torch
    from massccs_b200 import engine as E
    from massccs_b200 import host as H
    from massccs_b200 import synth
    torch.cuda.set_device(local)
    d = tempfile.mkdtemp(prefix=f"bench_batch_{rank}_")
    t0 = time.perf_counter()
    paths = synth.batch(d, nions=args.ions, ntraj=args.traj_per_ion, seed=2104 + 100000 * rank)
    systems = [H.System(p) for p in paths]
    engs = [S.engine(device=local) for S in systems]
    rnds = [S.predraw() for S in systems]
    natoms = [S.info["natoms"] for S in systems]
    log(f"[rank {rank}] {len(systems)} ions, {sum(natoms)} atoms, set-up {time.perf_counter() - t0:.1f} s")
    total = sum(r.shape[1] for r in rnds)
    for _ in range(args.warmup):
        E.run_batch(engs, rnds, want_steps=False, want_visits=False)
    kern, wall, last = [], [], None
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t = time.perf_counter()
            out, st = E.run_batch(engs, rnds, want_steps=False, want_visits=False)
            for S, o in zip(systems, out):
                H.reduce(S.info["niter"], S.info["nprobe"], o["status"], o["one_minus_cos"], S.info["bmax"])
            wall.append(time.perf_counter() - t)
            kern.append(st["kernel_ms"])
            last = st
    # one launch of each pass per ion (each context already tuned by a first run)
    for e, r in zip(engs, rnds):
        e.run(r, want_steps=False, want_visits=False)
    t = time.perf_counter()
    sep_kernel = 0.0
    for e, r in zip(engs, rnds):
        sep_kernel += e.run(r, want_steps=False, want_visits=False)["stats"]["kernel_ms"]
    sep_wall = time.perf_counter() - t
    ms = sum(kern) / len(kern)
    e2e_s = sum(wall) / len(wall)
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline_batch(paths, natoms)
        peak = E.measure_fp32_peak(local)
        fpv = FLOPS_PER_VISIT[("He", 4)]
        achieved = last["visits"] * fpv / (last["kernel_ms"] * 1e-3) / 1e12
        line = {
            "metric": METRIC + " (batched ions)", "value": world * total / (ms * 1e-3), "unit": "trajectories/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "batch_he", "description": CONFIGS["batch_he"]["desc"], "ions": len(systems),
                       "trajectories_per_ion": args.traj_per_ion, "atoms_total": int(sum(natoms)),
                       "atoms_min": int(min(natoms)), "atoms_max": int(max(natoms)),
                       "l2": "no flush: each step moves 72 B per trajectory host to device (3.7e8 B at 5.12e6)"},
            "e2e": {"value": world * total / e2e_s, "unit": "trajectories/s",
                    "h2d_bytes_per_step": 5 * 8 * total, "d2h_bytes_per_step": 9 * total,
                    "includes": "ccs_run_batch (H2D, both passes, D2H) and the per-ion reductions"},
            "one_launch_per_ion": {"kernel_ms": sep_kernel, "wall_s": sep_wall,
                                   "batch_speedup_kernel": sep_kernel / ms, "batch_speedup_wall": sep_wall / e2e_s},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if peak else None, "traffic": None,
                         "work": f"engine candidate visits x {fpv:g} flops per visit"},
            "cpu_baseline": cpu,
            # per run: watchdog arm, lane pass, warp pass (two launches), verdicts of the speculative tries
            "gpu_launches": 5 * args.steps,
            "engine": {"lane_ms": last["lane_ms"], "warp_ms": last["warp_ms"], "parked": last["parked"],
                       "lanes_per_force": last["lanes_per_traj"]},
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    for e in engs:
        e.close()
    shutil.rmtree(d, ignore_errors=True)


def run_field_bench(args, rank, world, local):
    """field_n2 / field_co2: the learned-field configuration.  The field is
    trained once (its set-up cost is reported, not timed as a step); each
    timed step runs the step's trajectories with plain FP32 forces and with
    the learned field, from the same device-resident random rows; accuracy:
    both against the FP64 plain path on the same initial conditions."""
    import numpy as np
    import torch
    from massccs_b200 import host as H
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    cfg = CONFIGS[args.config]
    d = tempfile.mkdtemp(prefix=f"bench_field_{rank}_")
    json_path = make_workload(args.config, d)
    S = H.System(json_path)
    n = args.ntraj if args.ntraj > 0 else cfg["ntraj"]
    seed = S.info["seed"] + rank
    rnd_host = S.predraw(n, seed=seed)
    eng = S.engine(device=local)
    t0 = time.perf_counter()
    rep = eng.field_train(**({"samples": args.field_samples} if args.field_samples else {}),
                          **({"iterations": args.field_iters} if args.field_iters else {}))
    train_s = time.perf_counter() - t0
    log(f"[rank {rank}] field trained in {train_s:.1f} s: " + json.dumps(
        {k: rep[k] for k in ("sample_ms", "label_ms", "train_ms", "validate_ms", "first_loss", "final_loss",
                             "val_force_rel_rms", "val_force_rel_p99", "exact_fraction", "err_voxels")}))
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    d_rnd = torch.from_numpy(rnd_host).to(dev)
    d_status = torch.empty(n, dtype=torch.int8, device=dev)
    d_omc = torch.empty(n, dtype=torch.float64, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def timed(on):
        eng.field_enable(on)
        for _ in range(args.warmup):
            eng.run_device(n, d_rnd.data_ptr(), n, d_status.data_ptr(), d_omc.data_ptr(), 0, 0, stream.cuda_stream)
        torch.cuda.synchronize()
        ms, st = [], None
        for _ in range(args.steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            eng.run_device(n, d_rnd.data_ptr(), n, d_status.data_ptr(), d_omc.data_ptr(), 0, 0, stream.cuda_stream)
            b.record(stream)
            st = eng.sync_stats()
            ms.append(a.elapsed_time(b))
        return sum(ms) / len(ms), st, d_status.cpu().numpy(), d_omc.cpu().numpy()

    with ClockSampler(local) as clocks:
        plain_ms, plain_st, p_status, p_omc = timed(False)
        field_ms, field_st, f_status, f_omc = timed(True)
    # e2e with the field on: host rows in, results out, through ccs_run
    eng.field_enable(True)
    t1 = time.perf_counter()
    for _ in range(args.steps):
        o = eng.run(rnd_host, want_steps=False, want_visits=False)
        H.reduce(1, n, o["status"], o["one_minus_cos"], S.info["bmax"])
    e2e_s = (time.perf_counter() - t1) / args.steps
    line = None
    if rank == 0:
        bmax = S.info["bmax"]
        m = min(n, args.fp64_check if args.fp64_check > 0 else 20000)
        e64 = S.engine(device=local, precision=1)
        r64 = e64.run(np.ascontiguousarray(rnd_host[:, :m]), want_steps=False, want_visits=False)
        e64.close()

        def paired(status, omc):
            a = np.pi * np.where(r64["status"] == 1, r64["one_minus_cos"], 0.0) * bmax ** 2
            b = np.pi * np.where(status[:m] == 1, omc[:m], 0.0) * bmax ** 2
            ok = (r64["status"] <= 1) & (status[:m] <= 1)
            dd = (b - a)[ok]
            ref = float(a[ok].mean())
            return {"ccs_fp64_A2": ref, "ccs_A2": float(b[ok].mean()), "rel_diff": float(dd.mean() / ref),
                    "rel_se": float(dd.std(ddof=1) / np.sqrt(len(dd)) / ref),
                    "status_agreement": float((r64["status"] == status[:m]).mean())}
        acc = {"trajectories": int(m), "vs": "FP64 plain engine mode, same initial conditions (paired)",
               "plain_fp32": paired(p_status, p_omc), "field": paired(f_status, f_omc)}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu, _ = cpu_baseline(json_path, args.config)
        value = world * n / (field_ms * 1e-3)
        line = {
            "metric": METRIC, "value": value, "unit": "trajectories/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": field_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 forces/integration, bf16 MLP with f32 accumulation", "data": "synthetic",
            "config": {"workload": args.config, "description": cfg["desc"], "trajectories_per_gpu": n,
                       "l2": "256 MiB buffer written between timed steps (outside the step events)"},
            "plain_fp32": {"value": world * n / (plain_ms * 1e-3), "ms_per_step": plain_ms,
                           "lane_ms": plain_st["lane_ms"], "warp_ms": plain_st["warp_ms"],
                           "visits_per_traj": plain_st["visits"] / n},
            "field": {"value": value, "ms_per_step": field_ms, "lane_ms": field_st["lane_ms"],
                      "warp_ms": field_st["warp_ms"], "exact_visits_per_traj": field_st["visits"] / n,
                      "gain_over_plain": plain_ms / field_ms},
            "training": {"wall_s": train_s, **{k: rep[k] for k in (
                "samples", "sample_ms", "label_ms", "train_ms", "validate_ms", "first_loss", "final_loss",
                "val_force_rel_rms", "val_force_rel_p99", "val_u_rel_rms", "exact_fraction", "err_voxels")}},
            "e2e": {"value": world * n / e2e_s, "unit": "trajectories/s",
                    "h2d_bytes_per_step": 9 * 8 * n, "d2h_bytes_per_step": 9 * n,
                    "includes": "ccs_run with the learned field (H2D, both passes, D2H) and the reduction; "
                                "training excluded (set-up, in `training`)"},
            # per step two runs (plain and field) of 5 kernels each: watchdog arm, lane pass,
            # warp pass (two launches), verdicts of the speculative tries
            "accuracy": acc, "cpu_baseline": cpu, "gpu_launches": 10 * args.steps,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    eng.close()
    shutil.rmtree(d, ignore_errors=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="globule_n2", choices=sorted(CONFIGS))
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ntraj", type=int, default=0,
                    help="trajectories per step (default: the workload's 3e5); smaller values are for profiling")
    ap.add_argument("--fp64-check", type=int, default=-1,
                    help="trajectories rerun in FP64 mode to report the FP32 CCS error (-1: all, 0: skip)")
    ap.add_argument("--ions", type=int, default=256, help="batch_he: number of ions")
    ap.add_argument("--traj-per-ion", type=int, default=20000, help="batch_he: trajectories per ion")
    ap.add_argument("--field-samples", type=int, default=0, help="field_*: training samples (0: default)")
    ap.add_argument("--field-iters", type=int, default=0, help="field_*: training steps (0: default)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":  # CPU only: rank 0 runs it, the other ranks have nothing to do
        run_reference_arm(args, rank, world)
        return
    if args.config == "batch_he":
        run_batch_bench(args, rank, world, local)
        return
    if args.config.startswith("field_"):
        run_field_bench(args, rank, world, local)
        return
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        import torch
        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
        dist = dist_mod

    import numpy as np
    import torch
    from massccs_b200 import engine as E
    from massccs_b200 import host as H

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    cfg = CONFIGS[args.config]
    d = tempfile.mkdtemp(prefix=f"bench_{rank}_")
    json_path = make_workload(args.config, d)
    S = H.System(json_path)
    n = args.ntraj if args.ntraj > 0 else cfg["ntraj"]
    # one job of world * n trajectories from one pre-draw; rank r runs the
    # contiguous slice [r n, (r + 1) n) (weak scaling: n per GPU is fixed)
    seed = S.info["seed"]
    job = world * n
    rnd_host = np.ascontiguousarray(S.predraw(job, seed=seed)[:, rank * n:(rank + 1) * n])
    eng = S.engine(device=local)
    stream = torch.cuda.Stream(dev)  # a real stream handle (0 would mean the engine's own stream)
    torch.cuda.set_stream(stream)
    d_rnd = torch.from_numpy(rnd_host).to(dev)
    d_status = torch.empty(n, dtype=torch.int8, device=dev)
    d_omc = torch.empty(n, dtype=torch.float64, device=dev)
    d_steps = torch.empty(n, dtype=torch.int32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2

    def step_device():
        eng.run_device(n, d_rnd.data_ptr(), n, d_status.data_ptr(), d_omc.data_ptr(), d_steps.data_ptr(), 0,
                       stream.cuda_stream)

    log(f"[rank {rank}] warmup x{args.warmup} on {cfg['desc']}")
    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()
    stats = eng.sync_stats()

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    per_step = []
    barrier()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            step_device()
            ev[k][1].record(stream)
            per_step.append(eng.sync_stats())  # host sync after the step's stop event
        barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    last = per_step[-1]
    log(f"[rank {rank}] steps (ms): " + ", ".join(f"{t:.1f} (lane {st['lane_ms']:.1f}, warp {st['warp_ms']:.1f},"
                                                  f" parked {st['parked']})" for t, st in zip(step_ms, per_step)))
    dev_ms = sum(step_ms)
    if dist:
        t = torch.tensor([dev_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms = float(t.item())
    ms_per_step = dev_ms / args.steps
    value = world * n / (ms_per_step * 1e-3)

    # e2e through the public API: pre-draw on the host into pinned memory,
    # ccs_run (H2D, both passes, D2H), the reduction; every step
    pin = torch.empty((9, job), dtype=torch.float64).pin_memory()
    pin_np = pin.numpy()
    st_pin = torch.empty(n, dtype=torch.int8).pin_memory().numpy()
    om_pin = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    import ctypes
    # this rank's slice of the job's rows
    rows = (ctypes.c_void_p * 9)(*[pin_np[k].ctypes.data + 8 * rank * n for k in range(9)])
    if dist:  # per-trajectory results of every rank, gathered for the fixed-order reduction
        g_st = torch.empty(job, dtype=torch.int8, device=dev)
        g_om = torch.empty(job, dtype=torch.float64, device=dev)
    L = E.load_library()
    HL = H.load_library()

    # the reduction's iterations x probes must cover exactly the job's
    # trajectories (a job smaller than the workload's, e.g. --ntraj, too)
    it_n = S.info["niter"] if job % S.info["niter"] == 0 else 1

    def step_e2e():
        HL.mh_predraw(S._h, seed, job, pin_np.ctypes.data_as(ctypes.c_void_p))
        stt = E.CcsStats()
        rc = L.ccs_run(eng._h, n, rows, st_pin.ctypes.data_as(ctypes.c_void_p),
                       om_pin.ctypes.data_as(ctypes.c_void_p), None, None, ctypes.byref(stt))
        if rc:
            raise E.CcsError(L.ccs_last_error(eng._h).decode())
        if dist:
            dist.all_gather_into_tensor(g_st, torch.from_numpy(st_pin).to(dev))
            dist.all_gather_into_tensor(g_om, torch.from_numpy(om_pin).to(dev))
            if rank == 0:
                H.reduce(it_n, job // it_n, g_st.cpu().numpy(), g_om.cpu().numpy(), S.info["bmax"])
        else:
            H.reduce(it_n, job // it_n, st_pin, om_pin, S.info["bmax"])

    step_e2e()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step_e2e()
    barrier()
    e2e_s = (time.perf_counter() - t0) / args.steps
    e2e_stats = eng.sync_stats()
    log(f"[rank {rank}] e2e step {e2e_s * 1e3:.1f} ms (kernel {e2e_stats['kernel_ms']:.1f}, lane {e2e_stats['lane_ms']:.1f},"
        f" warp {e2e_stats['warp_ms']:.1f}, h2d {e2e_stats['h2d_ms']:.2f}, d2h {e2e_stats['d2h_ms']:.2f})")
    if dist:
        t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * n / e2e_s

    if rank == 0:
        status = st_pin
        nscatter = int((status == 1).sum())
        m = (n if args.fp64_check < 0 else args.fp64_check) if world == 1 else 0  # N=1 line only
        accuracy = fp64_check(S, eng, pin_np, st_pin, om_pin, m, local) if m > 0 else None
        peak = E.measure_fp32_peak(local)
        engine_visits = last["visits"] / max(1, n)
        ref_visits = None
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu, ref_visits = cpu_baseline(json_path, args.config)
        fpv = FLOPS_PER_VISIT.get((cfg["gas"], cfg["ft"]), 30.0)
        kernel_s = ms_per_step * 1e-3
        alg_visits = ref_visits if ref_visits else engine_visits
        achieved = n * alg_visits * fpv / kernel_s / 1e12
        traffic = None
        prof = os.path.join(ROOT, "profiles", f"traffic_{args.config}.json")
        if os.path.exists(prof):
            traffic = json.load(open(prof)).get("bytes_per_launch")
        line = {
            "metric": METRIC, "value": value, "unit": "trajectories/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.config, "description": cfg["desc"], "trajectories_per_gpu": n,
                       "l2": "256 MiB buffer written between timed steps (outside the step events)",
                       "parallelism": f"one job of {world} x {n} trajectories (one pre-draw), rank r runs "
                                      f"trajectories [r n, (r+1) n); results gathered to rank 0 for the "
                                      f"fixed-order reduction"},
            "e2e": {"value": e2e_value, "unit": "trajectories/s",
                    "h2d_bytes_per_step": (9 if cfg["gas"] in ("N2", "CO2") else 5) * 8 * n,  # rows ccs_run copies
                    "d2h_bytes_per_step": 9 * n * (world if world > 1 else 1),
                    "includes": "host mt19937 pre-draw, H2D, lane+warp passes, D2H, reduction"},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if peak else None, "traffic": traffic,
                         "peak_source": "FP32 FMA-chain kernel (ccs_measure_fp32_peak) on this device",
                         "work": ("reference target-atom visits per trajectory (oracle, reference cells) "
                                  if ref_visits else "engine candidate visits per trajectory ") +
                                 f"{alg_visits:.4g} x {fpv:g} flops per visit",
                         "engine_visits_per_traj": engine_visits,
                         "engine_tflops": n * engine_visits * fpv / kernel_s / 1e12,
                         "frac_executed": (n * engine_visits * fpv / kernel_s / 1e12) / peak if peak else None},
            "cpu_baseline": cpu,
            "accuracy": accuracy,
            # per run: watchdog arm, lane pass, warp pass (two launches), verdicts of the speculative tries
            "gpu_launches": 5 * args.steps,
            "engine": {"lane_ms": last["lane_ms"], "warp_ms": last["warp_ms"], "parked": last["parked"],
                       "lanes_per_force": last["lanes_per_traj"], "scatter_fraction": nscatter / n,
                       "steps_per_traj": last["steps"] / n},
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    eng.close()
    shutil.rmtree(d, ignore_errors=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
