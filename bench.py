#!/usr/bin/env python
"""Throughput of the RTMC phonon transport hot path on B200.

Workload (the metric's configuration): a thin film 300 x 300 x 145 nm
(x transport between the two heat baths, z thickness, y periodic), pierced by
3 through-thickness cylindrical holes of radius 50 nm at seeded positions,
diffuse hole and z walls; a seeded Si-like 2000-mode spectrum with 64
frequency bins; every mode runs at its own bulk MFP (per-mode gray runs);
Nangle = 11 (10 simulated incident angles), 500 particles per (mode, angle):
10^7 trajectories per step and per GPU.

A step is one ptg_kappa call: the persistent FP32 transport kernel over all
10^7 trajectories plus the FP64 kappa / per-bin reduction.
  value : free flights / device time (CUDA events on the handle's stream
          around the transport and reduction kernels), inputs resident.
  e2e   : the same flights / wall time of the whole C-ABI call with host
          buffers (task tables and mode constants copied in, kappa, bins and
          EMFPs copied out).
The plain FP64 one-phonon-per-thread kernel is timed on the same workload as
the comparator, the CPU oracle (OpenMP, all host cores) on a bounded sample.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import datetime
import importlib.util
import json
import math
import os
import statistics
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "p-trans_b200")

METRIC = "phonon free-flights/s on 1 B200, batched FP32 vs plain FP64, at ≤1% κ std-err"
UNIT = "free-flights/s"
BYTES_PER_FLIGHT = 64       # FP32 SoA state: 32 B read + 32 B written per free flight
FLOPS_PER_FLIGHT_C2 = 702   # 6 box quads x 95 + 3 z-cylinders x 24 + 60 per event
FP32_PEAK_NOMINAL = 148 * 128 * 2 * 1.965e9 / 1e12   # TFLOP/s, 148 SMs x 128 lanes x FMA


def load_pkg():
    if "ptrans_b200" in sys.modules:
        return sys.modules["ptrans_b200"]
    spec = importlib.util.spec_from_file_location(
        "ptrans_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ptrans_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def workload(pkg, n_modes=2000, np_per_task=500, mfp_lo=1e-9):
    A, synth = pkg.abi, pkg.synth
    model = synth.film_with_holes(lx=300.0, ly=300.0, lz=145.0, nholes=3, radius=50.0, seed=0,
                                  periodic_y=True, p_hole=0.0, t_hole=0.0, p_z=0.0)
    spec = synth.spectrum(n_modes, seed=0, mfp_lo=mfp_lo)
    cfg = {"workload": "thin film 300x300x145 nm, 3 z-holes r=50 nm (voids, diffuse), y periodic, "
                       "z diffuse; 2000-mode Si-like spectrum, 64 bins; per-mode MFP runs",
           "modes": n_modes, "bins": 64, "nangle": 11, "particles_per_task": np_per_task,
           "samples_per_gpu": n_modes * 10 * np_per_task,
           "l2": "256 MiB written between timed steps"}
    return model, spec, cfg


def make_run(pkg, spec, np_total, rank, nranks, precision, seed=12345):
    A = pkg.abi
    return A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=11, np_=np_total, seed=seed, rank=rank,
                      nranks=nranks, precision=precision, temperature=300.0, nbins=64,
                      bin_omega=(0.0, 15.0 * 2 * math.pi * 1e12))


class ClockSampler:
    """SM clock and throttle reasons of one GPU, read through NVML every
    10 ms on a background thread (read-only queries)."""

    # NVML clocks-event reason bits
    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap"}

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.thread = None
        self.stop_flag = False

    def start(self):
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None
            return

        def loop():
            while not self.stop_flag:
                try:
                    sm = self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM)
                    rs = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                    self.samples.append((sm, rs))
                except Exception:
                    pass
                time.sleep(0.01)

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()

    def stop(self):
        if self.thread is None:
            return None
        self.stop_flag = True
        self.thread.join(timeout=5)
        if not self.samples:
            return None
        reasons = sorted({n for _, rs in self.samples for bit, n in self.REASONS.items() if rs & bit})
        return {"sm_mhz": statistics.median(sm for sm, _ in self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples), "source": "NVML, 10 ms"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dram_traffic(phase="drain"):
    """DRAM bytes of one launch of a transport phase (read + write) from the
    committed ncu summary, and the workload they were captured on."""
    p = os.path.join(ROOT, "profiles", "persistent_fp32_thinfilm_dram.json")
    if os.path.exists(p):
        d = json.load(open(p))
        e = d.get(phase, d)
        if "dram_bytes_read" in e:
            return float(e["dram_bytes_read"] + e["dram_bytes_write"]), e["workload"]
    return None, None


ORACLE_SEED = 777   # the oracle's seed: independent of the GPU run's 12345


def issue_profile(phase="drain"):
    """Warp instructions per free flight of a transport phase at the bench
    size, from the committed ncu summary (smsp__inst_executed.sum of one
    launch divided by the flights that launch took), with lanes active per
    warp instruction."""
    p = os.path.join(ROOT, "profiles", "persistent_fp32_thinfilm_issue.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p)).get(phase)
    return d if d and d.get("warp_inst_per_flight") else None


def cpu_leg(args):
    """The cpu_baseline leg in a process of its own (bench.py --cpu-leg; torch
    is never imported here: next to torch's OpenMP runtime the oracle ran
    about three times slower).  Two oracle runs (OpenMP, all host threads):
      - the timed baseline, sized exactly as the reference arm sizes a step
        (--impl reference: seed 12345, particles per task from a 2-particle
        probe so that the run takes about 5 s), so the two rates compare; the
        reference's schedule(static) loop makes the rate depend on where the
        few 10^5-flight trajectories fall, i.e. on the sample;
      - the parity run: the workload with this run's particles per task (or
        fewer, when that would take more than --cpu-target-s), seed 777,
        independent of the GPU run's draws, for kappa and the per-bin
        transmission with their standard errors.
    Prints one JSON line."""
    pkg = load_pkg()
    model, spec, _ = workload(pkg, np_per_task=args.np, mfp_lo=args.mfp_lo)
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from oracle import oracle as O
    o = O.Oracle(model=model, spectrum=spec)
    ntask = spec.nmode * 10
    # timed baseline: the reference arm's recipe
    _, _, r = o.counts(make_run(pkg, spec, 2, 0, 1, 0))
    probe_rate = r["flights"] / max(r["seconds"], 1e-6)
    nb = max(2, min(args.np, int(5.0 / max(r["seconds"] / 2, 1e-9))))
    _, _, rb = o.counts(make_run(pkg, spec, nb, 0, 1, 0))
    # parity run
    n = 2
    _, _, r = o.counts(make_run(pkg, spec, n, 0, 1, 0, seed=ORACLE_SEED))
    n = max(2, min(args.np, int(args.cpu_target_s / max(r["seconds"] / n, 1e-9))))
    run = make_run(pkg, spec, n, 0, 1, 0, seed=ORACLE_SEED)
    cnt, _, rp = o.counts(run)
    k = o.kappa(run, cnt)
    print(json.dumps({
        "value": rb["flights"] / rb["seconds"], "unit": UNIT, "cores": int(rb["threads"]), "kind": "port",
        "seconds": rb["seconds"], "flights": int(rb["flights"]), "probe_rate": probe_rate,
        "sample": (f"all {ntask} (mode, angle) tasks with {nb} particles each, seed 12345 (the reference "
                   f"arm's step)"),
        "parity_sample": (f"all {ntask} (mode, angle) tasks with {n} particles each, {rp['samples']} "
                          f"trajectories, seed {ORACLE_SEED}, {rp['seconds']:.1f} s"),
        "parity_run_rate": rp["flights"] / rp["seconds"],
        "kappa": k["kappa"], "kappa_stderr": k["kappa_stderr"],
        "bin_T": [float(x) for x in k["bin_T"]], "bin_T_stderr": [float(x) for x in k["bin_T_stderr"]]}))
    return 0


def cpu_baseline(args):
    """Runs the cpu_baseline leg (cpu_leg) as a child process with every host
    thread and returns its JSON record."""
    import subprocess
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-leg", "--np", str(args.np),
           "--mfp-lo", repr(args.mfp_lo), "--cpu-target-s", repr(args.cpu_target_s)]
    p = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=900)
    if p.returncode != 0:
        raise RuntimeError(f"cpu_baseline leg failed ({p.returncode}): {p.stderr[-2000:]}")
    return json.loads(p.stdout.strip().splitlines()[-1])


def parity(out, leg):
    """The FP32 GPU result against the FP64 oracle on the same workload
    (independent seeds): kappa and the per-bin transmission, with z-scores
    over the combined standard errors."""
    kg, sg = out["kappa"], out["kappa_stderr"]
    ko, so = leg["kappa"], leg["kappa_stderr"]
    se = math.hypot(sg, so)
    bg, bo = np.asarray(out["bin_T"], float), np.asarray(leg["bin_T"], float)
    eg, eo = np.asarray(out["bin_T_stderr"], float), np.asarray(leg["bin_T_stderr"], float)
    seb = np.hypot(eg, eo)
    live = seb > 0
    zb = np.zeros_like(bg)
    zb[live] = (bg[live] - bo[live]) / seb[live]
    d = bg - bo
    return {"reference": "FP64 CPU oracle (the cpu_baseline run)", "gpu_kappa": kg, "gpu_kappa_stderr": sg,
            "oracle_kappa": ko, "oracle_kappa_stderr": so, "z_kappa": (kg - ko) / se if se > 0 else None,
            "kappa_rel_diff": (kg - ko) / ko if ko else None,
            "kappa_rel_combined_stderr": se / ko if ko else None,
            "bins": int(bg.size), "bins_compared": int(live.sum()),
            "max_abs_z_bin": float(np.max(np.abs(zb))) if live.any() else None,
            "max_abs_bin_diff": float(np.max(np.abs(d))), "rms_bin_diff": float(np.sqrt(np.mean(d * d))),
            "bin_diff": [float(x) for x in d]}


def spawn_ranks(n, script, argv, timeout_s=3600, extra_env=None):
    """Runs `script argv` as n processes on this node, one per GPU, with the
    environment torchrun gives a rank (RANK, LOCAL_RANK, WORLD_SIZE,
    MASTER_ADDR = 127.0.0.1, a free MASTER_PORT).  Their output is passed
    through (rank 0 prints the result line); returns the largest exit code.
    A rank that fails ends the others."""
    import socket
    import subprocess
    sk = socket.socket()
    sk.bind(("127.0.0.1", 0))
    port = sk.getsockname()[1]
    sk.close()
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n), LOCAL_WORLD_SIZE=str(n),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        env.update(extra_env or {})
        procs.append(subprocess.Popen([sys.executable, script] + list(argv), env=env))
    rc = 0
    t0 = time.time()
    pending = list(procs)
    while pending:
        for pr in list(pending):
            code = pr.poll()
            if code is None:
                continue
            pending.remove(pr)
            rc = max(rc, abs(code))
            if code != 0:
                for other in pending:
                    other.kill()
        if time.time() - t0 > timeout_s:
            for pr in pending:
                pr.kill()
            rc = max(rc, 124)
        time.sleep(0.05)
    for pr in procs:
        pr.wait()
    return rc


def issue_ceiling(kernels, clocks):
    """Flights/s each phase would reach issuing one warp instruction per
    scheduler per clock (148 SMs x 4 schedulers x the sampled SM clock) at
    its measured warp instructions per flight, and the fraction reached."""
    sm_mhz = (clocks or {}).get("sm_mhz") or 1965.0
    out = {"issue_rate": "148 SMs x 4 warp instructions per clock", "sm_mhz": sm_mhz}
    for phase in ("drain", "tail"):
        prof = issue_profile(phase)
        k = kernels.get(phase) or {}
        if not prof or not k.get("flights_per_s"):
            out[phase] = None
            continue
        ceil = 148 * 4 * sm_mhz * 1e6 / prof["warp_inst_per_flight"]
        out[phase] = {"warp_inst_per_flight": prof["warp_inst_per_flight"],
                      "lanes_per_inst": prof.get("lanes_per_inst"), "ceiling_flights_per_s": ceil,
                      "achieved_flights_per_s": k["flights_per_s"], "frac": k["flights_per_s"] / ceil,
                      "source": prof.get("source")}
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    pkg = load_pkg()
    model, spec, cfg = workload(pkg)
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from oracle import oracle as O
    o = O.Oracle(model=model, spectrum=spec)
    # size each step to about 5 s of CPU work
    run = make_run(pkg, spec, 2, 0, 1, 0)
    _, _, r = o.counts(run)
    n = max(2, min(500, int(5.0 / max(r["seconds"] / 2, 1e-9))))
    run = make_run(pkg, spec, n, 0, 1, 0)
    for _ in range(args.warmup):
        o.counts(run)
    fl, sec = 0, 0.0
    for _ in range(args.steps):
        _, _, r = o.counts(run)
        fl += r["flights"]
        sec += r["seconds"]
    v = fl / sec
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": int(r["threads"]), "kind": "port",
                             "sample": f"all 20000 (mode, angle) tasks with {n} particles each per step"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_c5(args):
    """256 periodic films with one hole each, uneven sample counts (1e5-1e7),
    2000 modes, 64 bins: one batched persistent launch replayed as a CUDA graph
    against sequential plain FP64 launches (timed on a subset of films)."""
    import torch
    torch.cuda.set_device(0)
    pkg = load_pkg()
    A, synth = pkg.abi, pkg.synth
    models, nps = synth.film_batch(256, seed=0)
    spec = synth.spectrum(2000, seed=0)
    bufs = [A.GeomBuf(m) for m in models]
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=11, np_=1, temperature=300.0, nbins=64,
                     bin_omega=(0.0, 15.0 * 2 * math.pi * 1e12))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:0")
    with A.Batch([b.view for b in bufs], nps, list(range(256)), [0] * 256, spec, run) as bt:
        for _ in range(args.warmup):
            bt.run()
        ms = fl = 0.0
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            r = bt.run()
            ms += r["graph_ms"]
            fl += r["flights"]
        # per-geometry adjoint: one batched listing launch + one batched replay
        t0 = time.perf_counter()
        adj = bt.adjoint()
        adj_s = time.perf_counter() - t0
    batch_rate = fl / (ms * 1e-3)
    dks = np.concatenate([d for d in adj["dk_dp"]])
    dke = np.concatenate([e for e in adj["dk_dp_stderr"]])
    ok = ~np.isnan(dks)
    adjoint = {"wall_s": adj_s, "kernel_ms": adj["kernel_ms"], "replayed": adj["replayed"],
               "mismatched": adj["mismatched"], "geometries": len(adj["dk_dp"]),
               "surface_records": int(ok.sum()), "resolved_3sigma": int(np.sum(np.abs(dks[ok]) > 3 * dke[ok])),
               "dk_dscale_resolved_3sigma": int(np.sum(np.abs(adj["dk_dscale"]) > 3 * adj["dk_dscale_stderr"]))}
    # sequential plain FP64 runs of a subset of the films
    idx = list(range(0, 256, max(1, 256 // args.fp64_subset)))[: args.fp64_subset]
    f64_ms = f64_fl = 0.0
    for i in idx:
        with A.Handle(bufs[i].view, spec) as h:
            r64 = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=11, np_=nps[i], seed=i, precision=A.PREC_FP64,
                             temperature=300.0, nbins=64, bin_omega=(0.0, 15.0 * 2 * math.pi * 1e12))
            h.kappa(r64)
            st = h.stats()
            f64_ms += st["kernel_ms"] + st["reduce_ms"]
            f64_fl += st["flights"]
    f64_rate = f64_fl / (f64_ms * 1e-3)
    print(json.dumps({
        "metric": "phonon free-flights/s, 256-film batched screening (one CUDA-graph launch)",
        "value": batch_rate, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "256 periodic films, hole r~U(10,60) nm, period~U(100,400) nm, "
                               "thickness~U(50,300) nm, samples per film log-uniform 1e5-1e7, 2000 modes, 64 bins",
                   "samples_total": int(sum(nps) * 20000), "fp64_subset": len(idx)},
        "plain_fp64_sequential": {"value": f64_rate, "unit": UNIT, "films": len(idx),
                                  "speedup_batch_over_fp64": batch_rate / f64_rate},
        "adjoint": adjoint,
        "flights_per_step": fl / args.steps}))
    return 0


def run_structure(args):
    """C4 structures: 5 Voronoi grains in a 1 um cube (internal facets T = 0.5,
    p = 0, diffuse outer walls), or a simple-cubic lattice of 16^3 cubic voids
    (49152 triangles in the matrix grain, BVH).  20000-mode spectrum, 64 bins,
    per-mode MFP runs.  Device time of ptg_kappa (FP32 persistent kernel +
    reduction) against the plain FP64 kernel on a bounded sample (fewer
    particles per task) and, for the mesh, the FP32 kernel without the BVH."""
    import torch
    torch.cuda.set_device(0)
    pkg = load_pkg()
    A, synth = pkg.abi, pkg.synth
    if args.workload == "voronoi":
        model = synth.voronoi_box(5, box=(1000.0, 1000.0, 1000.0), seed=0, trans=0.5, spec=0.0, p_wall=0.0)
        desc = "5 Voronoi grains in a 1000^3 nm box, internal facets T=0.5 p=0, diffuse walls"
        np_default, np64 = 500, 5
    elif args.workload == "c4":
        model = synth.voronoi_box(5, box=(1000.0, 1000.0, 1000.0), seed=0, trans=0.5, spec=0.0, p_wall=0.0,
                                  tri_levels=4)
        desc = ("5 Voronoi grains in a 1000^3 nm box as a triangle mesh (43008 FP32 triangles, a BVH per "
                "grain), grain boundaries T=0.5 p=0, diffuse walls")
        np_default, np64 = 500, 1
    else:
        model = synth.cube_lattice(n=16, l=1000.0, fill=0.5, trans=0.0, spec=0.0, p_wall=0.0)
        desc = ("16^3 cubic voids (side 31.25 nm, pitch 62.5 nm) in a 1000^3 nm box, "
                "49152 triangles in the matrix grain, diffuse")
        np_default, np64 = 10, 1
    npt = args.np if args.np != 500 else np_default
    spec = synth.spectrum(20000, seed=0)
    gb = A.GeomBuf(model)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:0")

    def timed(opts, np_, prec, steps, warm):
        with A.Handle(gb.view, spec, **opts) as h:
            run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=11, np_=np_, seed=12345, precision=prec,
                             temperature=300.0, nbins=64, bin_omega=(0.0, 15.0 * 2 * math.pi * 1e12))
            for _ in range(warm):
                h.kappa(run)
            ms = fl = 0.0
            out = st = None
            for _ in range(steps):
                flush.zero_()
                torch.cuda.synchronize()
                out = h.kappa(run)
                st = h.stats()
                ms += st["kernel_ms"] + st["reduce_ms"]
                fl += st["flights"]
            return fl / (ms * 1e-3), ms / steps, fl / steps, out, st

    v, ms, fl, out, st = timed({}, npt, A.PREC_FP32, args.steps, args.warmup)
    line = {"metric": f"phonon free-flights/s, {args.workload} structure", "value": v, "unit": UNIT,
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "modes": 20000, "bins": 64, "nangle": 11,
                       "particles_per_task": npt, "samples": 20000 * 10 * npt},
            "flights_per_step": fl, "kappa": out["kappa"], "kappa_stderr": out["kappa_stderr"],
            "tests_per_flight": {"bvh_boxes": st["box_tests"] / max(st["flights"], 1),
                                 "surfaces": st["surface_tests"] / max(st["flights"], 1),
                                 "full_flight_fraction": st["full_flights"] / max(st["flights"], 1)},
            "tail": {"max_trajectory_flights": st["max_traj_flights"], "queue_drain_ms": st["drain_ms"],
                     "tail_ms": st["tail_ms"]}}
    if args.workload in ("mesh", "c4"):
        # the linear-scan comparators test every triangle of a grain per flight, one
        # trajectory per thread: a bounded sample of the 100 modes with the
        # longest MFP (short trajectories), one particle per (mode, angle) task,
        # timed for the BVH kernel too
        full = spec
        sel = np.argsort(full.mfp)[-100:]
        spec = A.Spectrum(omega=full.omega[sel], tau=full.tau[sel], vel=full.vel[sel],
                          weight=full.weight[sel], nbranch=1, rtemp=full.rtemp, vol=full.vol,
                          mfp=full.mfp[sel])
        sample = "the 100 longest-MFP modes, 1 particle per (mode, angle) task"
        vl, _, _, _, _ = timed({"bvh_leaf": -1}, np64, A.PREC_FP32, 1, 1)
        vb, _, _, _, _ = timed({}, np64, A.PREC_FP32, 1, 1)
        line["no_bvh_fp32"] = {"value": vl, "unit": UNIT, "sample": sample,
                               "bvh_speedup_same_sample": vb / vl}
    else:
        sample = f"all modes, {np64} particles per (mode, angle) task"
        vb, _, _, _, _ = timed({}, np64, A.PREC_FP32, 1, 1)
    v64, ms64, fl64, _, _ = timed({}, np64, A.PREC_FP64, 1, 0)
    line["plain_fp64"] = {"value": v64, "unit": UNIT, "sample": sample, "ms": ms64,
                          "fp32_same_sample": vb, "speedup_fp32_over_fp64_same_sample": vb / v64}
    print(json.dumps(line))
    return 0


def run_c1(args):
    """C1: the plain method on a square nanowire 100 x 100 x 1000 nm (x
    transport), fully diffuse side walls, 2000-mode spectrum, 10^5 samples
    (5 particles per (mode, angle) task), FP64 throughout, seed 0.  Timed
    three ways on the same workload: the plain FP64 GPU kernel (the
    configuration's precision), the persistent FP32 kernel, and the CPU
    oracle (OpenMP, all host threads, in a process without torch), with the
    FP64 GPU counts checked against the oracle's exactly."""
    import subprocess
    import torch
    torch.cuda.set_device(0)
    pkg = load_pkg()
    A, synth = pkg.abi, pkg.synth
    model = synth.nanowire(length=1000.0, width=100.0, height=100.0, p_side=0.0)
    spec = synth.spectrum(2000, seed=0)
    gb = A.GeomBuf(model)
    bins = dict(temperature=300.0, nbins=64, bin_omega=(0.0, 15.0 * 2 * math.pi * 1e12))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:0")
    res = {}
    with A.Handle(gb.view, spec) as h:
        for name, prec in (("fp64", A.PREC_FP64), ("fp32", A.PREC_FP32)):
            run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=11, np_=5, seed=0, precision=prec, **bins)
            for _ in range(args.warmup):
                h.kappa(run)
            ms = fl = 0.0
            for _ in range(args.steps):
                flush.zero_()
                torch.cuda.synchronize()
                out = h.kappa(run, want_counts=True)
                st = h.stats()
                ms += st["kernel_ms"] + st["reduce_ms"]
                fl += st["flights"]
            res[name] = {"value": fl / (ms * 1e-3), "ms_per_step": ms / args.steps, "kappa": out["kappa"],
                         "kappa_stderr": out["kappa_stderr"], "counts": out["counts"],
                         "flights": fl / args.steps}
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    p = subprocess.run([sys.executable, os.path.abspath(__file__), "--c1-oracle"], capture_output=True, text=True,
                       env=env, timeout=1800)
    if p.returncode != 0:
        raise RuntimeError(p.stderr[-2000:])
    orc = json.loads(p.stdout.strip().splitlines()[-1])
    counts_equal = orc["counts_sha"] == _sha(res["fp64"]["counts"])
    line = {"metric": "phonon free-flights/s, C1 square nanowire (plain method, FP64)",
            "value": res["fp64"]["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["fp64"]["ms_per_step"], "higher_is_better": True,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "nanowire 100x100x1000 nm, diffuse side walls, 2000-mode spectrum, "
                                   "64 bins, 5 particles per (mode, angle): 1e5 samples, seed 0",
                       "l2": "256 MiB written between timed steps"},
            "flights_per_step": res["fp64"]["flights"], "kappa": res["fp64"]["kappa"],
            "kappa_stderr": res["fp64"]["kappa_stderr"],
            "persistent_fp32": {"value": res["fp32"]["value"], "unit": UNIT,
                                "ms_per_step": res["fp32"]["ms_per_step"], "kappa": res["fp32"]["kappa"],
                                "kappa_stderr": res["fp32"]["kappa_stderr"]},
            "cpu_oracle": {"value": orc["value"], "unit": UNIT, "cores": orc["cores"], "seconds": orc["seconds"],
                           "kappa": orc["kappa"], "sample": "the whole C1 workload"},
            "fp64_counts_equal_oracle": counts_equal}
    print(json.dumps(line))
    return 0


def _sha(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint64).tobytes()).hexdigest()


def c1_oracle():
    """The CPU oracle on the whole C1 workload (bench.py --c1-oracle, a
    process without torch): rate, kappa and a digest of the counts."""
    pkg = load_pkg()
    A, synth = pkg.abi, pkg.synth
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from oracle import oracle as O
    model = synth.nanowire(length=1000.0, width=100.0, height=100.0, p_side=0.0)
    spec = synth.spectrum(2000, seed=0)
    o = O.Oracle(model=model, spectrum=spec)
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=11, np_=5, seed=0, precision=A.PREC_FP64,
                     temperature=300.0, nbins=64, bin_omega=(0.0, 15.0 * 2 * math.pi * 1e12))
    cnt, _, r = o.counts(run)
    k = o.kappa(run, cnt)
    print(json.dumps({"value": r["flights"] / r["seconds"], "cores": int(r["threads"]), "seconds": r["seconds"],
                      "kappa": k["kappa"], "counts_sha": _sha(cnt)}))
    return 0


def run_c3(args):
    """C3: 64 spheres (r ~ U(20, 80) nm) and 16 capped cylinders of random
    axis (r = 30 nm, length ~ U(100, 400) nm) as voids in a 1000^3 nm box,
    per-surface specularity p ~ U(0, 1), diffuse walls; 20000-mode spectrum,
    64 bins, per-mode MFP runs.  Forward kappa (device time) and the adjoint
    (forward listing pass + replay, wall time of the call) with the number of
    resolved derivatives dkappa/dp_k."""
    import torch
    torch.cuda.set_device(0)
    pkg = load_pkg()
    A, synth = pkg.abi, pkg.synth
    model = synth.spheres_cylinders_box(64, 16, l=1000.0, seed=0)
    spec = synth.spectrum(20000, seed=0)
    gb = A.GeomBuf(model)
    npt = args.np
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda:0")
    bins = dict(temperature=300.0, nbins=64, bin_omega=(0.0, 15.0 * 2 * math.pi * 1e12))
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=11, np_=npt, seed=12345, precision=A.PREC_FP32, **bins)
    with A.Handle(gb.view, spec) as h:
        for _ in range(args.warmup):
            h.kappa(run)
        ms = fl = 0.0
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            out = h.kappa(run)
            st = h.stats()
            ms += st["kernel_ms"] + st["reduce_ms"]
            fl += st["flights"]
        h.adjoint(run)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        adj = h.adjoint(run)
        adj_s = time.perf_counter() - t0
        h.kappa(A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=11, np_=2, seed=12345, precision=A.PREC_FP64, **bins))
        s64 = h.stats()
        h.kappa(A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=11, np_=2, seed=12345, precision=A.PREC_FP32, **bins))
        s32 = h.stats()
    v = fl / (ms * 1e-3)
    dk, de = adj["dk_dp"], adj["dk_dp_stderr"]
    v64 = s64["flights"] / ((s64["kernel_ms"] + s64["reduce_ms"]) * 1e-3)
    v32s = s32["flights"] / ((s32["kernel_ms"] + s32["reduce_ms"]) * 1e-3)
    print(json.dumps({
        "metric": "phonon free-flights/s, C3 spheres + random-axis capped cylinders, forward + adjoint",
        "value": v, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "64 spheres r~U(20,80) + 16 capped cylinders r=30, random axes, length~U(100,400), "
                               "voids in 1000^3 nm, per-surface p~U(0,1), diffuse walls; 20000 modes, 64 bins",
                   "particles_per_task": npt, "samples": 20000 * 10 * npt},
        "flights_per_step": fl / args.steps, "kappa": out["kappa"], "kappa_stderr": out["kappa_stderr"],
        "adjoint": {"wall_s": adj_s, "kappa": adj["kappa"], "replayed": adj["replayed"],
                    "mismatched": adj["mismatched"], "surface_records": int(dk.size),
                    "resolved_3sigma": int(np.sum(np.abs(dk) > 3 * de)), "dk_dscale": adj["dk_dscale"],
                    "dk_dscale_stderr": adj["dk_dscale_stderr"]},
        "plain_fp64": {"value": v64, "unit": UNIT, "sample": "all modes, 2 particles per (mode, angle) task",
                       "fp32_same_sample": v32s, "speedup_fp32_over_fp64_same_sample": v32s / v64}}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--np", type=int, default=500, help="particles per (mode, angle) per GPU")
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--mfp-lo", type=float, default=1e-9,
                    help="smallest bulk MFP of the spectrum [m]; 1e-9 is the metric's spectrum "
                         "(larger values remove the diffusive tail, for throughput diagnostics)")
    ap.add_argument("--workload", default="thinfilm",
                    choices=["thinfilm", "c1", "c3", "c4", "c5", "voronoi", "mesh"],
                    help="thinfilm: the metric's configuration; c3: spheres + capped cylinders with "
                         "the adjoint; c5: 256-film batched screening; c4: the Voronoi polycrystal as a "
                         "43k-triangle mesh with T=0.5 boundaries; voronoi / mesh: its polygon form and a "
                         "16^3 cube lattice of voids")
    ap.add_argument("--fp64-subset", type=int, default=16,
                    help="c5: films timed one by one with the plain FP64 kernel")
    ap.add_argument("--cpu-leg", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--c1-oracle", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--cpu-target-s", type=float, default=20.0,
                    help="seconds of CPU work the cpu_baseline leg is sized to")
    args = ap.parse_args()
    if args.cpu_leg:
        return cpu_leg(args)
    if args.c1_oracle:
        return c1_oracle()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "c5":
        return run_c5(args)
    if args.workload == "c1":
        return run_c1(args)
    if args.workload in ("voronoi", "mesh", "c4"):
        return run_structure(args)
    if args.workload == "c3":
        return run_c3(args)

    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # not launched by torchrun: start the ranks here, one per GPU
        return spawn_ranks(args.gpus, os.path.abspath(__file__), sys.argv[1:])
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        print(f"bench: WORLD_SIZE {world} differs from --gpus {args.gpus}", file=sys.stderr)
        return 2
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    pkg = load_pkg()
    A = pkg.abi
    model, spec, cfg = workload(pkg, np_per_task=args.np, mfp_lo=args.mfp_lo)
    if args.mfp_lo != 1e-9:
        cfg["workload"] += f"; bulk MFPs from {args.mfp_lo:g} m (diagnostic, not the metric's spectrum)"
    gb = A.GeomBuf(model)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def maxall(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sumall(x):
        if dist is None:
            return x
        t = torch.tensor([float(x)], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t)
        return float(t.item())

    h = A.Handle(gb.view, spec, device=local)
    run32 = make_run(pkg, spec, args.np * world, rank, world, A.PREC_FP32)
    for _ in range(args.warmup):
        h.kappa(run32)
    clk = ClockSampler(local)
    clk.start()
    barrier()
    dev_ms = kern_ms = wall = 0.0
    drain_k_ms = tail_k_ms = 0.0
    flights = tail_flights = tail_phonons = 0
    h2d = d2h = 0
    out = None
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = h.kappa(run32)
        t1 = time.perf_counter()
        st = h.stats()
        wall += t1 - t0
        kern_ms += st["kernel_ms"]
        dev_ms += st["kernel_ms"] + st["reduce_ms"]
        flights += st["flights"]
        drain_k_ms += st["drain_kernel_ms"]
        tail_k_ms += st["tail_kernel_ms"]
        tail_flights += st["tail_flights"]
        tail_phonons += st["tail_phonons"]
        h2d, d2h = st["h2d_bytes"], st["d2h_bytes"]
    barrier()
    clocks = clk.stop()
    launches_per_step = st["launches"]
    grid, block = st["grid"], st["block"]
    dev_ms, kern_ms, wall = maxall(dev_ms), maxall(kern_ms), maxall(wall)
    flights = sumall(flights)
    value = flights / (dev_ms * 1e-3)
    e2e = flights / wall

    # plain FP64 one-phonon-per-thread comparator on the same workload
    run64 = make_run(pkg, spec, args.np * world, rank, world, A.PREC_FP64)
    if args.fp64_steps > 0:
        h.kappa(run64)
    barrier()
    f64_ms, f64_flights = 0.0, 0
    for _ in range(args.fp64_steps):
        flush.zero_()
        torch.cuda.synchronize()
        h.kappa(run64)
        s64 = h.stats()
        f64_ms += s64["kernel_ms"] + s64["reduce_ms"]
        f64_flights += s64["flights"]
    barrier()
    f64_ms = maxall(f64_ms)
    f64_flights = sumall(f64_flights)
    fp64_value = f64_flights / (f64_ms * 1e-3) if f64_ms > 0 else None

    result = None
    if rank == 0:
        peak, peak_kind = measured_peaks()
        per_launch_flights = flights / world / args.steps
        # the transport is two launches of k_persistent per step: the drain
        # phase (queue) and the tail phase (handed-over phonons, after
        # two small kernels that order them, timed with the tail); the
        # roofline is the longer one's, with its own flights and CUDA-event time
        kernels = {
            "drain": {"ms_per_step": drain_k_ms / args.steps,
                      "flights_per_step": (flights / world - tail_flights) / args.steps},
            "tail": {"ms_per_step": tail_k_ms / args.steps, "flights_per_step": tail_flights / args.steps,
                     "phonons_per_step": tail_phonons / args.steps},
        }
        for k in kernels.values():
            k["flights_per_s"] = k["flights_per_step"] / (k["ms_per_step"] * 1e-3) if k["ms_per_step"] > 0 else None
        dom = "drain" if kernels["drain"]["ms_per_step"] >= kernels["tail"]["ms_per_step"] else "tail"
        launch_s = kernels[dom]["ms_per_step"] * 1e-3
        dom_flights = kernels[dom]["flights_per_step"]
        achieved = BYTES_PER_FLIGHT * dom_flights / launch_s / 1e9
        traffic, traffic_case = dram_traffic(dom)
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded film geometry and 2000-mode spectrum",
            "config": dict(cfg, samples_total=cfg["samples_per_gpu"] * world,
                           parallelism=f"{world} GPU(s), particle-strided shards, counts all-reduced"),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches_per_step * args.steps),
            "roofline": {"bound": "hbm",
                         "model": "state-traffic model of one free flight (64 B: 32 B of FP32 state read and "
                                  "written); the kernels keep the state in registers, so the measured DRAM "
                                  "traffic (traffic) is far below it and the model binds nothing: the phases "
                                  "are bound by instruction issue and latency (issue_ceiling)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": f"{peak_kind} hbm_gbs",
                         "bytes_per_flight": BYTES_PER_FLIGHT,
                         "traffic": traffic, "traffic_case": traffic_case,
                         "kernel": f"k_persistent ({dom} phase)", "launch_ms": launch_s * 1e3,
                         "flights_per_launch": dom_flights, "grid": grid, "block": block},
            "issue_ceiling": issue_ceiling(kernels, clocks),
            "fp32_roofline": {"flops_per_flight": FLOPS_PER_FLIGHT_C2,
                              "achieved_tflops": FLOPS_PER_FLIGHT_C2 * dom_flights / launch_s / 1e12,
                              "peak_tflops_nominal": FP32_PEAK_NOMINAL},
            "kernels": kernels,
            "plain_fp64": ({"value": fp64_value, "unit": UNIT, "ms_per_step": f64_ms / args.fp64_steps,
                            "speedup_fp32_over_fp64": value / fp64_value} if fp64_value else None),
            "flights_per_step": per_launch_flights,
            "tail": {"max_trajectory_flights": st["max_traj_flights"], "queue_drain_ms": st["drain_ms"],
                     "tail_ms": st["tail_ms"]},
            # how the flights were taken: with the full intersection test by
            # one lane, as p-p flights of cooperative rounds, or the rest (the
            # safe-ball fast path and the hit that ends a cooperative round)
            "paths": {"full_test": st["full_flights"], "cooperative": st["coop_flights"],
                      "fast_or_round_end": st["flights"] - st["full_flights"] - st["coop_flights"],
                      "coop_rounds": st["coop_rounds"], "safe_balls": st["safe_balls"]},
            "kappa": out["kappa"] if out else None,
            "kappa_stderr": out["kappa_stderr"] if out else None,
            "kappa_rel_stderr": (out["kappa_stderr"] / out["kappa"]) if out and out["kappa"] else None,
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu:
            leg = cpu_baseline(args)
            result["cpu_baseline"] = {k: leg[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                          "seconds", "flights", "probe_rate")}
            result["parity"] = dict(parity(out, leg), oracle_sample=leg["parity_sample"],
                                    oracle_run_rate=leg["parity_run_rate"])
    h.close()
    del flush
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if result is not None:
        print(json.dumps(result))
    return 0


if __name__ == "__main__":
    sys.exit(main())
