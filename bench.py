#!/usr/bin/env python
"""Benchmark of the B200 line-of-sight integrator.

Workload (default, "config3"): Nside 128/256/512/1024 over 4 shells
to 30 kpc with 0.01 kpc radial steps (21.6 G LOS samples per frequency),
512^3 FP32 random-field grids (B_rnd 3 components + lognormal n_e) on a
40 x 40 x 10 kpc box plus the analytic spiral B_reg and CRE_ana, three
frequencies 0.408 / 1.4 / 30 GHz in the reference's Pipeline order (the
first pass also produces DM and FD).  One step = the three frequency passes.

Reported: LOS samples/s of the FP32-compensated form (value, inputs resident
in HBM), ms per Nside-1024 map, the plain-FP64 GPU form on the same inputs,
the FP32C-vs-FP64 map errors, an end-to-end number through the host-buffer
C ABI (grid upload + maps download inside the timed region), the roofline of
the shell-integration kernel, and the reference CPU integrator timed on a
bounded sample on this host's cores.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LOS samples/s & ms per Nside-1024 map (FP32-comp vs FP64 GPU), adjoint/fwd ratio"
UNIT = "LOS samples/s"
BYTES_PER_SAMPLE = {"fp32c": 128, "fp64": 256}  # 8 corners x 4 gridded components

WORKLOADS = {
    "config3": dict(nside_shells=[128, 256, 512, 1024], r_max_kpc=30.0, res_kpc=0.01,
                    freqs_ghz=[0.408, 1.4, 30.0], grid_n=512, seeds=(3, 4)),
    "small": dict(nside_shells=[32, 64, 128, 256], r_max_kpc=30.0, res_kpc=0.01,
                  freqs_ghz=[0.408, 1.4, 30.0], grid_n=128, seeds=(3, 4)),
    # the case kernel captures run on: grid records (268 MB FP32) above L2,
    # an Nside-512 outer shell (one lane per pixel, as the config-3 outer
    # shells), about 15 ms per launch
    "profile": dict(nside_shells=[64, 128, 256, 512], r_max_kpc=30.0, res_kpc=0.01,
                    freqs_ghz=[0.408, 1.4, 30.0], grid_n=256, seeds=(3, 4)),
    # config 3's shells and output Nside on 0.5-kpc rays and a 64^3 grid: the
    # shell merges (the same launches and map sizes as config 3) take most
    # of the step; the case the merge kernels are captured on
    "merges": dict(nside_shells=[128, 256, 512, 1024], r_max_kpc=0.5, res_kpc=0.01,
                   freqs_ghz=[0.408, 1.4, 30.0], grid_n=64, seeds=(3, 4)),
}
# The bounded sample both arms time like for like: the first frequency pass
# (DM + FD + synchrotron) of the workload over its innermost shell only,
# with its own radii, Nside and sample positions, on the same grids (config
# 3: Nside 128, 0-3.75 kpc, 7.4e7 LOS samples, about 1.5 s of the
# reference on 16 host threads per step).
SUB_SHELLS = 1


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_figure(name, key):
    """A figure of the integration kernel from the committed ncu summary
    profiles/<name>: the number on its line '<key>: <value>', or None."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith(key + ":"):
            return float(line.split(":", 1)[1].split()[0])
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def setup_dist(args, gpu=True):
    from hammurabix_b200 import replicas
    ws, rank, local = replicas.env()
    if ws > 1 and gpu:
        import torch
        torch.cuda.set_device(local)
        return replicas.init("nccl", 120, torch.device("cuda", local))
    return replicas.init("gloo", 120) if ws > 1 else (ws, rank, local)


def make_passes(wl, nside_shells=None):
    from hammurabix_b200 import workloads as W
    return W.config_grid(nside_shells or wl["nside_shells"], wl["r_max_kpc"], wl["res_kpc"],
                         wl["freqs_ghz"])


def sub_workload(wl):
    """Obs of the bounded sample: pass 1 of the workload restricted to its
    SUB_SHELLS innermost shells (the same shell radii, Nsides and radial
    steps), output maps at the outermost of those Nsides."""
    from hammurabix_b200 import workloads as W
    full = make_passes(wl)[0]
    o = W.make_obs(wl["nside_shells"][:SUB_SHELLS], wl["r_max_kpc"], wl["res_kpc"],
                   freq_ghz=full.sync_freq / 1e9)
    for i in range(SUB_SHELLS + 1):
        o.radii_shell[i] = full.radii_shell[i]
    return o


def sub_workload_text(wl):
    from hammurabix_b200 import workloads as W
    from hammurabix_b200 import units as U
    o = sub_workload(wl)
    shells = "/".join(str(o.nside_shell[i]) for i in range(o.total_shell))
    what = "innermost shell" if SUB_SHELLS == 1 else f"{SUB_SHELLS} innermost shells"
    return (f"pass 1 ({o.sync_freq / 1e9:g} GHz with DM + FD) over the workload's {what} "
            f"(Nside {shells}, 0-{o.radii_shell[SUB_SHELLS] / U.kpc:g} kpc), "
            f"same {wl['grid_n']}^3 grids: {W.samples_of(o)} LOS samples, "
            f"Integrator::write_grid only")


def cpu_baseline(wl, host_fields, steps=1):
    """The reference's FP64 OpenMP integrator (oracle/_ref, compiled from the
    reference sources) on the bounded sample (sub_workload), all host cores:
    an exact subset of the workload's samples, which the GPU forms also time."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from hammurabix_b200 import workloads as W
    ref = pyoracle.Reference()
    threads = os.cpu_count()
    o = sub_workload(wl)
    grids = W.grids_dict(wl["grid_n"], *host_fields)
    m = W.grid_models()
    times = []
    for _ in range(steps):
        _, secs = ref.write_grid(o, m, grids, nthreads=threads)
        times.append(secs)
    return {"samples": W.samples_of(o), "seconds": times, "threads": threads,
            "sample": sub_workload_text(wl)}


def config_of(args, wl, ws, shard):
    """The workload's config entry, the same for both arms."""
    n = wl["grid_n"]
    passes = make_passes(wl)
    from hammurabix_b200 import workloads as W
    return {"workload": f"{args.workload}: Nside "
                        f"{'/'.join(str(s) for s in wl['nside_shells'])} x "
                        f"{len(wl['nside_shells'])} shells to {wl['r_max_kpc']:g} kpc, "
                        f"{wl['res_kpc']} kpc steps, {n}^3 FP32 grids, "
                        f"{'/'.join(str(f) for f in wl['freqs_ghz'])} GHz",
            "samples_per_step": sum(W.samples_of(o) for o in passes),
            "passes_per_step": len(passes),
            "l2": f"inputs larger than L2 (grids {4 * 4 * n ** 3 / 1e9:.2f} GB FP32)",
            "parallelism": (f"shell pixels split over {ws} GPUs, FD all-reduce per shell"
                            if shard else f"replicas x{ws}" if ws > 1 else "1 GPU")}


def run_reference_arm(args, wl):
    """The reference's own CPU integrator on the workload's config: each
    step is one Integrator::write_grid of the bounded sample (sub_workload)
    on all host cores; the value is its LOS samples/s."""
    # CPU only: no process group is needed; rank 0 alone runs and prints
    from hammurabix_b200 import replicas
    from hammurabix_b200 import workloads as W
    ws, rank, _ = replicas.env()
    if rank != 0:
        return
    b = W.random_grids_torch(wl["grid_n"], *wl["seeds"], device="cpu")
    host = [t.double().numpy().reshape(-1) for t in b]
    del b
    cb = cpu_baseline(wl, host, steps=args.warmup + args.steps)
    secs = cb["seconds"][args.warmup:]
    t = sum(secs) / len(secs)
    value = cb["samples"] / t
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "strong" if ws > 1 else "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_of(args, wl, ws, ws > 1 and args.mode == "shard"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cb["threads"],
                         "kind": "reference", "sample": cb["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def generators(args, dev, stream, torch):
    """Device time of the random-field generators on the config-3 grid
    geometry (--rfg-grid cells per axis, 512 by default, over the
    40 x 40 x 10 kpc box): Brnd_es with the
    template's spectrum (rms 0.8 muG, k0 10, k1 0.1, a0 1.7, rho 3) along the
    analytic spiral, and TErnd_dft (rms 0.01, k0 0.05, a0 -11/3).  Each call
    is synchronous: k-space fill, cuFFT transforms (6 for Brnd_es, 1 for
    TErnd_dft), the variance reduction and the real-space passes."""
    import time as _t
    from hammurabix_b200 import abi, workloads as W
    from hammurabix_b200 import units as U
    from hammurabix_b200.integrator import Integrator
    n = args.rfg_grid
    desc = W.grid_desc(n)
    obs = (-8.3 * U.kpc, 0.0, 0.006 * U.kpc)
    es = abi.BrndEs(rms=0.8 * U.muGauss, k0=10.0, k1=0.1, a0=1.7, a1=0.0, rho=3.0,
                    r0=8 * U.kpc, z0=1 * U.kpc)
    dft = abi.TerndDft(rms=0.01, k0=0.05, a0=-11.0 / 3.0, r0=8 * U.kpc, z0=1 * U.kpc)
    ig = Integrator("fp32c")
    ig.set_stream(stream.cuda_stream)
    ig.set_models(W.spiral_models())
    res = {}
    for name, fn in (("brnd_es", lambda k: ig.generate_brnd_es(desc, es, obs, 11 + k)),
                     ("ternd_dft", lambda k: ig.generate_ternd_dft(desc, dft, obs, 21 + k))):
        fn(0)                              # plans, workspace, first-touch
        ts = []
        for k in range(args.rfg_steps):
            torch.cuda.synchronize(dev)
            t0 = _t.perf_counter()
            fn(k + 1)                      # synchronous on the handle's stream
            ts.append(_t.perf_counter() - t0)
        res[f"{name}_ms"] = 1e3 * sum(ts) / len(ts)
    ig.close()
    res["grid"] = f"{n}^3"
    res["cells_per_s_brnd_es"] = n ** 3 / (res["brnd_es_ms"] / 1e3)
    return res


def adjoint_ratio(args, dev, stream, torch, prec="fp64"):
    """Adjoint vs forward device time on the config-4 workload: Nside
    64/128/256 over 3 shells to 30 kpc, 256^3 grids (B read as Grid_brnd,
    n_e fluctuations as Grid_ternd on the exponential disk), spiral B, CRE_ana,
    one 23 GHz pass with DM and FD; form `prec` with per-shell checkpointing.
    The adjoint produces dL/d(8 parameters) and dL/d(every B and n_e voxel)."""
    from hammurabix_b200 import abi, workloads as W
    from hammurabix_b200.integrator import Integrator
    n = 256
    bx, by, bz, ne = W.random_grids_torch(n, 1, 2, device=dev)
    grids = [t.double().reshape(-1).contiguous() for t in (bx, by, bz)]
    dne = (ne.double().reshape(-1) - 0.03).contiguous()
    del bx, by, bz, ne
    desc = W.grid_desc(n)
    m = W.spiral_models()
    m.brnd = abi.HXG_BRND_GRID
    m.tereg = abi.HXG_TEREG_EXPDISK
    m.ternd = abi.HXG_TERND_GRID
    o = W.make_obs([64, 128, 256], 30.0, 0.01, freq_ghz=23.0)
    ig = Integrator(prec)
    ig.set_stream(stream.cuda_stream)
    ig.set_models(m)
    ig.upload_grid_device(abi.HXG_FIELD_BRND, desc, grids)
    ig.upload_grid_device(abi.HXG_FIELD_TERND, desc, [dne])
    ig.set_checkpointing(True)
    npx = abi.npix(256)
    outs = [torch.zeros(npx, dtype=torch.float64, device=dev) for _ in range(5)]
    g = [torch.randn(npx, dtype=torch.float64, device=dev, generator=torch.Generator(
        device=dev).manual_seed(5 + k)) for k in range(5)]
    gpar = torch.zeros(abi.HXG_NUM_PARAMS, dtype=torch.float64, device=dev)
    gb = [torch.zeros(n ** 3, dtype=torch.float64, device=dev) for _ in range(3)]
    gne = torch.zeros(n ** 3, dtype=torch.float64, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    fwd, adj = [], []
    for it in range(1 + args.adjoint_steps):
        torch.cuda.synchronize(dev)
        ev[0].record(stream)
        ig.write_grid_device(o, *outs)
        ev[1].record(stream)
        ig.adjoint_device(o, *g, grad_params=gpar, grad_b=gb, grad_ne=gne)
        ev[2].record(stream)
        torch.cuda.synchronize(dev)
        if it > 0:
            fwd.append(ev[0].elapsed_time(ev[1]))
            adj.append(ev[1].elapsed_time(ev[2]))
    # the same forward without the checkpoint stores
    ig.set_checkpointing(False)
    plain = []
    for it in range(1 + args.adjoint_steps):
        torch.cuda.synchronize(dev)
        ev[0].record(stream)
        ig.write_grid_device(o, *outs)
        ev[1].record(stream)
        torch.cuda.synchronize(dev)
        if it > 0:
            plain.append(ev[0].elapsed_time(ev[1]))
    ig.close()
    f, a, fp = sum(fwd) / len(fwd), sum(adj) / len(adj), sum(plain) / len(plain)
    return {"workload": "config4: Nside 64/128/256 x 3 shells to 30 kpc, 256^3 grids, "
                        f"23 GHz + DM + FD, {prec.upper()} form",
            "forward_ms": f, "adjoint_ms": a, "ratio": a / f,
            "forward_plain_ms": fp, "ratio_vs_plain_forward": a / fp,
            "checkpoint_overhead": f / fp - 1.0,
            "samples": W.samples_of(o)}


def batch_config5(args, dev, stream, torch):
    """Config-5 batch: 256 parameter sets (seed 7: spiral b0 ~ U[2,8] muG,
    pitch ~ U[-40,-5] deg, h_B ~ U[0.5,2] kpc) x 3 frequencies (0.408, 1.4,
    30 GHz; the 30-GHz pass also makes DM and FD, as the reference pipeline
    runs its last frequency first with them), 1-3 shells of Nside 64/128/256
    to r_max ~ U[15,30] kpc at 0.01 kpc steps, one shared 256^3 FP32 random
    grid.  One graph-captured batch (persistent shell kernel per shell
    level, launch shape autotuned) against a loop of write_grid_device
    calls over the same 768 passes."""
    import numpy as np
    from hammurabix_b200 import abi, workloads as W
    from hammurabix_b200.integrator import Integrator
    n = 256
    bx, by, bz, ne = W.random_grids_torch(n, 5, 6, device=dev)
    f64 = [t.double().reshape(-1).contiguous() for t in (bx, by, bz, ne)]
    del bx, by, bz, ne
    rng = np.random.Generator(np.random.PCG64(7))
    entries = []
    for _ in range(args.batch_sets):
        m = W.grid_models(W.spiral_models(b0_muG=rng.uniform(2, 8), pitch_deg=rng.uniform(-40, -5),
                                          hb_kpc=rng.uniform(0.5, 2)))
        nsh = int(rng.integers(1, 4))
        rmax = rng.uniform(15, 30)
        for k, f in enumerate((30.0, 1.4, 0.408)):
            o = W.make_obs([64 * 2 ** s for s in range(nsh)], rmax, 0.01, freq_ghz=f,
                           do_dm=(k == 0), do_fd=(k == 0))
            ndm, nfd, nsy = abi.obs_output_sizes(o)
            z = lambda c: torch.zeros(c, dtype=torch.float64, device=dev) if c else None
            entries.append((m, o, {"dm": z(ndm), "fd": z(nfd), "is": z(nsy), "qs": z(nsy),
                                   "us": z(nsy)}))
    ig = Integrator("fp32c")
    ig.set_stream(stream.cuda_stream)
    ig.set_models(entries[0][0])
    ig.upload_grid_device(abi.HXG_FIELD_BRND, W.grid_desc(n), f64[:3])
    ig.upload_grid_device(abi.HXG_FIELD_TEREG, W.grid_desc(n), f64[3:])
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn, k):
        fn()
        torch.cuda.synchronize(dev)
        ev[0].record(stream)
        for _ in range(k):
            fn()
        ev[1].record(stream)
        torch.cuda.synchronize(dev)
        return ev[0].elapsed_time(ev[1]) / k

    def loop():
        for m, o, d in entries:
            ig.set_models(m)
            ig.write_grid_device(o, d["dm"], d["fd"], d["is"], d["qs"], d["us"])

    loop_ms = timed(loop, args.batch_steps)
    b = ig.batch(entries, tune=True)
    info = b.info()
    batch_ms = timed(b.run, args.batch_steps)
    b.close()
    ig.close()
    S = info["samples"]
    return {"workload": f"config5: {args.batch_sets} spiral parameter sets x 3 frequencies, 1-3 shells of "
                        "Nside 64/128/256 to 15-30 kpc, 0.01 kpc steps, 256^3 FP32 grid, FP32C",
            "passes": len(entries), "samples": S, "batch_ms": batch_ms, "loop_ms": loop_ms,
            "batch_samples_per_s": S / (batch_ms / 1e3), "loop_samples_per_s": S / (loop_ms / 1e3),
            "batch_speedup_vs_loop": loop_ms / batch_ms, "tuned_shape": info}


def rel_err(a, b):
    d = (a - b).abs().max().item()
    s = b.abs().max().item()
    return d / s if s > 0 else d


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="config3", choices=sorted(WORKLOADS))
    ap.add_argument("--fp64-steps", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=16)
    ap.add_argument("--e2e64-steps", type=int, default=3)
    ap.add_argument("--sub-steps", type=int, default=5,
                    help="timed repetitions of the bounded sample in each GPU form")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--adjoint-steps", type=int, default=2)
    ap.add_argument("--batch-steps", type=int, default=2)
    ap.add_argument("--batch-sets", type=int, default=256,
                    help="parameter sets of the config-5 batch (256 in config 5)")
    ap.add_argument("--rfg-steps", type=int, default=2)
    ap.add_argument("--rfg-grid", type=int, default=WORKLOADS["config3"]["grid_n"],
                    help="cells per axis of the generator timing grid")
    ap.add_argument("--mode", default="shard", choices=["shard", "replicas"],
                    help="N > 1: split each pass's shell pixels across the ranks with one FD "
                         "all-reduce per shell (shard, strong scaling) or run N independent "
                         "copies (replicas, weak scaling)")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference_arm(args, wl)

    import numpy as np
    import torch
    from hammurabix_b200 import abi, workloads as W
    from hammurabix_b200.integrator import Integrator

    from hammurabix_b200 import replicas, sharded
    ws, rank, local = setup_dist(args)
    shard = ws > 1 and args.mode == "shard"
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # a dedicated stream: the library launches on it and the CUDA events
    # that time the step are recorded on it
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    n = wl["grid_n"]
    t0 = time.time()
    fields = W.random_grids_torch(n, *wl["seeds"], device=dev)
    f64 = [t.double().reshape(-1).contiguous() for t in fields]
    del fields
    log(f"[rank {rank}] grids {n}^3 generated in {time.time() - t0:.1f}s")
    desc = W.grid_desc(n)
    models = W.grid_models()
    passes = make_passes(wl)
    samples_step = sum(W.samples_of(o) for o in passes)
    nout = max(wl["nside_shells"])
    npx = abi.npix(nout)

    def maps5():
        return [torch.zeros(npx, dtype=torch.float64, device=dev) for _ in range(5)]

    def outputs():
        """One set of the five maps per pass: the fused passes write theirs
        in the same traversal."""
        return [maps5() for _ in passes]

    def make_integ(prec):
        ig = Integrator(prec, device=local)
        ig.set_stream(stream.cuda_stream)
        ig.set_models(models)
        ig.upload_grid_device(abi.HXG_FIELD_BRND, desc, f64[:3])
        ig.upload_grid_device(abi.HXG_FIELD_TEREG, desc, f64[3:])
        return ig

    def sel(o, m):
        return [m[0] if o.do_dm else None, m[1] if o.do_fd else None, m[2], m[3], m[4]]

    # shard mode: shell maps for the per-shell exchange, summed with NCCL on
    # the launch stream (torch's current stream)
    shell_tmp = None
    if shard:
        import torch.distributed as dist
        nmax = max(abi.npix(n) for n in wl["nside_shells"])
        shell_tmp = sharded.make_shell_maps(
            nmax, lambda n: torch.zeros(n, dtype=torch.float64, device=dev))

        def reduce_sum(t):
            dist.all_reduce(t)

        def reduce_root(t):
            dist.reduce(t, dst=0)

    def step(ig, outs):
        """One config-3 step: the frequency passes in the Pipeline's order,
        fused into one traversal per shell where the form allows (FP32C)."""
        if shard:
            sharded.write_passes_sharded(ig, passes, [dict(zip(sharded.MAPS, m)) for m in outs],
                                         shell_tmp, rank, ws, reduce_sum, reduce_root)
        else:
            ig.write_grid_multi_device([(o, sel(o, m)) for o, m in zip(passes, outs)])

    def step_one_by_one(ig, outs):
        """The passes one write_grid each, as the reference's Pipeline runs
        them (the FP32C form's precision change alone)."""
        for o, m in zip(passes, outs):
            ig.write_grid_device(o, *sel(o, m))

    def barrier():
        torch.cuda.synchronize(dev)
        replicas.barrier(ws)

    def timed(ig, outs, k, fn=None):
        fn = fn or step
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        barrier()
        ev0.record(stream)
        for _ in range(k):
            fn(ig, outs)
        ev1.record(stream)
        barrier()
        return ev0.elapsed_time(ev1) / 1e3

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, ws, dev)

    # ---- FP32-compensated form: the product path ------------------------
    ig32 = make_integ("fp32c")
    out32 = outputs()
    for _ in range(args.warmup):
        step(ig32, out32)
    ig32.set_timing(True)
    lc0 = ig32.launch_count()
    with ClockSampler(local) as clk:
        t32 = max_over_ranks(timed(ig32, out32, args.steps))
    launches = ig32.launch_count() - lc0
    kms, klaunch, ksamples = ig32.get_timing()
    ig32.set_timing(False)
    # shard: the N ranks together did one job's steps; replicas: N jobs
    value = (samples_step * args.steps / t32 if shard
             else replicas.throughput(samples_step * args.steps, ws, t32))
    ms_step = t32 / args.steps * 1e3
    log(f"[rank {rank}] fp32c: {ms_step:.1f} ms/step, {value:.4g} samples/s")

    # ---- the same FP32C passes one by one (the precision change alone) ------
    one_by_one = None
    if not shard and args.fp64_steps > 0:
        step_one_by_one(ig32, out32)
        t1 = max_over_ranks(timed(ig32, out32, args.fp64_steps, step_one_by_one))
        ms1 = t1 / args.fp64_steps * 1e3
        one_by_one = {"ms_per_step": ms1, "ms_per_map": ms1 / len(passes),
                      "samples_per_s": ws * samples_step / (ms1 / 1e3)}
        log(f"[rank {rank}] fp32c passes one by one: {ms1:.1f} ms/step")

    # ---- plain FP64 GPU form on the same inputs ----------------------------
    fp64 = None
    errs = None
    if args.fp64_steps > 0:
        ig64 = make_integ("fp64")
        out64 = outputs()
        step(ig64, out64)
        ig64.set_timing(True)
        t64 = max_over_ranks(timed(ig64, out64, args.fp64_steps))
        k64ms, _, k64s = ig64.get_timing()
        ig64.set_timing(False)
        ms64 = t64 / args.fp64_steps * 1e3
        fp64 = {"ms_per_step": ms64, "ms_per_map": ms64 / len(passes),
                "samples_per_s": (1 if shard else ws) * samples_step / (ms64 / 1e3),
                "kernel_samples_per_s": k64s / (k64ms / 1e3) if k64ms > 0 else None}
        # errors of the last pass (0.408 GHz, sync only) and of the first
        # pass's DM/FD: rerun pass 0 and the last pass in both forms
        errs = {}
        for idx in (0, len(passes) - 1):
            o = passes[idx]
            a, b = out32[idx], maps5()      # the fused FP32C step's maps of this pass
            ig64.write_grid_device(o, *sel(o, b))
            torch.cuda.synchronize(dev)
            tag = f"{o.sync_freq / 1e9:g}GHz"
            for j, k in enumerate(("dm", "fd", "I", "Q", "U")):
                if (j == 0 and not o.do_dm) or (j == 1 and not o.do_fd):
                    continue
                errs[f"{k}@{tag}" if j >= 2 else k] = rel_err(a[j], b[j])
        ig64.close()
        del out64
        log(f"[rank {rank}] fp64: {ms64:.1f} ms/step; errors {errs}")

    # ---- the bounded sample, timed like for like with the CPU reference -----------
    sub = None
    if args.sub_steps > 0 and not shard:
        osub = sub_workload(wl)
        nsub = abi.npix(osub.nside_dm)
        sub = {"sample": sub_workload_text(wl), "samples": W.samples_of(osub),
               "valid_samples": sum(W.valid_samples(osub))}
        for prec in ("fp64", "fp32c"):
            ig_ = make_integ(prec)
            m5 = [torch.zeros(nsub, dtype=torch.float64, device=dev) for _ in range(5)]
            ig_.write_grid_device(osub, *m5)
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            barrier()
            ev0.record(stream)
            for _ in range(args.sub_steps):
                ig_.write_grid_device(osub, *m5)
            ev1.record(stream)
            barrier()
            ms = ev0.elapsed_time(ev1) / args.sub_steps
            ig_.close()
            sub[f"{prec}_ms"] = ms
            sub[f"{prec}_samples_per_s"] = sub["samples"] / (ms / 1e3)
        log(f"[rank {rank}] bounded sample: {sub}")

    # ---- end to end through the host-buffer C ABI -----------------------------
    def e2e_leg(prec, nsteps_timed):
        """Step throughput through the host-buffer C ABI in form `prec`:
        every step uploads its grids (the workload's FP32 grids, through
        hxg_upload_grid_f32) from pinned host memory and reads its maps back
        inside the timed region."""
        pinned = [torch.empty(t.numel(), dtype=torch.float32, pin_memory=True) for t in f64]
        for p, t in zip(pinned, f64):
            p.copy_(t)   # exact: the values are FP32 numbers
        hosts = [p.numpy() for p in pinned]
        keys = ("dm", "fd", "is", "qs", "us")

        def e2e_integ(s):
            ig_ = Integrator(prec, device=local)
            ig_.set_stream(s.cuda_stream)
            ig_.set_models(models)
            return ig_

        def read_back(outs, pinned_out):
            for o, m, po in zip(passes, outs, pinned_out):
                for k, t in zip(keys, sel(o, m)):
                    if t is not None:
                        torch.from_numpy(po[k]).copy_(t, non_blocking=True)

        def upload(ig_):
            ig_.upload_grid(abi.HXG_FIELD_BRND, desc, hosts[:3])
            ig_.upload_grid(abi.HXG_FIELD_TEREG, desc, hosts[3:])

        # sharded (N > 1): every rank takes the same collective steps in the
        # same order -- one handle, one stream, steps one after another,
        # device maps read back by torch copies
        e2e_streams = [stream]
        iges, e2e_outs, pinned_outs = [], [], []
        if shard:
            iges = [e2e_integ(s) for s in e2e_streams]
            e2e_outs = [outputs() for _ in iges]
            pinned_outs = [[{k: torch.empty(npx, dtype=torch.float64, pin_memory=True).numpy()
                             for k in keys} for _ in passes] for _ in iges]

        def e2e_run(nsteps):
            ig_, s_ = iges[0], e2e_streams[0]
            upload(ig_)
            for k in range(nsteps):
                with torch.cuda.stream(s_):
                    step(ig_, e2e_outs[0])
                    read_back(e2e_outs[0], pinned_outs[0])
                s_.synchronize()
                if k + 1 < nsteps:
                    upload(ig_)
            torch.cuda.synchronize(dev)

        # one process per GPU, N = 1 (the replicas mode too): the host-buffer
        # C ABI, as a host application calls it -- hxg_upload_grid_f32 from
        # pinned host grids and hxg_write_grid_multi_host into pinned host
        # maps, each call returning when its copies are done -- with two
        # handles driven by two host threads, so that one handle's upload
        # and read-back cross PCIe while the other one computes
        host_outs = ([[{k: torch.empty(npx, dtype=torch.float64, pin_memory=True).numpy()
                        for k in keys} for _ in passes] for _ in range(2)]
                     if not shard else [])

        def e2e_run_host(nsteps):
            import threading
            errs = []
            first_up = threading.Event()

            def worker(t):
                try:
                    ig_ = host_iges[t]
                    if t == 1:
                        first_up.wait()     # stagger: handle 1 uploads while 0 computes
                    for k in range(t, nsteps, 2):
                        upload(ig_)
                        if k == 0:
                            first_up.set()
                        ig_.write_grid_multi(passes, out=host_outs[t])
                except BaseException as e:  # noqa: BLE001 -- re-raised below
                    errs.append(e)
                    first_up.set()
            ths = [threading.Thread(target=worker, args=(t,)) for t in range(2)]
            for th in ths:
                th.start()
            for th in ths:
                th.join()
            if errs:
                raise errs[0]

        use_host = not shard
        if use_host:
            host_iges = []
            for _ in range(2):
                ig_ = Integrator(prec, device=local)
                ig_.set_models(models)
                host_iges.append(ig_)
            iges = host_iges
            run = e2e_run_host
        else:
            run = e2e_run
        run(2)
        barrier()
        te0 = time.perf_counter()
        run(nsteps_timed)
        barrier()
        te = max_over_ranks((time.perf_counter() - te0) / nsteps_timed)
        h2d = sum(h.nbytes for h in hosts)
        d2h = sum(8 * (abi.npix(o.nside_dm) * o.do_dm + abi.npix(o.nside_fd) * o.do_fd
                       + 3 * abi.npix(o.nside_sync)) for o in passes)
        res = {"value": (1 if shard else ws) * samples_step / te, "unit": UNIT,
               "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": te * 1e3,
               "api": ("hxg_upload_grid_f32 + hxg_write_grid_multi_host (host buffers)"
                       if use_host else
                       "hxg_upload_grid_f32 + sharded write_grid (device maps, torch D2H)"),
               "overlap": ("two handles driven by two host threads: one handle's upload and "
                           "read-back overlap the other's compute") if use_host
               else "none"}
        for ig_ in iges:
            ig_.close()
        del pinned, hosts, pinned_outs, host_outs
        log(f"[rank {rank}] e2e {prec}: {te * 1e3:.1f} ms/step")
        return res

    e2e = e2e_leg("fp32c", args.e2e_steps) if args.e2e_steps > 0 else None
    # the FP64 form end to end: the like-for-like counterpart of the
    # reference's FP64 integrator
    e2e64 = e2e_leg("fp64", args.e2e64_steps) if args.e2e64_steps > 0 else None

    # ---- adjoint / forward cost on the config-4 workload (FP64 form) -------
    adjoint = adjoint64 = None
    if args.adjoint_steps > 0:
        # the product form's adjoint, and the parity form's
        adjoint = adjoint_ratio(args, dev, stream, torch, "fp32c")
        adjoint64 = adjoint_ratio(args, dev, stream, torch, "fp64")
        log(f"[rank {rank}] adjoint: {adjoint} {adjoint64}")

    # ---- config-5 batch: one graph vs a per-pass loop --------------------------
    batch = None
    if args.batch_steps > 0:
        batch = batch_config5(args, dev, stream, torch)
        log(f"[rank {rank}] batch: {batch}")

    # ---- random-field generators (Brnd_es, TErnd_dft) on the config-3 grid -------
    rfg = None
    if args.rfg_steps > 0:
        rfg = generators(args, dev, stream, torch)
        log(f"[rank {rank}] generators: {rfg}")

    # ---- roofline of the shell-integration kernel -------------------------------
    # The kernel re-reads its voxels from L1/L2 (neighbouring samples and rays
    # share cells), so HBM is far from its roof; what bounds it is
    # instruction issue: one warp instruction per clock per SM sub-partition.
    # achieved = (warp instructions per integrated sample, from the ncu
    # capture of this kernel on this workload) x (integrated samples per
    # second of kernel time); integrated = passing the r / z cuts.
    peak_hbm, peak_kind = measured_peaks()
    per_launch_s = kms / 1e3 / max(klaunch, 1)
    samples_per_launch = ksamples / max(klaunch, 1)
    fused = len(passes) in (2, 3)
    kname = (f"hxg::shell_fp32c_multi_kernel<1,false,{len(passes)},true>" if fused
             else "hxg::shell_fp32c_kernel<1,false,true>")
    prof_name = "shell_fp32c_multi_config3.md" if fused else "shell_fp32c_config3.md"
    tps = profile_figure(prof_name, "dram_bytes_per_sample")
    ipv = profile_figure(prof_name, "warp_inst_per_valid_sample")
    # one traversal per shell serves all fused passes: its integrated samples
    # are those of one pass; launched one by one, every pass traverses
    # sharded (N > 1): this rank's launches covered its shard of the pixels;
    # the library's per-launch sample counts give the shard's share
    local_frac = ksamples / (samples_step * args.steps) if ksamples else 1.0
    valid_trav = (sum(W.valid_samples(passes[0])) * (1 if fused else len(passes))
                  * local_frac)
    valid_per_s = valid_trav * args.steps / (kms / 1e3) if kms > 0 else None
    clk_sum = clk.summary()
    mhz = clk_sum["sm_mhz"] if clk_sum else 1965.0
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    issue_peak = 4 * sms * mhz * 1e6 / 1e9          # G warp instructions / s
    achieved = ipv * valid_per_s / 1e9 if (ipv and valid_per_s) else None
    traffic = (tps * samples_per_launch) if tps else None
    dram_gbs = traffic / per_launch_s / 1e9 if traffic else None
    roofline = {"bound": "issue", "achieved": achieved, "peak": issue_peak,
                "unit": "G warp instructions/s",
                "frac": achieved / issue_peak if achieved else None,
                "peak_kind": f"4 warp instructions per clock per SM x {sms} SMs x "
                             f"{mhz:g} MHz (median sampled SM clock)",
                "warp_inst_per_valid_sample": ipv,
                "valid_samples_per_s": valid_per_s,
                "traffic": traffic, "dram_gbs": dram_gbs,
                "dram_frac": dram_gbs / peak_hbm if dram_gbs else None,
                "hbm_peak_gbs": peak_hbm, "hbm_peak_kind": peak_kind,
                "gather_gbs": samples_per_launch * BYTES_PER_SAMPLE["fp32c"] / per_launch_s / 1e9,
                "note": "bound: instruction issue. gather_gbs counts the 8-corner gather "
                        f"({BYTES_PER_SAMPLE['fp32c']} B per reference loop iteration), served "
                        "from L1/L2; traffic / dram_gbs / dram_frac are the DRAM bytes the "
                        "kernel moves (ncu) against the measured HBM copy bandwidth",
                "kernel": kname,
                "kernel_share_of_step": (kms / 1e3) / t32 if t32 > 0 else None,
                "kernel_samples_per_s": ksamples / (kms / 1e3) if kms > 0 else None}

    cpu = None
    # the CPU reference is timed at N = 1 only (the other ranks would wait)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        host = [t.cpu().numpy() for t in f64]
        cb = cpu_baseline(wl, host)
        v = cb["samples"] / cb["seconds"][0]
        cpu = {"value": v, "unit": UNIT, "cores": cb["threads"], "kind": "reference",
               "sample": cb["sample"]}
        if sub is not None:
            sub["cpu_ms"] = cb["seconds"][0] * 1e3
            sub["cpu_samples_per_s"] = v
            sub["fp64_gpu_vs_cpu"] = sub["fp64_samples_per_s"] / v
            sub["fp32c_gpu_vs_cpu"] = sub["fp32c_samples_per_s"] / v

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "strong" if shard else "weak", "vs_baseline": None, "dtype": "f32c",
            "data": "synthetic",
            "config": config_of(args, wl, ws, shard),
            "ms_per_map": ms_step / len(passes),
            "fp64": fp64,
            "fp32c_passes_one_by_one": one_by_one,
            # the product step (passes fused into one traversal per shell)
            # against the plain FP64 form, and the precision change alone
            # (both forms pass by pass)
            "fp32c_speedup_vs_fp64": (fp64["ms_per_step"] / ms_step) if fp64 else None,
            "fp32c_precision_speedup_vs_fp64": (fp64["ms_per_step"] / one_by_one["ms_per_step"]
                                                if fp64 and one_by_one else None),
            "fp32c_max_rel_err_vs_fp64": errs,
            "adjoint_fwd_ratio": adjoint["ratio"] if adjoint else None,
            "adjoint": adjoint,
            "adjoint_fp64": adjoint64,
            "batch": batch,
            "generators": rfg,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "e2e_fp64": e2e64,
            # the bounded sample of cpu_baseline, timed in both GPU forms
            "bounded_sample": sub,
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    ig32.close()
    replicas.finish(ws)


if __name__ == "__main__":
    main()
