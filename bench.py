"""Benchmark: batched Riemann2 512x512 eikonal solves on B200.

Workload (a "step"): one persistent launch solving a batch of independent
Riemann2 512^2 problems from a cold start (+inf values), with metrics
M = R(theta) diag(1, lambda) R(theta)^T, theta a smoothed random angle field
(sigma = 8 px at 512^2, i.e. the sigma = 16 px of the 1024^2 configuration in
the same physical units), lambda ~ U[1, 100] per pixel, 4 random seeds, cost 1,
gridScale 1/512, default tolerances.  Seeded synthetic data.

Reports solves/s (whole job), grid-updates/s, the HBM roofline of the
persistent solver kernel from its CUDA-event time and algorithmic bytes
(24.125 B per grid update), the end-to-end rate through the public API from
pinned host buffers, and a CPU baseline (the oracle, all host cores).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import gc
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

BYTES_PER_UPDATE = {"Riemann2": 24.125, "Riemann3": 36.125, "Isotropic2": 12.125, "Isotropic3": 12.125}
METRIC = "solves/s, Riemann2 512x512 batched cold-start solves (grid-updates/s in config)"


# (grid, batch, tile, niter_i, fim_front_width) -> DRAM bytes per solver launch, measured
MEASURED_TRAFFIC = {(512, 128, 8, 8, 4): 9.539e9 + 1.197e9}


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return 6650.0, "fallback"


def make_fields(n, batch, seed, sigma=8.0):
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    metrics, seeds = [], []
    for _ in range(batch):
        g1 = gaussian_filter(rng.standard_normal((n, n)), sigma, mode="wrap")
        g2 = gaussian_filter(rng.standard_normal((n, n)), sigma, mode="wrap")
        th = np.arctan2(g1, g2)
        lam = rng.uniform(1.0, 100.0, (n, n))
        c, s = np.cos(th), np.sin(th)
        metrics.append(np.stack([c * c + lam * s * s, c * s * (1 - lam), s * s + lam * c * c], -1).astype(np.float32))
        seeds.append(rng.uniform(0.05, 0.95, (4, 2)).astype(np.float32))
    return metrics, seeds


def make_iso256(seed, n=256, sigma=8.0):
    """The Isotropic2 256^2 configuration: g = white noise smoothed by a Gaussian
    of sigma pixels, renormalised to unit variance, cost = exp(0.5 g), one seed
    at the grid centre, gridScale 1/n, tolerance 1e-6 (case dictionary with the
    dictIn keys)."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    g = gaussian_filter(rng.standard_normal((n, n)), sigma, mode="wrap")
    g = (g - g.mean()) / g.std()
    return dict(model="Isotropic2", dims=np.array([n, n], np.float32), gridScales=np.full(2, 1.0 / n, np.float32),
                origin=np.zeros(2, np.float32), cost=np.exp(0.5 * g).astype(np.float32),
                seeds=np.array([[0.5, 0.5]], np.float32), tol=1e-6)


def dictins(metrics, seeds, n, to_device=True, pinned=False, traits=None):
    """One dictIn per instance; metrics and seeds are numpy arrays or (pinned)
    host tensors, moved to the device first if to_device."""
    import torch
    from adaptivegriddiscretizations_b200 import Eikonal
    out = []
    for m, s in zip(metrics, seeds):
        mt = m if isinstance(m, torch.Tensor) else torch.from_numpy(m)
        st = s if isinstance(s, torch.Tensor) else torch.from_numpy(s)
        if pinned and not mt.is_pinned():
            mt, st = mt.pin_memory(), st.pin_memory()
        if to_device:
            mt, st = mt.cuda(), st.cuda()
        d = {"model": "Riemann2", "mode": "gpu", "verbosity": 0, "dims": [n, n], "gridScale": 1.0 / n,
             "origin": [0.0, 0.0], "metric": mt, "seeds": st, "exportValues": True}
        d.update(traits or {})
        out.append(Eikonal.dictIn(d))
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index, self.proc, self.lines = index, None, []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:  # noqa: BLE001
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:  # noqa: BLE001
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_cases(n, count=4, seed=1234):
    """Oracle inputs of `count` instances of the benchmark's field distribution."""
    metrics, seeds = make_fields(n, count, seed)
    return [dict(model="Riemann2", dims=np.array([n, n], np.float32), gridScales=np.full(2, 1.0 / n, np.float32),
                 origin=np.zeros(2, np.float32), metric=m, seeds=s) for m, s in zip(metrics, seeds)]


def cpu_baseline(n, cases, seconds_budget=15.0, min_solves=1):
    """The oracle (C++ restatement of the scheme), OpenMP over all host cores,
    solving the prepared cases in turn (inputs made before the clock starts)
    until `seconds_budget` has passed; returns (solves/s, grid-updates/s, cores,
    sample, tile visits of each case solved)."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    solves, updates, visits = 0, 0, {}
    while True:
        k = solves % len(cases)
        r = O.run(cases[k], np.float32, nthreads=cores)
        solves += 1
        updates += r["tile_visits"] * 64
        visits[k] = int(r["tile_visits"])
        if solves >= min_solves and time.perf_counter() - t0 > seconds_budget:
            break
    dt = time.perf_counter() - t0
    return (solves / dt, updates / dt, cores,
            f"{solves} Riemann2 {n}^2 solves ({len(cases)} instances of the same field distribution in turn), "
            f"float32, {dt:.1f} s", visits)


def max_over_ranks(x, dist, device="cuda"):
    """The largest value of x over the ranks (every rank gets it); x itself
    without a process group.  Timings of several ranks are reported this way."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t)


def run_reference(args, rank):
    """The reference arm: the CPU scheme on the host cores, one solve per step.
    The inputs of the step's instances are made before the clock starts."""
    if rank != 0:
        return
    n = args.n
    cases = cpu_cases(n, 4, 1234)
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    for k in range(args.warmup):
        O.run(cases[k % len(cases)], np.float32, nthreads=cores)
    t0 = time.perf_counter()
    for k in range(args.steps):
        O.run(cases[k % len(cases)], np.float32, nthreads=cores)
    dt = time.perf_counter() - t0
    value = args.steps / dt
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": "solves/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"Riemann2 {n}x{n}, 1 instance per step on the host cores (oracle port)",
                   "grid": n, "seeds": 4},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": f"one Riemann2 {n}^2 solve per step, 4 prepared instances in turn (inputs made "
                                   "before the clock); the reference's own CPU path (the external HFM library) is "
                                   "not available, the oracle is the C++ restatement of its scheme"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_other_path(args):
    """The other two kernels of the path, timed on their configurations' sizes
    (one GPU, CUDA events): `--path geodesic`, the backtracking ODE from 64 tips
    on Riemann2 1024^2 (one warp per tip: latency-bound, so the figure is ODE
    steps/s, with the bytes an ODE step reads: 4 cells x (value, 2 flow planes,
    weight sum) x 4 B); `--path reverse`, the reverse adjoint (transpose and
    linear solve) of the arrival times at 128 receivers on Riemann3 200^3, with
    the algorithmic bytes of a linear tile visit point: 6 weights, 6 indices
    and the sensitivity read, the sensitivity written (56 B)."""
    import torch
    from scipy.ndimage import gaussian_filter
    from adaptivegriddiscretizations_b200 import Eikonal
    from adaptivegriddiscretizations_b200.Eikonal.HFM_CUDA import Interface
    torch.cuda.set_device(0)
    rng = np.random.default_rng(5)
    if args.path == "geodesic":
        n = args.path_size or 1024
        metrics, seeds = make_fields(n, 1, 21, sigma=16.0)
        tips = rng.uniform(0.02, 0.98, (64, 2)).astype(np.float32)
        d = dict(model="Riemann2", dims=np.array([n, n], np.float32), gridScales=np.full(2, 1.0 / n, np.float32),
                 origin=np.zeros(2, np.float32), metric=metrics[0], seeds=seeds[0], tips=tips, verbosity=0)
        workload = f"Riemann2 {n}x{n}, geodesics from 64 tips (flow already computed)"
    else:
        n = args.path_size or 200
        q = gaussian_filter(rng.standard_normal((4, n, n, n)).astype(np.float32), (0, 6, 6, 6), mode="wrap")
        q /= np.linalg.norm(q, axis=0, keepdims=True)
        w, x, y, z = q
        rot = np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
                        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
                        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], -2)
        ev = np.exp(rng.uniform(0, np.log(25.0), (n, n, n, 3))).astype(np.float32)
        M = rot @ (ev[..., :, None] * np.swapaxes(rot, -1, -2))
        metric = np.stack([M[..., i, j] for i in range(3) for j in range(i + 1)], -1).astype(np.float32)
        sens = np.zeros((n, n, n, 1), np.float32)
        sens.reshape(-1)[rng.choice(n ** 3, 128, replace=False)] = 1.0
        d = dict(model="Riemann3", dims=np.array([n] * 3, np.float32), gridScales=np.full(3, 1.0 / n, np.float32),
                 origin=np.zeros(3, np.float32), metric=metric, seeds=np.array([[0.5, 0.5, 0.5]], np.float32),
                 sensitivity=sens, verbosity=0)
        workload = f"Riemann3 {n}^3, reverse sensitivity of the arrival times at 128 receivers (flow already computed)"
    itf = Interface(Eikonal.dictIn(d))
    itf.SetKernelTraits()
    itf.SetGeometry()
    itf.SetArgs()
    itf.Solve()
    itf.PostProcess()
    import copy
    keys = copy.deepcopy(itf.hfmOut["keys"])  # each key is read once per Run: restored for every repetition
    call = itf.GetGeodesics if args.path == "geodesic" else itf.SolveAD

    def work():
        itf.hfmOut["keys"] = copy.deepcopy(keys)
        call()

    for _ in range(max(3, args.warmup)):
        work()
    torch.cuda.synchronize()
    ts = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        itf.hfmOut["keys"] = copy.deepcopy(keys)
        e0.record()
        call()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1) / 1e3)
    t = float(np.median(ts))
    hbm, peak_kind = peaks()
    if args.path == "geodesic":
        steps = sum(int(g.shape[1]) for g in itf.hfmOut["geodesics"])
        value, unit, nbytes = steps / t, "geodesic ODE steps/s", steps * 64
        extra = {"stops": {c: itf.hfmOut["geodesic_stopping_criteria"].count(c)
                           for c in set(itf.hfmOut["geodesic_stopping_criteria"])}, "points": steps}
    else:
        visits = int(itf.stats["reverseAD"]["nupdate_o_total"])
        value, unit, nbytes = 1.0 / t, "reverse solves/s", visits * itf.size_i * 56
        extra = {"tile_visits": visits, "epochs": int(itf.stats["reverseAD"]["niter_o"])}
    print(json.dumps({"metric": f"{args.path} path", "value": value, "unit": unit, "ms_per_step": 1e3 * t,
                      "steps": args.steps, "warmup": args.warmup, "data": "synthetic",
                      "config": dict({"workload": workload}, **extra),
                      "roofline": {"bound": "latency" if args.path == "geodesic" else "hbm",
                                   "achieved": nbytes / t / 1e9, "peak": hbm, "unit": "GB/s",
                                   "frac": nbytes / t / 1e9 / hbm, "peak_kind": peak_kind}}), flush=True)




def unet_flops(nb=128):
    """Forward FLOPs of the U-Net on one nb x nb block grid (the 3x3 convolutions)."""
    from adaptivegriddiscretizations_b200.WarmStart.unet import IN_CHANNELS, LEVELS
    c0, c1, c2, c3 = LEVELS
    convs = [(0, IN_CHANNELS, c0), (0, c0, c0), (1, c0, c1), (1, c1, c1), (2, c1, c2), (2, c2, c2), (3, c2, c3),
             (3, c3, c3), (2, c3 + c2, c2), (2, c2, c2), (1, c2 + c1, c1), (1, c1, c1), (0, c1 + c0, c0), (0, c0, c0)]
    return sum(2 * (nb >> lv) ** 2 * 9 * ci * co for lv, ci, co in convs)


def run_warm_start(args, peaks_tf):
    """The learned warm start on the benchmark's configuration: 20k solver-made
    training solutions, GPU training of the U-Net by the tensor-core kernels,
    then cold and warm batched solves of 1k held-out instances side by side
    (device time; the warm figure includes the network's prediction).  Returns
    the JSON object of the bench line."""
    import torch
    from adaptivegriddiscretizations_b200.WarmStart.warmstart import WarmStart, riemann2_fields
    n, B = args.n, args.batch
    ws = WarmStart(n=n, batch=B)
    gen = torch.Generator(device="cuda").manual_seed(1)
    t0 = time.perf_counter()
    X, T = ws.generate(args.warm_train, gen)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t0
    Xv, Tv = ws.generate(512, torch.Generator(device="cuda").manual_seed(99))
    fin = torch.isfinite(Tv)
    const_loss = float(((Tv - Tv[fin].mean()) ** 2)[fin].mean())
    hist = ws.train(X, T, args.warm_steps, batch=32, lr=2e-3, gen=torch.Generator(device="cuda").manual_seed(3))
    val_loss = ws.eval_loss(Xv, Tv)
    del X, T
    # inference throughput of the network (forward of a batch, CUDA events)
    m, sd = riemann2_fields(n, B, torch.Generator(device="cuda").manual_seed(7))
    x0, _ = ws.features(m, sd)
    for _ in range(3):
        ws.net.forward(x0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        ws.net.forward(x0)
    e1.record()
    torch.cuda.synchronize()
    t_fwd = e0.elapsed_time(e1) / 5e3
    flops = unet_flops(n // 4) * B
    best = ws.tune(m, sd)
    res = ws.evaluate(args.warm_eval, torch.Generator(device="cuda").manual_seed(11))
    res.update({
        "training": {"solutions": args.warm_train, "generate_s": t_gen, "steps": args.warm_steps, "batch": 32,
                     "train_s": ws.train_seconds, "ms_per_step": 1e3 * ws.train_seconds / args.warm_steps,
                     "final_train_loss": hist[-1][1] if hist else None},
        "validation_mse_log_ratio": val_loss, "constant_predictor_mse": const_loss,
        "release_epochs_tuned": {"epochs": best[0], "batch_solve_s": best[1]},
        "unet_forward": {"batch": B, "ms": 1e3 * t_fwd, "tflops": flops / t_fwd / 1e12,
                         "frac_of_bf16_peak": flops / t_fwd / 1e12 / peaks_tf, "peak_tflops": peaks_tf},
        "network": "U-Net 4 levels 32/64/128/256 channels, bf16, fp32 accumulation, 128x128 blocks of 4x4 points",
    })
    return res


def run_iso256(args):
    """The Isotropic2 256^2 configuration (one solve, tolerance 1e-6): solves/s
    through `dictIn(...).Run()` with host numpy inputs and the values read back
    (e2e: inputs copied in, preparation, solve, readback), the device time of
    the same call by CUDA events, and the oracle on all host cores timed on the
    same case (float32).  Parity: the largest relative difference of the GPU
    values from the float64 oracle's discrete solution."""
    import torch
    from adaptivegriddiscretizations_b200 import Eikonal
    from oracle import oracle as O
    torch.cuda.set_device(0)
    case = make_iso256(1)

    def solve(traits=None):
        d = dict(case, mode="gpu", verbosity=0, exportValues=True)
        if traits is not None:
            d["traits"] = traits
        out = Eikonal.dictIn(d).Run()
        return out["values"].cpu().numpy(), out["stats"]

    def timed(traits=None):
        for _ in range(max(3, args.warmup)):
            solve(traits)
        torch.cuda.synchronize()
        walls, devs = [], []
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record()
            v, stats = solve(traits)
            e1.record()
            torch.cuda.synchronize()
            walls.append(time.perf_counter() - t0)
            devs.append(e0.elapsed_time(e1) / 1e3)
        return v, stats, float(np.median(walls)), float(np.median(devs))

    v, _, t, tdev = timed()  # the reference's default traits (16x16 tiles, 16 local iterations)
    _, st_auto, t_auto, tdev_auto = timed("auto")  # the autotuner's choice
    exact = O.run(dict(case, atol=1e-14, rtol=1e-14), np.float64, nthreads=os.cpu_count() or 1)["values"]
    pos = np.isfinite(exact) & (exact > 0)  # (the seed's value is 0)
    err = float((np.abs(v[pos] - exact[pos]) / exact[pos]).max())
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    ncpu = 0
    while ncpu < 3 or time.perf_counter() - t0 < 5.0:
        r = O.run(case, np.float32, nthreads=cores)
        ncpu += 1
    tcpu = (time.perf_counter() - t0) / ncpu
    print(json.dumps({"metric": "iso256 path", "value": 1.0 / tdev, "unit": "solves/s",
                      "ms_per_step": 1e3 * tdev, "steps": args.steps, "warmup": args.warmup,
                      "data": "synthetic", "dtype": "f32",
                      "config": {"workload": "Isotropic2 256x256, cost exp(0.5 g) (g a sigma-8 Gaussian field), "
                                             "one seed at the centre, tolerance 1e-6, one solve per step"},
                      "e2e": {"value": 1.0 / t, "unit": "solves/s", "api": "dictIn(...).Run() from numpy inputs"},
                      "max_rel_diff_vs_discrete": err,
                      "traits_auto": {"solves_per_s": 1.0 / tdev_auto, "e2e_solves_per_s": 1.0 / t_auto,
                                      "traits": st_auto.get("autotune", {}).get("traits")},
                      "cpu_baseline": {"value": 1.0 / tcpu, "unit": "solves/s", "cores": cores, "kind": "port",
                                       "sample": f"{ncpu} solves of the same case, float32"}}))


def run_unet(args):
    """The learned warm start's network alone (`--path unet`): forward passes of
    a batch of 128 Riemann2 512^2 problems (128 x 128 blocks, 8 feature
    channels) with random weights, every 3x3 convolution timed by CUDA events:
    FLOPs = 2 x pixels x 9 cin x cout, against the measured dense bf16 peak."""
    import torch
    from adaptivegriddiscretizations_b200.WarmStart.unet import UNet
    torch.cuda.set_device(0)
    nb, B = (args.path_size or 512) // 4, args.batch
    net = UNet(seed=0)
    x0 = torch.randn((B, nb, nb, 8), device="cuda").to(torch.bfloat16)
    for _ in range(max(1, args.warmup)):
        net.forward(x0)
    torch.cuda.synchronize()
    orig, layers = net._conv, []

    def timed(layer, n, H, W, srcs, out_bf=None, out_f=None, relu=True, bias=True, weights=None):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        orig(layer, n, H, W, srcs, out_bf, out_f, relu, bias, weights)
        e1.record()
        cin = sum(sr[1] for sr in srcs)
        layers.append((H, cin, layer.cout, e0, e1, 2 * n * H * W * 9 * cin * layer.cout))

    net._conv = timed
    rows = []
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            layers.clear()
            net.forward(x0)
            torch.cuda.synchronize()
            rows.append([(H, ci, co, e0.elapsed_time(e1) / 1e3, fl) for H, ci, co, e0, e1, fl in layers])
    net._conv = orig
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f)["bf16_tflops"])
    except Exception:  # noqa: BLE001
        peak = 1590.0
    per = []
    for k in range(len(rows[0])):
        H, ci, co, _, fl = rows[0][k]
        t = float(np.median([r[k][3] for r in rows]))
        per.append({"H": H, "cin": ci, "cout": co, "us": 1e6 * t, "tflops": fl / t / 1e12})
    tot_t = sum(p["us"] for p in per) / 1e6
    tot_f = sum(r[4] for r in rows[0])
    print(json.dumps({"metric": "U-Net forward (3x3 convolutions on tcgen05)", "value": tot_f / tot_t / 1e12,
                      "unit": "TFLOP/s", "batch": B, "blocks": nb, "ms_per_forward_convs": 1e3 * tot_t,
                      "roofline": {"bound": "tensor", "achieved": tot_f / tot_t / 1e12, "peak": peak,
                                   "unit": "TFLOP/s", "frac": tot_f / tot_t / 1e12 / peak},
                      "clocks": clk.summary(), "layers": per}), flush=True)


def run_autotune(n, B, metrics, seeds):
    """Traits autotuner on the benchmark's batch: every candidate tile shape and
    local iteration count of Riemann2 (Eikonal/Autotune.py) timed on batched
    solves of the same instances (BatchSolver, device-resident inputs, CUDA
    events, best of two); the choice is cached like traits='auto' does."""
    import torch
    from adaptivegriddiscretizations_b200 import Eikonal
    from adaptivegriddiscretizations_b200.Eikonal.Autotune import Autotuner, bucket_key, candidates
    m = torch.from_numpy(np.stack(metrics)).cuda()
    sd = torch.from_numpy(np.stack(seeds)).cuda()

    def run(tr):
        tmpl = dictins(metrics[:1], seeds[:1], n, to_device=False, traits={"traits": dict(tr)})[0]
        solver = Eikonal.BatchSolver(tmpl, B, nbuffers=1)
        solver.submit(metric=m, seeds=sd).result()
        st = solver._bufs[0].stream
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        solver.submit(metric=m, seeds=sd)
        e1.record(st)
        e1.synchronize()
        del solver
        return e0.elapsed_time(e1) / 1e3

    key = bucket_key("Riemann2", (n, n), B, torch.cuda.get_device_name())
    tuner = Autotuner()
    choice, trials = tuner.tune(key, run, candidates("Riemann2"), repeats=2)
    t = {(tuple(c["shape_i"]), c["niter_i"]): tt for tt, c in trials}
    t_def = t[((8, 8), 8)]
    t_best = t[(tuple(choice["shape_i"]), choice["niter_i"])]
    return {"chosen": {"shape_i": list(choice["shape_i"]), "niter_i": choice["niter_i"]},
            "reference_default": {"shape_i": [8, 8], "niter_i": 8}, "gain_over_default": t_def / t_best,
            "solves_per_s_tuned": B / t_best, "solves_per_s_default": B / t_def,
            "trials_ms": [[list(c["shape_i"]), c["niter_i"], 1e3 * tt] for tt, c in trials]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--batch", type=int, default=128)
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--ctas", type=int, default=0)
    ap.add_argument("--wpc", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=24)
    ap.add_argument("--niter-i", type=int, default=0, help="local iterations per tile visit (0: the default, 8)")
    ap.add_argument("--front", type=int, default=0, help="FIM front width (0: the default, 4)")
    ap.add_argument("--tile", type=int, default=8, help="tile side (8: the default, or 16)")
    ap.add_argument("--path", default="solve", choices=["solve", "geodesic", "reverse", "unet", "iso256"],
                    help="solve: the benchmark (default); geodesic / reverse: the other kernels of the path; "
                         "unet: the learned warm start's network; iso256: the Isotropic2 256^2 configuration "
                         "with the oracle timed beside it")
    ap.add_argument("--path-size", type=int, default=0,
                    help="grid side for --path (0: 1024 for geodesic, 200 for reverse; smaller for profiler captures)")
    ap.add_argument("--warm-train", type=int, default=20000, help="training solutions of the learned warm start")
    ap.add_argument("--warm-steps", type=int, default=2000, help="training steps of the learned warm start")
    ap.add_argument("--warm-eval", type=int, default=1024, help="held-out instances of the warm/cold comparison")
    ap.add_argument("--no-warm", action="store_true", help="skip the learned warm start leg")
    ap.add_argument("--no-autotune", action="store_true", help="skip the traits autotuner leg")
    ap.add_argument("--warm-oracle", type=float, default=0.0,
                    help="experiment: warm start every solve from (1+eps) x its cold solution, all tiles active")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.path == "unet":
        run_unet(args)
        return
    if args.path == "iso256":
        run_iso256(args)
        return
    if args.path != "solve":
        run_other_path(args)
        return

    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from adaptivegriddiscretizations_b200 import Eikonal, _lib
    from adaptivegriddiscretizations_b200.Eikonal.HFM_CUDA import Interface, BatchPlan

    n, B = args.n, args.batch
    metrics, seeds = make_fields(n, B, 1000 + rank)
    traits = {}
    if args.niter_i or args.tile != 8:
        traits["traits"] = {"shape_i": (args.tile, args.tile), "niter_i": args.niter_i or 8}
    if args.front:
        traits["fim_front_width"] = args.front
    ins = dictins(metrics, seeds, n, to_device=True, traits=traits)
    itfs = [Interface(h) for h in ins]
    for it in itfs:
        it.SetKernelTraits()
        it.SetGeometry()
        it.SetArgs()
    size_tot = itfs[0].size_tot
    values = torch.full((B, size_tot), float("inf"), dtype=torch.float32, device="cuda")
    for i, it in enumerate(itfs):
        it.values_t = values[i]
    launch = _lib.AgdLaunch(ctas=args.ctas, warps_per_cta=args.wpc, timeout_ns=0)
    plan = BatchPlan(itfs, launch=launch)

    warm0 = None
    if args.warm_oracle:
        values.fill_(float("inf"))
        plan.run()
        torch.cuda.synchronize()
        cold = values.clone()
        warm0 = cold * (1.0 + args.warm_oracle)
        for it in itfs:
            it.activateAll = True
        plan = BatchPlan(itfs, launch=launch)

    def reset():
        if warm0 is None:
            values.fill_(float("inf"))
        else:
            values.copy_(warm0)

    def step():
        reset()
        plan.run()

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    niter, status, visits = plan.read_stats()
    assert not status.any(), f"solver status {status}"
    updates_per_step = int(visits.sum()) * args.tile ** 2

    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for k in range(args.steps):
            reset()
            evs[k][0].record()
            plan.run()
            evs[k][1].record()
        t1.record()
        torch.cuda.synchronize()
    elapsed = t0.elapsed_time(t1) / 1000.0
    kern = np.array([a.elapsed_time(b) / 1000.0 for a, b in evs])
    elapsed = max_over_ranks(elapsed, dist)
    niter, status, visits = plan.read_stats()
    assert not status.any()
    updates_per_step = int(visits.sum()) * args.tile ** 2
    warm_err = None
    if warm0 is not None:
        fin = torch.isfinite(cold)
        warm_err = float(((values - cold).abs()[fin] / cold.abs()[fin].clamp_min(1e-30)).max())
    total_solves = B * args.steps * world
    value = total_solves / elapsed
    hbm, peak_kind = peaks()
    # DRAM bytes (read + write) of one sched_worker launch of this workload,
    # from an ncu capture (dram__bytes_read.sum + dram__bytes_write.sum, one pass)
    traffic = MEASURED_TRAFFIC.get((n, B, args.tile, args.niter_i or 8, args.front or 4))
    achieved = updates_per_step * BYTES_PER_UPDATE["Riemann2"] / kern.mean() / 1e9

    # End to end, inputs in page-locked host memory, values read back to host
    # memory every step.  Primary: Eikonal.BatchSolver (repeated batched solves of
    # one configuration; batch k+1 is uploaded and prepared while batch k
    # solves).  Also reported: the dictIn path (one dictIn per instance,
    # Eikonal.SubmitBatch on two alternating streams).
    e2e = e2e_dictin = None
    if args.e2e_steps > 0:
        # The objects made so far (fields, prepared instances, torch and numpy
        # state) live to the end: kept out of the garbage collector's scans, a
        # generation-2 collection triggered by the dictIn made every step costs
        # well under a millisecond instead of about 34 ms (a serving process
        # does the same after its setup).
        gc.collect()
        gc.freeze()
        h2d = sum(m.nbytes + s.nbytes for m, s in zip(metrics, seeds))
        host_out = [torch.empty((B, n, n), dtype=torch.float32).pin_memory() for _ in range(2)]
        d2h = host_out[0].numel() * 4
        pin_metric = torch.from_numpy(np.stack(metrics)).pin_memory()
        pin_seeds = torch.from_numpy(np.stack(seeds)).pin_memory()
        template = dictins(metrics[:1], seeds[:1], n, to_device=False, traits=traits)[0]
        solver = Eikonal.BatchSolver(template, B, launch=launch)

        def run_solver(nsteps):
            pending = []
            for k in range(nsteps):
                pending.append(solver.submit(metric=pin_metric, seeds=pin_seeds, out=host_out[k % 2]))
                if len(pending) == 2:
                    pending.pop(0).result()
            for job in pending:
                job.result()

        run_solver(3)  # warm up both buffer sets
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t_e = time.perf_counter()
        run_solver(args.e2e_steps)
        te = max_over_ranks(time.perf_counter() - t_e, dist)
        e2e = {"value": B * args.e2e_steps * world / te, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "api": "Eikonal.BatchSolver.submit (two buffer sets)"}
        del solver

        pin_m = [torch.from_numpy(m).pin_memory() for m in metrics]
        pin_s = [torch.from_numpy(s).pin_memory() for s in seeds]
        streams = [torch.cuda.Stream(), torch.cuda.Stream()]

        def submit(k):
            with torch.cuda.stream(streams[k % 2]):
                return Eikonal.SubmitBatch(dictins(pin_m, pin_s, n, to_device=False, traits=traits))

        def collect(job):
            outs = job.result()
            with torch.cuda.stream(job.stream):  # copy engine only: no kernel behind the next solve
                for i, o in enumerate(outs):
                    host_out[0][i].copy_(o["values"], non_blocking=True)
            job.stream.synchronize()

        def run_dictin(nsteps):
            job = submit(0)
            for k in range(nsteps):
                nxt = submit(k + 1) if k + 1 < nsteps else None
                collect(job)
                job = nxt

        run_dictin(2)  # (its first SubmitBatch prepares the cached solver of the configuration)
        torch.cuda.synchronize()
        gc.collect()  # the objects made since the first freeze, out of the scans too
        gc.freeze()
        if dist:
            dist.barrier()
        t_e = time.perf_counter()
        run_dictin(args.e2e_steps)
        te = max_over_ranks(time.perf_counter() - t_e, dist)
        e2e_dictin = {"value": B * args.e2e_steps * world / te, "unit": "solves/s",
                      "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                      "api": "Eikonal.SubmitBatch of dictIn inputs (two streams)"}

    tuned = run_autotune(n, B, metrics, seeds) if rank == 0 and not args.no_autotune else None
    warm = None
    if rank == 0 and not args.no_warm:
        try:
            with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
                tf_peak = float(json.load(f)["bf16_tflops"])
        except Exception:  # noqa: BLE001
            tf_peak = 1590.0
        warm = run_warm_start(args, tf_peak)

    cpu = schedule = None
    if rank == 0 and not args.no_cpu_baseline:
        cases = cpu_cases(n, 4, 1234)
        v, gu, cores, sample, ref_visits = cpu_baseline(n, cases, min_solves=len(cases))
        cpu = {"value": v, "unit": "solves/s", "cores": cores, "kind": "port", "sample": sample,
               "grid_updates_per_s": gu}
        # Useful work: this solver's tile visits against the reference schedule's
        # (the oracle reproduces _solvers.fast_iterative_method's visit count) on
        # the same instances.
        sitfs = [Interface(h) for h in dictins([c["metric"] for c in cases], [c["seeds"] for c in cases], n,
                                               traits=traits)]
        for it in sitfs:
            it.SetKernelTraits()
            it.SetGeometry()
            it.SetArgs()
        splan = BatchPlan(sitfs, launch=launch)
        splan.run()
        gv = [int(x) for x in splan.read_stats()[2]]
        rv = [ref_visits[k] for k in range(len(cases))]
        schedule = {"instances": len(cases), "gpu_tile_visits": gv, "reference_schedule_tile_visits": rv,
                    "ratio": float(np.sum(gv) / np.sum(rv))}
        del splan, sitfs

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * elapsed / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"Riemann2 {n}x{n} cold-start solves, batch {B} per GPU per step, one "
                                   f"persistent launch", "batch_per_gpu": B, "grid": n, "seeds": 4,
                       "lambda": "U[1,100]", "theta_sigma_px": 8, "tile": f"{args.tile}x{args.tile}",
                       "niter_i": args.niter_i or 8, "fim_front_width": args.front or 4,
                       "grid_updates_per_step": updates_per_step,
                       "grid_updates_per_s": updates_per_step * args.steps * world / elapsed,
                       "mean_niter_o": float(niter.mean()), "max_niter_o": int(niter.max()),
                       "warm_oracle_eps": args.warm_oracle or None, "warm_max_rel_err": warm_err,
                       "l2": "inputs larger than L2 (batch working set %.0f MB)" % (B * size_tot * 24 / 1e6),
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "sched_worker<EikonalVisitor>", "kernel_ms": float(kern.mean() * 1000),
                         "bytes_per_update": BYTES_PER_UPDATE["Riemann2"]},
            "cpu_baseline": cpu, "schedule_vs_reference": schedule, "warm_start": warm, "autotune": tuned, "e2e": e2e, "e2e_dictin": e2e_dictin,
            # per solve step: stencil_kernel, setup_tiles, publish_first, publish_first_slots,
            # sched_worker, finish_stats (the values reset is a torch fill)
            "gpu_launches": 6 * args.steps,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
