#!/usr/bin/env python
"""Benchmark of the split-step spinor propagator on B200.

Workload (the q2D configuration the headline metric is quoted on): spin-2
SO-coupled real-time dynamics, NX=NY=512, DX=DY=0.05, DT=1e-4, Rb-87
(mass 87, a0/a2/a4 = 87.93/91.28/99.18 a_B), NATOMS=50000, NUX=NUY=20 Hz,
NUZ=500 Hz, ground state at GAMMAX=GAMMAY=1.0 quenched to GAMMAX=1.2.
Synthetic initial state: the reference's default Gaussian guess relaxed by
imaginary-time steps at gamma=(1,1) on the device, plus 1e-3 complex Gaussian
noise (numpy PCG64 seed 2), renormalised (no dataset is involved).

A step is one full Lie split step FFT->KE->SOC->BFT->SE->SP->NORMC of the
whole 512^2 x 5 spinor.  Metric: grid-pt*steps/s (higher is better).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision fp64|fp32]

value : device time (CUDA events on the launching stream) of K steps, L2
        flushed (256 MiB write) before every step, max over ranks.
e2e   : the same K steps through the C ABI with host buffers: pinned H2D of
        the state, every step's NORMC written by the step into a pinned host
        ring (fgpe_norms_sink), D2H of the final state; device-timed with the
        same flushes.
The reference arm (--impl reference) times the CPU restatement of the
reference (oracle/, OpenMP on all host cores) on the same workload: the
Fortran/FFTW/LAPACK reference cannot be compiled on this image.
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

WORKLOAD = dict(name="q2d-spin2-SO-realtime-512x512-quench", dim=2, spin=2, n=(512, 512),
                d=(0.05, 0.05), dt=1e-4, mass=87.0, a=(87.93, 91.28, 99.18), natoms=50000,
                nu=(20.0, 20.0, 500.0), gamma_gs=(1.0, 1.0), gamma=(1.2, 1.0))
METRIC = "grid-pt*steps/s"


def workload_config(gamma):
    from fortress_b200.config import RunConfig
    w = WORKLOAD
    c = RunConfig(dim=2, spin=2, n=(512, 512, 1), d=(0.05, 0.05, 1.0), dt=w["dt"], mass=w["mass"],
                  a=w["a"], natoms=w["natoms"], nu=w["nu"], switch_im=0,
                  gamma=(gamma[0], gamma[1], 0.0))
    return c


def gaussian_guess(cfg):
    """INITIALIZE default spin-2 guess, cgpe2d.f90:766-771."""
    import numpy as np
    nx, ny = cfg.n[0], cfg.n[1]
    x = (-1.0 + 2.0 * np.arange(nx) / nx) * nx * cfg.d[0] / 2.0
    y = (-1.0 + 2.0 * np.arange(ny) / ny) * ny * cfg.d[1] / 2.0
    ax, ay, _ = cfg.alpha
    g = np.sqrt(0.2) * np.exp(-(ax * x[:, None] ** 2 + ay * y[None, :] ** 2) / 2.0) / np.sqrt(np.pi)
    return np.repeat(g[:, :, None], 5, axis=2).astype(np.complex128)


def add_noise(phi, seed=2):
    import numpy as np
    rng = np.random.default_rng(seed)
    phi = phi + 1e-3 * (rng.standard_normal(phi.shape) + 1j * rng.standard_normal(phi.shape)) * np.abs(phi).max()
    return phi


def prepared_state(F, cfg_gs, prep_steps=3000):
    """Ground-state-like start: imaginary time on the device from the guess."""
    import numpy as np
    p = cfg_gs.params()
    p["imag_time"] = True
    p["dt"] = 1e-3
    prop = F.Propagator(**p)
    prop.set_state(gaussian_guess(cfg_gs))
    prop.normt()
    prop.step(prep_steps)
    phi = add_noise(prop.state().reshape(512, 512, 5))
    prop.close()
    # renormalise to the Simpson norm 1 (NORMT of the reference)
    from fortress_b200.config import simpson_weights
    w = simpson_weights(512, cfg_gs.d[0])
    tot = float(np.einsum("i,j,ijm->", w, w, np.abs(phi) ** 2))
    return phi / np.sqrt(tot)


# ------------------------------------------------------------------ clocks
def out_dir():
    """Directory for the bench's side files (clock samples, autotune cache):
    $FGPE_BENCH_OUT, else the system temporary directory."""
    import tempfile
    return os.environ.get("FGPE_BENCH_OUT") or tempfile.gettempdir()


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.path = os.path.join(out_dir(), f"clocks_rank{index}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1])); smax = max(smax, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def known_traffic(workload, precision, kernel):
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d.get(f"{workload}/{precision}/{kernel}")
    except Exception:
        return None


# --------------------------------------------------------------- CPU legs
def run_cpu(phi, cfg, steps, warmup, budget_s=None):
    from oracle import oracle as O
    t = cfg.tau()
    orc = O.Oracle(dim=2, spin=2, nx=512, ny=512, dx=cfg.d[0], dy=cfg.d[1], dt=cfg.dt, imag=0, tau=t,
                   gx=cfg.gamma[0], gy=cfg.gamma[1], ax=cfg.alpha[0], ay=cfg.alpha[1], az=cfg.alpha[2])
    orc.set_state(phi)
    for _ in range(warmup):
        orc.step(1)
    done, t0 = 0, time.perf_counter()
    while done < steps:
        orc.step(1)
        done += 1
        if budget_s is not None and time.perf_counter() - t0 > budget_s and done >= 2:
            break
    el = time.perf_counter() - t0
    return 512 * 512 * done / el, done, el, O.num_threads()


def capture(args):
    """The step kernels alone, for ncu launch lists and per-kernel captures
    (-k regex:k_row_fast / k_col_fast): warmup + steps split steps of the
    512^2 spin-2 real-time case from the noisy Gaussian guess, or with
    --workload 3d of the 3D spin-1 case on a 128^3 grid (the same kernel
    families, wide column tiles included, at an eighth of the 256^3 state:
    a small case for ncu)."""
    import numpy as np
    import fortress_b200 as F
    if args.workload == "fno":
        # training steps of the learned-guess network (64^2, batch 64)
        import torch
        from fortress_b200 import fno as FN
        net = FN.FNO(64, 64, seed=7)
        a = FN.input_channels(np.random.default_rng(0).uniform(-1, 1, (64, 5)), 64)
        tgt = torch.randn(6, 64 * 64 * 64, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
        net.forward(a)
        for _ in range(args.warmup + args.steps):
            net.forward(); net.loss(tgt); net.backward(); net.adam()
        torch.cuda.synchronize()
        assert not net.tc_error()
        print(json.dumps({"capture": "fno-train-64x64-b64", "steps": args.warmup + args.steps,
                          "loss": float(net.loss_dev.item())}))
        return
    if args.workload == "golden1d":
        with open(os.path.join(ROOT, "tests", "golden", "fortress_1d_spin2.json")) as f:
            golden = json.load(f)
        cfg = F.RunConfig.from_text(golden["input1D"], 1)
        prop = F.Propagator.from_config(cfg)
        x = (-1.0 + 2.0 * np.arange(cfg.n[0]) / cfg.n[0]) * cfg.n[0] * cfg.d[0] / 2.0
        prop.set_state(np.repeat(np.exp(-x * x / 2.0)[:, None], 5, axis=1).astype(np.complex128))
        prop.normt()
        prop.step(args.warmup + args.steps)
        en, mu, mz, rms = prop.observables()
        assert np.isfinite(en)
        print(json.dumps({"capture": "golden-1d-spin2-2048", "steps": args.warmup + args.steps, "en": en}))
        return
    if args.workload == "3d":
        from fortress_b200.config import RunConfig
        w = D3
        cfg = RunConfig(dim=3, spin=1, n=(128, 128, 128), d=(0.2, 0.2, 0.2), dt=w["dt"], mass=w["mass"],
                        a=w["a"], natoms=w["natoms"], nu=w["nu"], switch_im=1, gamma=w["gamma"])
        p = cfg.params(args.precision)
        prop = F.Propagator(**p)
        prop.set_state(gaussian_nd(p))
        prop.normt()
        prop.step(args.warmup + args.steps, snapshot=False)
        n = prop.normc()
        assert np.all(np.isfinite(n))
        print(json.dumps({"capture": "3d-spin1-SO-imag-128^3", "precision": args.precision,
                          "steps": args.warmup + args.steps, "norm": float(n.sum())}))
        return
    cfg = workload_config(WORKLOAD["gamma"])
    prop = F.Propagator(**cfg.params(args.precision))
    prop.set_state(add_noise(gaussian_guess(cfg)))
    prop.step(args.warmup + args.steps, snapshot=False)
    n = prop.normc()
    assert np.all(np.isfinite(n))
    print(json.dumps({"capture": WORKLOAD["name"], "precision": args.precision,
                      "steps": args.warmup + args.steps, "norm": float(n.sum())}))


def kernel_pass(prop, flush, steps):
    """Per-kernel device times: a second timed pass of the same steps with
    CUDA events recorded by the library around every kernel launch on its
    stream (fgpe_profile_*).  Returns (ms per class, launches per class)."""
    import torch
    prop.profile(True)
    prop.profile_read(reset=True)
    for _ in range(steps):
        flush.zero_()
        prop.step(1, snapshot=False)
    torch.cuda.synchronize()
    kms, kn = prop.profile_read(reset=True)
    prop.profile(False)
    return kms, kn


# -------------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--prep-steps", type=int, default=3000,
                    help="imaginary-time relaxation steps that build the initial state (untimed)")
    ap.add_argument("--workload", default="q2d", choices=["q2d", "3d", "sweep", "golden1d", "fno"],
                    help="q2d: 512^2 spin-2 real time (headline); 3d: 256^3 spin-1 imaginary time; "
                         "sweep: 512 ragged q2D spin-1 instances in one batched graph launch; "
                         "golden1d: the reference's published run (1D spin-2, 2048 points, to convergence); "
                         "fno: with --capture only, learned-guess training steps")
    ap.add_argument("--capture", action="store_true",
                    help="run only the workload's step kernels (warmup + steps launches of each, on the "
                         "unrelaxed guess, no timing, no other work) for profiler captures")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.capture:
        return capture(args)
    if args.workload == "fno" and not args.capture:
        ap.error("--workload fno is a profiling case: use it with --capture")
    if args.workload != "q2d" and args.impl == "ours":
        return other_workload(args)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return reference_arm(args, rank, world)

    import numpy as np
    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    import fortress_b200 as F

    cfg_gs = workload_config(WORKLOAD["gamma_gs"])
    cfg = workload_config(WORKLOAD["gamma"])
    phi0 = prepared_state(F, cfg_gs, args.prep_steps)

    prop = F.Propagator(**cfg.params(args.precision))
    # a real (non-default) stream shared by torch's events and the library
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    prop.set_stream(stream.cuda_stream)
    prop.set_state(phi0)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    npts = 512 * 512
    ms_comp, cs = 5, (16 if args.precision == "fp64" else 8)

    for _ in range(args.warmup):
        flush.zero_()
        prop.step(1, snapshot=False)
    torch.cuda.synchronize()

    # ---------------------------------------------------------- value
    # (per-kernel events cost about 10 us of device time per step, so the
    # value is timed without them; kernel_pass() below times the kernels)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = ClockSampler(local_rank)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = prop.kernel_launches()
    for k in range(args.steps):
        flush.zero_()
        evs[k][0].record(stream)
        prop.step(1, snapshot=False)
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    launches = prop.kernel_launches() - l0
    if dist:
        dist.barrier()
    clk = clocks.stop()
    total_ms = sum(a.elapsed_time(b) for a, b in evs)
    kms, kn = kernel_pass(prop, flush, args.steps)
    t_max = total_ms
    if dist:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    value = world * npts * args.steps / (t_max / 1e3)

    # --------------------------------------------------- e2e (host buffers)
    phi_host = torch.empty(npts * ms_comp * 2, dtype=torch.float64, pin_memory=True)
    phi_host.numpy()[:] = np.ascontiguousarray(phi0.reshape(-1, order="F")).view(np.float64)
    out_host = torch.empty_like(phi_host).pin_memory()
    norms_host = torch.empty(args.steps * ms_comp, dtype=torch.float64, pin_memory=True)
    # every step writes its NORMC straight into this pinned ring (the step's
    # device-to-host result read), without a call or a kernel of its own
    prop.norms_sink(norms_host.data_ptr(), args.steps)
    e2e_ms = 0.0
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps + 4)]
    flush.zero_()
    ev[0].record(stream)
    prop.set_state_host_ptr(phi_host.data_ptr())
    ev[1].record(stream)
    for k in range(args.steps):
        if k:
            flush.zero_()
        ev[2 + 2 * k].record(stream)
        prop.step(1, snapshot=(k == args.steps - 1))
        ev[3 + 2 * k].record(stream)
    flush.zero_()
    ev[2 * args.steps + 2].record(stream)
    prop.get_state_host_ptr(out_host.data_ptr())
    ev[2 * args.steps + 3].record(stream)
    torch.cuda.synchronize()
    prop.norms_sink(0, 0)
    e2e_ms = ev[0].elapsed_time(ev[1]) + ev[2 * args.steps + 2].elapsed_time(ev[2 * args.steps + 3])
    e2e_ms += sum(ev[2 + 2 * k].elapsed_time(ev[3 + 2 * k]) for k in range(args.steps))
    norms = norms_host.numpy().reshape(args.steps, ms_comp)
    # Real time conserves the discrete l2 norm; NORMC integrates with Simpson
    # weights, which the evolution does not conserve exactly once the state
    # carries grid-scale structure (the seeded noise), so the drift of that
    # norm is reported and only bounded loosely here.
    norm_drift = float(abs(norms[-1].sum() - norms[0].sum()) / norms[0].sum())
    assert np.all(np.isfinite(norms)) and norm_drift < 1e-2, norm_drift
    if dist:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * npts * args.steps / (e2e_ms / 1e3)
    state_bytes = npts * ms_comp * 16

    # ------------------------------------------------------------ roofline
    classes = ["row_x", "col_y", "col_z", "oned"]
    dom = int(np.argmax(kms))
    per_launch_ms = kms[dom] / max(kn[dom], 1)
    alg_bytes = 2 * ms_comp * npts * cs               # read + write of the spinor
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (per_launch_ms / 1e3) / 1e9
    kernels = {classes[i]: {"launches": int(kn[i]), "ms_per_launch": float(kms[i] / kn[i]),
                            "share": float(kms[i] / kms.sum())} for i in range(4) if kn[i]}

    result = {
        "metric": METRIC, "value": value, "unit": "grid-pt*steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128" if args.precision == "fp64" else "c64",
        "data": "synthetic (relaxed Gaussian guess + seeded noise)",
        "config": {"workload": WORKLOAD["name"], "grid": [512, 512], "spin": 2, "components": 5,
                   "time": "real", "dt": WORKLOAD["dt"], "precision": args.precision,
                   "parallelism": f"replicas{world}" if world > 1 else "single",
                   "l2": "flushed before every timed step (256 MiB write)",
                   "kernel_times": "second timed pass of the same steps with per-kernel CUDA events"},
        "e2e": {"value": e2e_value, "unit": "grid-pt*steps/s",
                "h2d_bytes_per_step": state_bytes / args.steps,
                "d2h_bytes_per_step": 8 * ms_comp + state_bytes / args.steps,
                "simpson_norm_drift": norm_drift},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": classes[dom], "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": known_traffic(WORKLOAD["name"], args.precision, classes[dom]),
                     "alg_bytes_per_launch": alg_bytes},
        "kernels": kernels,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, done, el, thr = run_cpu(phi0, cfg, steps=30, warmup=1, budget_s=12.0)
        result["cpu_baseline"] = {"value": rate, "unit": "grid-pt*steps/s", "cores": thr, "kind": "port",
                                  "sample": f"{done} steps of the same 512^2 workload ({el:.1f} s, oracle/ FP64 OpenMP)"}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result))


# ------------------------------------------------------- other workloads
D3 = dict(name="3d-spin1-SO-imag-256^3", n=(256, 256, 256), d=(0.1, 0.1, 0.1), dt=1e-3, mass=87.0,
          a=(101.8, 100.4, 0.0), natoms=100000, nu=(50.0, 50.0, 50.0), gamma=(0.5, 0.5, 0.5))


def sweep_instances(count=512, seed=4, precision="fp32"):
    """Seeded parameter box of the phase-diagram sweep: sizes from
    {128,192,256,384,512}^2, GAMMAX/GAMMAY in [0,2], c0 in [100,2000],
    c2/c0 in [-0.05,0.05], NUY/NUX in [1,2]; DX=0.1, DT=5e-4, spin-1, q2D,
    imaginary time.  c0, c2 are the printed TAU/2, so tau = 2c."""
    import numpy as np
    rng = np.random.default_rng(seed)
    sizes = rng.choice([128, 192, 256, 384, 512], size=count)
    out = []
    for k in range(count):
        g = rng.uniform(0, 2, 2)
        c0 = rng.uniform(100, 2000)
        c2 = c0 * rng.uniform(-0.05, 0.05)
        ay = rng.uniform(1, 2)
        n = int(sizes[k])
        out.append(dict(dim=2, spin=1, n=(n, n), d=(0.1, 0.1), dt=5e-4, imag_time=True,
                        tau=(2 * c0, 2 * c2, 0.0), gamma=(float(g[0]), float(g[1])), alpha=(1.0, ay, 1.0),
                        precision=precision))
    return out


def gaussian_nd(p):
    import numpy as np
    n = list(p["n"])
    axes = [(-1.0 + 2.0 * np.arange(m) / m) * m * d / 2.0 for m, d in zip(n, p["d"])]
    r2 = 0
    for a, x in enumerate(axes):
        shape = [1] * len(axes)
        shape[a] = -1
        r2 = r2 + p["alpha"][a] * x.reshape(shape) ** 2
    g = np.exp(-r2 / 2.0)
    ms = 2 * p["spin"] + 1
    return np.repeat(g[..., None], ms, axis=-1).astype(np.complex128)


# Wall time of the reference's own published run (its OUTPUT/ folder): 1D
# spin-2 SO-coupled imaginary time, NX=2048, run to CONV <= 1e-6.
GOLDEN_REF_S = 653.739042


def golden1d(args):
    """The reference's published run through the library's driver loop: the
    input records from the committed fixture, INITIALIZE's Gaussian, the
    reference's stop rule; one line with the wall time to convergence."""
    import numpy as np
    import torch
    import fortress_b200 as F
    from fortress_b200.driver import run
    with open(os.path.join(ROOT, "tests", "golden", "fortress_1d_spin2.json")) as f:
        golden = json.load(f)
    cfg = F.RunConfig.from_text(golden["input1D"], 1)
    x = (-1.0 + 2.0 * np.arange(cfg.n[0]) / cfg.n[0]) * cfg.n[0] * cfg.d[0] / 2.0
    g = np.sqrt(0.2) * np.exp(-cfg.alpha[0] * x * x / 2.0) / np.sqrt(np.sqrt(np.pi))
    phi = np.repeat(g[:, None], 5, axis=1).astype(np.complex128)
    clocks = ClockSampler(0)
    prop = F.Propagator.from_config(cfg)
    prop.set_state(phi)
    res = run(prop, 4 * cfg.stp, cfg.stp, cfg.tol, cfg.dt, 1)       # warm-up: graphs, first launches
    prop = F.Propagator.from_config(cfg)
    prop.set_state(phi)
    torch.cuda.synchronize()
    clocks.start()
    t0 = time.perf_counter()
    res = run(prop, cfg.niter, cfg.stp, cfg.tol, cfg.dt, 1)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    steps = res.final["ii_minus_1"] + 1
    print(json.dumps({"metric": "wall time to convergence (reference's published run)", "value": wall,
                      "unit": "s", "n_gpus": 1, "steps": steps, "warmup": 4 * cfg.stp,
                      "ms_per_step": 1e3 * wall / steps, "higher_is_better": False, "scaling": "weak",
                      "vs_baseline": wall / GOLDEN_REF_S, "dtype": "c128",
                      "data": "the reference's INPUT/input1D.dat (committed fixture) and INITIALIZE's guess",
                      "config": {"workload": "golden-1d-spin2-2048", "precision": "fp64",
                                 "exit_iteration": res.final["ii_minus_1"], "converged": bool(res.final["exited"]),
                                 "timing": "host wall clock around the driver loop (it syncs at every STP)"},
                      "clocks": clk}))


def other_workload(args):
    import numpy as np
    import torch
    import fortress_b200 as F
    if args.workload == "golden1d":
        return golden1d(args)
    from fortress_b200.config import RunConfig
    peak, peak_kind = measured_peaks()
    clocks = ClockSampler(0)
    if args.workload == "3d":
        w = D3
        cfg = RunConfig(dim=3, spin=1, n=w["n"], d=w["d"], dt=w["dt"], mass=w["mass"], a=w["a"],
                        natoms=w["natoms"], nu=w["nu"], switch_im=1, gamma=w["gamma"])
        prop = F.Propagator(**cfg.params(args.precision))
        s = torch.cuda.Stream(); torch.cuda.set_stream(s); prop.set_stream(s.cuda_stream)
        p = cfg.params(args.precision)
        phi = gaussian_nd(p)
        rng = np.random.default_rng(3)
        phi *= 1.0 + 1e-3 * rng.uniform(size=phi.shape)
        prop.set_state(phi)
        prop.normt()
        npts = int(np.prod(w["n"]))
        flush = torch.empty(256 * 2 ** 20, dtype=torch.uint8, device="cuda")
        for _ in range(args.warmup):
            flush.zero_(); prop.step(1, snapshot=False)
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        l0 = prop.kernel_launches()
        clocks.start()
        for k in range(args.steps):
            flush.zero_()
            evs[k][0].record(s); prop.step(1, snapshot=False); evs[k][1].record(s)
        torch.cuda.synchronize()
        clk = clocks.stop()
        total_ms = sum(a.elapsed_time(b) for a, b in evs)
        launches = prop.kernel_launches() - l0
        kms, kn = kernel_pass(prop, flush, args.steps)
        cs = 16 if args.precision == "fp64" else 8
        alg = 2 * 3 * npts * cs
        classes = ["row_x", "col_y", "col_z", "oned"]
        dom = int(np.argmax(kms))
        achieved = alg / (kms[dom] / kn[dom] / 1e3) / 1e9
        res = {"metric": METRIC, "value": npts * args.steps / (total_ms / 1e3), "unit": "grid-pt*steps/s",
               "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "c128" if args.precision == "fp64" else "c64", "data": "synthetic (seeded Gaussian guess)",
               "config": {"workload": w["name"], "precision": args.precision, "time": "imaginary",
                          "l2": "flushed before every timed step (state also larger than L2)",
                          "kernel_times": "second timed pass of the same steps with per-kernel CUDA events"},
               "gpu_launches": int(launches),
               "roofline": {"bound": "hbm", "kernel": classes[dom], "achieved": achieved, "peak": peak,
                            "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                            "alg_bytes_per_launch": alg},
               "kernels": {classes[i]: {"launches": int(kn[i]), "ms_per_launch": float(kms[i] / kn[i]),
                                        "share": float(kms[i] / kms.sum())} for i in range(4) if kn[i]},
               "clocks": clk}
        print(json.dumps(res))
        return 0
    # sweep
    from fortress_b200.batch import Batch
    insts = sweep_instances(precision=args.precision)
    b = Batch(insts)
    for i, p in enumerate(insts):
        b[i].set_state(gaussian_nd(p))
        b[i].normt()
    tune = b.autotune(trial_steps=4, cache_path=os.path.join(out_dir(), "autotune_cache.txt"))
    npts = sum(int(np.prod(p["n"])) for p in insts)
    b.step(max(args.warmup, 4))
    clocks.start()
    steps = args.steps + (1 if args.steps % tune[1] == 1 else 0)   # whole graph launches only
    el = b.step_timed(steps) / 1e3                                # CUDA events on the launch stream
    args.steps = steps
    clk = clocks.stop()
    cs = 16 if args.precision == "fp64" else 8
    res = {"metric": METRIC, "value": npts * args.steps / el, "unit": "grid-pt*steps/s", "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "c128" if args.precision == "fp64" else "c64", "data": "synthetic (seeded parameter box, seed 4)",
           "config": {"workload": "sweep-512-ragged-q2d-spin1-imag", "instances": len(insts),
                      "sizes": sorted(set(p["n"][0] for p in insts)), "precision": args.precision,
                      "autotuned": {"width": tune[0], "steps_per_graph": tune[1]},
                      "hbm_bytes_per_step_alg": 2 * 2 * 3 * npts * cs,
                      "l2": "batch state larger than L2"},
           "achieved_gbs_alg": 2 * 2 * 3 * npts * cs / (el / args.steps) / 1e9, "peak": peak,
           "clocks": clk}
    print(json.dumps(res))
    return 0


def reference_arm(args, rank, world):
    if rank != 0:
        return 0
    import numpy as np  # noqa: F401
    cfg = workload_config(WORKLOAD["gamma"])
    phi = add_noise(gaussian_guess(cfg))
    rate, done, el, thr = run_cpu(phi, cfg, steps=args.steps, warmup=args.warmup, budget_s=90.0)
    res = {"metric": METRIC, "value": rate, "unit": "grid-pt*steps/s", "n_gpus": world, "steps": done,
           "warmup": args.warmup, "ms_per_step": 1e3 * el / done, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "c128", "impl": "reference",
           "data": "synthetic (Gaussian guess + seeded noise)",
           "config": {"workload": WORKLOAD["name"], "grid": [512, 512], "spin": 2, "time": "real",
                      "precision": "fp64", "parallelism": "cpu"},
           "cpu_baseline": {"value": rate, "unit": "grid-pt*steps/s", "cores": thr, "kind": "port",
                            "sample": f"{done} timed steps after {args.warmup} warm-up steps"},
           "e2e": {"value": rate, "unit": "grid-pt*steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(res))
    return 0


if __name__ == "__main__":
    sys.exit(main() or 0)
