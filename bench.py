#!/usr/bin/env python
"""Benchmark of the split-step spinor propagator on B200.

Default workload (the largest configuration, the one the time-to-ground-state
target is stated on): 3D spin-1 SO-coupled imaginary-time propagation on a
256^3 grid, DX=DY=DZ=0.1, DT=1e-3, Rb-87 (mass 87, a0/a2 = 101.8/100.4 a_B),
NATOMS=100000, NUX=NUY=NUZ=50 Hz, GAMMAX=GAMMAY=GAMMAZ=0.5.  Synthetic
initial state, identical in both arms: INITIALIZE's 3D spin-1 Gaussian
(cgpe3d.f90:783-785) times (1 + 1e-3 u), u ~ U[0,1) from numpy PCG64 seed 3,
then NORMT.  No dataset is involved.

A step is one full Lie split step FFT->KE->SOC->BFT->SE->SP->NORMC->NORMT of
the whole 256^3 x 3 spinor.  Metric: grid-pt*steps/s (higher is better).
The arithmetic is FP64 complex (the reference's precision); the FP32-bulk
path (complex64 FFTs and exponentials, FP64 reductions) is reported beside it
under "fp32".

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload 3d|q2d|sweep|golden1d]

value : device time (CUDA events on the launching stream) of K steps back to
        back; the 805 MB state is larger than the 126 MB L2, so every step
        streams it from HBM; max over ranks.
e2e   : the same metric through the C ABI with host buffers, on a host wall
        clock: pinned host->device upload of the state, K steps with every
        step's NORMC written into a pinned host ring by the step itself
        (fgpe_norms_sink), device->host download of the final state, and a
        stream synchronisation, all inside the timed region.
The reference arm (--impl reference) times the CPU restatement of the
reference (oracle/, OpenMP on all host cores) on the same workload, the same
initial state and the same config: the Fortran/FFTW/LAPACK reference cannot
be compiled on this image.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "grid-pt*steps/s"

# 3D spin-1 SO-coupled imaginary time (the largest configuration)
D3 = dict(name="3d-spin1-SO-imag-256^3", dim=3, spin=1, n=(256, 256, 256), d=(0.1, 0.1, 0.1), dt=1e-3,
          mass=87.0, a=(101.8, 100.4, 0.0), natoms=100000, nu=(50.0, 50.0, 50.0), gamma=(0.5, 0.5, 0.5),
          switch_im=1, seed=3)
# q2D spin-2 SO-coupled real-time quench (GAMMAX 1.0 -> 1.2 at t = 0)
Q2D = dict(name="q2d-spin2-SO-realtime-512x512-quench", dim=2, spin=2, n=(512, 512, 1), d=(0.05, 0.05, 1.0),
           dt=1e-4, mass=87.0, a=(87.93, 91.28, 99.18), natoms=50000, nu=(20.0, 20.0, 500.0),
           gamma=(1.2, 1.0, 0.0), switch_im=0, seed=2)
WORKLOADS = {"3d": D3, "q2d": Q2D}


def run_config(w, n=None, d=None):
    from fortress_b200.config import RunConfig
    return RunConfig(dim=w["dim"], spin=w["spin"], n=n or w["n"], d=d or w["d"], dt=w["dt"], mass=w["mass"],
                     a=w["a"], natoms=w["natoms"], nu=w["nu"], switch_im=w["switch_im"], gamma=w["gamma"])


def initial_state(w, n=None, d=None):
    """The workload's synthetic start, PHI(NX,NY,NZ,M) complex128.
    3D: INITIALIZE's default spin-1 guess exp(-(x^2+y^2+z^2)/2)/pi^(3/4) in
    every component (cgpe3d.f90:783-785) times (1 + 1e-3 u), u ~ U[0,1).
    q2D: the spin-2 default sqrt(0.2) exp(-(ax x^2 + ay y^2)/2)/sqrt(pi)
    (cgpe2d.f90:766-771) plus 1e-3 of its peak in complex Gaussian noise."""
    import numpy as np
    n = n or w["n"]
    d = d or w["d"]
    ms = 2 * w["spin"] + 1
    rng = np.random.default_rng(w["seed"])
    ax = [(-1.0 + 2.0 * np.arange(n[a]) / n[a]) * n[a] * d[a] / 2.0 for a in range(w["dim"])]
    if w["dim"] == 3:
        r2 = ax[0][:, None, None] ** 2 + ax[1][None, :, None] ** 2 + ax[2][None, None, :] ** 2
        g = np.exp(-r2 / 2.0) / np.pi ** 0.75
        phi = np.empty(tuple(n) + (ms,), np.complex128)
        for m in range(ms):
            phi[..., m] = g * (1.0 + 1e-3 * rng.uniform(size=g.shape))
        return phi
    nu = w["nu"]
    al = (1.0, nu[1] / nu[0])
    g = np.sqrt(0.2) * np.exp(-(al[0] * ax[0][:, None] ** 2 + al[1] * ax[1][None, :] ** 2) / 2.0) / np.sqrt(np.pi)
    phi = np.repeat(g[:, :, None, None], ms, axis=3).astype(np.complex128)
    return phi + 1e-3 * np.abs(phi).max() * (rng.standard_normal(phi.shape) + 1j * rng.standard_normal(phi.shape))


def bench_config(w, precision="fp64", world=1, impl="ours"):
    """The config object both arms print (the driver compares them)."""
    return {"workload": w["name"], "grid": list(w["n"][:w["dim"]]), "spin": w["spin"],
            "components": 2 * w["spin"] + 1, "time": "imaginary" if w["switch_im"] else "real",
            "dt": w["dt"], "gamma": list(w["gamma"][:w["dim"]]), "precision": precision,
            "parallelism": f"replicas{world}" if world > 1 else "single",
            "l2": "state larger than L2 (not flushed)" if w is D3 else "flushed before every timed step (256 MiB write)"}


def data_string(w):
    if w is D3:
        return "synthetic: INITIALIZE's 3D spin-1 Gaussian x (1 + 1e-3 U[0,1), PCG64 seed 3), NORMT"
    return "synthetic: INITIALIZE's q2D spin-2 Gaussian + 1e-3 complex Gaussian noise (PCG64 seed 2), quench"

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


def profile_figures(workload, precision, kernel):
    """Per-launch DRAM traffic and FP64 pipe utilisation of a kernel, from
    the committed ncu summaries (profiles/traffic.json: dram__bytes_read.sum
    + dram__bytes_write.sum per launch, scaled to the bench grid where the
    capture ran on a smaller one, and sm__pipe_fp64_cycles_active in % of its
    peak).  (None, None) when not captured."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        e = d.get(f"{workload}/{precision}/{kernel}")
    except Exception:
        return None, None
    if e is None:
        return None, None
    if isinstance(e, dict):
        return e.get("dram_bytes"), e.get("fp64_pipe_pct")
    return e, None


def fp64_peak_tflops():
    """Measured FP64 FMA throughput of this device (fgpe_fp64_fma_rate)."""
    from fortress_b200 import _abi
    t = ctypes.c_double()
    rc = _abi.load().fgpe_fp64_fma_rate(200000, ctypes.byref(t))
    return float(t.value) if rc == 0 else None




# --------------------------------------------------------------- CPU legs
def oracle_for(w, phi):
    """The oracle on the workload's parameters, holding phi."""
    from oracle import oracle as O
    cfg = run_config(w)
    t = cfg.tau()
    n, d, g, al = cfg.n, cfg.d, cfg.gamma, cfg.alpha
    orc = O.Oracle(dim=w["dim"], spin=w["spin"], nx=n[0], ny=n[1], nz=n[2], dx=d[0], dy=d[1], dz=d[2],
                   dt=cfg.dt, imag=int(cfg.switch_im), tau=t, gx=g[0], gy=g[1], gz=g[2],
                   ax=al[0], ay=al[1], az=al[2])
    orc.set_state(phi)
    if cfg.switch_im:
        orc.normt()
    return orc, O.num_threads()


def run_cpu(w, phi, steps, warmup, budget_s):
    """Oracle split steps on the host cores: warm-up steps, then up to
    `steps` timed steps, stopping after budget_s seconds (at least one)."""
    orc, thr = oracle_for(w, phi)
    for _ in range(warmup):
        orc.step(1)
    npts = int(w["n"][0] * w["n"][1] * w["n"][2])
    done, t0 = 0, time.perf_counter()
    while done < steps:
        orc.step(1)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    el = time.perf_counter() - t0
    del orc
    return npts * done / el, done, el, thr


def capture(args):
    """The step kernels alone, for ncu launch lists and per-kernel captures
    (-k regex:k_row_fast / k_col_fast / k_obs ...): warmup + steps split
    steps of the workload on its initial state, no timing and no other work.
    --workload 3d runs the 3D spin-1 case on --grid^3 points (default 192:
    the same kernel families as 256^3, wide column tiles included, with a
    340 MB state that still exceeds L2, for DRAM figures that scale to the
    bench grid); --workload q2d the 512^2 spin-2 real-time case; --workload
    fno learned-guess training steps; --workload golden1d the reference's
    published 1D run."""
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
    if args.workload == "tour":
        return kernel_tour(args)
    if args.workload == "sweep":
        # a reduced phase-diagram batch in the grouped mode: 32 instances of
        # the seeded box, warmup + steps grouped steps
        from fortress_b200.batch import Batch
        insts = sweep_instances(count=32, precision=args.precision if args.precision_set else "fp32")
        b = Batch(insts)
        for i, p in enumerate(insts):
            b[i].set_state(gaussian_nd(p))
            b[i].normt()
        if args.batch_mode == "persistent":
            b.mode(persistent=True)
            b.variant(max(args.variant, 0))
        else:
            b.mode(grouped=True)
        b.config(32, 4)
        b.step(args.warmup + args.steps)
        obs = b.observables(with_conv=False)
        assert all(np.isfinite(o["en"]) for o in obs)
        print(json.dumps({"capture": "sweep-%s-32" % ("persistent" if args.batch_mode == "persistent" else "grouped"),
                          "steps": args.warmup + args.steps}))
        return
    w = WORKLOADS[args.workload]
    if w is D3:
        g = args.grid or 192
        n, d = (g, g, g), (25.6 / g,) * 3
    else:
        n, d = w["n"], w["d"]
    cfg = run_config(w, n, d)
    prop = F.Propagator(**cfg.params(args.precision))
    prop.set_state(initial_state(w, n, d))
    if cfg.switch_im:
        prop.normt()
    prop.step(args.warmup + args.steps, snapshot=False)
    if args.observables:
        en = prop.observables()[0]
        assert np.isfinite(en)
    nrm = prop.normc()
    assert np.all(np.isfinite(nrm))
    print(json.dumps({"capture": w["name"], "grid": list(n[:w["dim"]]), "precision": args.precision,
                      "steps": args.warmup + args.steps, "norm": float(nrm.sum())}))


def kernel_tour(args):
    """Every kernel family of the library once, each on a small case, for a
    per-kernel ncu capture (ncu -k regex:... -c <launches>): the observables
    (k_obs), state import/export (k_import, k_export), the NORMC read-back
    (k_norms_out), the 1D kernels (k_1d single block, k_cl1d cluster, k_r1d /
    k_c1d split), the generic row/column kernels (k_row, k_col on 160-point
    lines), the unfused operators (k_pointwise_op, k_permute), the
    handle-free NORMC (k_normc_noalloc) and the learned-guess kernels (GEMM,
    bias/GELU, dense tcgen05 layer, MSE, Adam)."""
    import ctypes
    import numpy as np
    import torch
    import fortress_b200 as F
    from fortress_b200 import _abi
    rng = np.random.default_rng(0)

    def rnd(shape):
        return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * 0.1

    # 3D 192^3 spin-1: import (FP32 handle), observables, export, NORMC read-back
    cfg = run_config(D3, (192, 192, 192), (25.6 / 192,) * 3)
    prop = F.Propagator(**cfg.params("fp32"))
    prop.set_state(initial_state(D3, (192, 192, 192), (25.6 / 192,) * 3))
    prop.normt()
    prop.step(2)
    prop.observables()
    pinned = torch.empty(8, dtype=torch.float64, pin_memory=True)
    prop.norms_async(pinned.data_ptr())
    prop.state()
    prop.close()
    # 1D: single block (spin-1, 256), cluster (spin-2, 2048), split (spin-2, 8192)
    for n, spin, d in ((256, 1, 0.1), (2048, 2, 0.05), (8192, 2, 0.02)):
        q = F.Propagator(dim=1, spin=spin, n=(n,), d=(d,), dt=1e-4, imag_time=True,
                         tau=(200.0, 5.0, -3.0), gamma=(0.5,), alpha=(1.0, 20.0, 20.0))
        x = (-1.0 + 2.0 * np.arange(n) / n) * n * d / 2.0
        q.set_state(np.repeat(np.exp(-x * x / 2)[:, None], 2 * spin + 1, axis=1).astype(complex))
        q.step(3)
        q.close()
    # generic 2D kernels (160-point lines) and the unfused operators
    q = F.Propagator(dim=2, spin=2, n=(160, 160), d=(0.15, 0.15), dt=1e-4, imag_time=False,
                     tau=(300.0, 10.0, -8.0), gamma=(0.5, 0.3), alpha=(1.0, 1.2, 1.0))
    q.set_state(rnd((160, 160, 5)))
    q.step(3)
    for op in ("FFT", "KE", "SOC", "BFT", "SE", "SP"):
        q.apply_op(op)
    q.close()
    # handle-free NORMC
    phi = torch.tensor(rnd((3, 128, 128)).astype(np.complex128), device="cuda")
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    rc = _abi.load().fgpe_normc_noalloc(2, 1, 128, 128, 1, 0.1, 0.1, 0.1, ctypes.c_void_p(phi.data_ptr()),
                                        ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 0
    # learned-guess kernels: one training step at 64^2, batch 16
    from fortress_b200 import fno as FN
    net = FN.FNO(64, 16, seed=7)
    a = FN.input_channels(rng.uniform(-1, 1, (16, 5)), 64)
    tgt = torch.randn(6, 16 * 64 * 64, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    net.forward(a); net.loss(tgt); net.backward(); net.adam()
    torch.cuda.synchronize()
    assert not net.tc_error()
    print(json.dumps({"capture": "kernel-tour"}))


def kernel_pass(prop, flush, steps):
    """Per-kernel device times: a second timed pass of the same steps with
    CUDA events recorded by the library around every kernel launch on its
    stream (fgpe_profile_*).  Returns (ms per class, launches per class)."""
    import torch
    prop.profile(True)
    prop.profile_read(reset=True)
    for _ in range(steps):
        if flush is not None:
            flush.zero_()
        prop.step(1, snapshot=False)
    torch.cuda.synchronize()
    kms, kn = prop.profile_read(reset=True)
    prop.profile(False)
    return kms, kn


KCLASS = ["row_x", "col_y", "col_z", "oned"]


def device_rate(F, w, phi, precision, steps, warmup, stream, flush, world, dist, kernels="auto"):
    """value of one precision: K split steps on the device between CUDA
    events on the launching stream (max over ranks), plus the per-kernel
    pass.  Returns a dict and the propagator."""
    import numpy as np
    import torch
    cfg = run_config(w)
    prop = F.Propagator(**cfg.params(precision), kernels=kernels)
    prop.set_stream(stream.cuda_stream)
    prop.set_state(phi)
    if cfg.switch_im:
        prop.normt()
    npts = int(np.prod(w["n"]))
    for _ in range(warmup):
        if flush is not None:
            flush.zero_()
        prop.step(1, snapshot=False)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = prop.kernel_launches()
    if flush is None:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            prop.step(1, snapshot=False)
        e1.record(stream)
        torch.cuda.synchronize()
        total_ms = e0.elapsed_time(e1)
    else:
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for k in range(steps):
            flush.zero_()
            evs[k][0].record(stream)
            prop.step(1, snapshot=False)
            evs[k][1].record(stream)
        torch.cuda.synchronize()
        total_ms = sum(a.elapsed_time(b) for a, b in evs)
    launches = prop.kernel_launches() - l0
    if dist:
        dist.barrier()
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    kms, kn = kernel_pass(prop, flush, steps)
    return {"value": world * npts * steps / (total_ms / 1e3), "ms_per_step": total_ms / steps,
            "launches": int(launches), "kms": kms, "kn": kn}, prop


def roofline(w, precision, kms, kn, peak, peak_kind, fp64_peak):
    """HBM roofline of the dominant kernel class (algorithmic bytes per
    launch = the spinor read and written once, 2*M*N*s) and its FP64
    compute fraction against the measured FP64 FMA peak."""
    import numpy as np
    npts = int(np.prod(w["n"]))
    ms_comp = 2 * w["spin"] + 1
    cs = 16 if precision == "fp64" else 8
    dom = int(np.argmax(kms))
    per_launch_ms = kms[dom] / max(kn[dom], 1)
    alg = 2 * ms_comp * npts * cs
    achieved = alg / (per_launch_ms / 1e3) / 1e9
    traffic, fp64_pct = profile_figures(w["name"], precision, KCLASS[dom])
    r = {"bound": "hbm", "kernel": KCLASS[dom], "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic, "alg_bytes_per_launch": alg,
         "ms_per_launch": per_launch_ms}
    if fp64_pct is not None:
        # compute side: the FP64 pipe's active fraction of its peak (ncu),
        # with this device's FP64 FMA peak measured in the same run
        r["fp64"] = {"frac": fp64_pct / 100.0, "basis": "sm__pipe_fp64_cycles_active (ncu capture in profiles/)",
                     "peak": fp64_peak, "unit": "TFLOP/s", "peak_kind": "measured (fgpe_fp64_fma_rate, this run)"}
    per_class = {}
    for i in range(4):
        if kn[i]:
            tr, pct = profile_figures(w["name"], precision, KCLASS[i])
            ms = kms[i] / kn[i]
            per_class[KCLASS[i]] = {"hbm_frac": alg / (ms / 1e3) / 1e9 / peak, "traffic": tr,
                                    "fp64_pipe_frac": (pct / 100.0) if pct is not None else None}
    r["per_kernel"] = per_class
    kernels = {KCLASS[i]: {"launches": int(kn[i]), "ms_per_launch": float(kms[i] / kn[i]),
                           "share": float(kms[i] / kms.sum())} for i in range(4) if kn[i]}
    return r, kernels


def e2e_rate(prop, w, phi_host, out_host, norms_host, steps, world, dist):
    """The public API with host buffers on a host wall clock: upload, K
    steps (each writes its NORMC into the pinned ring), download, sync."""
    import numpy as np
    import torch
    ms_comp = 2 * w["spin"] + 1
    npts = int(np.prod(w["n"]))
    prop.norms_sink(norms_host.data_ptr(), steps)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    prop.set_state_host_ptr(phi_host.data_ptr())
    if w["switch_im"]:
        prop.normt()
    prop.step(steps, snapshot=True)
    prop.get_state_host_ptr(out_host.data_ptr())     # synchronises the stream
    el = time.perf_counter() - t0
    prop.norms_sink(0, 0)
    norms = norms_host.numpy().reshape(steps, ms_comp)
    assert np.all(np.isfinite(norms)) and np.all(np.isfinite(out_host.numpy()[:1024]))
    if dist:
        t = torch.tensor([el], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        el = float(t.item())
    state_bytes = npts * ms_comp * 16
    return {"value": world * npts * steps / el, "unit": METRIC, "wall_s": el,
            "h2d_bytes_per_step": state_bytes / steps, "d2h_bytes_per_step": 8 * ms_comp + state_bytes / steps,
            "timing": "host wall clock around upload, steps, per-step NORMC ring and download"}


# -------------------------------------------------------------------- main
def ours(args, w, rank, world, local_rank):
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

    phi = initial_state(w)
    npts = int(np.prod(w["n"]))
    ms_comp = 2 * w["spin"] + 1
    # a real (non-default) stream shared by torch's events and the library
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = None if w is D3 else torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    peak, peak_kind = measured_peaks()
    fp64_peak = fp64_peak_tflops()

    clocks = ClockSampler(local_rank)
    clocks.start()
    main, prop = device_rate(F, w, phi, args.precision, args.steps, args.warmup, stream, flush, world, dist,
                             args.kernels)
    clk = clocks.stop()
    rl, kernels = roofline(w, args.precision, main["kms"], main["kn"], peak, peak_kind, fp64_peak)

    # e2e through the C ABI with host buffers (FP64 state in PHI layout)
    phi_host = torch.empty(npts * ms_comp * 2, dtype=torch.float64, pin_memory=True)
    phi_host.numpy()[:] = np.ascontiguousarray(phi.reshape(-1, order="F")).view(np.float64)
    out_host = torch.empty_like(phi_host).pin_memory()
    norms_host = torch.empty(args.steps * ms_comp, dtype=torch.float64, pin_memory=True)
    e2e = e2e_rate(prop, w, phi_host, out_host, norms_host, args.steps, world, dist)
    prop.close()

    result = {
        "metric": METRIC, "value": main["value"], "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": main["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c128" if args.precision == "fp64" else "c64", "data": data_string(w),
        "config": bench_config(w, args.precision, world),
        "e2e": e2e, "gpu_launches": main["launches"], "roofline": rl, "kernels": kernels, "clocks": clk,
    }
    if args.precision == "fp64" and not args.no_fp32:
        f32, p32 = device_rate(F, w, phi, "fp32", args.steps, args.warmup, stream, flush, world, dist, args.kernels)
        p32.close()
        rl32, k32 = roofline(w, "fp32", f32["kms"], f32["kn"], peak, peak_kind, fp64_peak)
        result["fp32"] = {"value": f32["value"], "ms_per_step": f32["ms_per_step"], "dtype": "c64",
                          "what": "FP32 bulk: complex64 FFTs and exponentials, FP64 reductions and NORMT",
                          "gpu_launches": f32["launches"], "roofline": rl32, "kernels": k32}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, done, el, thr = run_cpu(w, phi, steps=30, warmup=0, budget_s=20.0)
        result["cpu_baseline"] = {"value": rate, "unit": METRIC, "cores": thr, "kind": "port",
                                  "sample": f"{done} split steps of the same workload from the same state "
                                            f"({el:.1f} s, oracle/ FP64 OpenMP on {thr} threads)"}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result))


def reference_arm(args, w, rank, world):
    """The reference's algorithm on the host cores (the oracle port: the
    Fortran reference cannot be built here), same workload, state and
    config; each timed step is one whole split step of the full grid."""
    if rank != 0:
        return 0
    phi = initial_state(w)
    warm = min(args.warmup, 1)
    rate, done, el, thr = run_cpu(w, phi, steps=args.steps, warmup=warm, budget_s=90.0)
    res = {"metric": METRIC, "value": rate, "unit": METRIC, "n_gpus": world, "steps": done,
           "warmup": args.warmup, "ms_per_step": 1e3 * el / done, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "c128" if args.precision == "fp64" else "c64",
           "impl": "reference", "data": data_string(w), "config": bench_config(w, args.precision, world),
           "cpu_baseline": {"value": rate, "unit": METRIC, "cores": thr, "kind": "port",
                            "sample": f"{done} timed split steps after {warm} warm-up step(s), "
                                      f"at most 90 s (oracle/ FP64 OpenMP on {thr} threads)"},
           "e2e": {"value": rate, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(res))
    return 0


# ------------------------------------------------------- other workloads
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



def sweep(args):
    """512 ragged q2D spin-1 instances (seed 4) advanced by the batched
    launcher after its autotuner has picked the launch shape."""
    import numpy as np
    from fortress_b200.batch import Batch
    peak, _ = measured_peaks()
    clocks = ClockSampler(0)
    insts = sweep_instances(precision=args.precision if args.precision_set else "fp32")
    b = Batch(insts)
    for i, p in enumerate(insts):
        b[i].set_state(gaussian_nd(p))
        b[i].normt()
    cache = os.path.join(out_dir(), "autotune_cache.txt")
    tune = b.autotune(trial_steps=4, cache_path=cache)
    tuned_mode = {0: "branches", 1: "grouped", 2: "persistent"}.get(int(open(cache).read().split()[-2]), "?")
    if args.batch_mode != "auto":
        b.mode(grouped=args.batch_mode == "grouped", persistent=args.batch_mode == "persistent")
        if args.batch_mode == "persistent" and args.variant >= 0:
            b.variant(args.variant)
        b.config(tune[0], tune[1])
    npts = sum(int(np.prod(p["n"])) for p in insts)
    b.step(max(args.warmup, 4))
    clocks.start()
    steps = args.steps + (1 if args.steps % tune[1] == 1 else 0)   # whole graph launches only
    el = b.step_timed(steps) / 1e3                                # CUDA events on the launch stream
    clk = clocks.stop()
    prec = insts[0]["precision"]
    cs = 16 if prec == "fp64" else 8
    alg = 2 * 2 * 3 * npts * cs
    res = {"metric": METRIC, "value": npts * steps / el, "unit": METRIC, "n_gpus": 1,
           "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "c128" if prec == "fp64" else "c64", "data": "synthetic (seeded parameter box, seed 4)",
           "config": {"workload": "sweep-512-ragged-q2d-spin1-imag", "instances": len(insts),
                      "sizes": sorted(set(p["n"][0] for p in insts)), "precision": prec,
                      "autotuned": {"width": tune[0], "steps_per_graph": tune[1], "mode": tuned_mode,
                                    "variant": b.variant(), "variant_shape": Batch.variant_shapes()[b.variant()]},
                      "batch_mode": args.batch_mode,
                      "l2": "batch state larger than L2"},
           "roofline": {"bound": "hbm", "kernel": "whole batch step", "achieved": alg / (el / steps) / 1e9,
                        "peak": peak, "unit": "GB/s", "frac": alg / (el / steps) / 1e9 / peak,
                        "alg_bytes_per_step": alg},
           "clocks": clk}
    print(json.dumps(res))
    return 0


def time_to_ground_state(args):
    """Time to the 256^3 spin-1 ground state: wall time until
    |E - E*| <= 1e-8 |E*| holds for good (energy every 100 steps), E* the
    lowest final FP64 energy of the arms.  Arms (fortress_b200.experiments.
    time_to_gs): plain FP64 from INITIALIZE's seeded Gaussian (the
    reference's method); coarse (64^3 FP64 solve, spectral prolongation,
    FP32 to its stop rule, then FP64); learned (the trained 3D network's
    guess, FP32, then FP64) and learned_coarse (the guess on 64^3 as the
    coarse solve's start, then as coarse) when --fno3d names a saved
    parameter file."""
    import numpy as np
    import torch
    from fortress_b200.experiments import time_to_gs as T
    tp = T.target_point()
    arms = ["plain", "coarse"]
    infer = infer64 = None
    if args.fno3d:
        from fortress_b200 import fno3d as F3
        pz = dict(np.load(args.fno3d))
        W = pz["P"].shape[0]
        M = pz["Rr0"].shape[-1]
        layers = sum(1 for k in pz if k.startswith("Rr"))
        infer = F3.FNO3(256, 1, params=pz, width=W, modes=M, layers=layers, hidden=pz["Q1"].shape[0], train=False)
        infer64 = F3.FNO3(64, 1, params=pz, width=W, modes=M, layers=layers, hidden=pz["Q1"].shape[0], train=False)
        arms += ["learned", "learned_coarse"]
    clocks = ClockSampler(0)
    clocks.start()
    traces = {"plain": T.arm("plain", tp, 256, max_steps=args.tts_max_steps)}
    e_ref = traces["plain"][-1][3]
    for k in arms[1:]:
        traces[k] = T.arm(k, tp, 256, net=infer, max_steps=args.tts_max_steps, e_ref=e_ref, coarse_net=infer64)
    clk = clocks.stop()
    e_star = min(tr[-1][3] for tr in traces.values())
    res = {}
    for k, tr in traces.items():
        t = T.time_to(tr, e_star)
        res[k] = {"time_s": t[1] if t else None, "steps": t[0] if t else None,
                  "E_final_rel_to_Estar": (tr[-1][3] - e_star) / abs(e_star)}
    best = min((k for k in arms if k != "plain" and res[k]["time_s"]), key=lambda k: res[k]["time_s"], default=None)
    plain = res["plain"]["time_s"]
    out = {"metric": "time to |E-E*| <= 1e-8 |E*| (256^3 spin-1 SO ground state)",
           "value": res[best]["time_s"] if best else None, "unit": "s", "n_gpus": 1, "higher_is_better": False,
           "scaling": "weak", "vs_baseline": None, "dtype": "c64 then c128", "data": data_string(D3),
           "config": {"workload": "tts-3d-spin1-SO-256^3", "arm": best, "stp": T.STP, "tol_rel": T.TOL_REL},
           "E_star": e_star, "arms": res, "plain_fp64_s": plain,
           "speedup_vs_plain_fp64": (plain / res[best]["time_s"]) if (best and plain) else None, "clocks": clk}
    print(json.dumps(out))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=None, choices=["fp64", "fp32"],
                    help="arithmetic of the headline value (default fp64; the fp32 figure is added beside it)")
    ap.add_argument("--no-fp32", action="store_true", help="skip the FP32-bulk figure")
    ap.add_argument("--kernels", default="auto", choices=["auto", "generic", "warp-row", "block-row"],
                    help="kernel family of the timed propagators (fgpe_params.kernels)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="3d", choices=["3d", "q2d", "sweep", "golden1d", "tts", "fno", "tour"],
                    help="3d: 256^3 spin-1 imaginary time (headline); q2d: 512^2 spin-2 real-time quench; "
                         "sweep: 512 ragged q2D spin-1 instances in one batched graph launch; "
                         "golden1d: the reference's published run (1D spin-2, 2048 points, to convergence); "
                         "tts: time to the 256^3 spin-1 ground state (plain FP64 against coarse/learned + FP32); "
                         "fno: with --capture only, learned-guess training steps; "
                         "tour: with --capture only, every kernel family once")
    ap.add_argument("--capture", action="store_true",
                    help="run only the workload's step kernels (warmup + steps launches of each, no timing, "
                         "no other work) for profiler captures")
    ap.add_argument("--grid", type=int, default=0, help="with --capture --workload 3d: points per axis (192)")
    ap.add_argument("--observables", action="store_true", help="with --capture: also run ENERGY/RAD (k_obs)")
    ap.add_argument("--fno3d", default=None, help="with --workload tts: saved 3D network parameters (.npz)")
    ap.add_argument("--batch-mode", default="auto", choices=["auto", "grouped", "branches", "persistent"],
                    help="with --workload sweep: the autotuner's choice, or force grouped / per-instance branches / "
                         "one persistent launch")
    ap.add_argument("--variant", type=int, default=-1,
                    help="with --batch-mode persistent: the persistent kernel variant (default: the autotuner's)")
    ap.add_argument("--tts-max-steps", type=int, default=60000, help="with --workload tts: steps per FP64 stage")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    args.precision_set = args.precision is not None
    args.precision = args.precision or "fp64"
    if args.capture:
        return capture(args)
    if args.workload in ("fno", "tour"):
        ap.error(f"--workload {args.workload} is a profiling case: use it with --capture")
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload in WORKLOADS:
        w = WORKLOADS[args.workload]
        if args.impl == "reference":
            return reference_arm(args, w, rank, world)
        return ours(args, w, rank, world, local_rank)
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": f"--impl reference covers the 3d and q2d "
                                                                  f"workloads, not {args.workload}"}))
        return 0
    if args.workload == "golden1d":
        return golden1d(args)
    if args.workload == "tts":
        return time_to_ground_state(args)
    return sweep(args)


if __name__ == "__main__":
    sys.exit(main() or 0)
