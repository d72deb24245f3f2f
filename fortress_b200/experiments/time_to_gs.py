"""Time to the 3D spin-1 ground state: learned guess + FP32 against plain FP64.

Target problem (the largest configuration): 3D spin-1 SO-coupled imaginary
time on 256^3 points, DX=DY=DZ=0.1, DT=1e-3, Rb-87 a0/a2 = 101.8/100.4 a_B,
NATOMS=1e5, NU=(50,50,50) Hz, GAMMA=(0.5,0.5,0.5).  The quantity measured is
the wall time until |E - E*| <= 1e-8 |E*| holds for good (energy checked
every STP = 100 steps, as the reference's loop checks its stop rule,
cgpe3d.f90:497-508), with E* the FP64 energy after a long run past
convergence.  Arms, all on one B200 from the same seeded start where a start
is needed:

  plain      INITIALIZE's 3D spin-1 Gaussian (cgpe3d.f90:783-785) x (1 + 1e-3
             U[0,1), PCG64 seed 3), FP64 throughout: the reference's method.
  learned    the 3D Fourier neural operator (fortress_b200.fno3d), trained on
             ground states the solver computed on a 64^3 grid of the same box
             over a parameter box around the target, evaluated directly on the
             256^3 grid (inference time counted); then the FP32-bulk path to
             its own stop rule (CONV or CONV_EN <= 1e-6), then FP64.
  learned64  the same guess, FP64 throughout (the network's own gain).
  coarse     no network: the plain start solved on the 64^3 grid (FP64, to the
             stop rule at 1e-8), spectrally prolonged to 256^3 (the library's
             FFT on 64^3, zero padding of the spectrum, its BFT on 256^3),
             then FP32 and FP64 as in "learned" (the coarse-to-fine gain
             without learning).
  learned_coarse  the network's guess on the 64^3 grid as the start of the
             coarse solve, then as "coarse" (the network's gain on top of the
             coarse-to-fine method).

The target parameter point is held out of the training set (the training
points are drawn from the box with seed 5 and none coincides with it).

    python -m fortress_b200.experiments.time_to_gs [--train 192] [--epochs 60] [--out DIR]

Prints one JSON object per stage; the last one is the comparison.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

L_BOX = 25.6
STP = 100
TOL_REL = 1e-8


# ------------------------------------------------------------- parameters
def target_point():
    """(gamma, c0, c2/c0, NUZ/NUX) of the 256^3 workload (c0 = TAU(0)/2)."""
    from fortress_b200.config import RunConfig
    c = RunConfig(dim=3, spin=1, n=(256, 256, 256), d=(0.1, 0.1, 0.1), dt=1e-3, mass=87.0, a=(101.8, 100.4, 0.0),
                  natoms=100000, nu=(50.0, 50.0, 50.0), switch_im=1, gamma=(0.5, 0.5, 0.5))
    t = c.tau()
    return np.array([0.5, t[0] / 2.0, t[1] / t[0], 1.0])


def box_points(count, seed):
    from fortress_b200.fno3d import BOX3
    rng = np.random.default_rng(seed)
    lo = np.array([v[0] for v in BOX3.values()])
    hi = np.array([v[1] for v in BOX3.values()])
    return lo + (hi - lo) * rng.uniform(size=(count, 4))


def params(point, n, precision="fp64", dt=1e-3):
    g, c0, r2, az = (float(v) for v in point)
    d = L_BOX / n
    return dict(dim=3, spin=1, n=(n, n, n), d=(d, d, d), dt=dt, imag_time=True, tau=(2 * c0, 2 * c0 * r2, 0.0),
                gamma=(g, g, g), alpha=(1.0, 1.0, az), precision=precision)


def gaussian_start(n, seed=3):
    """INITIALIZE's 3D spin-1 default: the unweighted Gaussian in every
    component (cgpe3d.f90:783-785), times (1 + 1e-3 u), u ~ U[0,1)."""
    d = L_BOX / n
    x = (-1.0 + 2.0 * np.arange(n) / n) * n * d / 2.0
    g = np.exp(-(x[:, None, None] ** 2 + x[None, :, None] ** 2 + x[None, None, :] ** 2) / 2.0) / np.pi ** 0.75
    rng = np.random.default_rng(seed)
    phi = np.empty((n, n, n, 3), np.complex128)
    for m in range(3):
        phi[..., m] = g * (1.0 + 1e-3 * rng.uniform(size=g.shape))
    return phi


# ------------------------------------------------------------ training data
def ground_states(points, n, steps, precision="fp32", chunk=64):
    """Imaginary-time ground states of every point on the n^3 grid, in
    batches of `chunk` instances (fortress_b200.batch); returns complex64
    PHI arrays [count, n, n, n, 3] and the final CONV of each."""
    import torch
    from fortress_b200.batch import Batch
    start = gaussian_start(n)
    out = np.empty((len(points), n, n, n, 3), np.complex64)
    conv = np.empty(len(points))
    for c0 in range(0, len(points), chunk):
        pts = points[c0:c0 + chunk]
        b = Batch([params(p, n, precision) for p in pts])
        for i in range(len(pts)):
            b[i].set_state(start)
            b[i].normt()
        b.step(steps)
        torch.cuda.synchronize()
        obs = b.observables(with_conv=True)
        for i in range(len(pts)):
            out[c0 + i] = b[i].state()
            conv[c0 + i] = obs[i]["conv"] / (2.0 * params(pts[i], n)["dt"])
        b.close()
    return out, conv


def targets(states):
    """[6][B][Z][Y][X] float32 training targets from PHI arrays."""
    s = np.transpose(states, (4, 0, 3, 2, 1))           # [m][B][Z][Y][X]
    t = np.empty((6,) + s.shape[1:], np.float32)
    t[0::2] = s.real
    t[1::2] = s.imag
    return t


def train(points, states, n, epochs, batch, lr, seed=0, width=16, modes=8, layers=4, hidden=64):
    import torch
    from fortress_b200 import fno3d as F3
    net = F3.FNO3(n, batch, width=width, modes=modes, layers=layers, hidden=hidden, seed=seed)
    pn = np.stack([F3.normalise_params(*p) for p in points])
    tg = targets(states)
    rng = np.random.default_rng(seed)
    nb = len(points) // batch
    hist = []
    total = epochs * nb
    it = 0
    for ep in range(epochs):
        perm = rng.permutation(len(points))
        el = 0.0
        for k in range(nb):
            idx = perm[k * batch:(k + 1) * batch]
            a = F3.input_channels(pn[idx], n)
            t = torch.tensor(np.ascontiguousarray(tg[:, idx].reshape(6, -1)), device="cuda")
            net.forward(a)
            net.loss(t)
            net.backward()
            net.adam(lr=lr * 0.5 * (1.0 + math.cos(math.pi * it / total)))
            it += 1
            el += float(net.loss_dev.item())
        hist.append(el / nb)
    torch.cuda.synchronize()
    assert not net.tc_error()
    return net, hist


# --------------------------------------------------------------- the arms
class Clock:
    def __init__(self):
        import torch
        torch.cuda.synchronize()
        self.t0 = time.perf_counter()

    def __call__(self):
        return time.perf_counter() - self.t0


def run_to(prop, clock, trace, label, max_steps, stop_rule=None, dt=1e-3, settle=None):
    """STP-step blocks with ENERGY and CONV after each, appending
    (label, step, wall, E, CONV, CONV_EN) to trace; stops at max_steps, when
    stop_rule(conv, conv_en) holds, or, with settle = (E_ref, checks), once
    |E - E_ref| <= TOL_REL/2 |E_ref| has held for that many checks."""
    en_old = prop.observables()[0]
    done, held = 0, 0
    while done < max_steps:
        prop.step(STP)
        done += STP
        en = prop.observables()[0]
        c = prop.conv() / (STP * 2.0 * dt)
        ce = abs(en - en_old) / (STP * 2.0 * dt)
        en_old = en
        trace.append((label, done, clock(), en, c, ce))
        if stop_rule is not None and stop_rule(c, ce):
            break
        if settle is not None:
            held = held + 1 if abs(en - settle[0]) <= 0.5 * TOL_REL * abs(settle[0]) else 0
            if held >= settle[1]:
                break
    return done


def learned_guess_device(net, point, n):
    """Network output at n^3 as a device complex128 PHI array (x fastest)."""
    import torch
    from fortress_b200 import fno3d as F3
    net.set_inputs_device(F3.normalise_params(*point)[None, :])
    net.forward()
    o = net.out.reshape(6, n, n, n)
    return torch.complex(o[0::2].double(), o[1::2].double()).contiguous()   # [m][z][y][x] = PHI layout


def pad_spectrum(spec, n):
    """Zero padding of a natural-order device spectrum [m][z][y][x] of an
    m^3 grid to n^3 (the prolongation's only step outside the library's
    transforms: a device copy of the kept frequencies)."""
    import torch
    m = spec.shape[-1]
    h = m // 2
    big = torch.zeros((spec.shape[0], n, n, n), dtype=spec.dtype, device=spec.device)
    ii = torch.tensor(list(range(h)) + list(range(n - h, n)), device=spec.device)
    ss = torch.tensor(list(range(h)) + list(range(m - h, m)), device=spec.device)
    big[:, ii[:, None, None], ii[None, :, None], ii[None, None, :]] = \
        spec[:, ss[:, None, None], ss[None, :, None], ss[None, None, :]]
    return big


def arm(kind, point, n, clock_state=None, net=None, max_steps=60000, fp32_tol=1e-6, e_ref=None, coarse_net=None):
    """One arm on the n^3 grid; returns its trace.  e_ref: the plain arm's
    final energy; the other arms' FP64 stages stop once they have held
    within half the tolerance of it for 20 checks."""
    import fortress_b200 as F
    import torch
    trace = []
    clock = Clock()
    p64 = F.Propagator(**params(point, n, "fp64"))
    if kind == "plain":
        p64.set_state(gaussian_start(n))
        p64.normt()
        trace.append((kind, 0, clock(), p64.observables()[0], float("nan"), float("nan")))
        run_to(p64, clock, trace, "fp64", max_steps)
        p64.close()
        return trace
    if kind in ("learned", "learned64"):
        guess = learned_guess_device(net, point, n)
    else:   # coarse (learned_coarse): 64^3 FP64 solve to the stop rule at 1e-8, then prolong
        pc = F.Propagator(**params(point, 64, "fp64"))
        if kind == "learned_coarse":
            pc.set_state_device(learned_guess_device(coarse_net, point, 64).data_ptr())
        else:
            pc.set_state(gaussian_start(64))
        pc.normt()
        run_to(pc, clock, trace, "coarse64", 200000, stop_rule=lambda c, ce: c <= 1e-8 or ce <= 1e-8)
        # spectral prolongation with the library's transforms: the coarse
        # state's unnormalised spectrum (FFT, natural order), zero-padded to
        # n^3, taken back by the fine grid's BFT; NORMT then fixes the scale
        pc.FFT()
        buf = torch.empty((3, 64, 64, 64), dtype=torch.complex128, device="cuda")
        pc.get_state_device(buf.data_ptr())
        pc.close()
        guess = pad_spectrum(buf, n)
        del buf
    torch.cuda.synchronize()
    trace.append(("guess", 0, clock(), float("nan"), float("nan"), float("nan")))
    if kind != "learned64":
        p32 = F.Propagator(**params(point, n, "fp32"))
        p32.set_state_device(guess.data_ptr())
        if kind in ("coarse", "learned_coarse"):
            p32.BFT()
        p32.normt()
        run_to(p32, clock, trace, "fp32", max_steps, stop_rule=lambda c, ce: c <= fp32_tol or ce <= fp32_tol)
        buf = torch.empty_like(guess)
        p32.get_state_device(buf.data_ptr())
        p32.close()
        guess = buf
    p64.set_state_device(guess.data_ptr())
    p64.normt()
    del guess
    trace.append(("switch", 0, clock(), p64.observables()[0], float("nan"), float("nan")))
    run_to(p64, clock, trace, "fp64", max_steps, settle=(e_ref, 20) if e_ref is not None else None)
    p64.close()
    return trace


def time_to(trace, e_star, tol=TOL_REL):
    """(steps per stage, wall) at the first FP64 energy check after which
    every later check satisfies |E - E*| <= tol |E*|; None if never."""
    seen, out = {}, None
    for lab, st, wall, en, c, ce in trace:
        if st == 0:
            continue
        seen[lab] = st
        if lab == "fp64":
            ok = abs(en - e_star) <= tol * abs(e_star)
            if ok and out is None:
                out = (dict(seen), wall)
            elif not ok:
                out = None
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=192)
    ap.add_argument("--n-train", type=int, default=64)
    ap.add_argument("--gen-steps", type=int, default=30000)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--max-steps", type=int, default=60000)
    ap.add_argument("--arms", default="plain,learned,learned64,coarse,learned_coarse")
    ap.add_argument("--params", default=None, help="trained network parameters (.npz): skip data and training")
    ap.add_argument("--width", type=int, default=16)
    ap.add_argument("--modes", type=int, default=8)
    ap.add_argument("--layers", type=int, default=4)
    ap.add_argument("--hidden", type=int, default=64)
    ap.add_argument("--data", default=None, help="reuse training states saved by an earlier run (.npy)")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    out = args.out or os.environ.get("FGPE_BENCH_OUT") or "."
    os.makedirs(out, exist_ok=True)
    import torch
    tp = target_point()
    if args.params:
        params_np = {k: np.asarray(v, np.float64) for k, v in np.load(args.params).items()}
    else:
        pts = box_points(args.train, seed=5)
        t0 = time.perf_counter()
        if args.data:
            states = np.load(args.data)
        else:
            states, conv = ground_states(pts, args.n_train, args.gen_steps)
            np.save(os.path.join(out, "train_states.npy"), states)
            print(json.dumps({"stage": "data", "count": len(pts), "grid": args.n_train, "steps": args.gen_steps,
                              "seconds": time.perf_counter() - t0, "conv_median": float(np.median(conv)),
                              "conv_max": float(conv.max())}), flush=True)
        t0 = time.perf_counter()
        net, hist = train(pts, states, args.n_train, args.epochs, args.batch, args.lr, width=args.width,
                          modes=args.modes, layers=args.layers, hidden=args.hidden)
        print(json.dumps({"stage": "train", "epochs": args.epochs, "seconds": time.perf_counter() - t0,
                          "loss_first": hist[0], "loss_last": hist[-1]}), flush=True)
        params_np = net.params_numpy()
        np.savez(os.path.join(out, "fno3d_params.npz"), **{k: v.astype(np.float32) for k, v in params_np.items()})
        del net, states
        torch.cuda.empty_cache()
    from fortress_b200 import fno3d as F3
    shape = dict(width=params_np["P"].shape[0], modes=params_np["Rr0"].shape[-1], hidden=params_np["Q1"].shape[0],
                 layers=sum(1 for k in params_np if k.startswith("Rr")))
    infer = F3.FNO3(args.n, 1, params=params_np, train=False, **shape)
    infer64 = F3.FNO3(64, 1, params=params_np, train=False, **shape)
    traces = {}
    kinds = args.arms.split(",")
    kinds = (["plain"] if "plain" in kinds else []) + [k for k in kinds if k != "plain"]
    e_ref = None
    for kind in kinds:
        traces[kind] = arm(kind, tp, args.n, net=infer, max_steps=args.max_steps, e_ref=e_ref, coarse_net=infer64)
        if kind == "plain":
            e_ref = traces[kind][-1][3]
        last = traces[kind][-1]
        print(json.dumps({"stage": "arm", "arm": kind, "wall": last[2], "E_final": last[3],
                          "fp64_steps": last[1]}), flush=True)
    e_star = min(tr[-1][3] for tr in traces.values())
    res = {"stage": "result", "E_star": e_star, "tol_rel": TOL_REL, "grid": args.n, "arms": {}}
    for kind, tr in traces.items():
        t = time_to(tr, e_star)
        res["arms"][kind] = {"time_to_tol_s": t[1] if t else None, "steps": t[0] if t else None,
                             "E_final": tr[-1][3], "E_final_minus_Estar_rel": (tr[-1][3] - e_star) / abs(e_star)}
    plain = res["arms"].get("plain", {}).get("time_to_tol_s")
    for k, v in res["arms"].items():
        if k != "plain" and plain and v.get("time_to_tol_s"):
            v["speedup_vs_plain_fp64"] = plain / v["time_to_tol_s"]
    with open(os.path.join(out, "time_to_gs.json"), "w") as f:
        json.dump({"result": res, "traces": traces}, f)
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
