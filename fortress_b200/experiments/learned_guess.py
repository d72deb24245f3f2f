"""Learned initial guess for the q2D spin-1 parameter sweep: generate ground
states with the batched propagator, train the Fourier neural operator
(fortress_b200.fno) on them with the library's own kernels, and measure the
imaginary-time steps and wall time to convergence from the learned guess
against the Gaussian guess the reference starts from.

Parameter box (seeded): GAMMAX, GAMMAY in [0,2], c0 in [100,2000],
c2/c0 in [-0.05,0.05], NUY/NUX in [1,2]; spin-1, q2D, DT=5e-4, TOL=1e-8;
c0, c2 are the printed TAU/2 (tau = 2c).  Training states are computed in
the FP32 bulk path on a coarse grid of the same box (n_train x n_train points
over L = 25.6); the network is evaluated on the fine grid (256 x 256,
DX = 0.1), where both arms run in FP64 (the FP32 rounding floor keeps CONV
above 1e-8).

    python -m fortress_b200.experiments.learned_guess [--train 1024] [--heldout 64] [--out DIR]

Prints one JSON object per stage; the last one is the comparison.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

L_BOX = 25.6


def box(count, seed):
    """(gx, gy, c0, c2/c0, nuy/nux) rows."""
    rng = np.random.default_rng(seed)
    out = np.empty((count, 5))
    for k in range(count):
        g = rng.uniform(0, 2, 2)
        out[k] = (g[0], g[1], rng.uniform(100, 2000), rng.uniform(-0.05, 0.05), rng.uniform(1, 2))
    return out


def instance(row, n, dt=5e-4, precision="fp64"):
    gx, gy, c0, r2, ay = (float(v) for v in row)
    d = L_BOX / n
    return dict(dim=2, spin=1, n=(n, n), d=(d, d), dt=dt, imag_time=True, tau=(2 * c0, 2 * c0 * r2, 0.0),
                gamma=(gx, gy), alpha=(1.0, ay, 1.0), precision=precision)


def gaussian(p):
    """INITIALIZE's default spin-1 q2D guess (OPTION_FPC default): the same
    alpha-weighted Gaussian in every component (cgpe2d.f90:690-694, 723-726;
    the 1/sqrt(pi) factor drops out at the first NORMT)."""
    n, d = p["n"][0], p["d"][0]
    x = (-1.0 + 2.0 * np.arange(n) / n) * n * d / 2.0
    g = np.exp(-(p["alpha"][0] * x[:, None] ** 2 + p["alpha"][1] * x[None, :] ** 2) / 2.0)
    return np.repeat(g[:, :, None], 3, axis=2).astype(np.complex128)


def solve(insts, guesses, tol=1e-8, stp=100, max_steps=40000, run_all=False):
    """Imaginary time on every instance at once (one batch), STP steps per
    check.  Records per instance the energy after every STP block and the
    first step count at which the reference's stop rule holds (CONV <= TOL or
    CONV_EN <= TOL, cgpe2d.f90:489-496).  Stops when every instance has met
    the rule, unless run_all.  Returns a dict with the final states."""
    from fortress_b200.batch import Batch
    import torch
    b = Batch(insts)
    for i, g in enumerate(guesses):
        b[i].set_state(g)
        b[i].normt()
    torch.cuda.synchronize()
    n = len(insts)
    dt = insts[0]["dt"]
    stop = np.full(n, -1)
    en_old = np.array([o["en"] for o in b.observables(with_conv=False)])
    traj = []
    ii = 0
    t0 = time.perf_counter()
    while ii < max_steps:
        b.step(stp)
        ii += stp
        obs = b.observables(with_conv=True)
        en = np.array([o["en"] for o in obs])
        conv = np.array([o["conv"] for o in obs]) / (stp * 2.0 * dt)
        conv_en = np.abs(en - en_old) / (stp * 2.0 * dt)
        en_old = en
        traj.append(en)
        hit = (stop < 0) & ((conv <= tol) | (conv_en <= tol))
        stop[hit] = ii
        if not run_all and np.all(stop >= 0):
            break
    wall = time.perf_counter() - t0
    states = [b[i].state()[:, :, 0, :] for i in range(n)]
    b.close()
    return dict(stop=stop, traj=np.array(traj), stp=stp, steps=ii, wall=wall, states=states)


def first_within(traj, stp, e_star, rel):
    """First step count at which |E - E*| <= rel |E*| holds from then on."""
    ok = np.abs(traj - e_star[None, :]) <= rel * np.abs(e_star[None, :])
    out = np.full(traj.shape[1], -1)
    for i in range(traj.shape[1]):
        bad = np.nonzero(~ok[:, i])[0]
        last_bad = bad[-1] if len(bad) else -1
        if last_bad < traj.shape[0] - 1:
            out[i] = (last_bad + 2) * stp
    return out


def states_to_target(states):
    """[B] complex (n,n,3) -> float32 [6][B][n][n] (Re, Im per component)."""
    B = len(states)
    n = states[0].shape[0]
    t = np.empty((6, B, n, n), np.float32)
    for b, s in enumerate(states):
        for m in range(3):
            t[2 * m, b] = s[:, :, m].real
            t[2 * m + 1, b] = s[:, :, m].imag
    return t


def target_to_states(t):
    return [np.stack([t[2 * m, b] + 1j * t[2 * m + 1, b] for m in range(3)], axis=-1).astype(np.complex128)
            for b in range(t.shape[1])]


# The solver's states have unit Simpson norm over an L x L box, so their
# values are O(1/L) at every resolution; the network sees them times this.
TARGET_SCALE = 10.0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=1024)
    ap.add_argument("--heldout", type=int, default=32)
    ap.add_argument("--n-train", type=int, default=64)
    ap.add_argument("--n-eval", type=int, default=256)
    ap.add_argument("--gen-steps", type=int, default=25000)
    ap.add_argument("--gen-chunk", type=int, default=1024, help="instances per generation batch")
    ap.add_argument("--gen-dt", type=float, default=4e-3,
                    help="imaginary-time step of the training-data runs (a larger step relaxes faster; "
                         "its splitting error only shifts the targets slightly)")
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--max-steps", type=int, default=200000)
    ap.add_argument("--out", default="/tmp/learned_guess", help="training data and trained parameters")
    ap.add_argument("--params", default=None, help="trained parameters (.npz) to evaluate instead of training")
    ap.add_argument("--save-params", default=None, help="also write the trained parameters here")
    ap.add_argument("--fp32-tol", type=float, default=1e-6,
                    help="stop rule of the FP32 stage of the learned+FP32 arm (its rounding floor is above 1e-8)")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    import torch
    from fortress_b200 import fno as FN

    if args.params is not None:
        pfin = {k: np.asarray(v, np.float64) for k, v in np.load(args.params).items()}
        ptr, pho = None, box(args.heldout, 6)
    else:
        # ---------------------------------------------------------------- data
        ptr, pho = box(args.train, 5), box(args.heldout, 6)
        data_path = os.path.join(args.out, f"train_{args.train}_{args.n_train}_{args.gen_steps}_{args.gen_dt}.npz")
        if os.path.exists(data_path):
            tgt = np.load(data_path)["t"]
        else:
            # FP32 bulk: its rounding floor keeps CONV above 1e-8, so the training
            # states are a fixed number of imaginary-time steps from the guess
            # (in batches of --gen-chunk instances)
            t0 = time.perf_counter()
            parts, conv = [], 0
            for c0 in range(0, args.train, args.gen_chunk):
                insts = [instance(r, args.n_train, dt=args.gen_dt, precision="fp32") for r in ptr[c0:c0 + args.gen_chunk]]
                r = solve(insts, [gaussian(p) for p in insts], tol=1e-8, max_steps=args.gen_steps, run_all=True)
                parts.append(states_to_target(r["states"]) * TARGET_SCALE)
                conv += int((r["stop"] >= 0).sum())
            tgt = np.concatenate(parts, axis=1)
            np.savez_compressed(data_path, t=tgt)
            print(json.dumps({"stage": "generate", "instances": args.train, "grid": args.n_train, "dt": args.gen_dt,
                              "converged": conv, "steps": int(args.gen_steps),
                              "wall_s": time.perf_counter() - t0}), flush=True)

        # --------------------------------------------------------------- train
        a_all = FN.input_channels(np.array([FN.normalise_params(*row) for row in ptr]), args.n_train)
        B = args.batch
        net = FN.FNO(args.n_train, B, seed=7)
        nb = args.train // B
        t0 = time.perf_counter()
        rng = np.random.default_rng(8)
        tgt_dev = torch.tensor(tgt.reshape(6, args.train, -1), device="cuda")
        a_dev = torch.tensor(a_all.reshape(7, args.train, -1), device="cuda")
        losses = []
        steps_total = args.epochs * nb
        it = 0
        for ep in range(args.epochs):
            perm = torch.tensor(rng.permutation(args.train), device="cuda")
            tot = torch.zeros(1, dtype=torch.float64, device="cuda")
            for k in range(nb):
                idx = perm[k * B:(k + 1) * B]
                net.a.copy_(a_dev[:, idx, :].reshape(7, -1))
                tb = tgt_dev[:, idx, :].reshape(6, -1).contiguous()
                net.forward()
                tot += net.loss(tb)
                net.backward()
                lr = args.lr * 0.5 * (1 + np.cos(np.pi * it / steps_total))
                net.adam(lr=lr)
                it += 1
            losses.append(float(tot.item()) / nb)
        torch.cuda.synchronize()
        train_s = time.perf_counter() - t0
        pfin = net.params_numpy()
        np.savez_compressed(os.path.join(args.out, "fno_params.npz"), **{k: v.astype(np.float32) for k, v in pfin.items()})
        print(json.dumps({"stage": "train", "samples": args.train, "grid": args.n_train, "epochs": args.epochs,
                          "batch": B, "wall_s": train_s, "loss_first": losses[0], "loss_last": losses[-1]}), flush=True)
        if args.save_params:
            np.savez_compressed(args.save_params, **{k: v.astype(np.float32) for k, v in pfin.items()})

    # ---------------------------------------------------------------- eval
    ne = args.n_eval
    insts = [instance(r, ne) for r in pho]
    # learned guesses on the fine grid
    Be = 8
    guesses = []
    t0 = time.perf_counter()
    enet = FN.FNO(ne, Be, params=pfin)
    a_ev = FN.input_channels(np.array([FN.normalise_params(*row) for row in pho]), ne)
    for k in range(0, args.heldout, Be):
        blk = a_ev[:, k:k + Be]
        if blk.shape[1] < Be:
            blk = np.concatenate([blk, np.repeat(blk[:, -1:], Be - blk.shape[1], axis=1)], axis=1)
        out = enet.forward(blk).cpu().numpy().reshape(6, Be, ne, ne)
        guesses += target_to_states(out)[:min(Be, args.heldout - k)]
    torch.cuda.synchronize()
    infer_s = time.perf_counter() - t0
    g_run = solve(insts, [gaussian(p) for p in insts], max_steps=args.max_steps, run_all=True)
    l_run = solve(insts, guesses, max_steps=args.max_steps, run_all=True)
    # learned + FP32: the FP32 bulk path until its own stop rule at --fp32-tol
    # (its rounding floor keeps CONV above 1e-8), then FP64 from that state
    insts32 = [instance(r, ne, precision="fp32") for r in pho]
    a32 = solve(insts32, guesses, tol=args.fp32_tol, max_steps=args.max_steps)
    h64 = solve(insts, a32["states"], max_steps=args.max_steps, run_all=True)
    # E*: the lowest of the final energies (the FP64 arms ran max_steps)
    e_star = np.minimum(np.minimum(g_run["traj"][-1], l_run["traj"][-1]), h64["traj"][-1])
    res = {}
    for name, r in (("gaussian", g_run), ("learned", l_run)):
        reach = first_within(r["traj"], r["stp"], e_star, 1e-8).astype(float)
        reach[reach < 0] = np.nan
        stop = r["stop"].astype(float)
        stop[stop < 0] = np.nan
        per_step = r["wall"] / r["steps"]
        res[name] = dict(stop_median=float(np.nanmedian(stop)), stop_mean=float(np.nanmean(stop)),
                         stop_never=int(np.isnan(stop).sum()), reach_median=float(np.nanmedian(reach)),
                         reach_mean=float(np.nanmean(reach)), reach_never=int(np.isnan(reach).sum()),
                         batch_ms_per_step=1e3 * per_step,
                         wall_to_reach_all_s=float(np.nanmax(reach) * per_step) if np.any(~np.isnan(reach)) else None,
                         final_rel_above_estar_max=float(np.max((r["traj"][-1] - e_star) / np.abs(e_star))))
    # the hybrid arm: per instance FP32 steps to its stop rule, then FP64 steps
    s32 = a32["stop"].astype(float); s32[s32 < 0] = np.nan
    s64 = h64["stop"].astype(float); s64[s64 < 0] = np.nan
    r64 = first_within(h64["traj"], h64["stp"], e_star, 1e-8).astype(float); r64[r64 < 0] = np.nan
    t32, t64 = a32["wall"] / a32["steps"], h64["wall"] / h64["steps"]
    res["learned_fp32_then_fp64"] = dict(
        fp32_steps_median=float(np.nanmedian(s32)), fp32_never=int(np.isnan(s32).sum()),
        fp64_stop_median=float(np.nanmedian(s64)), fp64_stop_never=int(np.isnan(s64).sum()),
        fp64_reach_median=float(np.nanmedian(r64)), fp64_reach_never=int(np.isnan(r64).sum()),
        batch_ms_per_step_fp32=1e3 * t32, batch_ms_per_step_fp64=1e3 * t64,
        stop_time_median_batch_ms=float(np.nanmedian(s32 * t32 + s64 * t64) * 1e3),
        final_rel_above_estar_max=float(np.max((h64["traj"][-1] - e_star) / np.abs(e_star))))
    for name in ("gaussian", "learned"):
        res[name]["stop_time_median_batch_ms"] = res[name]["stop_median"] * res[name]["batch_ms_per_step"]
    print(json.dumps({"stage": "compare", "heldout": args.heldout, "grid": ne, "tol": 1e-8,
                      "steps_run": args.max_steps, "inference_s": infer_s, **res,
                      "reach_median_ratio": res["gaussian"]["reach_median"] / res["learned"]["reach_median"],
                      "stop_median_ratio": res["gaussian"]["stop_median"] / res["learned"]["stop_median"]}),
          flush=True)


if __name__ == "__main__":
    main()
