"""Shared case definitions for the parity tests (GPU path vs the oracle)."""
import numpy as np

# dim, spin, imag, grid: non-square grids with radix-3 and radix-5 factors
CASES = [
    (1, 1, 1, (96,)), (1, 2, 1, (64,)), (1, 1, 0, (120,)), (1, 2, 0, (80,)),
    (2, 1, 1, (32, 24)), (2, 2, 1, (32, 32)), (2, 1, 0, (48, 32)), (2, 2, 0, (32, 40)),
    (3, 1, 1, (16, 16, 12)), (3, 2, 1, (16, 12, 16)), (3, 1, 0, (12, 16, 16)), (3, 2, 0, (16, 16, 16)),
]


def case_id(c):
    dim, spin, imag, n = c
    return f"{dim}d-spin{spin}-{'im' if imag else 're'}-{'x'.join(map(str, n))}"


def case_params(c):
    dim, spin, imag, n = c
    d = {1: (0.3,), 2: (0.45, 0.5), 3: (0.6, 0.65, 0.7)}[dim]
    tau = (200.0, -5.0, 0.0) if spin == 1 else (300.0, 10.0, -8.0)
    return dict(dim=dim, spin=spin, n=n, d=d, dt=1e-3 if imag else 5e-4, imag_time=imag,
                tau=tau, gamma=(0.5, 0.3, 0.4)[:dim], alpha=(1.0, 1.3, 1.7))


def oracle_kwargs(p):
    n = list(p["n"]) + [1] * 3
    d = list(p["d"]) + [1.0] * 3
    g = list(p["gamma"]) + [0.0] * 3
    return dict(dim=p["dim"], spin=p["spin"], nx=n[0], ny=n[1], nz=n[2], dx=d[0], dy=d[1], dz=d[2],
                dt=p["dt"], imag=int(p["imag_time"]), tau=p["tau"], gx=g[0], gy=g[1], gz=g[2],
                ax=p["alpha"][0], ay=p["alpha"][1], az=p["alpha"][2])


def initial_state(orc, seed=0):
    """Default Gaussian guess of the reference times seeded amplitude noise
    and phases (so every operator sees a generic complex spinor)."""
    orc.initialize(4, 0.0)
    phi = orc.state()
    rng = np.random.default_rng(seed)
    phi = phi * (1.0 + 0.05 * rng.standard_normal(phi.shape)) * np.exp(1j * rng.uniform(-0.4, 0.4, phi.shape))
    return phi


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))

# Grids whose lines hit the size-specialised persistent kernels (128, 192,
# 256, 384, 512) on some axes and the generic ones on others.
FAST_CASES = [
    (2, 2, 1, (128, 192)), (2, 2, 0, (256, 128)), (2, 1, 1, (384, 128)), (2, 1, 0, (512, 96)),
    (3, 1, 1, (128, 128, 16)), (3, 2, 0, (16, 128, 128)), (3, 1, 0, (192, 16, 256)),
]
