"""FP64 numpy restatement of the Fourier neural operator used for the learned
initial guess, forward and backward (test infrastructure only: the oracle for
the GPU kernels' values and gradients).

Network (no reference counterpart; defined in fortress_b200/fno.py):
  input   a(x) = [p_1..p_5, X, Y]            7 channels on an N x N grid
  lift    h0 = P a + bP                        width W
  layer l h_{l+1} = act_l(W_l h_l + b_l + K_l h_l),  act = GELU(tanh), none
                                               after the last layer
  project q = GELU(Q1 h_L + c1), out = Q2 q + c2   (6 channels: Re/Im of the
                                               three spinor components)
  K h: H_c = Ex^T h_c Ey (modes kx in {0..M-1, N-M..N-1}, ky in {0..M-1});
       G_o = sum_c R_oc * H_c;  K_o = Re(conj(Ex) (w*G_o) conj(Ey)^T) / N^2
       with w = 1 for ky = 0 and 2 otherwise.
Loss: mean over all output values of (out - target)^2.
"""
from __future__ import annotations

import numpy as np


def gelu(x):
    c = np.sqrt(2.0 / np.pi)
    return 0.5 * x * (1.0 + np.tanh(c * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    c = np.sqrt(2.0 / np.pi)
    u = c * (x + 0.044715 * x ** 3)
    t = np.tanh(u)
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * c * (1.0 + 3 * 0.044715 * x ** 2)


def dft_mats(n, modes):
    kx = np.concatenate([np.arange(modes), np.arange(n - modes, n)])
    ky = np.arange(modes)
    i = np.arange(n)
    Ex = np.exp(-2j * np.pi * np.outer(i, kx) / n)     # [n, 2M]
    Ey = np.exp(-2j * np.pi * np.outer(i, ky) / n)     # [n, M]
    w = np.where(ky == 0, 1.0, 2.0)                     # [M]
    return Ex, Ey, w


def init_params(width=32, modes=16, layers=4, cin=7, hidden=128, cout=6, seed=0):
    rng = np.random.default_rng(seed)
    p = {"P": rng.standard_normal((width, cin)) / np.sqrt(cin), "bP": np.zeros(width)}
    for l in range(layers):
        p[f"W{l}"] = rng.standard_normal((width, width)) / np.sqrt(width)
        p[f"b{l}"] = np.zeros(width)
        sc = 1.0 / (width * width)
        p[f"Rr{l}"] = sc * rng.uniform(size=(width, width, 2 * modes, modes))
        p[f"Ri{l}"] = sc * rng.uniform(size=(width, width, 2 * modes, modes))
    p["Q1"] = rng.standard_normal((hidden, width)) / np.sqrt(width)
    p["c1"] = np.zeros(hidden)
    p["Q2"] = rng.standard_normal((cout, hidden)) / np.sqrt(hidden)
    p["c2"] = np.zeros(cout)
    return p


def spectral(h, Rr, Ri, Ex, Ey, w):
    """h [B, C, N, N] -> K h [B, O, N, N] and the mode coefficients H."""
    n = h.shape[-1]
    H = np.einsum("ia,bcij,jk->bcak", Ex, h, Ey)        # [B, C, 2M, M]
    R = Rr + 1j * Ri
    G = np.einsum("ocak,bcak->boak", R, H)
    Gt = G * w[None, None, None, :]
    K = np.einsum("ia,boak,jk->boij", np.conj(Ex), Gt, np.conj(Ey)).real / (n * n)
    return K, H


def spectral_bwd(dK, H, Rr, Ri, Ex, Ey, w):
    n = dK.shape[-1]
    R = Rr + 1j * Ri
    A = np.conj(Ex) / (n * n)                          # [N, 2M]
    Bm = np.conj(Ey).T                                  # [M, N]
    # gradient of K = Re(A Gt B): g_Gt = conj(A^T dK B^T)
    gGt = np.conj(np.einsum("ia,boij,kj->boak", A, dK, Bm))
    gG = gGt * w[None, None, None, :]
    gR = np.einsum("boak,bcak->ocak", gG, np.conj(H))
    gH = np.einsum("boak,ocak->bcak", gG, np.conj(R))
    dh = np.einsum("ia,bcak,jk->bcij", Ex, np.conj(gH), Ey).real
    return dh, gR.real, gR.imag


def forward(p, a, modes=16, layers=4, cache=False):
    """a [B, 7, N, N] -> out [B, 6, N, N]."""
    n = a.shape[-1]
    Ex, Ey, w = dft_mats(n, modes)
    h = np.einsum("oc,bcij->boij", p["P"], a) + p["bP"][None, :, None, None]
    st = {"a": a, "h": [h], "z": [], "H": []}
    for l in range(layers):
        K, H = spectral(h, p[f"Rr{l}"], p[f"Ri{l}"], Ex, Ey, w)
        z = np.einsum("oc,bcij->boij", p[f"W{l}"], h) + p[f"b{l}"][None, :, None, None] + K
        h = gelu(z) if l < layers - 1 else z
        st["z"].append(z); st["H"].append(H); st["h"].append(h)
    u = np.einsum("oc,bcij->boij", p["Q1"], h) + p["c1"][None, :, None, None]
    q = gelu(u)
    out = np.einsum("oc,bcij->boij", p["Q2"], q) + p["c2"][None, :, None, None]
    st.update(u=u, q=q)
    return (out, st) if cache else out


def loss_and_grad(p, a, target, modes=16, layers=4):
    out, st = forward(p, a, modes, layers, cache=True)
    n = a.shape[-1]
    Ex, Ey, w = dft_mats(n, modes)
    diff = out - target
    loss = float(np.mean(diff ** 2))
    g = {}
    dout = 2.0 * diff / diff.size
    g["c2"] = dout.sum(axis=(0, 2, 3))
    g["Q2"] = np.einsum("boij,bcij->oc", dout, st["q"])
    dq = np.einsum("oc,boij->bcij", p["Q2"], dout)
    du = dq * gelu_grad(st["u"])
    g["c1"] = du.sum(axis=(0, 2, 3))
    hL = st["h"][-1]
    g["Q1"] = np.einsum("boij,bcij->oc", du, hL)
    dh = np.einsum("oc,boij->bcij", p["Q1"], du)
    for l in reversed(range(layers)):
        z = st["z"][l]
        dz = dh * gelu_grad(z) if l < layers - 1 else dh
        hin = st["h"][l]
        g[f"b{l}"] = dz.sum(axis=(0, 2, 3))
        g[f"W{l}"] = np.einsum("boij,bcij->oc", dz, hin)
        dh_lin = np.einsum("oc,boij->bcij", p[f"W{l}"], dz)
        dh_sp, gRr, gRi = spectral_bwd(dz, st["H"][l], p[f"Rr{l}"], p[f"Ri{l}"], Ex, Ey, w)
        g[f"Rr{l}"], g[f"Ri{l}"] = gRr, gRi
        dh = dh_lin + dh_sp
    g["bP"] = dh.sum(axis=(0, 2, 3))
    g["P"] = np.einsum("boij,bcij->oc", dh, st["a"])
    return loss, g


# ------------------------------------------------------------------- 3D form
# The same network on an N x N x N grid (fortress_b200/fno3d.py):
#   K h: H_c = sum_{xyz} h_c(x,y,z) e^{-2 pi i (kx x + ky y + kz z)/N} over
#        kx in {0..M-1} and ky, kz in {0..M-1, N-M..N-1};
#        G_o = sum_c R_oc * H_c;  K_o = Re(sum_k w_kx G_o e^{+2 pi i k.r/N}) / N^3
#        with w = 1 for kx = 0 and 2 otherwise.
# Arrays are [B, C, Z, Y, X] (x fastest).
def dft_mats3(n, modes):
    kf = np.concatenate([np.arange(modes), np.arange(n - modes, n)])
    kh = np.arange(modes)
    i = np.arange(n)
    Ef = np.exp(-2j * np.pi * np.outer(i, kf) / n)     # [n, 2M]  (y and z)
    Eh = np.exp(-2j * np.pi * np.outer(i, kh) / n)     # [n, M]   (x)
    w = np.where(kh == 0, 1.0, 2.0)
    return Ef, Eh, w


def init_params3(width=16, modes=8, layers=4, cin=7, hidden=64, cout=6, seed=0):
    rng = np.random.default_rng(seed)
    p = {"P": rng.standard_normal((width, cin)) / np.sqrt(cin), "bP": np.zeros(width)}
    for l in range(layers):
        p[f"W{l}"] = rng.standard_normal((width, width)) / np.sqrt(width)
        p[f"b{l}"] = np.zeros(width)
        sc = 1.0 / (width * width)
        p[f"Rr{l}"] = sc * rng.uniform(size=(width, width, 2 * modes, 2 * modes, modes))
        p[f"Ri{l}"] = sc * rng.uniform(size=(width, width, 2 * modes, 2 * modes, modes))
    p["Q1"] = rng.standard_normal((hidden, width)) / np.sqrt(width)
    p["c1"] = np.zeros(hidden)
    p["Q2"] = rng.standard_normal((cout, hidden)) / np.sqrt(hidden)
    p["c2"] = np.zeros(cout)
    return p


def spectral3(h, Rr, Ri, Ef, Eh, w):
    """h [B, C, Z, Y, X] -> K h and the mode coefficients H [B, C, kz, ky, kx]."""
    n = h.shape[-1]
    H = np.einsum("zc,yb,xa,kizyx->kicba", Ef, Ef, Eh, h, optimize=True)
    G = np.einsum("oicba,kicba->kocba", Rr + 1j * Ri, H, optimize=True)
    Gt = G * w[None, None, None, None, :]
    K = np.einsum("zc,yb,xa,kocba->kozyx", np.conj(Ef), np.conj(Ef), np.conj(Eh), Gt, optimize=True).real
    return K / n ** 3, H


def spectral3_bwd(dK, H, Rr, Ri, Ef, Eh, w):
    n = dK.shape[-1]
    R = Rr + 1j * Ri
    # K = Re(A(Gt))/n^3 with A linear: grad wrt Gt = conj(A^T dK)/n^3
    gGt = np.conj(np.einsum("zc,yb,xa,kozyx->kocba", np.conj(Ef), np.conj(Ef), np.conj(Eh), dK,
                            optimize=True)) / n ** 3
    gG = gGt * w[None, None, None, None, :]
    gR = np.einsum("kocba,kicba->oicba", gG, np.conj(H), optimize=True)
    gH = np.einsum("kocba,oicba->kicba", gG, np.conj(R), optimize=True)
    dh = np.einsum("zc,yb,xa,kicba->kizyx", Ef, Ef, Eh, np.conj(gH), optimize=True).real
    return dh, gR.real, gR.imag


def _pw(Wm, x):
    return np.einsum("oc,bczyx->bozyx", Wm, x, optimize=True)


def _bias(b):
    return b[None, :, None, None, None]


def forward3(p, a, modes=8, layers=4, cache=False):
    """a [B, cin, N, N, N] -> out [B, 6, N, N, N]."""
    n = a.shape[-1]
    Ef, Eh, w = dft_mats3(n, modes)
    h = _pw(p["P"], a) + _bias(p["bP"])
    st = {"a": a, "h": [h], "z": [], "H": []}
    for l in range(layers):
        K, H = spectral3(h, p[f"Rr{l}"], p[f"Ri{l}"], Ef, Eh, w)
        z = _pw(p[f"W{l}"], h) + _bias(p[f"b{l}"]) + K
        h = gelu(z) if l < layers - 1 else z
        st["z"].append(z); st["H"].append(H); st["h"].append(h)
    u = _pw(p["Q1"], h) + _bias(p["c1"])
    q = gelu(u)
    out = _pw(p["Q2"], q) + _bias(p["c2"])
    st.update(u=u, q=q)
    return (out, st) if cache else out


def loss_and_grad3(p, a, target, modes=8, layers=4):
    out, st = forward3(p, a, modes, layers, cache=True)
    n = a.shape[-1]
    Ef, Eh, w = dft_mats3(n, modes)
    diff = out - target
    loss = float(np.mean(diff ** 2))
    g = {}
    red = (0, 2, 3, 4)
    dout = 2.0 * diff / diff.size
    g["c2"] = dout.sum(axis=red)
    g["Q2"] = np.einsum("bozyx,bczyx->oc", dout, st["q"], optimize=True)
    dq = np.einsum("oc,bozyx->bczyx", p["Q2"], dout, optimize=True)
    du = dq * gelu_grad(st["u"])
    g["c1"] = du.sum(axis=red)
    g["Q1"] = np.einsum("bozyx,bczyx->oc", du, st["h"][-1], optimize=True)
    dh = np.einsum("oc,bozyx->bczyx", p["Q1"], du, optimize=True)
    for l in reversed(range(layers)):
        z = st["z"][l]
        dz = dh * gelu_grad(z) if l < layers - 1 else dh
        hin = st["h"][l]
        g[f"b{l}"] = dz.sum(axis=red)
        g[f"W{l}"] = np.einsum("bozyx,bczyx->oc", dz, hin, optimize=True)
        dh_lin = np.einsum("oc,bozyx->bczyx", p[f"W{l}"], dz, optimize=True)
        dh_sp, gRr, gRi = spectral3_bwd(dz, st["H"][l], p[f"Rr{l}"], p[f"Ri{l}"], Ef, Eh, w)
        g[f"Rr{l}"], g[f"Ri{l}"] = gRr, gRi
        dh = dh_lin + dh_sp
    g["bP"] = dh.sum(axis=red)
    g["P"] = np.einsum("bozyx,bczyx->oc", dh, st["a"], optimize=True)
    return loss, g
