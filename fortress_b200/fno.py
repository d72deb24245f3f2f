"""Learned initial guess: a Fourier neural operator from the physical
parameters of a q2D spin-1 instance to its ground-state spinor, trained and
evaluated with the library's own kernels (include/fno.h).  No counterpart in
the reference, which starts every imaginary-time run from a fixed analytic
guess (INITIALIZE, cgpe2d.f90:707-790).

Network (width W, NM retained y modes, NA = 2 NM retained x modes):
  input   a = [p_1..p_5, X, Y]             7 channels on an N x N grid
  lift    h0 = P a + bP
  layer l z = W_l h + b_l + K_l h,  h' = GELU(z) (no GELU after the last layer)
  project out = Q2 GELU(Q1 h_L + c1) + c2  (6 channels: Re/Im of 3 components)
  K h     = Re(conj(Ex) (w * R(H)) conj(Ey)^T) / N^2, H_c = Ex^T h_c Ey,
          G_o = sum_c R_oc H_c per retained mode, w = 1 for ky = 0 else 2.

Layout on the device: channel-major activations [C][B][N][N] (float32), so a
pointwise channel mix is one GEMM over all B*N*N points; those dense layers
(and their input gradients) run on the tensor cores (fno_dense_tc: tcgen05,
BF16 operands, FP32 accumulation in tensor memory, bias and GELU fused).
Weights keep an FP32 master copy (Adam) and a BF16 copy that the GEMMs read.
The spectral convolution is five GEMM stages over real/imaginary planes
(truncated DFTs as dense matrices), the per-mode channel mix a batched GEMM
over the 2*NM*NM retained modes in the real block form [[Rr, -Ri], [Ri, Rr]].
With tensor_cores (the default) these stages and their backward and
weight-gradient products run on fno_gemm_tc: tcgen05 with each FP32 operand
split into a BF16 head and tail (about 16 significant bits), FP32
accumulation in tensor memory.

Device memory comes from torch (plumbing only); every arithmetic step is a
kernel of libfgpe.so.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi

FNO_EXPORTS = ("fno_gemm", "fno_bias_act", "fno_act_bwd", "fno_channel_sum", "fno_axpy", "fno_mse",
               "fno_adam", "fno_to_bf16", "fno_rbig_build", "fno_rbig_fold", "fno_dense_tc", "fno_gemm_tc")

_L = None


def lib():
    global _L
    if _L is not None:
        return _L
    L = _abi.load()
    vp, ip, ll, fl = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_float
    sig = {
        "fno_gemm": [ip, ip, ip, ip, fl, vp, ip, ll, ll, ll, vp, ll, ll, ll, fl, vp, ll, ll, ll, vp],
        "fno_bias_act": [vp, vp, vp, ll, ll, ll, ip, vp],
        "fno_act_bwd": [vp, vp, vp, ll, vp],
        "fno_channel_sum": [vp, vp, ll, ll, ll, fl, vp],
        "fno_axpy": [vp, vp, fl, ll, vp],
        "fno_mse": [vp, vp, vp, vp, vp, ll, vp],
        "fno_adam": [vp, vp, vp, vp, vp, ll, fl, fl, fl, fl, ip, vp],
        "fno_to_bf16": [vp, vp, ll, vp],
        "fno_rbig_build": [vp, vp, vp, ll, ip, ip, vp],
        "fno_rbig_fold": [vp, vp, vp, ll, ip, ip, vp],
        "fno_dense_tc": [vp, ip, vp, vp, vp, vp, ip, ip, ll, ip, vp, vp],
        "fno_gemm_tc": [ip, ip, ip, ip, fl, vp, ip, ll, ll, ll, vp, ll, ll, ll, fl, vp, ll, ll, ll, vp, vp],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ip
    _L = L
    return L


def _ck(rc, what):
    if rc != 0:
        raise _abi.FgpeError(rc, f"{what}: {_abi.load().fgpe_last_error(None).decode(errors='replace')}")


PARAM_NAMES_SCALED = ("gx", "gy", "c0", "c2_over_c0", "ay")


def normalise_params(gx, gy, c0, c2_over_c0, ay):
    """Map the sweep box (gamma in [0,2], c0 in [100,2000], c2/c0 in
    [-0.05,0.05], nu_y/nu_x in [1,2]) onto about [-1, 1]."""
    return np.array([gx - 1.0, gy - 1.0, (c0 - 1050.0) / 950.0, c2_over_c0 / 0.05, (ay - 1.5) / 0.5])


def input_channels(params_norm, n):
    """a [7][B][n][n]: the five normalised parameters as constant planes, then
    X and Y in units of the box half-width (the grid points INITIALIZE places,
    cgpe2d.f90:692-699, divided by NX*DX/2)."""
    pn = np.asarray(params_norm, np.float64).reshape(-1, 5)
    B = pn.shape[0]
    x = (-1.0 + 2.0 * np.arange(n) / n)
    a = np.empty((7, B, n, n), np.float32)
    for q in range(5):
        a[q] = pn[:, q][:, None, None]
    a[5] = x[None, :, None]
    a[6] = x[None, None, :]
    return a


class FNO:
    """Forward, backward and Adam on the device for one grid size n and
    batch size B.  The parameters do not depend on n (the truncated DFT
    matrices do), so a network trained at one resolution runs at another."""

    def __init__(self, n, batch, width=32, modes=16, layers=4, cin=7, hidden=128, cout=6, seed=0,
                 params=None, device="cuda", tensor_cores=True):
        import torch
        self.torch = torch
        # dense (pointwise) layers on tcgen05 (BF16 operands, FP32 accumulation)
        # when their channel counts fit one 128-row tile, and the spectral
        # stages on the split-BF16 tcgen05 GEMM (fno_gemm_tc); else the FP32 GEMM
        self.tensor_cores = tensor_cores
        self.tc_err = torch.zeros(1, dtype=torch.int32, device=device)
        self.L = lib()
        self.n, self.B, self.W, self.NM, self.NA = n, batch, width, modes, 2 * modes
        self.layers, self.cin, self.hidden, self.cout = layers, cin, hidden, cout
        self.S = n * n
        self.dev = device
        if params is None:
            from_np = init_params(width, modes, layers, cin, hidden, cout, seed)
        else:
            from_np = params
        self.p = {}       # FP32 master weights (device)
        self.pb = {}      # BF16 copies of the matrices the GEMMs read
        self.g = {}       # gradients
        self.m, self.v = {}, {}
        for k, val in self._to_device_layout(from_np).items():
            t = torch.tensor(val, dtype=torch.float32, device=device).contiguous()
            self.p[k] = t
            self.g[k] = torch.zeros_like(t)
            self.m[k] = torch.zeros_like(t)
            self.v[k] = torch.zeros_like(t)
        self.t = 0
        nm = self.NA * self.NM
        for k in self._matrices():
            self.pb[k] = torch.empty(self.p[k].numel(), dtype=torch.bfloat16, device=device)
        for l in range(layers):
            self.pb[f"Rbig{l}"] = torch.empty(nm * 4 * width * width, dtype=torch.bfloat16, device=device)
        self.g_rbig = torch.empty(nm * 4 * width * width, dtype=torch.float32, device=device)
        self.refresh_bf16()
        self._dft()
        self._alloc()
        self.loss_dev = torch.zeros(1, dtype=torch.float64, device=device)
        self.loss_part = torch.zeros(256, dtype=torch.float64, device=device)

    # ------------------------------------------------------------ layout
    def _matrices(self):
        return ["P", "Q1", "Q2"] + [f"W{l}" for l in range(self.layers)]

    def _to_device_layout(self, p):
        """Oracle layout -> device layout (R: [o,c,a,k] -> [a,k][o][c])."""
        out = {}
        for k, v in p.items():
            if k.startswith("Rr") or k.startswith("Ri"):
                out[k] = np.ascontiguousarray(np.transpose(v, (2, 3, 0, 1)))
            else:
                out[k] = np.asarray(v)
        return out

    def params_numpy(self):
        """Device parameters back in the oracle layout (float64)."""
        out = {}
        for k, t in self.p.items():
            v = t.detach().cpu().numpy().astype(np.float64)
            if k.startswith("Rr") or k.startswith("Ri"):
                v = np.transpose(v, (2, 3, 0, 1))
            out[k] = v
        return out

    def grads_numpy(self):
        out = {}
        for k, t in self.g.items():
            v = t.detach().cpu().numpy().astype(np.float64)
            if k.startswith("Rr") or k.startswith("Ri"):
                v = np.transpose(v, (2, 3, 0, 1))
            out[k] = v
        return out

    def _dft(self):
        torch, n, NM, NA = self.torch, self.n, self.NM, self.NA
        kx = np.concatenate([np.arange(NM), np.arange(n - NM, n)])
        ky = np.arange(NM)
        i = np.arange(n)
        thx = 2 * np.pi * np.outer(i, kx) / n          # Ex = exp(-i thx)  [n, NA]
        thy = 2 * np.pi * np.outer(i, ky) / n          # Ey = exp(-i thy)  [n, NM]
        exr, exi = np.cos(thx), -np.sin(thx)
        eyr, eyi = np.cos(thy), -np.sin(thy)
        w = np.where(ky == 0, 1.0, 2.0)
        f = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device=self.dev)
        self.Ey = [f(eyr), f(eyi)]                                      # [n][NM]
        self.ExS = [f(np.concatenate([exr.T, -exi.T], axis=1)),         # [NA][2n]
                    f(np.concatenate([exi.T, exr.T], axis=1))]
        self.ExA = [f(np.concatenate([exr, -exi], axis=0)),             # [2n][NA]
                    f(np.concatenate([exi, exr], axis=0))]
        self.EywT = [f((w[:, None] * eyr.T)), f((w[:, None] * eyi.T))]  # [NM][n]
        self.Eyw = [f(eyr * w[None, :]), f(eyi * w[None, :])]           # [n][NM]

    def _alloc(self):
        torch, B, W, S, n, NM, NA = self.torch, self.B, self.W, self.S, self.n, self.NM, self.NA
        z = lambda *s: torch.zeros(*s, dtype=torch.float32, device=self.dev)
        self.a = z(self.cin, B * S)
        self.h = [z(W, B * S) for _ in range(self.layers + 1)]
        self.zs = [z(W, B * S) for _ in range(self.layers)]
        self.u = z(self.hidden, B * S)
        self.q = z(self.hidden, B * S)
        self.out = z(self.cout, B * S)
        self.T = z(W * B * 2 * n * NM)
        self.Hm = [z(NA * NM * 2 * W * B) for _ in range(self.layers)]
        self.Gm = z(NA * NM * 2 * W * B)
        self.U = z(W * B * 2 * n * NM)
        # backward scratch
        self.dout = z(self.cout, B * S)
        self.dq = z(self.hidden, B * S)
        self.dh = z(W, B * S)
        self.dh2 = z(W, B * S)
        self.dz = z(W, B * S)
        self.da = z(self.cin, B * S)
        self.chunk = S                      # a divisor of B*S of at most ~2048 points
        while self.chunk > 2048 and self.chunk % 2 == 0:
            self.chunk //= 2
        self.part = z((B * S // self.chunk) * max(self.hidden, W) * max(self.hidden, W, self.cin))
        self.dHm = z(NA * NM * 2 * W * B)

    def refresh_bf16(self):
        st = self._st()
        for k in self._matrices():
            _ck(self.L.fno_to_bf16(self._p(self.p[k]), self._p(self.pb[k]), self.p[k].numel(), st), "to_bf16")
        self._rbig()

    def _rbig(self):
        nm = self.NA * self.NM
        for l in range(self.layers):
            _ck(self.L.fno_rbig_build(self._p(self.p[f"Rr{l}"]), self._p(self.p[f"Ri{l}"]),
                                      self._p(self.pb[f"Rbig{l}"]), nm, self.W, self.W, self._st()), "rbig")

    # ----------------------------------------------------------- helpers
    def _st(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    @staticmethod
    def _p(t, off=0):
        return ctypes.c_void_p(t.data_ptr() + t.element_size() * off)

    def gemm(self, batch, M, N, K, A, sA, B_, sB, C, sC, alpha=1.0, beta=0.0, a_bf16=False, aoff=0, boff=0, coff=0):
        ea = 2 if a_bf16 else 4
        args = (batch, M, N, K, alpha, ctypes.c_void_p(A.data_ptr() + ea * aoff), int(a_bf16),
                sA[0], sA[1], sA[2], ctypes.c_void_p(B_.data_ptr() + 4 * boff), sB[0], sB[1], sB[2],
                beta, ctypes.c_void_p(C.data_ptr() + 4 * coff), sC[0], sC[1], sC[2])
        if self.tensor_cores:
            _ck(self.L.fno_gemm_tc(*args, self._p(self.tc_err), self._st()), "gemm_tc")
        else:
            _ck(self.L.fno_gemm(*args, self._st()), "gemm")

    def _use_tc(self, M, K):
        return self.tensor_cores and M <= 128 and K <= 128

    def pointwise(self, wname, x, out, O, C, bias=None, act_out=None, act=False):
        """out[O][BS] = W[O][C] x[C][BS] (+ bias); act_out = GELU(out) or out
        when given."""
        BS = self.B * self.S
        if self._use_tc(O, C):
            _ck(self.L.fno_dense_tc(self._p(self.pb[wname]), 0, self._p(x), self._p(bias) if bias is not None else None,
                                    self._p(out), self._p(act_out) if act_out is not None else None, O, C, BS,
                                    int(act), self._p(self.tc_err), self._st()), "dense_tc")
            return
        self.gemm(1, O, BS, C, self.pb[wname], (0, C, 1), x, (0, BS, 1), out, (0, BS, 1), a_bf16=True)
        if bias is not None or act_out is not None:
            self.bias_act(out, act_out, bias, O, act)

    def tc_error(self):
        """True if a tensor-core layer's wait for its accumulator ran out."""
        return bool(self.tc_err.item())

    def bias_act(self, z, h, bias, C, act):
        BS = self.B * self.S
        _ck(self.L.fno_bias_act(self._p(z), self._p(h) if h is not None else None,
                                self._p(bias) if bias is not None else None, C, BS, C * BS, int(act), self._st()),
            "bias_act")

    # ----------------------------------------------------------- spectral
    def spectral(self, l, h, z):
        """z[O][B][n][n] += K_l h (h [C][B][n][n])."""
        B, W, n, NM, NA = self.B, self.W, self.n, self.NM, self.NA
        CB, OB, nm = W * B, W * B, NA * NM
        T, Hm, Gm, U = self.T, self.Hm[l], self.Gm, self.U
        for p in range(2):   # T[z1][p] = h_z1 Ey_p
            self.gemm(CB, n, NM, n, h, (n * n, n, 1), self.Ey[p], (0, NM, 1), T, (2 * n * NM, NM, 1), coff=p * n * NM)
        for p in range(2):   # Hm[a][k][p][c][b] = ExS_p Tstack_z1
            self.gemm(CB, NA, NM, 2 * n, self.ExS[p], (0, 2 * n, 1), T, (2 * n * NM, NM, 1),
                      Hm, (1, NM * 2 * CB, 2 * CB), coff=p * CB)
        # Gm[mode][p][o][b] = Rbig[mode] Hm[mode]
        self.gemm(nm, 2 * W, B, 2 * W, self.pb[f"Rbig{l}"], (4 * W * W, 2 * W, 1), Hm, (2 * W * B, B, 1),
                  Gm, (2 * W * B, B, 1), a_bf16=True)
        for q in range(2):   # U[z4][p][i][k] = sum_q ExA_q G_q
            self.gemm(OB, 2 * n, NM, NA, self.ExA[q], (0, NA, 1), Gm, (1, NM * 2 * OB, 2 * OB),
                      U, (2 * n * NM, NM, 1), beta=float(q), boff=q * OB)
        for p in range(2):   # z_z4 += U_p EywT_p / n^2
            self.gemm(OB, n, n, NM, U, (2 * n * NM, NM, 1), self.EywT[p], (0, n, 1), z, (n * n, n, 1),
                      alpha=1.0 / (n * n), beta=1.0, aoff=p * n * NM)

    def spectral_bwd(self, l, dz, dh):
        """dh += K_l^T dz; gradients of Rr_l, Ri_l."""
        B, W, n, NM, NA = self.B, self.W, self.n, self.NM, self.NA
        CB, OB, nm = W * B, W * B, NA * NM
        T, Hm, Gm, U = self.T, self.Hm[l], self.Gm, self.U     # reused as dT, -, dGm, dU
        for p in range(2):   # dU_p = dz Eyw_p / n^2
            self.gemm(OB, n, NM, n, dz, (n * n, n, 1), self.Eyw[p], (0, NM, 1), U, (2 * n * NM, NM, 1),
                      alpha=1.0 / (n * n), coff=p * n * NM)
        for q in range(2):   # dG_q = ExA_q^T dUstack
            self.gemm(OB, NA, NM, 2 * n, self.ExA[q], (0, 1, NA), U, (2 * n * NM, NM, 1),
                      Gm, (1, NM * 2 * OB, 2 * OB), coff=q * OB)
        # dRbig = dG Hm^T ; dHm = Rbig^T dG
        self.gemm(nm, 2 * W, 2 * W, B, Gm, (2 * W * B, B, 1), Hm, (2 * W * B, 1, B),
                  self.g_rbig, (4 * W * W, 2 * W, 1))
        _ck(self.L.fno_rbig_fold(self._p(self.g_rbig), self._p(self.g[f"Rr{l}"]), self._p(self.g[f"Ri{l}"]),
                                 nm, W, W, self._st()), "rbig_fold")
        dHm = self.dHm
        self.gemm(nm, 2 * W, B, 2 * W, self.pb[f"Rbig{l}"], (4 * W * W, 1, 2 * W), Gm, (2 * W * B, B, 1),
                  dHm, (2 * W * B, B, 1), a_bf16=True)
        for p in range(2):   # dTstack = sum_p ExS_p^T dH_p
            self.gemm(CB, 2 * n, NM, NA, self.ExS[p], (0, 1, 2 * n), dHm, (1, NM * 2 * CB, 2 * CB),
                      T, (2 * n * NM, NM, 1), beta=float(p), boff=p * CB)
        for p in range(2):   # dh += dT_p Ey_p^T
            self.gemm(CB, n, n, NM, T, (2 * n * NM, NM, 1), self.Ey[p], (0, 1, NM), dh, (n * n, n, 1),
                      beta=1.0, aoff=p * n * NM)

    # ------------------------------------------------------------ passes
    def forward(self, a_host=None):
        torch = self.torch
        if a_host is not None:
            self.a.copy_(torch.from_numpy(np.ascontiguousarray(a_host.reshape(self.cin, -1))))
        W = self.W
        self.pointwise("P", self.a, self.h[0], W, self.cin, bias=self.p["bP"])
        for l in range(self.layers):
            z = self.zs[l]
            self.pointwise(f"W{l}", self.h[l], z, W, W)
            self.spectral(l, self.h[l], z)
            last = l == self.layers - 1
            self.bias_act(z, self.h[l + 1], self.p[f"b{l}"], W, not last)
        self.pointwise("Q1", self.h[-1], self.u, self.hidden, W, bias=self.p["c1"], act_out=self.q, act=True)
        self.pointwise("Q2", self.q, self.out, self.cout, self.hidden, bias=self.p["c2"])
        return self.out

    def loss(self, target, want_grad=True):
        n = self.out.numel()
        _ck(self.L.fno_mse(self._p(self.out), self._p(target), self._p(self.dout) if want_grad else None,
                           self._p(self.loss_dev), self._p(self.loss_part), n, self._st()), "mse")
        return self.loss_dev

    def _wgrad(self, gname, dy, x, O, C):
        """g[O][C] = dy[O][BS] x[C][BS]^T: the BS points split into chunks
        (one GEMM batch entry each), then the chunk partials summed."""
        BS = self.B * self.S
        ch = self.chunk
        nch = BS // ch
        self.gemm(nch, O, C, ch, dy, (ch, BS, 1), x, (ch, 1, BS), self.part, (O * C, C, 1))
        _ck(self.L.fno_channel_sum(self._p(self.g[gname]), self._p(self.part), nch, O * C, 1, 0.0, self._st()),
            "csum")

    def _bgrad(self, gname, dy, O):
        _ck(self.L.fno_channel_sum(self._p(self.g[gname]), self._p(dy), 1, O, self.B * self.S, 0.0, self._st()),
            "csum")

    def _dinput(self, wname, dy, dx, O, C):
        """dx[C][BS] = W^T dy"""
        BS = self.B * self.S
        if self._use_tc(C, O):
            _ck(self.L.fno_dense_tc(self._p(self.pb[wname]), 1, self._p(dy), None, self._p(dx), None, C, O, BS, 0,
                                    self._p(self.tc_err), self._st()), "dense_tc")
            return
        self.gemm(1, C, BS, O, self.pb[wname], (0, 1, C), dy, (0, BS, 1), dx, (0, BS, 1), a_bf16=True)

    def backward(self):
        W, hid = self.W, self.hidden
        n_all = lambda t: t.numel()
        self._bgrad("c2", self.dout, self.cout)
        self._wgrad("Q2", self.dout, self.q, self.cout, hid)
        self._dinput("Q2", self.dout, self.dq, self.cout, hid)
        _ck(self.L.fno_act_bwd(self._p(self.dq), self._p(self.dq), self._p(self.u), n_all(self.dq), self._st()), "act")
        self._bgrad("c1", self.dq, hid)
        self._wgrad("Q1", self.dq, self.h[-1], hid, W)
        self._dinput("Q1", self.dq, self.dh, hid, W)
        for l in reversed(range(self.layers)):
            if l < self.layers - 1:
                _ck(self.L.fno_act_bwd(self._p(self.dz), self._p(self.dh), self._p(self.zs[l]), n_all(self.dz),
                                       self._st()), "act")
            else:
                self.dz.copy_(self.dh)
            self._bgrad(f"b{l}", self.dz, W)
            self._wgrad(f"W{l}", self.dz, self.h[l], W, W)
            self._dinput(f"W{l}", self.dz, self.dh2, W, W)
            self.spectral_bwd(l, self.dz, self.dh2)
            self.dh, self.dh2 = self.dh2, self.dh
        self._bgrad("bP", self.dh, W)
        self._wgrad("P", self.dh, self.a, W, self.cin)

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.t += 1
        st = self._st()
        for k, w in self.p.items():
            wb = self.pb.get(k)
            _ck(self.L.fno_adam(self._p(w), self._p(wb) if wb is not None else None, self._p(self.g[k]),
                                self._p(self.m[k]), self._p(self.v[k]), w.numel(), lr, b1, b2, eps, self.t, st),
                "adam")
        self._rbig()


def init_params(width=32, modes=16, layers=4, cin=7, hidden=128, cout=6, seed=0):
    """Random initial parameters in the oracle's layout (float64 arrays)."""
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
