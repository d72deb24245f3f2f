"""Learned initial guess in 3D: a Fourier neural operator from the physical
parameters of a 3D spin-1 instance to its ground-state spinor, trained and
evaluated with the library's own kernels (include/fno.h).  No counterpart in
the reference, which starts every 3D imaginary-time run from INITIALIZE's
fixed Gaussian (cgpe3d.f90:747-837; spin-1 default 783-785).

Network (width W, M retained x modes, F = 2M retained y and z modes):
  input   a = [p_1..p_4, X, Y, Z]           7 channels on an N x N x N grid
  lift    h0 = P a + bP
  layer l z = W_l h + b_l + K_l h,  h' = GELU(z) (no GELU after the last layer)
  project out = Q2 GELU(Q1 h_L + c1) + c2  (6 channels: Re/Im of 3 components)
  K h     = Re(sum_k w_kx G_o(k) e^{+2 pi i k.r/N}) / N^3, G_o = sum_c R_oc H_c,
          H_c(k) = sum_r h_c(r) e^{-2 pi i k.r/N}, kx in {0..M-1}, ky and kz
          in {0..M-1, N-M..N-1}, w = 1 for kx = 0 else 2.
The parameters do not depend on N (only the truncated DFT matrices do): the
network is trained on a coarse grid and evaluated on the fine one.

Layout on the device: channel-major activations [C][B][Z][Y][X] (float32),
so a pointwise channel mix is one GEMM over all B*N^3 points, run on the
tensor cores (fno_dense_tc: tcgen05, BF16 operands, FP32 accumulation in
tensor memory, bias and GELU fused).  The spectral convolution is the
truncated DFT along x, then y, then z (three batched GEMM stages over
real/imaginary planes), a per-mode channel mix (batched GEMM over the F*F*M
modes in the real block form [[Rr, -Ri], [Ri, Rr]]), and the inverse stages
in reverse order; the backward pass runs the transposed stages by strides.
With tensor_cores (the default) those stages run on fno_gemm_tc (tcgen05,
FP32 operands split into BF16 head and tail, FP32 accumulation).
Device memory comes from torch (plumbing only); every arithmetic step is a
kernel of libfgpe.so.
"""
from __future__ import annotations

import numpy as np

from .fno import _ck, lib


def init_params(width=16, modes=8, layers=4, cin=7, hidden=64, cout=6, seed=0):
    """Random initial parameters (float64 arrays); R_l is [o, c, kz, ky, kx]."""
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


# Parameter box of the 3D learned guess (around the 256^3 spin-1 ground
# state of Rb-87 with a0/a2 = 101.8/100.4 a_B, N = 1e5, 50 Hz, gamma = 0.5):
# isotropic SO strength gamma, c0 = TAU(0)/2, c2/c0 = TAU(1)/TAU(0), NUZ/NUX.
BOX3 = {"gamma": (0.3, 0.7), "c0": (3500.0, 5300.0), "c2_over_c0": (-0.012, 0.0), "az": (0.8, 1.25)}


def normalise_params(gamma, c0, c2_over_c0, az):
    """Map BOX3 onto about [-1, 1]."""
    lo = np.array([v[0] for v in BOX3.values()])
    hi = np.array([v[1] for v in BOX3.values()])
    x = np.array([gamma, c0, c2_over_c0, az], float)
    return 2.0 * (x - lo) / (hi - lo) - 1.0


def input_channels(params_norm, n):
    """a [7][B][n][n][n]: the four normalised parameters as constant fields,
    then X, Y, Z in units of the box half-width (INITIALIZE's grid points,
    cgpe3d.f90:726-735, divided by N*D/2)."""
    pn = np.asarray(params_norm, np.float64).reshape(-1, 4)
    B = pn.shape[0]
    x = (-1.0 + 2.0 * np.arange(n) / n).astype(np.float32)
    a = np.empty((7, B, n, n, n), np.float32)
    for q in range(4):
        a[q] = pn[:, q][:, None, None, None]
    a[4] = x[None, None, None, :]          # X varies fastest
    a[5] = x[None, None, :, None]
    a[6] = x[None, :, None, None]
    return a


class FNO3:
    """Forward, backward and Adam on the device for one grid size n and
    batch size B (train=False: forward only, no gradient buffers)."""

    def __init__(self, n, batch, width=16, modes=8, layers=4, cin=7, hidden=64, cout=6, seed=0, params=None,
                 device="cuda", tensor_cores=True, train=True):
        import torch
        self.torch = torch
        self.tensor_cores = tensor_cores
        self.tc_err = torch.zeros(1, dtype=torch.int32, device=device)
        self.L = lib()
        self.n, self.B, self.W, self.M, self.F = n, batch, width, modes, 2 * modes
        self.layers, self.cin, self.hidden, self.cout = layers, cin, hidden, cout
        self.S = n ** 3
        self.NMODE = self.F * self.F * self.M
        self.dev = device
        self.train = train
        src = init_params(width, modes, layers, cin, hidden, cout, seed) if params is None else params
        self.p, self.pb, self.g, self.m, self.v = {}, {}, {}, {}, {}
        for k, val in self._to_device_layout(src).items():
            t = torch.tensor(val, dtype=torch.float32, device=device).contiguous()
            self.p[k] = t
            if train:
                self.g[k] = torch.zeros_like(t)
                self.m[k] = torch.zeros_like(t)
                self.v[k] = torch.zeros_like(t)
        self.t = 0
        for k in self._matrices():
            self.pb[k] = torch.empty(self.p[k].numel(), dtype=torch.bfloat16, device=device)
        for l in range(layers):
            self.pb[f"Rbig{l}"] = torch.empty(self.NMODE * 4 * width * width, dtype=torch.bfloat16, device=device)
        if train:
            self.g_rbig = torch.empty(self.NMODE * 4 * width * width, dtype=torch.float32, device=device)
        self.refresh_bf16()
        self._dft()
        self._alloc()
        self.loss_dev = torch.zeros(1, dtype=torch.float64, device=device)
        self.loss_part = torch.zeros(256, dtype=torch.float64, device=device)

    # ------------------------------------------------------------ layout
    def _matrices(self):
        return ["P", "Q1", "Q2"] + [f"W{l}" for l in range(self.layers)]

    @staticmethod
    def _to_device_layout(p):
        """R: [o, c, kz, ky, kx] -> [mode = (kz, ky, kx)][o][c]."""
        out = {}
        for k, v in p.items():
            v = np.asarray(v)
            if k.startswith("Rr") or k.startswith("Ri"):
                o, c = v.shape[:2]
                out[k] = np.ascontiguousarray(np.transpose(v, (2, 3, 4, 0, 1)).reshape(-1, o, c))
            else:
                out[k] = v
        return out

    def _from_device(self, t, k):
        v = t.detach().cpu().numpy().astype(np.float64)
        if k.startswith("Rr") or k.startswith("Ri"):
            W, F, M = self.W, self.F, self.M
            v = np.transpose(v.reshape(F, F, M, W, W), (3, 4, 0, 1, 2))
        return v

    def params_numpy(self):
        return {k: self._from_device(t, k) for k, t in self.p.items()}

    def grads_numpy(self):
        return {k: self._from_device(t, k) for k, t in self.g.items()}

    def _dft(self):
        torch, n, M, F = self.torch, self.n, self.M, self.F
        kf = np.concatenate([np.arange(M), np.arange(n - M, n)])
        kh = np.arange(M)
        i = np.arange(n)
        thf = 2 * np.pi * np.outer(i, kf) / n          # E = exp(-i th)
        thh = 2 * np.pi * np.outer(i, kh) / n
        efr, efi = np.cos(thf), -np.sin(thf)            # [n][F]
        ehr, ehi = np.cos(thh), -np.sin(thh)            # [n][M]
        w = np.where(kh == 0, 1.0, 2.0)
        dt = getattr(self, "mat_dtype", torch.float32)
        f = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=dt, device=self.dev)
        # stage x: T1_p[cbz][y][kx] = sum_x h[cbz][y][x] Ex_p[x][kx]
        self.Ex = [f(ehr), f(ehi)]
        # stage y: T2_p'[cbz][ky][kx] = sum_(p,y) EyS_p'[ky][(p,y)] T1[cbz][(p,y)][kx]
        self.EyS = [f(np.concatenate([efr.T, -efi.T], axis=1)), f(np.concatenate([efi.T, efr.T], axis=1))]
        # stage z: K index interleaved (z, p'): k = 2 z + p'
        ezs_r = np.empty((F, 2 * n)); ezs_i = np.empty((F, 2 * n))
        ezs_r[:, 0::2], ezs_r[:, 1::2] = efr.T, -efi.T
        ezs_i[:, 0::2], ezs_i[:, 1::2] = efi.T, efr.T
        self.EzS = [f(ezs_r), f(ezs_i)]
        # inverse stages multiply by conj(E): [[Er, Ei], [-Ei, Er]] for (p, q)
        self.EfI = [[f(efr), f(efi)], [f(-efi), f(efr)]]   # [n][F], used for y and z
        # last stage, real part with the kx weights: ExWT_p[kx][x]
        self.ExWT = [f(w[:, None] * ehr.T), f(w[:, None] * ehi.T)]

    def _alloc(self):
        torch, B, W, S, n, M, F = self.torch, self.B, self.W, self.S, self.n, self.M, self.F
        z = lambda *s: torch.zeros(*s, dtype=torch.float32, device=self.dev)
        BS = B * S
        self.a = z(self.cin, BS)
        self.h = [z(W, BS) for _ in range(self.layers + 1)]
        self.zs = [z(W, BS) for _ in range(self.layers)]
        self.u = z(self.hidden, BS)
        self.q = z(self.hidden, BS)
        self.out = z(self.cout, BS)
        CB = W * B
        self.T1 = z(CB * n * 2 * n * M)          # [cbz][p][y][kx]
        self.T2 = z(CB * n * 2 * F * M)          # [cb][z][p][ky][kx]
        nh = self.layers if self.train else 1
        self.Hm = [z(self.NMODE * 2 * CB) for _ in range(nh)]    # [mode][p][c][b]
        self.Gm = z(self.NMODE * 2 * CB)
        self.U1 = z(CB * n * 2 * F * M)          # [(o,b)][z][p][ky][kx]
        self.U2 = z(CB * n * 2 * n * M)          # [(o,b,z)][p][y][kx]
        if self.train:
            self.dout = z(self.cout, BS)
            self.dq = z(self.hidden, BS)
            self.dh = z(W, BS)
            self.dh2 = z(W, BS)
            self.dz = z(W, BS)
            self.chunk = S
            while self.chunk > 2048 and self.chunk % 2 == 0:
                self.chunk //= 2
            self.part = z((BS // self.chunk) * max(self.hidden, W) * max(self.hidden, W, self.cin))
            self.dHm = z(self.NMODE * 2 * CB)

    def refresh_bf16(self):
        st = self._st()
        for k in self._matrices():
            _ck(self.L.fno_to_bf16(self._p(self.p[k]), self._p(self.pb[k]), self.p[k].numel(), st), "to_bf16")
        self._rbig()

    def _rbig(self):
        for l in range(self.layers):
            _ck(self.L.fno_rbig_build(self._p(self.p[f"Rr{l}"]), self._p(self.p[f"Ri{l}"]),
                                      self._p(self.pb[f"Rbig{l}"]), self.NMODE, self.W, self.W, self._st()), "rbig")

    # ----------------------------------------------------------- helpers
    def _st(self):
        import ctypes
        return ctypes.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    @staticmethod
    def _p(t, off=0):
        import ctypes
        return ctypes.c_void_p(t.data_ptr() + t.element_size() * off)

    def gemm(self, batch, M, N, K, A, sA, B_, sB, C, sC, alpha=1.0, beta=0.0, a_bf16=False, aoff=0, boff=0, coff=0):
        import ctypes
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
        """out[O][BS] = W[O][C] x[C][BS] (+ bias); act_out = GELU(out) or out."""
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
        return bool(self.tc_err.item())

    def bias_act(self, z, h, bias, C, act):
        BS = self.B * self.S
        _ck(self.L.fno_bias_act(self._p(z), self._p(h) if h is not None else None,
                                self._p(bias) if bias is not None else None, C, BS, C * BS, int(act), self._st()),
            "bias_act")

    # ----------------------------------------------------------- spectral
    def spectral(self, l, h, z):
        """z[O][B][n^3] += K_l h."""
        n, M, F, W, B = self.n, self.M, self.F, self.W, self.B
        CB, FM, NM = W * B, F * M, self.NMODE
        T1, T2, Gm, U1, U2 = self.T1, self.T2, self.Gm, self.U1, self.U2
        Hm = self.Hm[l if self.train else 0]
        for p in range(2):   # T1_p[cbz][y][kx] = h[cbz][y][:] Ex_p
            self.gemm(CB * n, n, M, n, h, (n * n, n, 1), self.Ex[p], (0, M, 1), T1, (2 * n * M, M, 1),
                      coff=p * n * M)
        for p in range(2):   # T2[cb][z][p][ky][kx] = EyS_p T1[cbz]
            self.gemm(CB * n, F, M, 2 * n, self.EyS[p], (0, 2 * n, 1), T1, (2 * n * M, M, 1),
                      T2, (2 * FM, M, 1), coff=p * FM)
        for p in range(2):   # Hm[mode][p][cb] = EzS_p T2[cb]
            self.gemm(CB, F, FM, 2 * n, self.EzS[p], (0, 2 * n, 1), T2, (n * 2 * FM, FM, 1),
                      Hm, (1, FM * 2 * CB, 2 * CB), coff=p * CB)
        # Gm[mode][(p,o)][b] = Rbig[mode] Hm[mode]
        self.gemm(NM, 2 * W, B, 2 * W, self.pb[f"Rbig{l}"], (4 * W * W, 2 * W, 1), Hm, (2 * W * B, B, 1),
                  Gm, (2 * W * B, B, 1), a_bf16=True)
        for p in range(2):   # U1_p[(o,b)][z][(ky,kx)] = sum_q conj(Ez)_pq G_q
            for q in range(2):
                self.gemm(CB, n, FM, F, self.EfI[p][q], (0, F, 1), Gm, (1, FM * 2 * CB, 2 * CB),
                          U1, (n * 2 * FM, 2 * FM, 1), beta=float(q), boff=q * CB, coff=p * FM)
        for p in range(2):   # U2_p[(o,b,z)][y][kx] = sum_q conj(Ey)_pq U1_q
            for q in range(2):
                self.gemm(CB * n, n, M, F, self.EfI[p][q], (0, F, 1), U1, (2 * FM, M, 1),
                          U2, (2 * n * M, M, 1), beta=float(q), boff=q * FM, coff=p * n * M)
        for p in range(2):   # z += Re part along x, kx weights, 1/n^3
            self.gemm(CB * n, n, n, M, U2, (2 * n * M, M, 1), self.ExWT[p], (0, n, 1), z, (n * n, n, 1),
                      alpha=1.0 / n ** 3, beta=1.0, aoff=p * n * M)

    def spectral_bwd(self, l, dz, dh):
        """dh += K_l^T dz; gradients of Rr_l, Ri_l."""
        n, M, F, W, B = self.n, self.M, self.F, self.W, self.B
        CB, FM, NM = W * B, F * M, self.NMODE
        T1, T2, Gm, U1, U2, Hm, dHm = self.T1, self.T2, self.Gm, self.U1, self.U2, self.Hm[l], self.dHm
        for p in range(2):   # dU2_p = dz ExWT_p^T / n^3
            self.gemm(CB * n, n, M, n, dz, (n * n, n, 1), self.ExWT[p], (0, 1, n), U2, (2 * n * M, M, 1),
                      alpha=1.0 / n ** 3, coff=p * n * M)
        for q in range(2):   # dU1_q = sum_p conj(Ey)_pq^T dU2_p
            for p in range(2):
                self.gemm(CB * n, F, M, n, self.EfI[p][q], (0, 1, F), U2, (2 * n * M, M, 1),
                          U1, (2 * FM, M, 1), beta=float(p), boff=p * n * M, coff=q * FM)
        for q in range(2):   # dG_q = sum_p conj(Ez)_pq^T dU1_p
            for p in range(2):
                self.gemm(CB, F, FM, n, self.EfI[p][q], (0, 1, F), U1, (n * 2 * FM, 2 * FM, 1),
                          Gm, (1, FM * 2 * CB, 2 * CB), beta=float(p), boff=p * FM, coff=q * CB)
        # dRbig = dG Hm^T ; dHm = Rbig^T dG
        self.gemm(NM, 2 * W, 2 * W, B, Gm, (2 * W * B, B, 1), Hm, (2 * W * B, 1, B),
                  self.g_rbig, (4 * W * W, 2 * W, 1))
        self._rbig_fold(l)
        self.gemm(NM, 2 * W, B, 2 * W, self.pb[f"Rbig{l}"], (4 * W * W, 1, 2 * W), Gm, (2 * W * B, B, 1),
                  dHm, (2 * W * B, B, 1), a_bf16=True)
        for p in range(2):   # dT2[cb][(z,p')][(ky,kx)] = sum_p EzS_p^T dH_p
            self.gemm(CB, 2 * n, FM, F, self.EzS[p], (0, 1, 2 * n), dHm, (1, FM * 2 * CB, 2 * CB),
                      T2, (n * 2 * FM, FM, 1), beta=float(p), boff=p * CB)
        for p in range(2):   # dT1[cbz][(p,y)][kx] = sum_p' EyS_p'^T dT2_p'
            self.gemm(CB * n, 2 * n, M, F, self.EyS[p], (0, 1, 2 * n), T2, (2 * FM, M, 1),
                      T1, (2 * n * M, M, 1), beta=float(p), boff=p * FM)
        for p in range(2):   # dh += dT1_p Ex_p^T
            self.gemm(CB * n, n, n, M, T1, (2 * n * M, M, 1), self.Ex[p], (0, 1, M), dh, (n * n, n, 1),
                      beta=1.0, aoff=p * n * M)

    def _rbig_fold(self, l):
        _ck(self.L.fno_rbig_fold(self._p(self.g_rbig), self._p(self.g[f"Rr{l}"]), self._p(self.g[f"Ri{l}"]),
                                 self.NMODE, self.W, self.W, self._st()), "rbig_fold")

    # ------------------------------------------------------------ passes
    def set_inputs_device(self, params_norm):
        """The input channels of input_channels(), written on the device
        (no host array of B*n^3 values)."""
        torch, n = self.torch, self.n
        pn = np.asarray(params_norm, np.float64).reshape(-1, 4)
        a = self.a.view(self.cin, self.B, n, n, n)
        for b in range(self.B):
            for q in range(4):
                a[q, b].fill_(float(pn[b, q]))
        x = -1.0 + 2.0 * torch.arange(n, dtype=torch.float32, device=self.dev) / n
        a[4].copy_(x.view(1, 1, 1, n).expand(self.B, n, n, n))
        a[5].copy_(x.view(1, 1, n, 1).expand(self.B, n, n, n))
        a[6].copy_(x.view(1, n, 1, 1).expand(self.B, n, n, n))

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
        BS = self.B * self.S
        if self._use_tc(C, O):
            _ck(self.L.fno_dense_tc(self._p(self.pb[wname]), 1, self._p(dy), None, self._p(dx), None, C, O, BS, 0,
                                    self._p(self.tc_err), self._st()), "dense_tc")
            return
        self.gemm(1, C, BS, O, self.pb[wname], (0, 1, C), dy, (0, BS, 1), dx, (0, BS, 1), a_bf16=True)

    def backward(self):
        W, hid = self.W, self.hidden
        self._bgrad("c2", self.dout, self.cout)
        self._wgrad("Q2", self.dout, self.q, self.cout, hid)
        self._dinput("Q2", self.dout, self.dq, self.cout, hid)
        _ck(self.L.fno_act_bwd(self._p(self.dq), self._p(self.dq), self._p(self.u), self.dq.numel(), self._st()), "act")
        self._bgrad("c1", self.dq, hid)
        self._wgrad("Q1", self.dq, self.h[-1], hid, W)
        self._dinput("Q1", self.dq, self.dh, hid, W)
        for l in reversed(range(self.layers)):
            if l < self.layers - 1:
                _ck(self.L.fno_act_bwd(self._p(self.dz), self._p(self.dh), self._p(self.zs[l]), self.dz.numel(),
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

    def spinor(self, b=0):
        """Network output of batch entry b as PHI(NX,NY,NZ,3) complex128 (the
        layout fgpe_set_state takes): out channels are Re/Im of the three
        components, arrays [Z][Y][X]."""
        n = self.n
        o = self.out.detach().reshape(self.cout, self.B, n, n, n)[:, b].double().cpu().numpy()
        phi = np.empty((n, n, n, 3), np.complex128)
        for m in range(3):
            phi[..., m] = np.transpose(o[2 * m] + 1j * o[2 * m + 1], (2, 1, 0))
        return phi
