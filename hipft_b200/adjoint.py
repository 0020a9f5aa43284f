"""Discrete adjoint of the flux-transport step: gradients of a map misfit.

Beside the reference-facing C-ABI path, this PyTorch binding returns the
gradient of an area-weighted L2 misfit between the final map and a target
map with respect to the initial field, the per-realization diffusion
coefficient constant and the analytic flow-profile coefficients
(differential rotation p0, p2, p4 and meridional flow p1, p3, p5, in the
namelist's m/s units; v0 and A, B, C follow by the chain rule).  HipFT has
no adjoint; the forward operators are diffusion_operator_cd
(src/hipft.f90:7927-7990) and advection_operator_weno3 (src/hipft.f90:
7711-7925) inside flux_transport_step (src/hipft.f90:4463-4507).

Method.  The forward run goes through the library's own fused step
(hipft_gpu_flux_transport_step) and keeps the field every
`checkpoint_every` steps on the device, and every step input of the last
segment.  The reverse pass walks the checkpoint segments backwards: it
recomputes a segment's step inputs from its checkpoint (all but the last
segment), then, step by step from the last, calls hipft_adj_step,
which replays that one step with every stage input kept and runs the
hand-written adjoint kernels (csrc/adjoint.cuh: transposed Laplacian with its
pole rings and seam, WENO3 face derivatives including the nonlinear weights,
the SSPRK(4,3) and RKG2 stage recurrences run backwards).  The schedule
(step dts, PTL subcycle dts, RKG2 stage counts) is the forward's and is held
fixed: the result is the gradient of the discrete map at that schedule.

Flow cotangents come back per cell from the kernels; the reduction to the
1-D profiles and the chain through the LLF alpha (max of |v| over the
set_lf_alpha stencil, src/hipft.f90:6940-7048) and the analytic profile
formulas (src/hipft.f90:7219-7285) is done here with torch autograd on 1-D
tensors.
"""
from __future__ import annotations

import ctypes
import time
from typing import Sequence

import numpy as np

from .gpu import HipftError, HipftGPU

M_S_TO_RS_HR = 5.172413793103448e-06  # m_s_to_rs_hr, src/hipft.f90:126
FLOW_KEYS = ("p0", "p2", "p4", "p1", "p3", "p5")


def mesh_1d(t: np.ndarray, p: np.ndarray) -> dict:
    """The 1-D mesh quantities set_mesh builds (src/hipft.f90:6495-6653), 1-based
    (index 0 unused), for the flow profiles and the misfit's area weights."""
    t = np.asarray(t, dtype=np.float64)
    p = np.asarray(p, dtype=np.float64)
    ntm, npm1 = len(t), len(p)
    npm, nt, np_ = npm1 + 1, ntm + 1, npm1 + 1
    T = np.zeros(ntm + 1)
    T[1:] = t
    P = np.zeros(npm + 1)
    P[1:npm1 + 1] = p
    P[npm] = P[2] + 2.0 * np.pi
    th = np.zeros(nt + 1)
    dth = np.zeros(nt + 1)
    for i in range(2, ntm + 1):
        th[i] = 0.5 * (T[i] + T[i - 1])
        dth[i] = T[i] - T[i - 1]
    th[1] = th[2] - dth[2]
    th[nt] = th[ntm] + dth[ntm]
    dth[1] = dth[2]
    dth[nt] = dth[ntm]
    dt = np.zeros(ntm + 1)
    for i in range(1, ntm + 1):
        dt[i] = th[i + 1] - th[i]
    st = np.sin(T)
    st[1] = st[ntm] = 0.0
    ct = np.cos(T)
    ct[1] = ct[ntm] = 1.0
    sth = np.sin(np.abs(th))
    cth = np.cos(th)
    ph = np.zeros(np_ + 1)
    dph = np.zeros(np_ + 1)
    for i in range(2, np_ + 1):
        ph[i] = 0.5 * (P[i] + P[i - 1])
        dph[i] = P[i] - P[i - 1]
    ph[1] = ph[npm1] - 2.0 * np.pi
    dph[1] = dph[npm1]
    dp = np.zeros(npm + 1)
    for i in range(1, npm):
        dp[i] = ph[i + 1] - ph[i]
    dp[npm] = dp[2]
    return dict(ntm=ntm, npm=npm, nt=nt, t=T, dth=dth, dt=dt, st=st, ct=ct, sth=sth, cth=cth, dph=dph, dp=dp)


def misfit_weights(mesh: dict) -> np.ndarray:
    """(npm, ntm) area weights of the misfit: get_flux's cell areas
    (src/hipft.f90:8672-8750; quarter cells at the poles, half-width columns
    at phi = 0 and 2 pi), zero in the seam column npm."""
    ntm, npm = mesh["ntm"], mesh["npm"]
    t, dth, dt, st, dph, dp = (mesh[k] for k in ("t", "dth", "dt", "st", "dph", "dp"))
    da_t = np.array([0.0] + [st[j] * dt[j] for j in range(1, ntm + 1)])
    da_t[1] = 0.25 * np.sin(0.5 * (t[1] + t[2])) * dth[2]
    da_t[ntm] = 0.25 * np.sin(0.5 * (t[ntm] + t[ntm - 1])) * dth[ntm]
    da_p = np.array([0.0] + [dp[k] for k in range(1, npm + 1)])
    da_p[1] = 0.5 * dph[1]
    da_p[npm - 1] = 0.5 * dph[npm - 1]
    w = np.zeros((npm, ntm))
    for k in range(1, npm):
        w[k - 1, :] = da_p[k] * da_t[1:]
    return w


def flow_profiles(mesh: dict, coef: dict):
    """Differentiable 1-D flows and LLF alphas for (nr,) tensors coef[p0..p5]:
    vt (nr, nt+1), at (nr, ntm+1), vp (nr, ntm+1), ap (nr, ntm+1), 1-based.
    add_flow_mf_analytic / add_flow_dr_analytic (src/hipft.f90:7243-7283)
    and set_lf_alpha's stencils (src/hipft.f90:6940-7048)."""
    import torch
    ntm, nt = mesh["ntm"], mesh["nt"]
    kw = dict(dtype=torch.float64, device=coef["p0"].device)
    cth = torch.tensor(mesh["cth"], **kw)
    sth = torch.tensor(mesh["sth"], **kw)
    ct = torch.tensor(mesh["ct"], **kw)
    st = torch.tensor(mesh["st"], **kw)
    c = lambda name: coef[name][:, None]
    vt = -M_S_TO_RS_HR * sth[None, :] * (c("p1") * cth + c("p3") * cth ** 3 + c("p5") * cth ** 5)
    vt = torch.cat([torch.zeros_like(vt[:, :1]), vt[:, 1:]], dim=1)
    vp = M_S_TO_RS_HR * st[None, :] * (c("p0") + c("p2") * ct ** 2 + c("p4") * ct ** 4)
    vp = torch.cat([torch.zeros_like(vp[:, :1]), vp[:, 1:]], dim=1)
    avt = vt.abs()

    def vmax(lo, hi):  # max |vt(lo..hi)| per realization
        return avt[:, lo:hi + 1].max(dim=1).values

    at_cols = [torch.zeros_like(vt[:, 0])]
    for j in range(1, ntm + 1):
        if j == 1:
            at_cols.append(vmax(1, 4))
        elif j == 2:
            at_cols.append(vmax(1, 5))
        elif j == nt - 2:
            at_cols.append(vmax(j - 2, j + 2))
        elif j == nt - 1:
            at_cols.append(vmax(j - 2, j + 1))
        else:
            at_cols.append(vmax(j - 2, j + 3))
    at = torch.stack(at_cols, dim=1)
    ap = vp.abs()  # the six phi neighbours of a 1-D profile are equal
    return vt, at, vp, ap


class MisfitAdjoint:
    """Gradient of L = 1/2 sum_{j,k} w(j,k) (f_N - g)^2 over N flux-transport
    steps of sizes `dts`, where w are misfit_weights and g the target field.

    gpu: a HipftGPU handle configured for the run (flows set with
    gpu.set_flow); D: the diffusion_coef_constants it was built with; flow:
    dict of (nr,) arrays p0, p2, p4, p1, p3, p5 as given to gpu.set_flow."""

    def __init__(self, gpu: HipftGPU, D: Sequence[float], flow: dict, checkpoint_every: int = 64):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("the adjoint runs on the GPU (libhipft_gpu); no CUDA device is visible")
        self.gpu = gpu
        self.nr, self.npm, self.ntm = gpu.nr, gpu.npm, gpu.ntm
        self.D = np.asarray(D, dtype=np.float64).reshape(self.nr)
        self.flow = {k: np.asarray(flow.get(k, 0.0), dtype=np.float64).reshape(-1) * np.ones(self.nr)
                     for k in FLOW_KEYS}
        self.k = max(1, int(checkpoint_every))
        self.mesh = mesh_1d(gpu.t, gpu.p)
        self.w = misfit_weights(self.mesh)
        self.timing = {}

    def _dev(self):
        return self.gpu.field_tensor()

    def _set(self, x):
        self.gpu._ck(self.gpu.L.hipft_gpu_set_field_device(self.gpu.h, ctypes.c_void_p(x.data_ptr())),
                     "set_field_device")

    def loss_and_cotangent(self, fN: np.ndarray, target: np.ndarray):
        """Misfit and its folded cotangent (nr, npm, ntm)."""
        r = fN - target
        loss = 0.5 * float(np.sum(self.w[None] * r * r))
        g = self.w[None] * r
        gb = np.zeros_like(g)
        gb[:, 1:self.npm - 1] = g[:, 1:self.npm - 1]
        gb[:, self.npm - 2] += g[:, 0]  # column 1 is the seam copy of column npm-1
        return loss, gb

    def run(self, f0: np.ndarray, target: np.ndarray, dts: Sequence[float]) -> tuple:
        """Forward, misfit, reverse.  Returns (loss, grads) with grads["f0"]
        (nr, npm, ntm) (folded: seam columns zero, their share in columns
        npm-1 and 2), grads["D"] (nr,) and grads["p0".."p5"] (nr,).
        self.timing holds the wall seconds of the forward and reverse parts."""
        import torch
        g = self.gpu
        dts = [float(d) for d in dts]
        n = len(dts)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.set_field(f0)
        g.update_flow()
        ckpt = {}
        last0 = ((n - 1) // self.k) * self.k  # the last segment's inputs are kept, not recomputed
        kept = []
        for s, dt in enumerate(dts):
            if s % self.k == 0:
                ckpt[s] = self._dev().clone()
            if s >= last0:
                kept.append(ckpt[s] if s == last0 else self._dev().clone())
            g.flux_transport_step(dt)
        fN = g.get_field()
        t1 = time.perf_counter()
        loss, gb = self.loss_and_cotangent(fN, np.asarray(target, dtype=np.float64))
        ldt = self._dev().shape[-1]
        dev = torch.device("cuda")
        fbar = torch.zeros((self.nr, self.npm, ldt), dtype=torch.float64, device=dev)
        fbar[:, :, :self.ntm] = torch.from_numpy(gb).to(dev)
        dacc = torch.zeros(self.nr, dtype=torch.float64, device=dev)
        gflow = torch.zeros((5, self.nr, self.npm, ldt), dtype=torch.float64, device=dev)
        for s0 in sorted(ckpt, reverse=True):
            s1 = min(s0 + self.k, n)
            states = kept if s0 == last0 else [ckpt[s0]]
            if s0 != last0 and s1 - s0 > 1:
                self._set(ckpt[s0])
                for s in range(s0, s1 - 1):
                    g.flux_transport_step(dts[s])
                    states.append(self._dev().clone())
            for s in range(s1 - 1, s0 - 1, -1):
                rc = g.L.hipft_adj_step(g.h, dts[s], ctypes.c_void_p(states[s - s0].data_ptr()),
                                        ctypes.c_void_p(fbar.data_ptr()), ctypes.c_void_p(dacc.data_ptr()),
                                        ctypes.c_void_p(gflow.data_ptr()))
                g._ck(rc, "hipft_adj_step")
        torch.cuda.synchronize()
        grads = {"f0": fbar[:, :, :self.ntm].cpu().numpy().copy()}
        grads["f0"][:, 0] = 0.0
        grads["f0"][:, self.npm - 1] = 0.0
        grads["D"] = dacc.cpu().numpy() / self.D
        grads.update(self._flow_grads(gflow))
        t2 = time.perf_counter()
        self.timing = {"forward_s": t1 - t0, "reverse_s": t2 - t1}
        return loss, grads

    def _flow_grads(self, gflow) -> dict:
        import torch
        ntm, npm = self.ntm, self.npm
        G = gflow[:, :, 1:npm - 1, :ntm].sum(dim=2).cpu()  # (5, nr, ntm), theta index j-1
        gln_t, glp_t, gup_t, gln_p, glp_p = G
        nt = ntm + 1
        vt_bar = torch.zeros((self.nr, nt + 1), dtype=torch.float64)
        vt_bar[:, 1:ntm + 1] += gln_t + gup_t
        vt_bar[:, 2:nt + 1] += glp_t
        at_bar = torch.zeros((self.nr, ntm + 1), dtype=torch.float64)
        at_bar[:, 1:] = gln_t - glp_t
        vp_bar = torch.zeros((self.nr, ntm + 1), dtype=torch.float64)
        vp_bar[:, 1:] = gln_p + glp_p
        ap_bar = torch.zeros((self.nr, ntm + 1), dtype=torch.float64)
        ap_bar[:, 1:] = gln_p - glp_p
        coef = {k: torch.tensor(self.flow[k], dtype=torch.float64, requires_grad=True) for k in FLOW_KEYS}
        vt, at, vp, ap = flow_profiles(self.mesh, coef)
        torch.autograd.backward([vt, at, vp, ap], [vt_bar, at_bar, vp_bar, ap_bar])
        return {k: coef[k].grad.numpy().copy() for k in FLOW_KEYS}


def chain_physical(grads: dict) -> dict:
    """Gradients with respect to v0 (p1 = 2 v0, p3 = -2 v0) and A, B, C in
    deg/day (p0, p2, p4 = 140.596... x A, B, C)."""
    from .synthetic import DEG_DAY_TO_M_S
    return {"v0": 2.0 * grads["p1"] - 2.0 * grads["p3"], "A": DEG_DAY_TO_M_S * grads["p0"],
            "B": DEG_DAY_TO_M_S * grads["p2"], "C": DEG_DAY_TO_M_S * grads["p4"]}


__all__ = ["MisfitAdjoint", "mesh_1d", "misfit_weights", "flow_profiles", "chain_physical", "HipftError"]
