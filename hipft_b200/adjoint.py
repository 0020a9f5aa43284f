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

Method.  The forward run keeps the field every `checkpoint_every` steps on
the device and tapes the steps of the last segment as it runs them
(hipft_adj_record: the library's own step, the same bits as
hipft_gpu_flux_transport_step, with every stage input kept on a tape stack).
The reverse pass walks the segments backwards: a segment other than the last
is recomputed once from its checkpoint, taped; then its steps are reversed
from the last (hipft_adj_reverse: the hand-written adjoint kernels of
csrc/adjoint.cuh -- transposed Laplacian with its pole rings and seam, WENO3
face derivatives including the nonlinear weights, the SSPRK(4,3) and RKG2
stage recurrences run backwards).  Steps for which the device has no room
left keep their input field instead and are taped one at a time in the
reverse pass.  The schedule (step dts, PTL subcycle dts, RKG2 stage counts)
is the forward's and is held fixed: the result is the gradient of the
discrete map at that schedule.

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
import torch

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
    dict of (nr,) arrays p0, p2, p4, p1, p3, p5 as given to gpu.set_flow;
    assim: optional {step index s: (map3, options)}, an assimilation of the
    (3, ntm, npm1) map with HipftGPU.assimilate's keyword options right after
    step s (apply_data_assimilation, src/hipft.f90:4148-4306), differentiated
    by hipft_adj_assimilate_at (blend and additive forms, and the balanced
    increment, for which the field before each such assimilation of the
    segment being reversed is kept: one field per balanced assimilation).

    Flows: analytic (gradients of f0, D and p0..p5), or a 2-D flow from
    files with or without analytic parts (gpu.set_flow_from_files; gradients
    of f0 and D only: the flow is a constant of the step, and the LLF alpha
    of a 2-D flow is not chained to the coefficients).  Attenuated flows,
    which depend on the field, are not differentiated.

    Device memory: one field per checkpoint (every `checkpoint_every` steps)
    and the tapes of one segment's steps, as many as fit while
    `reserve_frac` of the device memory stays free (the other steps of the
    segment keep one input field each); each step's tape is bounded by
    hipft_adj_set_tape_limit; release() frees the tape."""

    def __init__(self, gpu: HipftGPU, D: Sequence[float], flow: dict, checkpoint_every: int = 64,
                 assim: dict | None = None, reserve_frac: float = 0.15):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("the adjoint runs on the GPU (libhipft_gpu); no CUDA device is visible")
        self.gpu = gpu
        self.nr, self.npm, self.ntm = gpu.nr, gpu.npm, gpu.ntm
        self.D = np.asarray(D, dtype=np.float64).reshape(self.nr)
        self.flow = {k: np.asarray(flow.get(k, 0.0), dtype=np.float64).reshape(-1) * np.ones(self.nr)
                     for k in FLOW_KEYS}
        self.k = max(1, int(checkpoint_every))
        self.assim = dict(assim or {})
        self._preda = {}  # step -> field before its balanced assimilation
        self.mesh = mesh_1d(gpu.t, gpu.p)
        self.w = misfit_weights(self.mesh)
        self.timing = {}
        self._fwd = None
        self.reserve_frac = float(reserve_frac)
        self._fbytes = 0
        self._est_fields = 16
        self._budget = 0.0
        self._free = self._total = self._tape0 = 0

    def _dev(self):
        return self.gpu.field_tensor()

    def _snapshot(self):
        """A copy of the current field, complete on return: the library's
        stream does not wait for torch's, and its next launch may overwrite
        the field in place."""
        import torch
        x = self._dev().clone()
        torch.cuda.current_stream().synchronize()
        return x

    def _set(self, x):
        self.gpu._ck(self.gpu.L.hipft_gpu_set_field_device(self.gpu.h, ctypes.c_void_p(x.data_ptr())),
                     "set_field_device")

    def _da_opts(self, opts: dict):
        from .gpu import DAOpts, _p, _vec
        v = [_vec(opts.get(k, dflt), self.nr) for k, dflt in (("mu_power", 4.0), ("mu_limit", 0.1),
                                                               ("lat_limit", 0.0))]
        o = DAOpts(int(opts.get("add", False)), int(opts.get("custom_from_mu", False)),
                   int(opts.get("balance_flux", False)), float(opts.get("mult_fac", 1.0)), *[_p(a) for a in v])
        return o, v

    def _assimilate(self, s: int, keep: bool):
        """The assimilation after step s, if any; keep: hold the field before
        a balanced increment for the reverse pass."""
        if s in self.assim:
            m3, opts = self.assim[s]
            if keep and opts.get("balance_flux", False) and not opts.get("add", False):
                self._preda[s] = self._snapshot()
            self.gpu.assimilate(m3, **opts)

    def _step(self, s: int, dt: float, keep: bool = False):
        self.gpu.flux_transport_step(dt)
        self._assimilate(s, keep)

    def loss_and_cotangent(self, fN: np.ndarray, target: np.ndarray):
        """Misfit and its folded cotangent (nr, npm, ntm)."""
        r = fN - target
        loss = 0.5 * float(np.sum(self.w[None] * r * r))
        g = self.w[None] * r
        return loss, fold_cotangent(g)

    # -- taping: a recorded step is a forward step whose tape stays on the
    # library's stack until its reverse; a segment is recorded while the
    # device has room for it (beyond `reserve_frac` of its memory) and its
    # remaining steps keep their input fields instead, to be recorded one at a
    # time in the reverse pass.
    def _recorded(self):
        n, used = ctypes.c_int64(0), ctypes.c_int64(0)
        self.gpu._ck(self.gpu.L.hipft_adj_recorded(self.gpu.h, ctypes.byref(n), ctypes.byref(used)),
                     "hipft_adj_recorded")
        return n.value, used.value

    def _tape_fields(self):
        n = ctypes.c_int64(0)
        self.gpu._ck(self.gpu.L.hipft_adj_tape_fields(self.gpu.h, ctypes.byref(n)), "hipft_adj_tape_fields")
        return n.value

    def _segment_budget(self):
        """Bytes a segment's tapes may take: the device memory free at the
        start of the run (queried once, in forward()) plus the allocated,
        unused tape slots, less the reserve; each recorded step then draws on
        it."""
        _, used = self._recorded()
        # free now = free at the start - tape grown since; spare = tape - used
        self._budget = self._free + (self._tape0 - used) * self._fbytes - self.reserve_frac * self._total

    def _room_to_record(self) -> bool:
        return self._budget >= self._est_fields * self._fbytes

    def _record(self, s: int, dt: float):
        _, u0 = self._recorded()
        self.gpu._ck(self.gpu.L.hipft_adj_record(self.gpu.h, float(dt)), "hipft_adj_record")
        _, u1 = self._recorded()
        self._est_fields = max(self._est_fields, u1 - u0)
        self._budget -= (u1 - u0) * self._fbytes
        self._assimilate(s, True)

    def forward(self, f0: np.ndarray, dts: Sequence[float]) -> np.ndarray:
        """The forward run with its checkpoints, the last segment taped;
        returns f_N (nr, npm, ntm)."""
        import torch
        g = self.gpu
        dts = [float(d) for d in dts]
        n = len(dts)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g._ck(g.L.hipft_adj_clear(g.h), "hipft_adj_clear")  # steps left by an earlier run; the tape memory stays
        self._preda = {}
        g.set_field(f0)
        g.update_flow()
        self._fbytes = self._dev().numel() * 8
        self._est_fields = 16
        if not self._total:  # the first run; later runs find the same free memory (the tape is kept)
            self._free, self._total = torch.cuda.mem_get_info()
            self._tape0 = self._tape_fields()
        ckpt, recorded, states = {}, set(), {}
        last0 = ((n - 1) // self.k) * self.k
        taping = True
        self._budget = 0.0
        for s, dt in enumerate(dts):
            if s % self.k == 0:
                ckpt[s] = self._snapshot()
            if s == last0:
                torch.cuda.synchronize()
                t_last = time.perf_counter()
                self._segment_budget()
            if s >= last0 and taping and self._room_to_record():
                self._record(s, dt)
                recorded.add(s)
                continue
            if s >= last0:
                taping = False
                states[s] = self._snapshot()
            self._step(s, dt, keep=s >= last0)
        fN = g.get_field()
        self._fwd = dict(dts=dts, ckpt=ckpt, recorded=recorded, states=states, last0=last0)
        t1 = time.perf_counter()
        # forward_parts: seconds before the last segment, and of the (taped) last segment
        self.timing = {"forward_s": t1 - t0, "forward_parts": (t_last - t0, t1 - t_last)}
        return fN

    def backward(self, gb) -> dict:
        """Reverse pass from the folded cotangent gb (nr, npm, ntm) of f_N
        (numpy or torch; seam columns ignored).  Returns grads["f0"] (nr,
        npm, ntm) (folded: seam columns zero, their share in columns npm-1
        and 2), grads["D"] (nr,) and, for analytic flows, grads["p0".."p5"]
        (nr,)."""
        import torch
        if self._fwd is None:
            raise RuntimeError("backward() needs a forward() first")
        g = self.gpu
        dts, ckpt, last0 = (self._fwd[k] for k in ("dts", "ckpt", "last0"))
        n = len(dts)
        t1 = time.perf_counter()
        ldt = self._dev().shape[-1]
        dev = torch.device("cuda")
        fbar = torch.zeros((self.nr, self.npm, ldt), dtype=torch.float64, device=dev)
        gbt = torch.as_tensor(gb, dtype=torch.float64).to(dev)
        fbar[:, 1:self.npm - 1, :self.ntm] = gbt[:, 1:self.npm - 1]
        dacc = torch.zeros(self.nr, dtype=torch.float64, device=dev)
        gflow = torch.zeros((5, self.nr, self.npm, ldt), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()  # the library's stream reads these next
        ptr = lambda x: ctypes.c_void_p(x.data_ptr())
        seg_times = []
        for s0 in sorted(ckpt, reverse=True):
            s1 = min(s0 + self.k, n)
            ta = time.perf_counter()
            if s0 == last0:
                recorded, states = self._fwd["recorded"], self._fwd["states"]
            else:
                # recompute the segment from its checkpoint, taped while there is room
                recorded, states = set(), {}
                self._set(ckpt[s0])
                self._segment_budget()
                taping = True
                for s in range(s0, s1):
                    if taping and self._room_to_record():
                        self._record(s, dts[s])
                        recorded.add(s)
                        continue
                    taping = False
                    states[s] = self._snapshot()
                    if s < s1 - 1:
                        self._step(s, dts[s], keep=True)
            torch.cuda.synchronize()
            tb = time.perf_counter()
            for s in range(s1 - 1, s0 - 1, -1):
                if s in self.assim:
                    m3, opts = self.assim[s]
                    o, keep = self._da_opts(opts)
                    m3 = np.ascontiguousarray(m3, dtype=np.float64)
                    fpre = self._preda.pop(s, None)
                    if (fpre is None and opts.get("balance_flux", False) and not opts.get("add", False)
                            and s in states):
                        # a step the recompute did not run (taping stopped before
                        # the segment's last step): its output, once more
                        self._set(states[s])
                        g.flux_transport_step(dts[s])
                        fpre = self._snapshot()
                    g._ck(g.L.hipft_adj_assimilate_at(g.h, m3.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                      ctypes.byref(o), None if fpre is None else ptr(fpre),
                                                      ptr(fbar)), "hipft_adj_assimilate_at")
                if s not in recorded:
                    self._set(states.pop(s))
                    g._ck(g.L.hipft_adj_record(g.h, float(dts[s])), "hipft_adj_record")
                g._ck(g.L.hipft_adj_reverse(g.h, ptr(fbar), ptr(dacc), ptr(gflow)), "hipft_adj_reverse")
            torch.cuda.synchronize()
            seg_times.append((s0, tb - ta, time.perf_counter() - tb))
        torch.cuda.synchronize()
        nrec, _ = self._recorded()
        if nrec:
            raise RuntimeError(f"adjoint: {nrec} recorded steps left after the reverse pass")
        grads = {"f0": fbar[:, :, :self.ntm].cpu().numpy().copy()}
        grads["f0"][:, 0] = 0.0
        grads["f0"][:, self.npm - 1] = 0.0
        grads["D"] = dacc.cpu().numpy() / self.D
        if not getattr(g, "file_flow", False):
            grads.update(self._flow_grads(gflow))
        self.timing["reverse_s"] = time.perf_counter() - t1
        # per segment: (first step, recompute seconds, reverse seconds)
        self.timing["segments"] = seg_times
        self._fwd = None
        return grads

    def run(self, f0: np.ndarray, target: np.ndarray, dts: Sequence[float]) -> tuple:
        """Forward, misfit, reverse: (loss, grads) as backward() returns them.
        self.timing holds the wall seconds of the forward and reverse parts."""
        fN = self.forward(f0, dts)
        loss, gb = self.loss_and_cotangent(fN, np.asarray(target, dtype=np.float64))
        return loss, self.backward(gb)

    def release(self):
        """Frees the checkpoints and the library's tape."""
        self._fwd = None
        self.gpu._ck(self.gpu.L.hipft_adj_release(self.gpu.h), "hipft_adj_release")

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
        # the profile chain needs autograd even inside a Function's backward,
        # where grad mode is off
        with torch.enable_grad():
            coef = {k: torch.tensor(self.flow[k], dtype=torch.float64, requires_grad=True) for k in FLOW_KEYS}
            vt, at, vp, ap = flow_profiles(self.mesh, coef)
            torch.autograd.backward([vt, at, vp, ap], [vt_bar, at_bar, vp_bar, ap_bar])
        return {k: coef[k].grad.numpy().copy() for k in FLOW_KEYS}


def fold_cotangent(g):
    """Folds a cotangent (nr, npm, ntm) of a periodic field: the seam columns
    1 and npm are copies of columns npm-1 and 2, so their entries move there
    and the seam entries become zero (numpy or torch)."""
    gb = g.clone() if hasattr(g, "clone") else np.array(g, dtype=np.float64, copy=True)
    npm = gb.shape[1]
    gb[:, npm - 2] += gb[:, 0]
    gb[:, 1] += gb[:, npm - 1]
    gb[:, 0] = 0.0
    gb[:, npm - 1] = 0.0
    return gb


class FluxTransport:
    """f_N = F(f0; D, p0, p2, p4, p1, p3, p5): N flux-transport steps of the
    library (flux_transport_step, src/hipft.f90:4463-4507) as a differentiable
    PyTorch function.

        run = FluxTransport(t, p, dts, assim=..., checkpoint_every=64)
        fN = run(f0, D, {"p0": ..., "p2": ..., ...})   # torch tensors, FP64
        loss = ((fN - target) ** 2 * w).sum(); loss.backward()

    The forward runs the CUDA library (WENO3 + SSPRK(4,3) Strang-split with
    RKG2); backward runs its hand-written adjoint (hipft_adj_reverse,
    hipft_adj_assimilate) through MisfitAdjoint.backward.  f0 must be periodic
    (columns 1, npm copy columns npm-1, 2), as the reference's fields are; its
    gradient is folded onto the core columns.  Handle options (diffusion
    subcycles and so on) are HipftGPU keyword arguments."""

    def __init__(self, t, p, dts, *, assim: dict | None = None, checkpoint_every: int = 64, device: int = 0,
                 **handle_kw):
        self.t = np.asarray(t, dtype=np.float64)
        self.p = np.asarray(p, dtype=np.float64)
        self.dts = [float(d) for d in dts]
        self.assim = assim
        self.k = checkpoint_every
        self.device = device
        self.kw = dict(advance_flow=True, flow_num_method=4, strang_splitting=True, advance_diffusion=True,
                       diffusion_num_method=3)
        self.kw.update(handle_kw)

    def __call__(self, f0, D, coef: dict):
        return _FluxTransportFn.apply(f0, D, *[torch.as_tensor(coef.get(k, 0.0), dtype=torch.float64)
                                             .reshape(-1).expand(f0.shape[0]).contiguous() for k in FLOW_KEYS],
                                      self)


class _FluxTransportFn(torch.autograd.Function):
    """The autograd node of FluxTransport: forward through the library's
    steps with checkpoints, backward through its adjoint."""

    @staticmethod
    def forward(ctx, f0, D, p0, p2, p4, p1, p3, p5, run):
        nr = f0.shape[0]
        Dn = D.detach().cpu().numpy().astype(np.float64).reshape(nr)
        flow = {k: v.detach().cpu().numpy().astype(np.float64).reshape(nr)
                for k, v in zip(FLOW_KEYS, (p0, p2, p4, p1, p3, p5))}
        g = HipftGPU(run.t, run.p, nr, device=run.device, diffusion_coef_constants=Dn, **run.kw)
        g.set_flow(dr_model=1, mf_model=1, dr_p0=flow["p0"], dr_p2=flow["p2"], dr_p4=flow["p4"],
                   mf_p1=flow["p1"], mf_p3=flow["p3"], mf_p5=flow["p5"])
        A = MisfitAdjoint(g, Dn, flow, checkpoint_every=run.k, assim=run.assim)
        fN = A.forward(f0.detach().cpu().numpy().astype(np.float64), run.dts)
        ctx.A = A
        return torch.as_tensor(fN, dtype=torch.float64, device=f0.device)

    @staticmethod
    def backward(ctx, gN):
        A = ctx.A
        grads = A.backward(fold_cotangent(gN.detach().to(torch.float64).cpu().numpy()))
        A.gpu.close()
        ctx.A = None
        dev = gN.device
        out = [torch.as_tensor(grads["f0"], device=dev), torch.as_tensor(grads["D"], device=dev)]
        out += [torch.as_tensor(grads[k], device=dev) for k in FLOW_KEYS]
        return (*out, None)


def chain_physical(grads: dict) -> dict:
    """Gradients with respect to v0 (p1 = 2 v0, p3 = -2 v0) and A, B, C in
    deg/day (p0, p2, p4 = 140.596... x A, B, C)."""
    from .synthetic import DEG_DAY_TO_M_S
    return {"v0": 2.0 * grads["p1"] - 2.0 * grads["p3"], "A": DEG_DAY_TO_M_S * grads["p0"],
            "B": DEG_DAY_TO_M_S * grads["p2"], "C": DEG_DAY_TO_M_S * grads["p4"]}


__all__ = ["MisfitAdjoint", "FluxTransport", "fold_cotangent", "mesh_1d", "misfit_weights", "flow_profiles",
           "chain_physical", "HipftError"]
