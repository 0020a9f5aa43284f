"""FP64 pure-PyTorch restatement of the flux-transport step, differentiated by
torch autograd: the reference the hand-written adjoint kernels are checked
against (test infrastructure; small grids only).

It restates, vectorised over (realization, phi, theta) tensors of shape
(nr, npm, ntm), the forward scheme the adjoint differentiates:
diffusion_operator_cd (src/hipft.f90:7927-7990, coefficients of
load_diffusion_matrix 4927-4983 with per-realization constant D),
advection_operator_weno3 (7711-7925; WENO weights of load_weno 6846-6938),
advection_step_ssprk43 (7515-7582), the RKG2 super-step
diffusion_step_sts_cd (5163-5242) with load_sts_rkg2 (5361-5475), fixed
diffusion subcycles (4551-4695) and Strang splitting (4463-4507).  The
schedule (step dts, RKG2 stage counts) is fixed up front, as in the adjoint.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from hipft_b200.adjoint import flow_profiles, mesh_1d, misfit_weights

DIFF_FACTOR = 7.43162901307967e-09  # diffusion_coef_factor default, src/hipft.f90


def _t(a, dev):
    return torch.as_tensor(np.asarray(a, dtype=np.float64), dtype=torch.float64, device=dev)


class RefScheme:
    def __init__(self, t, p, nr, upwind=1.0, factor=DIFF_FACTOR, device="cpu"):
        self.m = mesh_1d(t, p)
        m = self.m
        self.nr, self.ntm, self.npm, self.nt = nr, m["ntm"], m["npm"], m["nt"]
        self.np = self.npm
        self.up = float(upwind)
        self.factor = float(factor)
        self.dev = torch.device(device)
        ntm, npm, nt, np_ = self.ntm, self.npm, self.nt, self.np
        dt, dth, dp, dph = m["dt"], m["dth"], m["dp"], m["dph"]
        self.dt_i = 1.0 / np.where(dt == 0, 1, dt)
        self.dth_i = 1.0 / np.where(dth == 0, 1, dth)
        self.dp_i = 1.0 / np.where(dp == 0, 1, dp)
        self.dph_i = 1.0 / np.where(dph == 0, 1, dph)
        st_i = np.zeros(ntm + 1)
        st_i[2:ntm] = 1.0 / m["st"][2:ntm]
        self.st_i = st_i
        self.bcn = (1.0 / math.pi) * self.dth_i[2] * self.dth_i[2]
        self.bcs = (1.0 / math.pi) * self.dth_i[nt - 1] * self.dth_i[nt - 1]
        self.bcfn = 2.0 * self.dth_i[2] / math.pi
        self.bcfs = 2.0 * self.dth_i[nt - 1] / math.pi
        # load_weno
        wt = {k: np.zeros(nt + 1) for k in ("cp", "mc", "m", "cpt", "p", "mct")}
        for j in range(2, nt - 1):
            tot = dt[j - 1] + dt[j] + dt[j + 1]
            wt["cp"][j] = dt[j] / (dt[j] + dt[j + 1])
            wt["mc"][j] = dt[j] / (dt[j - 1] + dt[j])
            wt["m"][j] = dt[j - 1] / tot
            wt["cpt"][j] = (dt[j] + dt[j + 1]) / tot
            wt["p"][j] = dt[j + 1] / tot
            wt["mct"][j] = (dt[j - 1] + dt[j]) / tot
        wp = {k: np.zeros(np_ + 1) for k in ("cp", "mc", "m", "cpt", "p", "mct")}
        for k in range(2, np_):
            tot = dp[k - 1] + dp[k] + dp[k + 1]
            wp["cp"][k] = dp[k] / (dp[k] + dp[k + 1])
            wp["mc"][k] = dp[k] / (dp[k - 1] + dp[k])
            wp["m"][k] = dp[k - 1] / tot
            wp["cpt"][k] = (dp[k] + dp[k + 1]) / tot
            wp["p"][k] = dp[k + 1] / tot
            wp["mct"][k] = (dp[k - 1] + dp[k]) / tot
        for a in wp.values():
            a[1] = a[np_ - 1]
            a[np_] = a[2]
        self.wt, self.wp = wt, wp
        self.eps_t = dt.copy()
        self.eps_p = dp.copy()

    # ------------------------------------------------------------- diffusion
    def coefs(self, D):
        """coef1..5 on interior cells (nr, npm-2, ntm-2) for D (nr,) tensor."""
        ntm, npm = self.ntm, self.npm
        dfac = self.factor * D
        Dh = (0.5 * (dfac + dfac))[:, None, None]
        j = np.arange(2, ntm)
        k = np.arange(2, npm)
        sti = self.st_i[j]
        T = lambda a: _t(a, self.dev)
        ones = torch.ones((1, npm - 2, 1), dtype=torch.float64, device=self.dev)
        c1 = Dh * T(self.dph_i[k] * self.dp_i[k])[None, :, None] * T(sti * sti)[None, None, :]
        c2 = Dh * T(self.dth_i[j] * self.dt_i[j] * sti * self.m["sth"][j])[None, None, :] * ones
        c4 = Dh * T(self.dth_i[j + 1] * self.dt_i[j] * sti * self.m["sth"][j + 1])[None, None, :] * ones
        c5 = Dh * T(self.dph_i[k + 1] * self.dp_i[k])[None, :, None] * T(sti * sti)[None, None, :]
        c3 = -(c1 + c2 + c4 + c5)
        return c1, c2, c3, c4, c5, dfac

    def diffusion_op(self, x, D):
        ntm, npm = self.ntm, self.npm
        c1, c2, c3, c4, c5, dfac = self.coefs(D)
        xc = x[:, 1:npm - 1, 1:ntm - 1]
        y = (c1 * x[:, 0:npm - 2, 1:ntm - 1] + c2 * x[:, 1:npm - 1, 0:ntm - 2] + c3 * xc +
             c4 * x[:, 1:npm - 1, 2:ntm] + c5 * x[:, 2:npm, 1:ntm - 1])
        dp = _t(self.m["dp"][2:npm], self.dev)[None, :]
        dd = (dfac + dfac)[:, None]
        fn = (dd * (x[:, 1:npm - 1, 1] - x[:, 1:npm - 1, 0]) * dp).sum(dim=1)
        fs = (dd * (x[:, 1:npm - 1, ntm - 1] - x[:, 1:npm - 1, ntm - 2]) * dp).sum(dim=1)
        north = (fn * self.bcn)[:, None, None].expand(-1, npm - 2, 1)
        south = (-fs * self.bcs)[:, None, None].expand(-1, npm - 2, 1)
        return self._seam(torch.cat([north, y, south], dim=2))

    @staticmethod
    def _seam(core):
        return torch.cat([core[:, -1:], core, core[:, :1]], dim=1)

    def euler_dt(self, D):
        with torch.no_grad():
            c = self.coefs(_t(D, self.dev))[:5]
            g = sum(ci.abs() for ci in c)
        return 0.95 * (2.0 / float(g.max()))

    # ------------------------------------------------------------- advection
    @staticmethod
    def _weno(LNm2, LNm1, LN0, LPm1, LP0, LPp1, W, e_m1, e_0):
        (mc_m1, mc_0, cp_m1, cp_0, p_m1, mct_m1, m_0, cpt_0) = W
        p0m = (1.0 + mc_m1) * LNm1 - mc_m1 * LNm2
        p1m = mc_0 * LNm1 + cp_m1 * LN0
        p0p = (1.0 + cp_0) * LP0 - cp_0 * LPp1
        p1p = cp_m1 * LP0 + mc_0 * LPm1
        t0 = mc_m1 * (LNm1 - LNm2)
        t1 = cp_m1 * (LN0 - LNm1)
        t2 = cp_0 * (LPp1 - LP0)
        t3 = mc_0 * (LP0 - LPm1)
        e0 = e_m1 + 4.0 * t0 * t0
        e1 = e_m1 + 4.0 * t1 * t1
        e2 = e_0 + 4.0 * t2 * t2
        e3 = e_0 + 4.0 * t3 * t3
        w0m = p_m1 / (e0 * e0)
        w1m = mct_m1 / (e1 * e1)
        w0p = m_0 / (e2 * e2)
        w1p = cpt_0 / (e3 * e3)
        um = (w0m / (w0m + w1m)) * p0m + (w1m / (w0m + w1m)) * p1m
        upv = (w0p / (w0p + w1p)) * p0p + (w1p / (w0p + w1p)) * p1p
        return upv + um

    def advection_op(self, x, vt, at, vp, ap):
        ntm, npm, nt = self.ntm, self.npm, self.nt
        T = lambda a: _t(a, self.dev)
        xc = x[:, 1:npm - 1, :]
        # theta: LLF split and faces 2..ntm of the core columns
        LP = 0.5 * xc * (vt[:, 2:nt + 1] - at[:, 1:ntm + 1])[:, None, :]
        LN = 0.5 * xc * (vt[:, 1:ntm + 1] + at[:, 1:ntm + 1])[:, None, :]
        jf = np.arange(3, ntm)
        wt = self.wt
        W = [T(a)[None, None, :] for a in (wt["mc"][jf - 1], wt["mc"][jf], wt["cp"][jf - 1], wt["cp"][jf],
                                           wt["p"][jf - 1], wt["mct"][jf - 1], wt["m"][jf], wt["cpt"][jf])]
        Fw = self._weno(LN[..., 0:ntm - 3], LN[..., 1:ntm - 2], LN[..., 2:ntm - 1], LP[..., 1:ntm - 2],
                        LP[..., 2:ntm - 1], LP[..., 3:ntm], W, T(self.eps_t[jf - 1])[None, None, :],
                        T(self.eps_t[jf])[None, None, :])

        def upwind(v, xhi, xlo):
            cct = torch.where(v >= 0, torch.full_like(v, self.up), torch.full_like(v, -self.up))
            return v * 0.5 * ((1.0 - cct) * xhi + (1.0 + cct) * xlo)

        F2 = upwind(vt[:, 2][:, None], xc[..., 1], xc[..., 0])[..., None]
        Fn = upwind(vt[:, ntm][:, None], xc[..., ntm - 1], xc[..., ntm - 2])[..., None]
        ft = torch.cat([F2, Fw, Fn], dim=2)  # faces 2..ntm, index jf-2
        # phi: rows 2..ntm-1, cells 1..npm-1 with the periodic pad
        xr = x[:, 0:npm - 1, 1:ntm - 1]
        LPk = 0.5 * xr * (vp[:, 2:ntm] - ap[:, 2:ntm])[:, None, :]
        LNk = 0.5 * xr * (vp[:, 2:ntm] + ap[:, 2:ntm])[:, None, :]
        pad = lambda L: torch.cat([L[:, npm - 3:npm - 2], L, L[:, 1:2]], dim=1)  # indices 0..npm
        LPp, LNp = pad(LPk), pad(LNk)
        kf = np.arange(2, npm)
        wp = self.wp
        Wp = [T(a)[None, :, None] for a in (wp["mc"][kf - 1], wp["mc"][kf], wp["cp"][kf - 1], wp["cp"][kf],
                                            wp["p"][kf - 1], wp["mct"][kf - 1], wp["m"][kf], wp["cpt"][kf])]
        fp = self._weno(LNp[:, 0:npm - 2], LNp[:, 1:npm - 1], LNp[:, 2:npm], LPp[:, 1:npm - 1], LPp[:, 2:npm],
                        LPp[:, 3:npm + 1], Wp, T(self.eps_p[kf - 1])[None, :, None], T(self.eps_p[kf])[None, :, None])
        fp = torch.cat([fp, fp[:, :1]], dim=1)  # faces 2..npm (face npm = face 2)
        j = np.arange(2, ntm)
        sth = T(self.m["sth"])
        div_t = ((sth[j + 1][None, None, :] * ft[..., j - 1] - sth[j][None, None, :] * ft[..., j - 2]) *
                 T(self.st_i[j] * self.dt_i[j])[None, None, :])
        div_p = (fp[:, 1:, :] - fp[:, :-1, :]) * T(self.st_i[j])[None, None, :] * T(self.dp_i[2:npm])[None, :, None]
        aint = div_t + div_p
        dp = T(self.m["dp"][2:npm])[None, :]
        fn = (ft[..., 0] * dp).sum(dim=1)
        fs = (ft[..., ntm - 2] * dp).sum(dim=1)
        north = (fn * self.bcfn)[:, None, None].expand(-1, npm - 2, 1)
        south = (-fs * self.bcfs)[:, None, None].expand(-1, npm - 2, 1)
        return self._seam(torch.cat([north, aint, south], dim=2))

    # ------------------------------------------------------------------ steps
    def ssprk43(self, f, dtl, flows):
        L = lambda y: self.advection_op(y, *flows)
        f1 = f - 0.5 * dtl * L(f)
        f1 = f1 - 0.5 * dtl * L(f1)
        f1 = (2.0 / 3.0) * f + (1.0 / 3.0) * f1 - (1.0 / 6.0) * dtl * L(f1)
        return f1 - 0.5 * dtl * L(f1)

    @staticmethod
    def rkg2_coefs(s):
        w = 6.0 / ((s + 4) * (s - 1))
        b = [0.0] * (s + 1)
        uj, vj, ubj, gj = ([0.0] * (s + 1) for _ in range(4))
        b[1], b[2] = 1.0 / 3.0, 1.0 / 15.0
        uj[1], ubj[1] = 1.0, w
        uj[2], vj[2], ubj[2], gj[2] = 0.5, -0.1, 0.5 * w, 0.0
        for j in range(3, s + 1):
            b[j] = (4.0 * (j - 1) * (j + 4)) / (3.0 * j * (j + 1) * (j + 2) * (j + 3))
            uj[j] = b[j] / b[j - 1] * (2.0 + 1.0 / j)
            vj[j] = -b[j] / b[j - 2] * (1.0 / j + 1.0)
            ubj[j] = uj[j] * w
            gj[j] = (0.5 * j * (j + 1.0) * b[j - 1] - 1.0) * ubj[j]
        return uj, vj, ubj, gj

    @staticmethod
    def rkg2_stages(dtl, dt_euler):
        s = math.ceil(0.5 * (math.sqrt(25.0 + 24.0 * (dtl / dt_euler)) - 3.0))
        s = max(s, 3)
        return s + 1 if s % 2 == 0 else s

    def rkg2(self, f, dtl, D, s):
        uj, vj, ubj, gj = self.rkg2_coefs(s)
        A = lambda y: self.diffusion_op(y, D)
        u0 = f
        dty0 = dtl * A(u0)
        ykm2, ykm1 = u0, u0 + ubj[1] * dty0
        for k in range(2, s + 1):
            y = uj[k] * ykm1 + vj[k] * ykm2 + (1.0 - uj[k] - vj[k]) * u0 + ubj[k] * dtl * A(ykm1) + gj[k] * dty0
            ykm2, ykm1 = ykm1, y
        return ykm1

    def step(self, f, dt, D, flows, subcycles, dt_euler, strang=True, sub_dts=None):
        """One step; sub_dts, when given, are the diffusion subcycle dts (a
        PTL schedule recorded from a forward run), else `subcycles` equal ones."""
        f = self.ssprk43(f, 0.5 * dt if strang else dt, flows)
        for dtl2 in (sub_dts if sub_dts is not None else [dt / subcycles] * subcycles):
            f = self.rkg2(f, dtl2, D, self.rkg2_stages(dtl2, dt_euler))
        if strang:
            f = self.ssprk43(f, 0.5 * dt, flows)
        return f

    def run(self, f0, dts, D, coef, subcycles, dt_euler, strang=True, sched=None):
        flows = flow_profiles(self.m, coef)
        f = f0
        for n, dt in enumerate(dts):
            f = self.step(f, float(dt), D, flows, subcycles, dt_euler, strang, None if sched is None else sched[n])
        return f

    def misfit(self, f, target):
        w = _t(misfit_weights(self.m), self.dev)[None]
        r = f - target
        return 0.5 * (w * r * r).sum()
