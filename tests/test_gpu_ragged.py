"""Ragged batches: every realization advanced with its own schedule.

The reference keeps one schedule for all realizations (global MIN/MAX
reductions, src/hipft.f90:5036, 5103, 5141, 7345).  A ragged batch gives each
realization the schedule it would have alone, so its parity oracle is the
oracle run of that realization alone at the same dt sequence:

* diffusion + advection, per-realization D and flows: every realization's
  final field within 1e-12 of its own single-realization oracle run, and its
  stage counts and subcycles equal to that run's history;
* advection substeps: a step longer than some realizations' CFL limits
  splits into ceil(dt / limit) substeps for those realizations, which equals
  the oracle run of that realization alone with dt_max = dt / n_i;
* identical realizations: ragged and plain mode give the same field bit for
  bit (the schedules coincide).
"""
import numpy as np
import pytest

import test_gpu_refined as R
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-12

NTM, NPM1 = 96, 129
D = [80.0, 300.0, 900.0, 150.0]
P1 = [22.0, 30.0, 12.0, 40.0]
P2 = [-262.0, -300.0, -200.0, -340.0]


def _grid(ntm=NTM, npm1=NPM1):
    from hipft_b200 import synthetic as S
    t = S.refined_theta(ntm)
    p = S.uniform_phi(npm1)
    return t, p, R.smooth_map(t, p, 17)


def _handle(t, p, nr, diffusion=True, **kw):
    import hipft_b200 as H
    g = H.HipftGPU(t, p, nr, advance_flow=True, flow_num_method=4, strang_splitting=True,
                   advance_diffusion=diffusion, diffusion_coef_constants=D[:nr] if diffusion else None, **kw)
    g.set_flow(dr_model=1, mf_model=1, dr_p2=P2[:nr], mf_p1=P1[:nr])
    return g


def _oracle_alone(i, t, p, br, dt_max, time_end, diffusion=True):
    raw = dict(n_realizations=1, advance_flow=True, flow_num_method=4, strang_splitting=True, flow_dr_model=1,
               flow_mf_model=1, advance_diffusion=diffusion, time_end=time_end, dt_max=dt_max,
               flow_dr_coef_p2_values=[P2[i]], flow_mf_coef_p1_values=[P1[i]],
               # the handle's set_flow leaves the other coefficients at zero
               flow_dr_coef_p0_values=[0.0], flow_dr_coef_p4_values=[0.0],
               flow_mf_coef_p3_values=[0.0], flow_mf_coef_p5_values=[0.0],
               diffusion_coef_constants=[D[i]])
    prm = O.process_parameters(raw)
    return O.run(prm, map_pt=br[None], s1=p, s2=t)


def _dt_sequence(dt, nsteps):
    """The dt of each step as the oracle's update_timestep picks it when
    time_end is the sum of nsteps steps of dt and dt_max = dt."""
    tend = 0.0
    for _ in range(nsteps):
        tend += dt
    seq, time = [], 0.0
    for _ in range(nsteps):
        d = tend - time if time + dt >= tend else dt
        seq.append(d)
        time += d
    return seq, tend


def test_ragged_matches_each_realization_alone():
    t, p, br = _grid()
    nr, nsteps = 4, 3
    with _handle(t, p, nr) as g:
        g.load_initial_map(br[None])
        g.update_flow()
        g.set_ragged(True)
        dt = g.flow_dtmax()  # the shared step: every realization within its own CFL limit
        seq, tend = _dt_sequence(dt, nsteps)
        for d in seq:
            g.flux_transport_step(d)
        sched = g.ragged_schedule()
        f = g.get_field()
    assert len(set(sched["sts_s"].tolist())) > 1, "the realizations should need different stage counts"
    for i in range(nr):
        r = _oracle_alone(i, t, p, br, dt, tend)
        assert r["nsteps"] == nsteps
        err = np.abs(f[i] - r["f"][0]).max() / np.abs(r["f"][0]).max()
        assert err <= FIELD_TOL, f"realization {i}: field rel max-norm {err:.3e}"
        last = r["num"][-1, 0, :]
        assert int(last[6]) == sched["sts_s"][i], f"realization {i}: stage count {sched['sts_s'][i]} vs {last[6]}"
        assert int(last[7]) == sched["subcycles"][i], f"realization {i}: subcycles"
        assert np.isclose(last[5], sched["dt_euler"][i], rtol=1e-14, atol=0), f"realization {i}: Euler limit"


def test_ragged_advection_substeps():
    t, p, br = _grid()
    nr, nsteps = 3, 2
    with _handle(t, p, nr, diffusion=False) as g:
        g.load_initial_map(br[None])
        g.update_flow()
        g.set_ragged(True)
        lim = g.flow_dtmax_each()
        dt = 2.5 * lim.min()
        for _ in range(nsteps):
            g.flux_transport_step(dt)
        sched = g.ragged_schedule()
        f = g.get_field()
    n = np.maximum(1, np.ceil(dt / lim)).astype(int)
    assert np.array_equal(sched["adv_substeps"], n)
    assert n.max() >= 2 and len(set(n.tolist())) > 1
    for i in range(nr):
        dtm = dt / n[i]
        tend = 0.0
        for _ in range(nsteps * n[i]):
            tend += dtm
        r = _oracle_alone(i, t, p, br, dtm, tend, diffusion=False)
        assert r["nsteps"] == nsteps * n[i]
        err = np.abs(f[i] - r["f"][0]).max() / np.abs(r["f"][0]).max()
        assert err <= FIELD_TOL, f"realization {i} ({n[i]} substeps): field rel max-norm {err:.3e}"


def test_ragged_equals_plain_for_identical_realizations():
    import hipft_b200 as H
    t, p, br = _grid()
    nr = 3
    out = []
    for ragged in (False, True):
        g = H.HipftGPU(t, p, nr, advance_flow=True, flow_num_method=4, strang_splitting=True,
                       advance_diffusion=True, diffusion_coef_constants=[300.0] * nr)
        g.set_flow(dr_model=1, mf_model=1, dr_p2=-262.0, mf_p1=22.0)
        g.load_initial_map(br[None])
        g.update_flow()
        if ragged:
            g.set_ragged(True)
        dt = g.flow_dtmax()
        for _ in range(3):
            g.flux_transport_step(dt)
        out.append(g.get_field())
        g.close()
    assert np.array_equal(out[0], out[1])


def test_ragged_rejects_unsupported_methods():
    import hipft_b200 as H
    from hipft_b200 import gpu
    t, p, br = _grid()
    with H.HipftGPU(t, p, 2, advance_diffusion=True, diffusion_num_method=1, diffusion_coef_constants=100.0) as g:
        with pytest.raises(gpu.HipftError) as e:
            g.set_ragged(True)
        assert e.value.code == gpu.HIPFT_EINVAL


_CHILD = r"""
import sys, numpy as np
sys.path.insert(0, %(root)r); sys.path.insert(0, %(tests)r)
import test_gpu_ragged as T
t, p, br = T._grid(%(ntm)d, %(npm1)d)
g = T._handle(t, p, %(nr)d)
g.load_initial_map(br[None]); g.update_flow(); g.set_ragged(True)
dt = g.flow_dtmax()
seq, tend = T._dt_sequence(dt, %(nsteps)d)
for d in seq:
    g.flux_transport_step(d)
sched = g.ragged_schedule()
np.savez(%(out)r, f=g.get_field(), s=sched["sts_s"], c=sched["subcycles"], dt=dt, tend=tend, desc=g.describe())
g.close()
"""


@pytest.mark.parametrize("kind", ["7", "5"])
def test_ragged_four_stage_path(tmp_path, kind):
    """A grid with interior theta blocks (ntm = 300), so that ragged
    super-steps take four-stage passes for the realizations with two stage
    pairs left and two-stage launches for the rest (HIPFT_STS_PAIR=7), and
    the same with two-stage launches only (=5): every realization against the
    oracle run of that realization alone."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = str(tmp_path / "r.npz")
    nr, nsteps, ntm, npm1 = 4, 2, 300, 65
    code = _CHILD % dict(root=root, tests=os.path.join(root, "tests"), ntm=ntm, npm1=npm1, nr=nr, nsteps=nsteps,
                         out=out)
    env = {k: v for k, v in os.environ.items() if k not in ("HIPFT_STS_PAIR", "HIPFT_TUNE")}
    env["HIPFT_STS_PAIR"] = kind
    res = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    z = np.load(out)
    if kind == "7":
        assert "ws-quad" in str(z["desc"]), str(z["desc"])
    t, p, br = _grid(ntm, npm1)
    assert len(set(z["s"].tolist())) > 1
    for i in range(nr):
        r = _oracle_alone(i, t, p, br, float(z["dt"]), float(z["tend"]))
        err = np.abs(z["f"][i] - r["f"][0]).max() / np.abs(r["f"][0]).max()
        assert err <= FIELD_TOL, f"realization {i}: field rel max-norm {err:.3e}"
        assert int(r["num"][-1, 0, 6]) == z["s"][i]


def test_driver_ragged_namelist(tmp_path):
    """The standalone driver with ragged_realizations = .true.: each
    realization's final field and its history rows, including its own Euler
    limit, stage count and subcycle columns, against the oracle run of that
    realization alone (dt_max below every realization's CFL limit, so the
    step sequence is the same)."""
    import cases
    import hipft_b200 as H
    import test_gpu_features as F
    Ds, p1s, p2s = [80.0, 300.0, 900.0], [20.0, 30.0, 12.0], [-262.0, -300.0, -200.0]
    base = dict(F.BASE, advance_flow=True, flow_dr_model=1, flow_mf_model=1, advance_diffusion=True,
                strang_splitting=True, validation_run=1, time_end=24.0, dt_max=6.0)
    d = dict(base, n_realizations=3, diffusion_coef_constants=Ds, flow_mf_coef_p1_values=p1s,
             flow_dr_coef_p2_values=p2s, ragged_realizations=True)
    text = F._namelist(d)
    (tmp_path / "hipft.in").write_text(text)
    prm = O.process_parameters(O.parse_namelist(text))
    shape = (3, prm["res_np"] + 1, prm["res_nt"])
    f = H.run_field(str(tmp_path / "hipft.in"), str(tmp_path), shape)
    sol, num = cases.read_run_histories(str(tmp_path), 3)
    assert len(set(num[:, -1, 6].tolist())) > 1, "the realizations should run different stage counts"
    for i in range(3):
        di = dict(base, n_realizations=1, diffusion_coef_constants=[Ds[i]], flow_mf_coef_p1_values=[p1s[i]],
                  flow_dr_coef_p2_values=[p2s[i]])
        r = O.run(O.process_parameters(O.parse_namelist(F._namelist(di))))
        err = np.abs(f[i] - r["f"][0]).max() / np.abs(r["f"][0]).max()
        assert err <= FIELD_TOL, f"realization {i}: field rel max-norm {err:.3e}"
        e = cases.col_errors(sol[i], r["sol"][:, 0, :])
        bad = {cases.COLS[c - 2]: float(e[c]) for c in range(2, 16)
               if e[c] > (1e-10 if c < 15 else max(1e-10, cases.VALERR_TOL))}
        assert not bad, f"realization {i}: {bad}"
        o = r["num"][:, 0, :]
        rel = np.abs(num[i][:, :6] - o[:, :6]) / np.maximum(np.abs(o[:, :6]), 1e-300)
        assert rel.max() <= 1e-10, f"realization {i} num columns: {rel.max(0)}"
        assert np.array_equal(num[i][:, 6:], o[:, 6:]), f"realization {i}: stage/cycle counts differ"
