"""A small advection + diffusion run (two realizations, analytic flows,
RKG2 with fixed subcycles, Strang splitting) shared by the adjoint tests."""
import numpy as np

import test_gpu_features as F
from oracle import oracle as O

CASE = dict(res_nt=24, res_np=41, n_realizations=2, time_end=120.0, dt_max=40.0, advance_flow=True,
            flow_dr_model=1, flow_mf_model=1, flow_dr_coef_p0_values=[10.0, -5.0],
            flow_dr_coef_p2_values=[-337.43, -300.0], flow_dr_coef_p4_values=[-253.07, -240.0],
            flow_mf_coef_p1_values=[300.0, 240.0], flow_mf_coef_p3_values=[-300.0, -240.0],
            flow_mf_coef_p5_values=[0.0, 30.0], advance_diffusion=True, diffusion_coef_constants=[3000.0, 8000.0],
            diffusion_subcycles=2, strang_splitting=True, validation_run=1)
FLOW = {"p0": "flow_dr_coef_p0_values", "p2": "flow_dr_coef_p2_values", "p4": "flow_dr_coef_p4_values",
        "p1": "flow_mf_coef_p1_values", "p3": "flow_mf_coef_p3_values", "p5": "flow_mf_coef_p5_values"}


def oracle_run(case=CASE):
    """Oracle run of the case: parameters, results (with the initial field
    in map_initial) and the step dts it took."""
    p = O.process_parameters(O.parse_namelist(F._namelist(case)))
    r = O.run(p, map_cap=1)
    dts = r["num"][1:, 0, 2]
    return p, r, dts


def rough_run(case=CASE, seed=7):
    """Oracle run of the case from a noisy map (10 cos(theta) G plus unit
    Gaussian noise) with automatic PTL subcycling, which then takes several
    subcycles per step: parameters, results and step dts."""
    c = {k: v for k, v in case.items() if k not in ("res_nt", "res_np")}
    c.update(diffusion_subcycles=0, validation_run=0)
    p = O.process_parameters(O.parse_namelist(F._namelist(c)))
    t, ph = mesh_tp(case)
    rng = np.random.default_rng(seed)
    nr = case["n_realizations"]
    m = 10.0 * np.cos(t)[None, :, None] * np.ones((nr, len(t), len(ph))) + rng.standard_normal((nr, len(t), len(ph)))
    r = O.run(p, map_pt=m, s1=ph, s2=t, map_cap=1)
    return p, r, r["num"][1:, 0, 2]


def mesh_tp(case=CASE):
    nt, np_ = case["res_nt"], case["res_np"]
    return np.linspace(0.0, np.pi, nt), np.linspace(0.0, 2.0 * np.pi, np_)


def target_field(f0):
    """A smooth target: the initial field scaled and shifted by one phi column."""
    g = 0.7 * np.roll(f0, 1, axis=1)
    g[:, 0] = g[:, -2]
    g[:, -1] = g[:, 1]
    return g
