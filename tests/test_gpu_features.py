"""GPU parity on feature combinations the testsuite does not cover.

Small synthetic namelists drive the standalone GPU driver (hipft_run_field)
and the CPU oracle on identical inputs; the final fields must agree to
FIELD_TOL in relative max-norm and every history row to HIST_TOL (column
max-norm).  Grid sizes are chosen to hit the kernels' edge paths: theta
counts with row ntm-1 on a warp's last lane (ntm = 33, 161), phi counts
that leave partial phi blocks, and tiny grids.

The rotated rigid rotation (flow_rigid_omega, src/hipft.f90:3450-3486) is
built exactly as the reference writes it, but its square roots go negative
on most of the sphere, so its fields are NaN in both implementations and it
has no field-parity case here.
"""
import numpy as np
import pytest

import cases
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-12
HIST_TOL = 1e-10

BASE = dict(res_nt=45, res_np=91, n_realizations=2, time_end=6.0, dt_max=1.0, verbose=0)

CASES = {
    # diffusion methods and subcycling
    "rkg2_auto_ntm33": dict(res_nt=33, res_np=70, advance_diffusion=True, diffusion_coef_constants=[400.0, 90.0],
                            validation_run=1),
    "rkg2_auto_ntm161": dict(res_nt=161, res_np=101, n_realizations=3, advance_diffusion=True,
                             diffusion_coef_constants=[300.0, 600.0, 50.0], validation_run=1),
    # theta rows 128 | 129 and 129 | 130 straddle a 128-row tile boundary at the south pole
    "rkg2_ntm129_np65": dict(res_nt=129, res_np=65, advance_diffusion=True, diffusion_coef_constants=[500.0, 120.0],
                             validation_run=1),
    "rkg2_ntm130_np96": dict(res_nt=130, res_np=96, advance_diffusion=True, diffusion_coef_constants=[80.0, 700.0],
                             validation_run=1),
    # three full 128-row blocks (north pole, interior, south pole) and full
    # phi tiles at both seams: every tile of the two-stage kernel takes its
    # widest path
    "rkg2_ntm384_np45": dict(res_nt=384, res_np=45, advance_diffusion=True, diffusion_coef_constants=[150.0, 900.0],
                             validation_run=1),
    # five interior 128-row blocks between the pole blocks: the four-stage
    # path (interior blocks) meets the two-stage path (pole blocks) at both
    # block edges
    "rkg2_ntm900_np70": dict(res_nt=900, res_np=70, advance_diffusion=True, diffusion_coef_constants=[200.0, 800.0],
                             validation_run=1, time_end=3.0),
    "rkl2_fixed_sc": dict(advance_diffusion=True, diffusion_num_method=2, diffusion_subcycles=3,
                          diffusion_coef_constants=[250.0, 500.0], validation_run=1),
    "euler_fixed_sc": dict(res_nt=20, res_np=37, advance_diffusion=True, diffusion_num_method=1,
                           diffusion_subcycles=2, diffusion_coef_constants=[20.0, 40.0], time_end=2.0,
                           validation_run=1),
    "rkg2_grid_coef": dict(advance_diffusion=True, diffusion_coef_grid=True, diffusion_coef_constants=[100.0, 0.0],
                           validation_run=1),
    # advection methods
    "fe_upwind": dict(advance_flow=True, flow_num_method=1, flow_dr_model=1, flow_mf_model=1, validation_run=2,
                      flow_vp_rigid_omega=1.0, dt_max=0.5),
    "ssprk33_upwind_half": dict(advance_flow=True, flow_num_method=2, upwind=0.5, flow_dr_model=1, validation_run=2,
                                flow_vt_const=1.0),
    "ssprk33_weno_eps": dict(advance_flow=True, flow_num_method=3, weno_eps=0.01, flow_dr_model=1, flow_mf_model=1,
                             validation_run=2, flow_vp_rigid_omega=1.0, flow_vt_const=1.0),
    # flow + diffusion, Strang and Lie, attenuation, per-realization coefficients
    "strang_dr_mf_diff": dict(advance_flow=True, flow_dr_model=1, flow_mf_model=1, advance_diffusion=True,
                              strang_splitting=True, diffusion_coef_constants=[150.0, 450.0],
                              flow_dr_coef_p2_values=[-250.0, -300.0], flow_mf_coef_p1_values=[20.0, 30.0],
                              validation_run=1),
    "attenuated_lie": dict(advance_flow=True, flow_dr_model=1, flow_mf_model=1, flow_attenuate=True,
                           flow_attenuate_values=[0.6, 2.0], advance_diffusion=True,
                           diffusion_coef_constants=[100.0, 200.0], validation_run=1),
    "cadence_balance": dict(advance_flow=True, flow_dr_model=1, advance_diffusion=True,
                            diffusion_coef_constants=[300.0, 300.0], validation_run=1,
                            initial_map_flux_balance=True, initial_map_mult_fac=2.5,
                            output_history_time_cadence=1.5, output_map_time_cadence=2.5, verbose=2),
}


def _namelist(d: dict) -> str:
    def fmt(v):
        if isinstance(v, str):
            return "'" + v + "'"
        if isinstance(v, bool):
            return ".true." if v else ".false."
        if isinstance(v, (list, tuple)):
            return ", ".join(str(float(x)) for x in v)
        return str(v)
    body = "\n".join(f"  {k} = {fmt(v)}" for k, v in d.items())
    return "&hipft_input_parameters\n" + body + "\n/\n"


@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_feature_parity(name, tmp_path):
    import hipft_b200 as H
    d = dict(BASE)
    d.update(CASES[name])
    text = _namelist(d)
    (tmp_path / "hipft.in").write_text(text)
    p = O.process_parameters(O.parse_namelist(text))
    r = O.run(p)
    f = H.run_field(str(tmp_path / "hipft.in"), str(tmp_path), r["f"].shape)
    ferr = np.abs(f - r["f"]).max() / np.abs(r["f"]).max()
    assert ferr <= FIELD_TOL, f"{name}: field rel max-norm {ferr:.3e}"
    sol, num = cases.read_run_histories(str(tmp_path), p["n_realizations"])
    assert sol.shape[1] == r["sol"].shape[0], "history row count differs"
    for i in range(p["n_realizations"]):
        err = cases.col_errors(sol[i], r["sol"][:, i, :])
        tol = [HIST_TOL] * 15 + [max(HIST_TOL, cases.VALERR_TOL)]
        bad = {cases.COLS[c - 2]: float(err[c]) for c in range(2, 16) if err[c] > tol[c]}
        assert not bad, f"{name} r{i + 1}: {bad}"
        o = r["num"][:, i, :]
        rel = np.abs(num[i][:, :6] - o[:, :6]) / np.maximum(np.abs(o[:, :6]), 1e-300)
        assert rel.max() <= HIST_TOL, f"num columns: {rel.max(0)}"
        assert np.array_equal(num[i][:, 6:], o[:, 6:])
