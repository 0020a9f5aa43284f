"""The phi-marching WENO3 advection stage (k_adv_weno_march) against the
tile kernel (k_advection_stage) and the oracle.  HIPFT_ADV_KERNEL=march and
=tile force either kernel (the library otherwise picks by grid size: the
tile kernel on grids too small to fill the GPU with the marching kernel's
32-column chunks).

Both kernels evaluate every face, divergence and combine with the same
expressions, so their final fields must be bitwise equal; each must also
match the oracle to FIELD_TOL.  Grid sizes put theta row counts on and
around the marching kernel's 31-row groups (lane 0 of a group is the row
below it, lanes 31, 0 and 1 load the halo rows j0-2, j0+31, j0+32) and phi
counts on and around its column chunks (8 columns on the small grids, 32 and
64 on the two 256 x 512 batches); the cases cover 1-D (analytic)
and 2-D (attenuated) flows, SSPRK(3,3) and SSPRK(4,3), Strang and Lie
splitting and a set weno_eps.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import test_gpu_features as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-12
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

ADV = dict(advance_flow=True, flow_dr_model=1, flow_mf_model=1, validation_run=1)
CASES = {
    "g31_np66": dict(ADV, res_nt=31, res_np=66, n_realizations=2, time_end=4.0),
    "g32_np67": dict(ADV, res_nt=32, res_np=67, n_realizations=1, time_end=4.0),
    "g62_np9": dict(ADV, res_nt=62, res_np=9, n_realizations=2, time_end=8.0),
    "g63_np66": dict(ADV, res_nt=63, res_np=66, n_realizations=1, time_end=8.0),
    "g64_np131": dict(ADV, res_nt=64, res_np=131, n_realizations=3, time_end=3.0,
                      flow_dr_coef_p2_values=[-250.0, -300.0, -200.0],
                      flow_mf_coef_p1_values=[20.0, 30.0, 12.0]),
    "g97_np130_strang": dict(ADV, res_nt=97, res_np=130, n_realizations=2, time_end=3.0, advance_diffusion=True,
                             strang_splitting=True, diffusion_coef_constants=[150.0, 450.0]),
    "g45_attenuated": dict(ADV, res_nt=45, res_np=91, n_realizations=2, time_end=4.0, flow_attenuate=True,
                           flow_attenuate_values=[0.6, 2.0], advance_diffusion=True,
                           diffusion_coef_constants=[100.0, 200.0]),
    "g94_np70_attenuated": dict(ADV, res_nt=94, res_np=70, n_realizations=1, time_end=3.0, flow_attenuate=True,
                                flow_attenuate_values=[1.0]),
    # enough warps for 64- and 32-column chunks
    "g256_np512_nr64": dict(ADV, res_nt=256, res_np=512, n_realizations=64, time_end=2.0),
    "g256_np512_nr32": dict(ADV, res_nt=256, res_np=512, n_realizations=32, time_end=2.0,
                            flow_attenuate=True, flow_attenuate_values=[1.0] * 32),
    "ssprk33_weno_eps": dict(ADV, res_nt=45, res_np=91, n_realizations=2, time_end=4.0, flow_num_method=3,
                             weno_eps=0.01, flow_vp_rigid_omega=1.0, flow_vt_const=1.0, validation_run=2),
}


def _run(name, tmp_path, env_extra):
    d = dict(F.BASE)
    d.update(CASES[name])
    text = F._namelist(d)
    (tmp_path / "hipft.in").write_text(text)
    r = O.run(O.process_parameters(O.parse_namelist(text)))
    out = tmp_path / ("f_%s.npy" % "_".join(env_extra.values()))
    code = ("import sys, numpy as np; sys.path.insert(0, %r); import hipft_b200 as H; "
            "np.save(%r, H.run_field(%r, %r, %r))" % (ROOT, str(out), str(tmp_path / "hipft.in"), str(tmp_path),
                                                      tuple(r["f"].shape)))
    env = {k: v for k, v in os.environ.items() if k != "HIPFT_ADV_KERNEL"}
    env.update(env_extra)
    res = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    return r["f"], np.load(out)


@pytest.mark.parametrize("name", sorted(CASES))
def test_marching_advection_matches_tile_kernel_and_oracle(name, tmp_path):
    ref, f_march = _run(name, tmp_path, {"HIPFT_ADV_KERNEL": "march"})
    _, f_tile = _run(name, tmp_path, {"HIPFT_ADV_KERNEL": "tile"})
    assert np.isfinite(f_march).all()
    assert np.array_equal(f_march.view(np.uint64), f_tile.view(np.uint64)), (
        f"{name}: marching and tile kernels differ (max |diff| {np.abs(f_march - f_tile).max():.3e})")
    err = np.abs(f_march - ref).max() / np.abs(ref).max()
    assert err <= FIELD_TOL, f"{name}: field rel max-norm vs oracle {err:.3e}"
