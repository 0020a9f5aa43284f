"""Parity of every two-stage RKG2 kernel the autotuner may pick, and of one
stage per launch, against the oracle.

The library fixes its RKG2 kernel from the environment when asked
(HIPFT_STS_PAIR=4: persistent warp-specialised CTAs with one theta row per
consumer thread; =5: two rows per thread; =6: the same with the outputs
leaving by bulk stores; =7: four stages per pass on the interior theta
blocks; =0: one stage per launch), so each variant runs the standalone
driver in a fresh subprocess; final fields must match the oracle to
FIELD_TOL.  The "tuned"
variant lets the autotuner choose."""
import os
import subprocess
import sys

import numpy as np
import pytest

import cases
import test_gpu_features as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-12
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
VARIANTS = {"pair_ws": {"HIPFT_STS_PAIR": "4"}, "pair_ws_rowpairs": {"HIPFT_STS_PAIR": "5"},
            "pair_ws_bulkst": {"HIPFT_STS_PAIR": "6"}, "quad_ws": {"HIPFT_STS_PAIR": "7"},
            "single_v3": {"HIPFT_STS_PAIR": "0"}, "tuned": {}}
RUNS = ["diffuse_soccer", "rkg2_auto_ntm33", "rkg2_auto_ntm161", "rkg2_ntm129_np65", "rkg2_ntm130_np96",
        "rkg2_ntm384_np45", "rkg2_ntm900_np70", "strang_dr_mf_diff"]


def _setup(name, tmp_path):
    if name in cases.CASES:
        src = cases.input_dir(name)
        text = open(os.path.join(src, "hipft.in")).read()
        r = cases.oracle_case(name)
    else:
        d = dict(F.BASE)
        d.update(F.CASES[name])
        text = F._namelist(d)
        r = O.run(O.process_parameters(O.parse_namelist(text)))
    (tmp_path / "hipft.in").write_text(text)
    return r


@pytest.mark.parametrize("variant", sorted(VARIANTS))
@pytest.mark.parametrize("name", RUNS)
def test_stage_kernel_variant_parity(variant, name, tmp_path):
    r = _setup(name, tmp_path)
    out = tmp_path / "f.npy"
    code = ("import sys, numpy as np; sys.path.insert(0, %r); import hipft_b200 as H; "
            "np.save(%r, H.run_field(%r, %r, %r))" % (ROOT, str(out), str(tmp_path / "hipft.in"), str(tmp_path),
                                                      tuple(r["f"].shape)))
    env = {k: v for k, v in os.environ.items() if k not in ("HIPFT_STS_PAIR", "HIPFT_TUNE")}
    env.update(VARIANTS[variant])
    res = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    f = np.load(out)
    err = np.abs(f - r["f"]).max() / np.abs(r["f"]).max()
    assert err <= FIELD_TOL, f"{variant}/{name}: field rel max-norm {err:.3e}"
