"""Map output of the standalone driver against the oracle (write_map,
output_map and the validation maps, src/hipft.f90:2700-2917, 1891-2102).

The driver writes <root>_initial.h5, numbered maps in output_map_directory
at the output cadence with their list file, <root>_final.h5 and, for
validation runs, the analytic maps.  Each map must hold the oracle's field at
the same moment (flux-balanced on a copy when output_map_flux_balance) in the
reference's PT layout with one-point phi overlap: to FIELD_TOL for float64
files and to one float32 rounding step for float32 files; the scales must be
the run's phi and theta meshes (and 1..nr for 3-D files).
"""
import os

import numpy as np
import pytest

import test_gpu_features as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-12
F32_TOL = 2.0 ** -23  # one rounding step of a float32, relative to the map's scale


def _pt(f_tp):
    """(nr, npm, ntm) field -> (nr, ntm, npm1) PT map."""
    return np.ascontiguousarray(np.transpose(f_tp[:, :-1, :], (0, 2, 1)))


def _check(path, ref_pt, single, two_d, t, p):
    import hipft_b200 as H
    data, sc = H.h5_read(path)
    if two_d:
        assert data.shape == ref_pt.shape[1:], path
        ref = ref_pt[0]
        assert len(sc) == 2
    else:
        assert data.shape == ref_pt.shape, path
        ref = ref_pt
        assert np.array_equal(sc[2], np.arange(1, ref_pt.shape[0] + 1, dtype=float))
    scale = np.abs(ref).max()
    if single:
        err = np.abs(data - ref.astype(np.float32).astype(np.float64)).max() / scale
        assert err <= F32_TOL, f"{path}: {err:.3e}"
        assert np.array_equal(sc[0], p.astype(np.float32).astype(np.float64))
        assert np.array_equal(sc[1], t.astype(np.float32).astype(np.float64))
    else:
        err = np.abs(data - ref).max() / scale
        assert err <= FIELD_TOL, f"{path}: {err:.3e}"
        assert np.array_equal(sc[0], p) and np.array_equal(sc[1], t)


def _run(d, tmp_path):
    import hipft_b200 as H
    text = F._namelist(d)
    (tmp_path / "hipft.in").write_text(text)
    prm = O.process_parameters(O.parse_namelist(text))
    r = O.run(prm, map_cap=64)
    H.run_field(str(tmp_path / "hipft.in"), str(tmp_path), r["f"].shape)
    return prm, r


CASES = {
    # 3-D float64 maps of two realizations, flux-balanced, time cadence
    "cadence_f64_balanced": dict(F.BASE, advance_flow=True, flow_dr_model=1, advance_diffusion=True,
                                 diffusion_coef_constants=[300.0, 300.0], validation_run=1,
                                 output_map_time_cadence=1.5, output_map_flux_balance=True,
                                 output_single_precision=False),
    # 2-D float32 maps of one realization, index cadence, own directory and root name
    "idx_f32_2d": dict(F.BASE, n_realizations=1, res_nt=33, res_np=70, advance_diffusion=True,
                       diffusion_coef_constants=[400.0], validation_run=1, output_map_idx_cadence=2,
                       output_map_directory="maps/out", output_map_root_filename="br"),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_driver_maps_match_oracle(name, tmp_path):
    d = CASES[name]
    prm, r = _run(d, tmp_path)
    nr = prm["n_realizations"]
    single = bool(prm["output_single_precision"])
    two_d = bool(prm["output_map_2d"]) and nr == 1
    root = prm["output_map_root_filename"]
    mdir = prm["output_map_directory"]
    ntm, npm1 = r["f"].shape[2], r["f"].shape[1] - 1
    t = np.linspace(0.0, np.pi, ntm)
    p = np.linspace(0.0, 2.0 * np.pi, npm1)
    _check(str(tmp_path / f"{root}_initial.h5"), _pt(r["map_initial"]), single, two_d, t, p)
    _check(str(tmp_path / f"{root}_final.h5"), _pt(r["map_final"]), single, two_d, t, p)
    # numbered maps and their list
    lines = (tmp_path / "hipft_output_map_list.out").read_text().splitlines()
    assert lines[0].split() == ["IDX", "TIME", "FILENAME"]
    rows = [ln.split() for ln in lines[1:]]
    assert len(rows) == len(r["map_idx"]) > 1
    for row, idx, tm, m in zip(rows, r["map_idx"], r["map_time"], r["maps"]):
        assert int(row[0]) == idx
        assert abs(float(row[1]) - tm) <= 1e-12 * max(1.0, abs(tm))
        assert row[2] == f"{root}_idx{idx:06d}.h5"
        _check(str(tmp_path / mdir / row[2]), _pt(m), single, two_d, t, p)


def test_validation_maps(tmp_path):
    """_initial_0.h5 and _final_analytic.h5 of validation runs 1 and 2."""
    import hipft_b200 as H
    d = dict(F.BASE, n_realizations=2, advance_diffusion=True, diffusion_coef_constants=[250.0, 500.0],
             validation_run=1, output_single_precision=False)
    prm, r = _run(d, tmp_path)
    u0 = _pt(r["map_initial"])  # the validation map itself (mult_fac 1, no balance)
    ntm, npm1 = u0.shape[1], u0.shape[2]
    t = np.linspace(0.0, np.pi, ntm)
    p = np.linspace(0.0, 2.0 * np.pi, npm1)
    data, sc = H.h5_read(str(tmp_path / "hipft_brmap_initial_0.h5"))
    # the analytic map is made on the host; the field went through the GPU's pole averaging
    assert np.abs(data - u0)[:, 1:-1, :].max() <= FIELD_TOL * np.abs(u0).max()
    fa, _ = H.h5_read(str(tmp_path / "hipft_brmap_final_analytic.h5"))
    dk = np.asarray(prm["diffusion_coef_constants"])[:, None, None]
    expect = data * np.exp(-42.0 * dk * prm["diffusion_coef_factor"] * prm["time_end"])
    assert np.abs(fa - expect).max() <= 1e-14 * np.abs(expect).max()

    tmp2 = tmp_path / "v2"
    tmp2.mkdir()
    d2 = dict(F.BASE, n_realizations=1, advance_flow=True, flow_vt_const=1.0, validation_run=2, dt_max=0.5,
              output_single_precision=False)
    prm2, r2 = _run(d2, tmp2)
    fa2, sc2 = H.h5_read(str(tmp2 / "hipft_brmap_final_analytic.h5"))
    s1, s2 = sc2
    w = prm2["validation_run_width"]
    st_i = np.zeros_like(s2)
    st_i[1:-1] = 1.0 / np.sin(s2[1:-1])
    e = (s2 - 3.0 * np.pi / 4.0)[:, None] ** 2 / w
    g = (-st_i[:, None] * np.exp(-e - (s1 - np.pi / 2)[None, :] ** 2 / w)
         + st_i[:, None] * np.exp(-e - (s1 - 3.0 * np.pi / 2)[None, :] ** 2 / w))
    assert fa2.shape == g.shape
    assert np.abs(fa2 - g).max() <= 1e-12 * np.abs(g).max()
