"""Data assimilation from files, end to end through the standalone driver.

The reference's input path (load_data_assimilation src/hipft.f90:3949-4081,
assimilate_new_data 4083-4146, apply_data_assimilation 4148-4306): a map list
read with the fixed format (A19,1X,A19,1X,F13.5,1X,A), map times in hours
from the first map's Julian day, and 3-slice [data, weight, mu] HDF5 maps
(float32, as observed maps come) under assimilate_data_map_root_dir.  Here
the maps are written with the library's own HDF5 writer; the oracle gets the
same (float32-rounded) slices and times, and the final fields and every
history row must agree as in the feature-parity tests.
"""
import numpy as np
import pytest

import cases
import test_gpu_features as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("sep", [" ", ","])
def test_da_from_files_matches_oracle(tmp_path, sep):
    import hipft_b200 as H
    d = dict(F.BASE, advance_flow=True, flow_dr_model=1, flow_mf_model=1, advance_diffusion=True,
             diffusion_coef_constants=[300.0, 150.0], validation_run=1, strang_splitting=True,
             assimilate_data=True, assimilate_data_map_list_filename="da/map_list.csv",
             assimilate_data_map_root_dir="da", assimilate_data_custom_from_mu=True,
             assimilate_data_mu_powers=[4.0, 2.0], assimilate_data_mu_limits=[0.1, 0.2],
             assimilate_data_lat_limits=[0.0, 60.0], assimilate_data_balance_flux=True,
             assimilate_data_mult_fac=1.2)
    ntm, npm1 = d["res_nt"], d["res_np"]
    t = np.linspace(0.0, np.pi, ntm)
    p = np.linspace(0.0, 2.0 * np.pi, npm1)
    rng = np.random.default_rng(21)
    (tmp_path / "da").mkdir()
    jd0 = 2459580.5
    jds = jd0 + 0.0625 * np.arange(4)  # every 1.5 h
    maps = []
    rows = ["target_datetime_utc,obs_datetime_utc,obs_jd,path"]
    for q, jd in enumerate(jds):
        data = rng.normal(size=(ntm, npm1)) * 3.0 + 1.0
        weight = rng.uniform(0.0, 1.0, size=(ntm, npm1))
        mu = np.sin(t)[:, None] * np.cos(p[None, :] - 0.3 * q)
        slab = np.stack([data, weight, mu])  # Fortran (npm1, ntm, 3)
        name = f"obs_{q:03d}.h5"
        H.h5_write(str(tmp_path / "da" / name), slab, [p, t, np.arange(1.0, 4.0)], single_precision=True)
        maps.append(slab.astype(np.float32).astype(np.float64))
        date = f"2022-01-01T{int(1.5 * q):02d}:{int(90 * q) % 60:02d}:00"
        rows.append(date + sep + date + sep + f"{jd:13.5f}" + sep + name)
    (tmp_path / "da" / "map_list.csv").write_text("\n".join(rows) + "\n")
    text = F._namelist(d)
    (tmp_path / "hipft.in").write_text(text)
    prm = O.process_parameters(O.parse_namelist(text))
    times = 24.0 * jds - 24.0 * jds[0]
    r = O.run(prm, da_times=times, da_maps=np.stack(maps))
    f = H.run_field(str(tmp_path / "hipft.in"), str(tmp_path), r["f"].shape)
    ferr = np.abs(f - r["f"]).max() / np.abs(r["f"]).max()
    assert ferr <= F.FIELD_TOL, f"field rel max-norm {ferr:.3e}"
    sol, num = cases.read_run_histories(str(tmp_path), prm["n_realizations"])
    assert sol.shape[1] == r["sol"].shape[0]
    for i in range(prm["n_realizations"]):
        err = cases.col_errors(sol[i], r["sol"][:, i, :])
        tol = [F.HIST_TOL] * 15 + [max(F.HIST_TOL, cases.VALERR_TOL)]
        bad = {cases.COLS[c - 2]: float(err[c]) for c in range(2, 16) if err[c] > tol[c]}
        assert not bad, f"r{i + 1}: {bad}"
    # the assimilation cut the steps at the map times
    assert set(np.round(times, 9)).issubset(set(np.round(r["sol"][:, 0, 1], 9)))
