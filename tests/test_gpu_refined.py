"""GPU parity on nonuniform theta grids and on the benchmark configurations.

HipFT builds only uniform meshes itself; a nonuniform theta mesh enters
through the dim2 scale of the initial map file (set_mesh, src/hipft.f90:
6495-6653, reads the file's scales).  On such a mesh the half-mesh spacings
dt(j) = th(j+1) - th(j) and dth(j) = t(j) - t(j-1) differ, so a slip between
them in any coefficient table (diffusion coefficients src/hipft.f90:4927-4983,
WENO weights 6893-6932, CFL 7287-7350) shows up here and not on the uniform
testsuite grids.

* every feature combination of test_gpu_features on a refined theta scale
  (spacing halved within 15 degrees of each pole), initial map from a file;
* the plain dipole diffusion configuration in full (256 x 512 uniform,
  D = 500 km^2/s, 27.27 days, daily histories);
* the single-realization advection + diffusion configuration (1024 x 2048
  refined, 200 bipoles from seed 0) for its first 24 model hours;
* the 64-realization configuration (seed 1) for two steps across one
  assimilation.  The GPU runs all 64 realizations; the oracle runs the
  realizations that set the shared schedule (largest D: Euler limit, RKG2
  stage count and PTL cells; smallest CFL limit: dt) plus a few others, and
  the test first checks that the schedules (dt, stage counts, subcycles)
  agree exactly, which shows that the subset reproduces the full run's
  schedule, then compares those realizations' fields and histories.

Bars as elsewhere: final fields 1e-12 relative max-norm, history columns
1e-10, stage and cycle counts exact.
"""
import zlib

import numpy as np
import pytest

import cases
import test_gpu_features as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-12
HIST_TOL = 1e-10


def smooth_map(t, p, seed):
    """A smooth, periodic, pole-regular random field (ntm, npm1), Gauss."""
    rng = np.random.default_rng(seed)
    st, ct = np.sin(t)[:, None], np.cos(t)[:, None]
    f = 3.0 * ct + 0.0 * p[None, :]
    for _ in range(10):
        m = int(rng.integers(0, 5))
        n = int(rng.integers(0, 4))
        f = f + rng.normal() * st ** m * ct ** n * np.cos(m * p[None, :] + rng.uniform(0, 2 * np.pi))
    f[:, -1] = f[:, 0]
    return f


def write_map(path, t, p, br):
    import hipft_b200 as H
    H.h5_write(str(path), br, [p, t], single_precision=False)


def compare(tag, f, r, sol, num, realizations=None, oracle_index=None):
    """Field and history comparison of GPU realizations `realizations` with
    oracle realizations `oracle_index` (same order; default all)."""
    nr = r["f"].shape[0]
    gi = list(range(nr)) if realizations is None else list(realizations)
    oi = list(range(nr)) if oracle_index is None else list(oracle_index)
    ff = f[gi]
    ferr = np.abs(ff - r["f"][oi]).max() / np.abs(r["f"][oi]).max()
    assert ferr <= FIELD_TOL, f"{tag}: field rel max-norm {ferr:.3e}"
    assert sol.shape[1] == r["sol"].shape[0], f"{tag}: history row count differs"
    for g, o in zip(gi, oi):
        err = cases.col_errors(sol[g], r["sol"][:, o, :])
        tol = [HIST_TOL] * 15 + [max(HIST_TOL, cases.VALERR_TOL)]
        bad = {cases.COLS[c - 2]: float(err[c]) for c in range(2, 16) if err[c] > tol[c]}
        assert not bad, f"{tag} r{g + 1}: {bad}"
        on = r["num"][:, o, :]
        rel = np.abs(num[g][:, :6] - on[:, :6]) / np.maximum(np.abs(on[:, :6]), 1e-300)
        assert rel.max() <= HIST_TOL, f"{tag} r{g + 1} num columns: {rel.max(0)}"
        assert np.array_equal(num[g][:, 6:], on[:, 6:]), f"{tag} r{g + 1}: stage/cycle counts differ"
    return ferr


# ---------------------------------------------------------------- features
REFINED = {name: dict(c) for name, c in F.CASES.items()}


@pytest.mark.parametrize("name", sorted(REFINED))
def test_refined_theta_feature_parity(name, tmp_path):
    import hipft_b200 as H
    from hipft_b200 import synthetic as S
    d = dict(F.BASE)
    d.update(REFINED[name])
    ntm, npm1 = int(d.pop("res_nt")), int(d.pop("res_np"))
    d.pop("validation_run", None)
    t = S.refined_theta(ntm)
    p = S.uniform_phi(npm1)
    assert np.ptp(np.diff(t)) > 0.3 * np.diff(t).max(), "theta scale must be visibly nonuniform"
    br = smooth_map(t, p, zlib.crc32(name.encode()) % 1000)
    write_map(tmp_path / "map.h5", t, p, br)
    d["initial_map_filename"] = "map.h5"
    text = F._namelist(d)
    (tmp_path / "hipft.in").write_text(text)
    prm = O.process_parameters(O.parse_namelist(text))
    nr = prm["n_realizations"]
    r = O.run(prm, map_pt=np.broadcast_to(br, (nr,) + br.shape), s1=p, s2=t)
    f = H.run_field(str(tmp_path / "hipft.in"), str(tmp_path), r["f"].shape)
    sol, num = cases.read_run_histories(str(tmp_path), nr)
    compare(name, f, r, sol, num)


# ------------------------------------------------- benchmark configurations
def test_config_dipole_diffusion_full(tmp_path):
    """256 x 512 uniform, Br = 10 cos(theta) G, D = 500 km^2/s, RKG2 with PTL
    subcycles, 27.27 days in daily steps (dt_max = 24 h), daily history."""
    import hipft_b200 as H
    ntm, npm1 = 256, 513
    t = np.linspace(0.0, np.pi, ntm)
    p = np.linspace(0.0, 2.0 * np.pi, npm1)
    br = 10.0 * np.cos(t)[:, None] * np.ones((1, npm1))
    write_map(tmp_path / "map.h5", t, p, br)
    d = dict(initial_map_filename="map.h5", n_realizations=1, advance_diffusion=True,
             diffusion_coef_constant=500.0, diffusion_num_method=3, time_end=654.48, dt_max=24.0,
             output_history_time_cadence=24.0, verbose=0)
    text = F._namelist(d)
    (tmp_path / "hipft.in").write_text(text)
    prm = O.process_parameters(O.parse_namelist(text))
    r = O.run(prm, map_pt=br[None], s1=p, s2=t)
    f = H.run_field(str(tmp_path / "hipft.in"), str(tmp_path), r["f"].shape)
    sol, num = cases.read_run_histories(str(tmp_path), 1)
    assert sol.shape[1] >= 28, "daily histories over 27.27 days"
    compare("dipole_256x512", f, r, sol, num)


def _bench_namelist(prm, idx, time_end, extra=None):
    """Namelist of the benchmark physics for realizations `idx` of the
    per-realization parameter set `prm` (hipft_b200.synthetic)."""
    vals = lambda key: [float(prm[key][i]) for i in idx]
    d = dict(initial_map_filename="map.h5", n_realizations=len(idx), advance_flow=True, flow_num_method=4,
             flow_dr_model=1, flow_mf_model=1, advance_diffusion=True, strang_splitting=True,
             diffusion_num_method=3, time_end=time_end, verbose=0,
             diffusion_coef_constants=vals("diffusion_coef_constants"),
             flow_dr_coef_p0_values=vals("dr_p0"), flow_dr_coef_p2_values=vals("dr_p2"),
             flow_dr_coef_p4_values=vals("dr_p4"), flow_mf_coef_p1_values=vals("mf_p1"),
             flow_mf_coef_p3_values=vals("mf_p3"), flow_mf_coef_p5_values=vals("mf_p5"))
    if extra:
        d.update(extra)
    return F._namelist(d)


@pytest.mark.slow
def test_config_single_1024x2048_refined_24h(tmp_path):
    """1024 x 2048 with theta refined x2 near the poles, 200 bipoles (seed 0),
    DR + MF + D = 300 km^2/s, WENO3 + SSPRK(4,3) Strang-split with RKG2:
    the first 24 model hours."""
    import hipft_b200 as H
    from hipft_b200 import synthetic as S
    t = S.refined_theta(1024)
    p = S.uniform_phi(2049)
    br = S.bipole_map(t, p, 0)
    write_map(tmp_path / "map.h5", t, p, br)
    text = _bench_namelist(S.plain_params(), [0], 24.0)
    (tmp_path / "hipft.in").write_text(text)
    prm = O.process_parameters(O.parse_namelist(text))
    r = O.run(prm, map_pt=br[None], s1=p, s2=t)
    assert r["nsteps"] >= 10
    f = H.run_field(str(tmp_path / "hipft.in"), str(tmp_path), r["f"].shape)
    sol, num = cases.read_run_histories(str(tmp_path), 1)
    compare("single_1024x2048", f, r, sol, num)


def _cfl_rank(prm, t):
    """Per-realization analytic-flow speed measure max_j |v| / spacing (larger
    = smaller CFL limit), used only to pick the oracle subset."""
    c = np.cos(t)
    s = np.sin(t)
    dth = np.gradient(t)
    out = []
    for i in range(len(prm["diffusion_coef_constants"])):
        vt = s * np.abs(prm["mf_p1"][i] * c + prm["mf_p3"][i] * c ** 3 + prm["mf_p5"][i] * c ** 5)
        vp = np.abs(prm["dr_p0"][i] + prm["dr_p2"][i] * c ** 2 + prm["dr_p4"][i] * c ** 4)
        out.append(np.max(vt[1:-1] / dth[1:-1] + vp[1:-1] / (2 * np.pi / 2048)))
    return np.array(out)


@pytest.mark.slow
def test_config_batched64_two_steps_across_assimilation(tmp_path):
    """64 realizations (seed 1) on 1024 x 2048 refined with synthetic observed
    maps (mu^4 weights, mu > 0.1) at 0 h and 1.5 h, to 2.5 h.  As in the
    reference (load_data_assimilation, src/hipft.f90:4010-4042), a map at the
    start time makes the first step zero-length, so the run takes three steps:
    0 h (assimilate map 0), 0 -> 1.5 h (assimilate map 1), 1.5 -> 2.5 h.  The
    map list holds Julian dates to five decimals; 1.5 h (1/16 day) is exact
    there, so the oracle's map times equal the driver's.  The oracle runs the
    schedule-setting realizations and two others."""
    import hipft_b200 as H
    from hipft_b200 import synthetic as S
    nr = 64
    t = S.refined_theta(1024)
    p = S.uniform_phi(2049)
    br = S.bipole_map(t, p, 1)
    prm = S.batched_params(nr, 1)
    write_map(tmp_path / "map.h5", t, p, br)
    (tmp_path / "da").mkdir()
    jd0 = 2459580.5
    jds = [jd0, jd0 + 0.0625]
    dates = ["2022-01-01T00:00:00", "2022-01-01T01:30:00"]
    maps = []
    rows = ["target_datetime_utc,obs_datetime_utc,obs_jd,path"]
    for q, jd in enumerate(jds):
        slab = S.observed_map(t, p, 24.0 * (jd - jd0), 1)
        name = f"obs_{q:03d}.h5"
        H.h5_write(str(tmp_path / "da" / name), slab, [p, t, np.arange(1.0, 4.0)], single_precision=False)
        maps.append(slab)
        rows.append(f"{dates[q]} {dates[q]} {jd:13.5f} {name}")
    (tmp_path / "da" / "map_list.csv").write_text("\n".join(rows) + "\n")
    da = dict(assimilate_data=True, assimilate_data_map_list_filename="da/map_list.csv",
              assimilate_data_map_root_dir="da", assimilate_data_custom_from_mu=True,
              assimilate_data_mu_power=4.0, assimilate_data_mu_limit=0.1)
    text = _bench_namelist(prm, range(nr), 2.5, da)
    (tmp_path / "hipft.in").write_text(text)
    D = np.asarray(prm["diffusion_coef_constants"])
    speed = _cfl_rank(prm, t)
    subset = sorted({int(np.argmax(D)), int(np.argmax(speed)), int(np.argsort(speed)[-2]), 0, 37})
    sub_text = _bench_namelist(prm, subset, 2.5, da)
    sub = O.process_parameters(O.parse_namelist(sub_text))
    times = [24.0 * (jd - jd0) for jd in jds]
    r = O.run(sub, map_pt=np.broadcast_to(br, (len(subset),) + br.shape), s1=p, s2=t, da_times=times,
              da_maps=np.stack(maps))
    assert r["nsteps"] == 3, f"expected three steps, the oracle took {r['nsteps']}"
    shape = (nr,) + r["f"].shape[1:]
    f = H.run_field(str(tmp_path / "hipft.in"), str(tmp_path), shape)
    sol, num = cases.read_run_histories(str(tmp_path), nr)
    # the subset reproduces the shared schedule of all 64 realizations
    assert np.array_equal(num[0][:, 6:], r["num"][:, 0, 6:]), "stage/cycle counts of the subset differ"
    rel = np.abs(num[0][:, :6] - r["num"][:, 0, :6]) / np.maximum(np.abs(r["num"][:, 0, :6]), 1e-300)
    assert rel.max() <= HIST_TOL, f"dt columns of the subset differ: {rel.max(0)}"
    compare("batched64", f, r, sol, num, realizations=subset, oracle_index=range(len(subset)))
