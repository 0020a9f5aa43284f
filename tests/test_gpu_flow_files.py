"""Flows from files (use_flow_from_files) through the standalone driver.

The reference's path (load_flow_from_files src/hipft.f90:3675-3800,
add_flow_from_files 3525-3673, the 'flowfile' time-step cut 4415-4426): a
flow list read with (F11.5,1X,A11,1X,A11), a 2-D theta velocity (npm1, nt)
and phi velocity (np, ntm) per entry in m/s, shared by all realizations,
the next pair read when the time reaches it and the list wrapping around at
its end; the analytic models are added on top (and attenuation applied) at
every step.  The files are written with the library's HDF5 writer; the
oracle gets the same float32-rounded flows; the final field and every
history row (including the time steps the file times cut) must agree.
"""
import numpy as np
import pytest

import cases
import test_gpu_features as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _flows(tmp_path, ntm, npm1, n):
    import hipft_b200 as H
    nt, np_ = ntm + 1, npm1 + 1
    t = np.linspace(0.0, np.pi, ntm)
    th = np.concatenate([[t[0] - 0.5 * (t[1] - t[0])], 0.5 * (t[1:] + t[:-1]), [t[-1] + 0.5 * (t[1] - t[0])]])
    p = np.linspace(0.0, 2.0 * np.pi, npm1)
    ph = np.concatenate([0.5 * (p[1:] + p[:-1]), [p[-1] + 0.5 * (p[1] - p[0])], [p[-1] + 1.5 * (p[1] - p[0])]])
    (tmp_path / "flows").mkdir()
    jd = 0.0625 * np.arange(n)  # every 1.5 h, starting at 0
    rows = ["JD                 VT          VP"]
    vts, vps = [], []
    for q in range(n):
        vt = 40.0 * np.sin(2.0 * th)[:, None] * (1.0 + 0.3 * np.cos(p + q)[None, :])  # (nt, npm1)
        vp = 120.0 * np.sin(t)[:, None] * (1.0 + 0.2 * np.sin(2.0 * ph[:np_] - q)[None, :])  # (ntm, np)
        a, b = f"vt_{q:03d}.h5", f"vp_{q:03d}.h5"
        H.h5_write(str(tmp_path / "flows" / a), vt, [p, np.arange(1.0, nt + 1)], single_precision=True)
        H.h5_write(str(tmp_path / "flows" / b), vp, [np.arange(1.0, np_ + 1), t], single_precision=True)
        vts.append(vt.astype(np.float32).astype(np.float64))
        vps.append(vp.astype(np.float32).astype(np.float64))
        rows.append(f"{jd[q]:11.5f} {a:<11s} {b:<11s}")
    (tmp_path / "flows" / "list.txt").write_text("\n".join(rows) + "\n")
    return dict(jd=jd, vt=np.stack(vts), vp=np.stack(vps))


CASES = {
    "files_plus_models": dict(advance_diffusion=True, diffusion_coef_constants=[300.0, 150.0],
                              flow_dr_model=1, flow_mf_model=1, strang_splitting=True),
    "files_attenuated_upwind": dict(flow_attenuate=True, flow_attenuate_values=[0.8, 3.0], flow_num_method=2,
                                    flow_vp_rigid_omega=0.5, flow_vt_const=0.3),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_flow_from_files_matches_oracle(name, tmp_path):
    import hipft_b200 as H
    d = dict(F.BASE, advance_flow=True, use_flow_from_files=True, flow_list_filename="flows/list.txt",
             flow_root_dir="flows", validation_run=1, time_end=6.0, dt_max=1.0)
    d.update(CASES[name])
    flows = _flows(tmp_path, d["res_nt"], d["res_np"], 3)
    text = F._namelist(d)
    (tmp_path / "hipft.in").write_text(text)
    prm = O.process_parameters(O.parse_namelist(text))
    r = O.run(prm, flows=flows)
    f = H.run_field(str(tmp_path / "hipft.in"), str(tmp_path), r["f"].shape)
    ferr = np.abs(f - r["f"]).max() / np.abs(r["f"]).max()
    assert ferr <= F.FIELD_TOL, f"{name}: field rel max-norm {ferr:.3e}"
    sol, num = cases.read_run_histories(str(tmp_path), prm["n_realizations"])
    assert sol.shape[1] == r["sol"].shape[0], "history row count differs"
    for i in range(prm["n_realizations"]):
        err = cases.col_errors(sol[i], r["sol"][:, i, :])
        tol = [F.HIST_TOL] * 15 + [max(F.HIST_TOL, cases.VALERR_TOL)]
        bad = {cases.COLS[c - 2]: float(err[c]) for c in range(2, 16) if err[c] > tol[c]}
        assert not bad, f"{name} r{i + 1}: {bad}"
        o = r["num"][:, i, :]
        rel = np.abs(num[i][:, :6] - o[:, :6]) / np.maximum(np.abs(o[:, :6]), 1e-300)
        assert rel.max() <= F.HIST_TOL, f"num columns: {rel.max(0)}"
    # the steps were cut at the flow times 1.5, 3.0 and, after the wrap, 4.5
    times = set(np.round(r["sol"][:, 0, 1], 9))
    assert {1.5, 3.0, 4.5}.issubset(times)


def test_file_flow_survives_a_later_set_flow():
    """The flow from files stays the base of vt, vp whichever of
    hipft_gpu_set_flow and hipft_gpu_set_flow_from_files is called first:
    both orders give bitwise the same step, and it differs from the step
    without the file flow."""
    import hipft_b200 as H
    ntm, npm1, nr = 40, 81, 2
    t = np.linspace(0.0, np.pi, ntm)
    p = np.linspace(0.0, 2.0 * np.pi, npm1)
    th = np.concatenate([[t[0]], 0.5 * (t[1:] + t[:-1]), [t[-1]]])
    vt = 30.0 * np.sin(th)[:, None] ** 2 * np.cos(p)[None, :]
    vp = 60.0 * np.sin(t)[:, None] * np.ones((1, npm1 + 1))
    core = np.cos(t)[None, None, :] * (1.0 + 0.1 * np.sin(3.0 * p[:-1]))[None, :, None] * np.ones((nr, 1, 1))
    f0 = np.concatenate([core[:, -1:], core, core[:, :1]], axis=1)  # (nr, npm, ntm), periodic seam
    flow = dict(dr_model=1, mf_model=1, dr_p2=-300.0, mf_p1=20.0, mf_p3=-20.0)
    out = []
    for order in ("flow_first", "files_first", "no_files"):
        with H.HipftGPU(t, p, nr, advance_flow=True) as g:
            if order == "files_first":
                g.set_flow_from_files(vt, vp)
            g.set_flow(**flow)
            if order == "flow_first":
                g.set_flow_from_files(vt, vp)
            g.set_field(f0)
            g.update_flow()
            g.advection_step(0.5)
            out.append(g.get_field())
    assert np.array_equal(out[0].view(np.uint64), out[1].view(np.uint64))
    assert np.abs(out[0] - out[2]).max() > 1e-6
