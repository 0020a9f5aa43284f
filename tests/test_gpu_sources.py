"""Sources (advance_source) through the standalone driver.

The reference's source path: load_source (src/hipft.f90:7050-7213) with the
source file interpolated onto the mesh by interp2d and the random flux
emergence frames of generate_rfe (8809-8921, flux-balanced), update_source's
time blend of two frames (3875-3947) with a new frame every
source_rfe_lifetime, the 'rfeswap' time-step cut (4431-4442) and source_step
in flux_transport_step (4463-4507, 4697-4732).  The random deviates come from
the generator both the driver and the oracle use (seeded); the source file is
written with the library's HDF5 writer on a coarser grid of its own.  Final
fields and every history row must agree with the oracle.

Seams: every operator here leaves the phi seam columns as periodic copies.
The reference recomputes them in its stage combines, which is the same thing
while the field is periodic; a source that is not periodic at the seams (the
reference's interpolation of a one-point-overlap file leaves column npm at
zero) makes the reference's seam columns drift, and this library does not
reproduce that drift.
"""
import numpy as np
import pytest

import cases
import test_gpu_features as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _source_file(tmp_path):
    """A source on a coarser grid of its own with the two-point phi overlap
    (last column at the second one plus 2 pi) and periodic data, so that the
    interpolated source is periodic at the seams: the reference's map files
    with a one-point overlap leave the source's last phi column at zero, a case
    whose seam handling differs by design (see the module docstring)."""
    import hipft_b200 as H
    n0, nft = 64, 30
    p0 = np.linspace(0.0, 2.0 * np.pi, n0)
    pf = np.concatenate([p0, [p0[1] + 2.0 * np.pi]])
    tf = np.linspace(0.0, np.pi, nft)
    data = 0.02 * np.cos(2.0 * tf)[:, None] * np.sin(pf + 0.4)[None, :] + 0.005  # (nft, nfp) C order
    data[:, n0 - 1] = data[:, 0]
    data[:, n0] = data[:, 1]
    H.h5_write(str(tmp_path / "source.h5"), data, [pf, tf], single_precision=False)
    return dict(data=data, pf=pf, tf=tf)


CASES = {
    "rfe1_strang_diffusion": dict(advance_diffusion=True, diffusion_coef_constants=[300.0, 150.0],
                                  strang_splitting=True, source_rfe_model=1, source_rfe_seed=1234,
                                  source_rfe_lifetime=0.8,
                                  source_rfe_total_unsigned_flux_per_hours=[2.0e3, 5.0e3]),
    "rfe2_file_flow_lie": dict(advance_flow=True, flow_dr_model=1, flow_mf_model=1, source_rfe_model=2,
                               source_rfe_seed=77, source_rfe_lifetime=1.3, source_rfe_total_unsigned_flux_per_hour=8.0e3,
                               source_from_file=True, source_filename="source.h5"),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_sources_match_oracle(name, tmp_path):
    import hipft_b200 as H
    d = dict(F.BASE, advance_source=True, validation_run=1, time_end=6.0, dt_max=1.0)
    d.update(CASES[name])
    src = _source_file(tmp_path) if d.get("source_from_file") else None
    text = F._namelist(d)
    (tmp_path / "hipft.in").write_text(text)
    prm = O.process_parameters(O.parse_namelist(text))
    r = O.run(prm, source=src)
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
    # the frames were swapped inside the run: the steps were cut at the lifetime
    lt = prm["source_rfe_lifetime"]
    assert np.any(np.isclose(r["sol"][:, 0, 1], lt)), "no step ended at the first RFE swap"
