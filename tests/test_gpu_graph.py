"""Graph-run steps (hipft_gpu_set_graph) against host-driven steps.

A graph-run flux_transport_step takes its schedule decisions (PTL subcycle
lengths, stage counts and coefficients, advection substeps) on the device,
with the host path's arithmetic, inside one captured CUDA graph.  The bar is
bit-for-bit equality with the host-driven step of the same handle
configuration, plain and ragged, for every advection and diffusion method the
graph supports, and the same schedule record; one case is also checked
against the oracle directly.
"""
import numpy as np
import pytest

import test_gpu_ragged as RG
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _run(t, p, br, nr, steps, graph, ragged=False, flow=True, diffusion=True, dt_scale=1.0, D=None, **kw):
    import hipft_b200 as H
    g = H.HipftGPU(t, p, nr, advance_flow=flow, advance_diffusion=diffusion,
                   diffusion_coef_constants=(D or RG.D[:nr]) if diffusion else None, **kw)
    if flow:
        g.set_flow(dr_model=1, mf_model=1, dr_p2=RG.P2[:nr], mf_p1=RG.P1[:nr])
    g.load_initial_map(br[None])
    if flow:
        g.update_flow()
    if ragged:
        g.set_ragged(True)
    if graph:
        g.set_graph(True)
    dt = (g.flow_dtmax() if flow else 6.0) * dt_scale
    infos = []
    for _ in range(steps):
        i = g.flux_transport_step(dt)
        infos.append((i.sts_s, i.subcycles, i.total_stages))
    sched = g.ragged_schedule() if ragged else None
    f = g.get_field()
    g.close()
    return f, infos, sched, dt


CASES = {
    # name: (nr, ragged, kwargs)
    "plain_ptl_ssprk43_strang": (3, False, dict(flow_num_method=4, strang_splitting=True)),
    "plain_fixed3_rkl2_lie_ssprk33": (2, False, dict(flow_num_method=2, strang_splitting=False,
                                                    diffusion_num_method=2, diffusion_subcycles=3)),
    "plain_fe_upwind": (2, False, dict(flow_num_method=1, strang_splitting=True)),
    "ragged_ptl": (4, True, dict(flow_num_method=4, strang_splitting=True)),
    "ragged_fixed2_lie": (3, True, dict(flow_num_method=4, strang_splitting=False, diffusion_subcycles=2)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_graph_step_equals_host_step(name):
    nr, ragged, kw = CASES[name]
    t, p, br = RG._grid()
    fh, ih, sh, _ = _run(t, p, br, nr, 3, False, ragged=ragged, **kw)
    fg, ig, sg, _ = _run(t, p, br, nr, 3, True, ragged=ragged, **kw)
    assert ih == ig, f"schedules differ: host {ih}, graph {ig}"
    assert np.array_equal(fh, fg), f"fields differ: max {np.abs(fh - fg).max():.3e}"
    if ragged:
        for k in ("sts_s", "subcycles", "adv_substeps"):
            assert np.array_equal(sh[k], sg[k]), (k, sh[k], sg[k])


def test_graph_ragged_advection_substeps():
    """A step longer than some realizations' CFL limits: ceil(dt / limit)
    substeps for those, decided on the device."""
    t, p, br = RG._grid()
    fh, ih, sh, _ = _run(t, p, br, 3, 2, False, ragged=True, diffusion=False, dt_scale=2.5,
                         flow_num_method=4, strang_splitting=True)
    fg, ig, sg, _ = _run(t, p, br, 3, 2, True, ragged=True, diffusion=False, dt_scale=2.5,
                         flow_num_method=4, strang_splitting=True)
    assert sh["adv_substeps"].max() >= 2 and np.array_equal(sh["adv_substeps"], sg["adv_substeps"])
    assert np.array_equal(fh, fg)


def test_graph_diffusion_only_steps():
    t, p, br = RG._grid()
    fh, ih, _, _ = _run(t, p, br, 2, 4, False, flow=False)
    fg, ig, _, _ = _run(t, p, br, 2, 4, True, flow=False)
    assert ih == ig
    assert np.array_equal(fh, fg)


def test_graph_interior_blocks_grid():
    """ntm = 300 (interior theta blocks, several stage-pair iterations per
    subcycle with realizations ending at different pairs)."""
    t, p, br = RG._grid(300, 65)
    fh, ih, sh, _ = _run(t, p, br, 4, 2, False, ragged=True, flow_num_method=4, strang_splitting=True)
    fg, ig, sg, _ = _run(t, p, br, 4, 2, True, ragged=True, flow_num_method=4, strang_splitting=True)
    assert len(set(sh["sts_s"].tolist())) > 1
    assert np.array_equal(fh, fg)


def test_graph_step_against_oracle():
    """Ragged graph-run steps, each realization against the oracle run of that
    realization alone (as the host-driven ragged test does)."""
    t, p, br = RG._grid()
    nr, nsteps = 4, 3
    import hipft_b200 as H
    with RG._handle(t, p, nr) as g:
        g.load_initial_map(br[None])
        g.update_flow()
        g.set_ragged(True)
        g.set_graph(True)
        dt = g.flow_dtmax()
        seq, tend = RG._dt_sequence(dt, nsteps)
        for d in seq:
            g.flux_transport_step(d)
        sched = g.ragged_schedule()
        f = g.get_field()
    for i in range(nr):
        r = RG._oracle_alone(i, t, p, br, dt, tend)
        assert r["nsteps"] == nsteps
        err = np.abs(f[i] - r["f"][0]).max() / np.abs(r["f"][0]).max()
        assert err <= RG.FIELD_TOL, f"realization {i}: field rel max-norm {err:.3e}"
        assert int(r["num"][-1, 0, 6]) == sched["sts_s"][i]


def test_graph_rejects_what_it_does_not_run():
    import hipft_b200 as H
    from hipft_b200 import gpu
    t, p, br = RG._grid()
    with H.HipftGPU(t, p, 2, advance_diffusion=True, diffusion_num_method=1, diffusion_coef_constants=100.0) as g:
        with pytest.raises(gpu.HipftError) as e:
            g.set_graph(True)
        assert e.value.code == gpu.HIPFT_EINVAL
    with H.HipftGPU(t, p, 2, advance_diffusion=True, diffusion_coef_constants=100.0) as g:
        g.load_initial_map(br[None])
        g.set_graph(True)
        with pytest.raises(gpu.HipftError) as e:
            g.flux_transport_step(1.0, cb=lambda *a: None)
        assert e.value.code == gpu.HIPFT_ESTATE
