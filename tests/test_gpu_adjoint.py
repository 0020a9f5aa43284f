"""The hand-written adjoint (hipft_adj_step + hipft_b200.adjoint) against
torch autograd through the pure-PyTorch restatement of the same discrete
scheme, and against central finite differences of the library's own
forward; checkpoint spacing must not change the result."""
import numpy as np
import pytest
import torch

import adjoint_cases as C
from adjoint_ref import RefScheme
from hipft_b200 import gpu as G
from hipft_b200.adjoint import FLOW_KEYS, FluxTransport, MisfitAdjoint, chain_physical, misfit_weights, mesh_1d

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-9     # relative max-norm, adjoint vs autograd of the restatement
FD_TOL = 1e-6       # relative, adjoint vs central differences (h = 1e-6 relative)


def _handle(D, coef, subcycles=C.CASE["diffusion_subcycles"]):
    t, p = C.mesh_tp()
    g = G.HipftGPU(t, p, C.CASE["n_realizations"], advance_flow=True, flow_num_method=4, strang_splitting=True,
                   advance_diffusion=True, diffusion_num_method=3, diffusion_subcycles=subcycles,
                   diffusion_coef_constants=D)
    g.set_flow(dr_model=1, mf_model=1, dr_p0=coef["p0"], dr_p2=coef["p2"], dr_p4=coef["p4"], mf_p1=coef["p1"],
               mf_p3=coef["p3"], mf_p5=coef["p5"])
    return g


def _inputs():
    p, r, dts = C.oracle_run()
    D = np.array(C.CASE["diffusion_coef_constants"])
    coef = {k: np.array(C.CASE[v]) for k, v in C.FLOW.items()}
    f0 = r["map_initial"]
    return f0, C.target_field(f0), dts, D, coef


def _reference_grads(f0, target, dts, D, coef, sched=None):
    t, p = C.mesh_tp()
    S = RefScheme(t, p, len(D))
    f0v = torch.tensor(f0, requires_grad=True)
    Dv = torch.tensor(D, requires_grad=True)
    cv = {k: torch.tensor(v, requires_grad=True) for k, v in coef.items()}
    f = S.run(f0v, dts, Dv, cv, C.CASE["diffusion_subcycles"], S.euler_dt(D), sched=sched)
    L = S.misfit(f, torch.tensor(target))
    L.backward()
    g = {"f0": f0v.grad.numpy(), "D": Dv.grad.numpy()}
    g.update({k: cv[k].grad.numpy() for k in FLOW_KEYS})
    return L.item(), g


def _rel(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300)


def _check_against_reference(loss, grads, Lr, gr):
    assert abs(loss - Lr) <= 1e-12 * abs(Lr), (loss, Lr)
    # the restatement's f0 gradient carries the seam columns separately; fold them
    fr = gr["f0"].copy()
    npm = fr.shape[1]
    fr[:, npm - 2] += fr[:, 0]
    fr[:, 1] += fr[:, npm - 1]
    fr[:, 0] = fr[:, npm - 1] = 0.0
    assert _rel(grads["f0"], fr) < GRAD_TOL, _rel(grads["f0"], fr)
    for k in ["D"] + list(FLOW_KEYS):
        assert _rel(grads[k], gr[k]) < GRAD_TOL, (k, grads[k], gr[k])
    phys = chain_physical(grads)
    assert all(np.all(np.isfinite(v)) for v in phys.values())


def test_adjoint_matches_autograd_of_restatement():
    f0, target, dts, D, coef = _inputs()
    with _handle(D, coef) as g:
        loss, grads = MisfitAdjoint(g, D, coef, checkpoint_every=2).run(f0, target, dts)
    _check_against_reference(loss, grads, *_reference_grads(f0, target, dts, D, coef))


def test_adjoint_with_ptl_subcycles_matches_autograd_of_restatement():
    """Automatic (PTL) subcycling: the adjoint replays the forward's subcycle
    dts, which the restatement takes from the step callback."""
    _, r, dts = C.rough_run()
    D = np.array(C.CASE["diffusion_coef_constants"])
    coef = {k: np.array(C.CASE[v]) for k, v in C.FLOW.items()}
    f0 = r["map_initial"]
    target = C.target_field(f0)
    sched = []
    with _handle(D, coef, subcycles=0) as g:
        g.set_field(f0)
        g.update_flow()
        for dt in dts:
            sub = []
            g.flux_transport_step(float(dt), cb=lambda c, ts, dtl2, s, sc: sub.append(dtl2))
            sched.append(sub)
    assert max(len(s) for s in sched) > 1
    with _handle(D, coef, subcycles=0) as g:
        loss, grads = MisfitAdjoint(g, D, coef, checkpoint_every=2).run(f0, target, dts)
    _check_against_reference(loss, grads, *_reference_grads(f0, target, dts, D, coef, sched=sched))


def test_checkpoint_spacing_does_not_change_the_gradient():
    f0, target, dts, D, coef = _inputs()
    out = []
    for k in (1, 2, 64):
        with _handle(D, coef) as g:
            out.append(MisfitAdjoint(g, D, coef, checkpoint_every=k).run(f0, target, dts))
    for loss, grads in out[1:]:
        assert loss == out[0][0]
        for key in grads:
            assert np.array_equal(grads[key], out[0][1][key]), key


def test_adjoint_matches_finite_differences_of_library_forward():
    f0, target, dts, D, coef = _inputs()
    with _handle(D, coef) as g:
        A = MisfitAdjoint(g, D, coef, checkpoint_every=1)
        loss, grads = A.run(f0, target, dts)

    def loss_at(Dd, cd, f0d):
        with _handle(Dd, cd) as g:
            g.set_field(f0d)
            g.update_flow()
            for dt in dts:
                g.flux_transport_step(float(dt))
            return A.loss_and_cotangent(g.get_field(), target)[0]

    for name, i in (("D", 0), ("D", 1), ("p0", 0), ("p2", 0), ("p4", 1), ("p1", 1), ("p3", 0), ("p5", 1)):
        base = D if name == "D" else coef[name]
        h = 1e-6 * abs(base[i])
        vals = []
        for s in (1.0, -1.0):
            Dd, cd = D.copy(), {k: v.copy() for k, v in coef.items()}
            (Dd if name == "D" else cd[name])[i] += s * h
            vals.append(loss_at(Dd, cd, f0))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(grads[name][i] - fd) <= FD_TOL * abs(fd), (name, i, grads[name][i], fd)
    dirn = np.random.default_rng(5).standard_normal(f0.shape)
    dirn[:, 0] = dirn[:, -2]
    dirn[:, -1] = dirn[:, 1]
    h = 1e-6 * np.max(np.abs(f0))
    fd = (loss_at(D, coef, f0 + h * dirn) - loss_at(D, coef, f0 - h * dirn)) / (2 * h)
    assert abs(float(np.sum(grads["f0"] * dirn)) - fd) <= FD_TOL * abs(fd), (np.sum(grads["f0"] * dirn), fd)


def _file_flow(t, p):
    """A smooth 2-D flow in m/s on the test grid: vt (nt, npm1) on theta
    faces, vp (ntm, np) on phi faces (set_flow_from_files' shapes)."""
    th = np.concatenate([[t[0]], 0.5 * (t[1:] + t[:-1]), [t[-1]]])   # nt faces
    ph = np.concatenate([p, [p[-1] + (p[-1] - p[-2])]])               # np faces
    vt = 25.0 * np.sin(th)[:, None] ** 2 * np.sin(2.0 * p + 0.3)[None, :]
    vp = 40.0 * np.sin(t)[:, None] * np.cos(ph - 0.7)[None, :] ** 2
    return vt, vp


def test_adjoint_with_flows_from_files_matches_finite_differences():
    """A 2-D flow from files added to the analytic flows (a constant of the
    step): the gradients of f0 (a random direction) and D against central
    differences of the library's forward with the same flows."""
    f0, target, dts, D, coef = _inputs()
    t, p = C.mesh_tp()
    vt, vp = _file_flow(t, p)
    with _handle(D, coef) as g:
        g.set_flow_from_files(vt, vp)
        A = MisfitAdjoint(g, D, coef, checkpoint_every=2)
        loss, grads = A.run(f0, target, dts)
    assert set(grads) == {"f0", "D"}

    def loss_at(Dd, f0d):
        with _handle(Dd, coef) as g:
            g.set_flow_from_files(vt, vp)
            g.set_field(f0d)
            g.update_flow()
            for dt in dts:
                g.flux_transport_step(float(dt))
            return A.loss_and_cotangent(g.get_field(), target)[0]

    for i in range(len(D)):
        h = 1e-6 * abs(D[i])
        Dp, Dm = D.copy(), D.copy()
        Dp[i] += h
        Dm[i] -= h
        fd = (loss_at(Dp, f0) - loss_at(Dm, f0)) / (2 * h)
        assert abs(grads["D"][i] - fd) <= FD_TOL * abs(fd), (i, grads["D"][i], fd)
    dirn = np.random.default_rng(11).standard_normal(f0.shape)
    dirn[:, 0] = dirn[:, -2]
    dirn[:, -1] = dirn[:, 1]
    h = 1e-6 * np.max(np.abs(f0))
    fd = (loss_at(D, f0 + h * dirn) - loss_at(D, f0 - h * dirn)) / (2 * h)
    assert abs(float(np.sum(grads["f0"] * dirn)) - fd) <= FD_TOL * abs(fd), (np.sum(grads["f0"] * dirn), fd)


def test_autograd_function_matches_restatement():
    """FluxTransport (torch.autograd.Function over the library's forward and
    adjoint) inside an ordinary torch loss: its gradients equal the
    restatement's autograd gradients."""
    f0, target, dts, D, coef = _inputs()
    t, p = C.mesh_tp()
    run = FluxTransport(t, p, dts, checkpoint_every=2, diffusion_subcycles=C.CASE["diffusion_subcycles"])
    f0v = torch.tensor(f0, requires_grad=True)
    Dv = torch.tensor(D, requires_grad=True)
    cv = {k: torch.tensor(v, requires_grad=True) for k, v in coef.items()}
    fN = run(f0v, Dv, cv)
    w = torch.tensor(misfit_weights(mesh_1d(t, p)))[None]
    loss = 0.5 * (w * (fN - torch.tensor(target)) ** 2).sum()
    loss.backward()
    grads = {"f0": f0v.grad.numpy(), "D": Dv.grad.numpy()}
    grads.update({k: cv[k].grad.numpy() for k in FLOW_KEYS})
    _check_against_reference(loss.item(), grads, *_reference_grads(f0, target, dts, D, coef))


def _da_map(seed=3):
    t, p = C.mesh_tp()
    rng = np.random.default_rng(seed)
    data = 5.0 * np.cos(t)[:, None] * np.ones((1, len(p))) + rng.standard_normal((len(t), len(p)))
    mu = np.sin(t)[:, None] * np.cos(p[None, :] - 0.4)
    data[:, -1] = data[:, 0]
    mu[:, -1] = mu[:, 0]
    return np.stack([data, np.zeros_like(mu), mu])


@pytest.mark.parametrize("balance", [False, True])
def test_adjoint_through_assimilation_matches_restatement(balance):
    """An assimilation blend (mu^4 weights, mu > 0.1) after the first step,
    with and without flux balancing of the increment (balance_flux,
    src/hipft.f90:8752-8807): the hand-written reverse
    (hipft_adj_assimilate_at) against autograd of the restatement with the
    same blend."""
    f0, target, dts, D, coef = _inputs()
    t, p = C.mesh_tp()
    m3 = _da_map()
    opts = dict(custom_from_mu=True, mu_power=4.0, mu_limit=0.1, balance_flux=balance)
    with _handle(D, coef) as g:
        A = MisfitAdjoint(g, D, coef, checkpoint_every=2, assim={0: (m3, opts)})
        loss, grads = A.run(f0, target, dts)
    # the restatement, split at the assimilation
    S = RefScheme(t, p, len(D))
    f0v = torch.tensor(f0, requires_grad=True)
    Dv = torch.tensor(D, requires_grad=True)
    cv = {k: torch.tensor(v, requires_grad=True) for k, v in coef.items()}
    sc = C.CASE["diffusion_subcycles"]
    f = S.run(f0v, dts[:1], Dv, cv, sc, S.euler_dt(D))
    mu = m3[2]
    w = np.where(mu > 0.1, mu ** 4.0, 0.0)          # (ntm, npm1): map column c is field column c (0-based)
    Wc = torch.tensor(w[:, 1:].T)[None]             # core field columns 1..npm-2 (0-based)
    Dd = torch.tensor(m3[0][:, 1:].T)[None]
    delta = Wc * (Dd - f[:, 1:-1])
    if balance:
        # get_flux's areas over columns 1..npm-1 (column 1 the seam copy of npm-1)
        A = torch.tensor(misfit_weights(mesh_1d(t, p)))[None]
        full = S._seam(delta)
        pos = full > 0
        fp = (full * A * pos).sum(dim=(1, 2))
        fm = (full * A * ~pos).sum(dim=(1, 2))
        assert (fp > 0).all() and (fm < 0).all()
        r = torch.sqrt(torch.abs(fp / fm))[:, None, None]
        delta = torch.where(delta > 0, delta / r, delta * r)
    core = f[:, 1:-1] + delta
    f = S._seam(core)
    f = S.run(f, dts[1:], Dv, cv, sc, S.euler_dt(D))
    L = S.misfit(f, torch.tensor(target))
    L.backward()
    gr = {"f0": f0v.grad.numpy(), "D": Dv.grad.numpy()}
    gr.update({k: cv[k].grad.numpy() for k in FLOW_KEYS})
    _check_against_reference(loss, grads, L.item(), gr)


def test_balanced_assimilation_without_room_to_tape():
    """A balanced assimilation after the last step of a recomputed segment,
    with no device memory left for tapes (every step recorded one at a time
    in the reverse pass, so the recompute never runs that step and its output
    is computed again for the balance's reverse): the same gradient as with
    the segment taped."""
    f0, target, dts, D, coef = _inputs()
    assert len(dts) >= 3
    m3 = _da_map()
    opts = dict(custom_from_mu=True, mu_power=4.0, mu_limit=0.1, balance_flux=True)
    out = []
    for reserve in (0.15, 0.9999):
        with _handle(D, coef) as g:
            A = MisfitAdjoint(g, D, coef, checkpoint_every=2, assim={1: (m3, opts)}, reserve_frac=reserve)
            out.append(A.run(f0, target, dts))
    (l0, g0), (l1, g1) = out
    assert l0 == l1
    for k in g0:
        np.testing.assert_allclose(g1[k], g0[k], rtol=1e-13, atol=0.0, err_msg=k)


def test_stage_checkpoints_do_not_change_the_gradient():
    """Stage checkpoints inside the RKG2 super-steps (the reverse recomputes
    each block of q stages from its pair) give bitwise the gradient of the
    full tape, with fewer tape fields."""
    _, r, dts = C.rough_run()
    D = np.array(C.CASE["diffusion_coef_constants"])
    coef = {k: np.array(C.CASE[v]) for k, v in C.FLOW.items()}
    f0 = r["map_initial"]
    target = C.target_field(f0)
    out, tapes = [], []
    for q in (0, 2, 4):
        with _handle(D, coef, subcycles=0) as g:
            g.L.hipft_adj_set_tape_limit(g.h, 0, q)
            A = MisfitAdjoint(g, D, coef, checkpoint_every=2)
            out.append(A.run(f0, target, dts))
            n = __import__("ctypes").c_int64(0)
            g.L.hipft_adj_tape_fields(g.h, __import__("ctypes").byref(n))
            tapes.append(n.value)
            A.release()
            g.L.hipft_adj_tape_fields(g.h, __import__("ctypes").byref(n))
            assert n.value == 0
    for loss, grads in out[1:]:
        assert loss == out[0][0]
        for key in grads:
            assert np.array_equal(grads[key], out[0][1][key]), key
    assert tapes[1] < tapes[0], tapes


def test_adjoint_matches_restatement_128x256():
    """The restatement comparison on a 128 x 256 grid (the adjoint
    configuration's small grid)."""
    case = dict(C.CASE, res_nt=128, res_np=257, time_end=40.0, dt_max=20.0,
                diffusion_coef_constants=[600.0, 1500.0])
    p_, r, dts = C.oracle_run(case)
    D = np.array(case["diffusion_coef_constants"])
    coef = {k: np.array(case[v]) for k, v in C.FLOW.items()}
    f0 = r["map_initial"]
    target = C.target_field(f0)
    t, p = C.mesh_tp(case)
    g = G.HipftGPU(t, p, case["n_realizations"], advance_flow=True, flow_num_method=4, strang_splitting=True,
                   advance_diffusion=True, diffusion_num_method=3, diffusion_subcycles=case["diffusion_subcycles"],
                   diffusion_coef_constants=D)
    g.set_flow(dr_model=1, mf_model=1, dr_p0=coef["p0"], dr_p2=coef["p2"], dr_p4=coef["p4"], mf_p1=coef["p1"],
               mf_p3=coef["p3"], mf_p5=coef["p5"])
    with g:
        loss, grads = MisfitAdjoint(g, D, coef, checkpoint_every=1).run(f0, target, dts)
    S = RefScheme(t, p, len(D))
    f0v = torch.tensor(f0, requires_grad=True)
    Dv = torch.tensor(D, requires_grad=True)
    cv = {k: torch.tensor(v, requires_grad=True) for k, v in coef.items()}
    f = S.run(f0v, dts, Dv, cv, case["diffusion_subcycles"], S.euler_dt(D))
    L = S.misfit(f, torch.tensor(target))
    L.backward()
    gr = {"f0": f0v.grad.numpy(), "D": Dv.grad.numpy()}
    gr.update({k: cv[k].grad.numpy() for k in FLOW_KEYS})
    _check_against_reference(loss, grads, L.item(), gr)
