"""The pure-PyTorch restatement behind the adjoint checks (CPU).

Its forward must reproduce the oracle's final field (the same scheme in C,
itself pinned to the reference's golden histories), and its autograd
gradients must agree with central finite differences of its own forward;
the GPU adjoint is then checked against these gradients."""
import numpy as np
import torch

import adjoint_cases as C
from adjoint_ref import RefScheme
from hipft_b200.adjoint import FLOW_KEYS

FIELD_TOL = 1e-12   # relative max-norm, forward vs oracle
FD_TOL = 1e-6       # relative, autograd vs central differences (h = 1e-6 relative)


def _setup():
    p, r, dts = C.oracle_run()
    t, ph = C.mesh_tp()
    S = RefScheme(t, ph, C.CASE["n_realizations"])
    D = np.array(C.CASE["diffusion_coef_constants"])
    coef = {k: np.array(C.CASE[v]) for k, v in C.FLOW.items()}
    return S, r, dts, D, coef, S.euler_dt(D)


def _loss(S, f0, target, dts, D, coef, dte):
    f = S.run(f0, dts, D, coef, C.CASE["diffusion_subcycles"], dte)
    return S.misfit(f, target)


def _tensors(D, coef):
    return torch.tensor(D), {k: torch.tensor(v) for k, v in coef.items()}


def test_reference_forward_matches_oracle():
    S, r, dts, D, coef, dte = _setup()
    Dt, ct = _tensors(D, coef)
    f = S.run(torch.tensor(r["map_initial"]), dts, Dt, ct, C.CASE["diffusion_subcycles"], dte).numpy()
    err = np.max(np.abs(f - r["f"])) / np.max(np.abs(r["f"]))
    assert err < FIELD_TOL, err


def test_reference_gradients_match_finite_differences():
    S, r, dts, D, coef, dte = _setup()
    f0 = torch.tensor(r["map_initial"])
    target = torch.tensor(C.target_field(r["map_initial"]))
    f0v = f0.clone().requires_grad_(True)
    Dv = torch.tensor(D, requires_grad=True)
    cv = {k: torch.tensor(v, requires_grad=True) for k, v in coef.items()}
    L = _loss(S, f0v, target, dts, Dv, cv, dte)
    L.backward()
    Lval = L.item()
    # a direction in the initial field with the seam copies kept
    dirn = np.random.default_rng(3).standard_normal(f0.shape)
    dirn[:, 0] = dirn[:, -2]
    dirn[:, -1] = dirn[:, 1]
    dirn = torch.tensor(dirn)
    g_f = float((f0v.grad * dirn).sum())
    h = 1e-6 * float(f0.abs().max())
    with torch.no_grad():
        Dt, ct = _tensors(D, coef)
        fd = float(_loss(S, f0 + h * dirn, target, dts, Dt, ct, dte) -
                   _loss(S, f0 - h * dirn, target, dts, Dt, ct, dte)) / (2 * h)
    assert abs(g_f - fd) <= FD_TOL * abs(fd), (g_f, fd)
    for name in ["D"] + list(FLOW_KEYS):
        for i in range(len(D)):
            base = D if name == "D" else coef[name]
            if base[i] == 0.0:
                continue
            h = 1e-6 * abs(base[i])

            def L_at(delta):
                Dd, cd = D.copy(), {k: v.copy() for k, v in coef.items()}
                (Dd if name == "D" else cd[name])[i] += delta
                with torch.no_grad():
                    return float(_loss(S, f0, target, dts, *_tensors(Dd, cd), dte))
            fd = (L_at(h) - L_at(-h)) / (2 * h)
            g = float((Dv.grad if name == "D" else cv[name].grad)[i])
            assert abs(g - fd) <= FD_TOL * abs(fd) + 1e-12 * abs(Lval), (name, i, g, fd)
