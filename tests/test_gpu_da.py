"""GPU parity of the data-assimilation blend (hipft_gpu_assimilate) against
the oracle's restatement of apply_data_assimilation + assimilate_new_data
(src/hipft.f90:4228-4271, 4083-4146): blend and add modes, mu^p weights with
per-realization powers and limits, latitude caps, multiplication factor and
multiplicative flux balance of the increment.  The PT map is read through a
shared-memory transpose on the GPU; a ragged grid (ntm = 67, npm1 = 101)
exercises partial tiles."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.mark.parametrize("add,custom,balance", [(False, True, False), (False, False, True), (True, True, True),
                                                (False, True, True)])
def test_gpu_da_blend_matches_oracle(add, custom, balance):
    import hipft_b200 as H
    ntm, npm1, nr = 67, 101, 3
    rng = np.random.default_rng(5)
    t = np.linspace(0.0, np.pi, ntm)
    p = np.linspace(0.0, 2.0 * np.pi, npm1)
    mu_power, mu_limit, lat_limit = [4.0, 2.0, 3.0], [0.1, 0.25, 0.0], [0.0, 60.0, 75.0]
    prm = O.process_parameters({
        "n_realizations": nr, "res_nt": ntm, "res_np": npm1, "assimilate_data": True,
        "assimilate_data_add": add, "assimilate_data_custom_from_mu": custom,
        "assimilate_data_balance_flux": balance, "assimilate_data_mult_fac": 1.5,
        "assimilate_data_mu_powers": mu_power, "assimilate_data_mu_limits": mu_limit,
        "assimilate_data_lat_limits": lat_limit})
    with H.HipftGPU(t, p, nr) as g:
        g.load_initial_map(rng.normal(size=(nr, ntm, npm1)) * 5.0)
        f0 = g.get_field()
        data = rng.normal(size=(ntm, npm1)) * 3.0 + 1.0
        weight = rng.uniform(0.0, 1.0, size=(ntm, npm1))
        mu = np.sin(t)[:, None] * np.cos(p[None, :] - 1.0)
        map3 = np.stack([data, weight, mu])
        g.assimilate(map3, add=add, custom_from_mu=custom, balance_flux=balance, mult_fac=1.5, mu_power=mu_power,
                     mu_limit=mu_limit, lat_limit=lat_limit)
        f_gpu = g.get_field()
    f_ref = np.ascontiguousarray(f0.copy())
    O.da_blend(prm, t, p, f_ref, map3)
    assert np.abs(f_ref - f0).max() > 1e-3  # the blend changed the field
    err = np.abs(f_gpu - f_ref).max() / np.abs(f_ref).max()
    assert err <= TOL, f"DA blend rel max-norm {err:.3e}"
