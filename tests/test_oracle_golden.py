"""The CPU oracle against the reference testsuite's golden histories.

Pins the oracle (oracle/hipft_oracle.c) to the reference: every history row
of every realization of the seven testsuite cases
(testsuite/*/reference/hipft_history_{sol,num}_r*.out) must agree within
cases.GOLDEN_TOL, and the step/time/dt/stage-count columns exactly.
"""
import numpy as np
import pytest

import cases


@pytest.mark.parametrize("case", cases.CASES)
def test_oracle_matches_golden(case):
    rows, gsol, gnum, nrows = cases.golden(case)
    r = cases.oracle_case(case)
    sol, num = r["sol"], r["num"]
    assert sol.shape[0] == nrows, f"history row count {sol.shape[0]} != golden {nrows}"
    for i in range(gsol.shape[0]):
        err = cases.col_errors(sol[rows, i, :], gsol[i])
        tol = [cases.GOLDEN_TOL[case]] * 15 + [max(cases.VALERR_TOL, cases.GOLDEN_TOL[case])]
        bad = {cases.COLS[c - 2]: float(err[c]) for c in range(2, 16) if err[c] > tol[c]}
        assert not bad, f"{case} realization {i + 1}: {bad}"
        n = num[rows, i, :]
        g = gnum[i]
        # step, time, dt, flow dt, adv dt, Euler dt: relative; stage counts exact
        rel = np.abs(n[:, :6] - g[:, :6]) / np.maximum(np.abs(g[:, :6]), 1e-300)
        assert rel.max() <= max(cases.GOLDEN_TOL[case], 1e-13), f"num columns differ: {rel.max(0)}"
        if case != "diffuse_dipole":
            assert np.array_equal(n[:, 6:], g[:, 6:]), "stage / cycle counts differ"
