"""Regenerate the golden fixtures from the reference testsuite.

Copies each testsuite case's hipft.in and input map, and stores a subsample of
its golden history rows (16-digit values from
testsuite/<case>/reference/hipft_history_{sol,num}_rNNNNNN.out) as .npz, so the
GPU tests can run where the reference tree is absent.  Run from the repo root:
    python tests/golden/make_golden.py /root/reference/testsuite
"""
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["advect_gaussians_phi", "advect_gaussians_theta", "advect_gaussians_phi_theta", "diffuse_soccer",
         "diffuse_advect_soccer", "diffuse_dipole", "diffuse_advect_atten_map_1cr"]


def read_history(path):
    rows = []
    with open(path) as fh:
        next(fh)
        for line in fh:
            if line.strip():
                rows.append([float(x) for x in line.split()])
    return np.array(rows)


def main(src):
    for case in CASES:
        d = os.path.join(src, case)
        out = os.path.join(HERE, case)
        os.makedirs(out, exist_ok=True)
        for f in os.listdir(os.path.join(d, "input")):
            shutil.copy(os.path.join(d, "input", f), os.path.join(out, f))
        sol, num, idx = [], [], None
        r = 1
        while os.path.exists(os.path.join(d, "reference", f"hipft_history_sol_r{r:06d}.out")):
            s = read_history(os.path.join(d, "reference", f"hipft_history_sol_r{r:06d}.out"))
            n = read_history(os.path.join(d, "reference", f"hipft_history_num_r{r:06d}.out"))
            if idx is None:
                m = len(s)
                idx = np.unique(np.r_[np.arange(min(m, 8)), np.arange(0, m, 32), np.arange(max(m - 4, 0), m)])
            sol.append(s[idx])
            num.append(n[idx])
            r += 1
        np.savez_compressed(os.path.join(out, "golden_history.npz"), rows=idx, nrows=m, sol=np.stack(sol),
                            num=np.stack(num))
        print(case, "realizations:", len(sol), "rows kept:", len(idx), "of", m)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/testsuite")
