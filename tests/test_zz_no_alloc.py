"""The allocation-free flux integral, hipft_get_flux_noalloc, through the C ABI.

It serves callers that hold all device memory themselves (e.g. maps kept on
the GPU by OpenMP target data mappings and passed as device addresses) and
therefore cannot let the library call cudaMalloc.  Its results must match the
handle-based hipft_gpu_get_flux on the same field, on two calls in a row with
different fields (the fixed scratch keeps the previous call's contents, which
must not leak into the next result).  This file is collected last so that a
failing run that stops at the first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def test_noalloc_flux_matches_handle_twice():
    import torch
    import hipft_b200 as H
    from hipft_b200 import gpu

    L = gpu.lib()
    ntm, npm1, nr = 181, 361, 3
    t = np.linspace(0.0, np.pi, ntm)
    p = np.linspace(0.0, 2.0 * np.pi, npm1)
    rng = np.random.default_rng(11)
    with H.HipftGPU(t, p, nr) as g:
        ldt = g.info().ldt
        npm = npm1 + 1
        stream = torch.cuda.current_stream()
        for scale in (1.0, -3.5):
            g.load_initial_map(scale * rng.normal(size=(nr, ntm, npm1)) + 0.3)
            fp_ref, fm_ref = g.get_flux()
            field = g.get_field()
            dev = torch.zeros((nr, npm, ldt), dtype=torch.float64, device="cuda")
            dev[:, :, :ntm] = torch.from_numpy(field).cuda()
            stream.synchronize()
            fp, fm = np.full(nr, np.nan), np.full(nr, np.nan)
            err = ctypes.create_string_buffer(256)
            rc = L.hipft_get_flux_noalloc(ctypes.c_void_p(dev.data_ptr()), ntm, npm1, nr, ldt, _dp(t), _dp(p),
                                          _dp(fp), _dp(fm), ctypes.c_void_p(stream.cuda_stream), err, 256)
            assert rc == 0, err.value.decode()
            np.testing.assert_allclose(fp, fp_ref, rtol=RTOL, atol=0)
            np.testing.assert_allclose(fm, fm_ref, rtol=RTOL, atol=0)


def test_noalloc_flux_matches_oracle_refined_theta():
    """Independent check on a nonuniform theta scale (spacing halved near the
    poles): the entry point against the oracle's get_flux, two calls in a row."""
    import torch
    from hipft_b200 import gpu
    from hipft_b200 import synthetic as S
    from oracle import oracle as O

    L = gpu.lib()
    ntm, npm1, nr = 200, 257, 4
    t = S.refined_theta(ntm)
    p = S.uniform_phi(npm1)
    npm = npm1 + 1
    ldt = 208
    rng = np.random.default_rng(5)
    stream = torch.cuda.current_stream()
    for shift in (0.2, -0.7):
        f = rng.normal(size=(nr, npm, ntm)) + shift
        f[:, 0, :] = f[:, npm - 2, :]
        f[:, npm - 1, :] = f[:, 1, :]
        fp_ref, fm_ref = O.get_flux(t, p, f)
        dev = torch.zeros((nr, npm, ldt), dtype=torch.float64, device="cuda")
        dev[:, :, :ntm] = torch.from_numpy(f).cuda()
        stream.synchronize()
        fp, fm = np.full(nr, np.nan), np.full(nr, np.nan)
        err = ctypes.create_string_buffer(256)
        rc = L.hipft_get_flux_noalloc(ctypes.c_void_p(dev.data_ptr()), ntm, npm1, nr, ldt, _dp(t), _dp(p),
                                      _dp(fp), _dp(fm), ctypes.c_void_p(stream.cuda_stream), err, 256)
        assert rc == 0, err.value.decode()
        np.testing.assert_allclose(fp, fp_ref, rtol=RTOL, atol=0)
        np.testing.assert_allclose(fm, fm_ref, rtol=RTOL, atol=0)


def test_noalloc_rejects_oversize_grid():
    import torch
    from hipft_b200 import gpu

    L = gpu.lib()
    ntm, npm1, nr = 20000, 8, 1  # theta count above the fixed scratch
    t = np.linspace(0.0, np.pi, ntm)
    p = np.linspace(0.0, 2.0 * np.pi, npm1)
    dev = torch.zeros(8, dtype=torch.float64, device="cuda")
    fp, fm = np.zeros(nr), np.zeros(nr)
    err = ctypes.create_string_buffer(256)
    rc = L.hipft_get_flux_noalloc(ctypes.c_void_p(dev.data_ptr()), ntm, npm1, nr, ntm, _dp(t), _dp(p), _dp(fp),
                                  _dp(fm), None, err, 256)
    assert rc == gpu.HIPFT_EINVAL
    assert b"too large" in err.value
