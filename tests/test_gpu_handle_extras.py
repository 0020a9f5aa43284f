"""Handle extras: the zero-copy field view and the bounded-wait error path.

hipft_gpu_field_device_ptr must expose exactly the field hipft_gpu_get_field
copies out.  hipft_gpu_check_bounded_wait runs a kernel whose wait on an
mbarrier can never complete: it must give up after its poll limit, the call
must report HIPFT_ETIMEOUT (the status a stalled tile copy would give), and
the handle must stay usable (a diffusion step afterwards succeeds and matches
a handle that never saw the error).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _handle(H):
    ntm, npm1, nr = 45, 91, 2
    t = np.linspace(0.0, np.pi, ntm)
    p = np.linspace(0.0, 2.0 * np.pi, npm1)
    g = H.HipftGPU(t, p, nr, advance_diffusion=True, diffusion_coef_constants=[300.0, 600.0])
    rng = np.random.default_rng(3)
    g.load_initial_map(rng.normal(size=(nr, ntm, npm1)))
    return g


def test_field_device_view_matches_get_field():
    import hipft_b200 as H
    with _handle(H) as g:
        v = g.field_tensor()
        f = g.get_field()
        assert np.array_equal(v[:, :, :g.ntm].cpu().numpy(), f)


def test_bounded_wait_reports_timeout_and_handle_recovers():
    import hipft_b200 as H
    from hipft_b200 import gpu
    with _handle(H) as a, _handle(H) as b:
        rc = a.L.hipft_gpu_check_bounded_wait(a.h, 64)
        assert rc == gpu.HIPFT_ETIMEOUT
        a.diffusion_step(2.0)
        b.diffusion_step(2.0)
        assert np.array_equal(a.get_field(), b.get_field())
