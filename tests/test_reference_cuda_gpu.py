"""The reference's own CUDA backend (CudaBackend::run, backend_cuda.cu:99-195,
built unchanged for sm_100a from its sources) on the B200: its maps equal the
CPU backend's and the device pass's here, bit for bit, so the timing the
benchmark reports beside the stack kernel is of the same work."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_reference_cuda_pass_equals_cpu_and_device(reference, backend, oracle):
    import fainttrail_b200 as ftb
    R = reference
    if not R.cuda_available():
        pytest.fail("the reference CUDA backend sees no device")
    rng = np.random.default_rng(3)
    n, h, w = 18, 96, 130
    frames = rng.standard_normal((n, h, w)).astype(np.float32)
    frames[2, 40, 50] = np.nan
    t = np.sort(rng.uniform(-0.3, 0.3, n))
    g = np.arange(-10, 11) * 4.0
    vel = np.array([(vx, vy) for vy in g for vx in g if 5.0 <= np.hypot(vx, vy) <= 40.0])
    mc = 13
    got = R.stack_cuda_timed(frames, t, vel, mc)
    ms_cpu, bv_cpu = R.stack(frames, t_h=t, vel=vel, min_count=mc, which=0)
    r = backend.run(ftb.StackPass(frames, t_h=t, velocities=vel, min_count=mc))
    assert np.array_equal(got["max_snr"], ms_cpu, equal_nan=True) and np.array_equal(got["best_v"], bv_cpu)
    assert np.array_equal(r.max_snr, ms_cpu, equal_nan=True) and np.array_equal(r.best_v, bv_cpu)
    assert got["kernel"] > 0.0
