"""The "b200" SearchBackend registered into the reference library: the
reference's own search() (prepare, real pass, time-shuffled null passes, tail
fit, refinement, candidates) run with backend "b200" must give exactly what it
gives with its CPU backend -- threshold, pooled null peaks, detection map and
every candidate field."""
import ctypes as C
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADAPTER = os.path.join(ROOT, "fainttrail_b200", "adapter", "libft_b200_adapter.so")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref_b200(reference):
    if not os.path.exists(ADAPTER):
        pytest.skip("adapter not built (needs the reference headers)")
    lib = C.CDLL(ADAPTER, mode=C.RTLD_GLOBAL)
    assert lib.ft_b200_register_backend() == 0
    return reference


def compare(a, b):
    assert a["threshold"] == b["threshold"] and a["method"] == b["method"]
    assert np.array_equal(a["null_peaks"], b["null_peaks"])
    assert np.array_equal(a["max_snr"], b["max_snr"])
    assert len(a["candidates"]) == len(b["candidates"])
    for (va, fa), (vb, fb) in zip(a["candidates"], b["candidates"]):
        assert np.array_equal(va, vb) and fa == fb


@pytest.mark.parametrize("seed,w,h,n,nmovers", [(5, 96, 80, 12, 2), (21, 160, 128, 24, 4)])
def test_reference_search_with_b200_backend(ref_b200, seed, w, h, n, nmovers):
    R = ref_b200
    frames, mjd, exp = R.simulate(width=w, height=h, nframes=n, nstars=60, nmovers=nmovers, seed=seed,
                                  rate_min_arcsec_min=0.3, rate_max_arcsec_min=0.8)
    prep = R.prepare(frames, mjd, exp, fwhm_px=2.5, null_runs=2)
    cpu = prep.search(fwhm_px=2.5, null_runs=2, backend="cpu", threshold_snr=0.0)
    gpu = prep.search(fwhm_px=2.5, null_runs=2, backend="b200", threshold_snr=0.0)
    compare(cpu, gpu)
    # a fixed, low threshold so that candidates are refined and compared too
    cpu = prep.search(fwhm_px=2.5, null_runs=0, backend="cpu", threshold_snr=4.5)
    gpu = prep.search(fwhm_px=2.5, null_runs=0, backend="b200", threshold_snr=4.5)
    compare(cpu, gpu)
    if n >= 24:
        assert len(cpu["candidates"]) > 0


def test_reference_check_backend_conformance(ref_b200):
    """The reference's own conformance procedure (check-backend: a 72 x 52 x 12
    sequence against the naive contract, the same frames with a curved shift
    table, a 384 x 320 x 40 sequence against the simple reference;
    cli/main.cpp:697-741, backend.cpp:281-314) run on the "b200" backend: every
    check conforms, and every map is bit-identical, not merely within the
    contract's 1e-4 tolerance."""
    ok, total, same, text = ref_b200.check_backend("b200")
    assert total == 3 and ok == total and same == total, text
    ok, total, same, text = ref_b200.check_backend("cpu")
    assert ok == total == same == 3, text
