"""The reference's real-data regression cases through the device search: the
three committed sequences (real sky noise, 16-bit registered crops with their
registration offsets; tests/regression/*-cut.case) searched by ft_b200_search
with the case's settings, the PSF width estimated and the detector test on,
must give the reference's search outputs bit for bit: threshold and tail fit,
pooled null peaks, detection map, every candidate field and flag (the
leo-triplet crop holds 81 candidates, among them the asteroid and rejected edge
artefacts)."""
import pytest

from regression_cases import CASES, load_case, same_search

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", CASES)
def test_device_search_equals_reference_on_real_data(device, case):
    g = load_case(case)
    got = device.search(g["frames"], g["mjd"], g["exptime"], reg_dx=g["reg_dx"], reg_dy=g["reg_dy"], **g["params"])
    assert got["n_velocities"] == g["n_velocities"]
    same_search(got, g)
