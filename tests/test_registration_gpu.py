"""The registration check on the device (ft_b200_check_registration and _dev)
and inside a search (align): bit-identical to the reference's
check_registration (registration.cpp:260-312) on the golden cases and on
rendered star fields (drift, rotation, scale, meridian flip, tied peaks, NaN
blanks, tied and unsorted times, a frame large enough to sample every other
pixel); a search with align "check" refuses frames that are not registered with
the reference's message (preprocess.cpp:618-619) and otherwise equals the same
search without the check."""
import numpy as np
import pytest

from test_registration import FIELDS, field, golden_cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", range(5))
def test_golden_cases(device, case):
    name, frames, t, want = golden_cases()[case]
    assert device.check_registration(frames, t) == want, name


@pytest.mark.parametrize("name", list(FIELDS))
def test_rendered_fields_match_reference(device, reference, name):
    frames, t = field(**FIELDS[name])
    assert device.check_registration(frames, t) == reference.check_registration(frames, t)


def test_device_frames_with_row_pitch(device, reference):
    import torch
    frames, t = field(**FIELDS["drift"])
    n, h, w = frames.shape
    pitch = w + 13
    buf = torch.zeros((n, h, pitch), dtype=torch.float32, device="cuda")
    buf[:, :, :w] = torch.from_numpy(frames).cuda()
    torch.cuda.synchronize()
    got = device.check_registration_dev(buf.data_ptr(), w, h, pitch, n, t)
    assert got == reference.check_registration(frames, t)


def _sequence(name):
    frames, t = field(**FIELDS[name])
    mjd = 60000.0 + t / 24.0
    return frames, mjd, np.full(t.size, 30.0)


def test_search_refuses_unregistered_frames(device, reference):
    frames, mjd, exp = _sequence("drift")
    want = reference.check_registration(frames, (mjd - mjd[0]) * 24.0)
    assert want["registered"] == 0
    with pytest.raises(RuntimeError) as e:
        device.search(frames, mjd, exp, fwhm_px=2.0, null_runs=1, align="check")
    assert want["message"] in str(e.value)
    with pytest.raises(RuntimeError, match="does not align frames"):
        device.search(frames, mjd, exp, fwhm_px=2.0, null_runs=1, align="auto")


def test_search_with_check_equals_search_without(device, reference):
    """Registered frames given in shuffled order: the search sorts them by time,
    checks the sorted sequence as the reference does, and returns what the
    search without the check returns, plus the check."""
    frames, mjd, exp = _sequence("registered")
    perm = np.random.default_rng(3).permutation(mjd.size)
    kw = dict(fwhm_px=2.0, null_runs=1)
    plain = device.search(frames[perm], mjd[perm], exp[perm], **kw)
    checked = device.search(frames[perm], mjd[perm], exp[perm], align="check", **kw)
    assert checked["registration"] == reference.check_registration(frames, (mjd - mjd[0]) * 24.0)
    assert checked["registration"]["measured"] == 1 and checked["registration"]["registered"] == 1
    assert plain["registration"]["measured"] == 0 and plain["registration"]["registered"] == 1
    assert checked["threshold"] == plain["threshold"] and checked["peaks"] == plain["peaks"]
    assert np.array_equal(checked["max_snr"], plain["max_snr"], equal_nan=True)
    assert np.array_equal(checked["best_v"], plain["best_v"])
