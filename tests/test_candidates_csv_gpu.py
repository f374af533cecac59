"""The candidate file of a device search (ft_b200_result_candidates_csv,
ft_b200_write_candidates_csv) is the reference's write_candidates_csv
(io.cpp:82-115) text byte for byte, and its track points
(ft_b200_result_track_point) are the reference's ft_get_track_point values: on
the golden cases (the frames made again by the reference's simulate()), and
against the live reference."""
import json

import numpy as np
import pytest

from conftest import golden
from test_candidates_csv import csv_cases

pytestmark = pytest.mark.gpu


def _setup(name):
    return json.loads(str(golden("candidates_csv_small.npz")[name + "_setup"]))


@pytest.mark.parametrize("case", range(2))
def test_search_file_matches_golden(device, reference, case, tmp_path):
    name, _, _, _, _, want = csv_cases()[case]
    setup = _setup(name)
    frames, mjd, exp = reference.simulate(**setup["simulate"])
    path = tmp_path / "candidates.csv"
    got = device.search(frames, mjd, exp, csv_path=path, **setup["search"])
    assert got["candidates_csv"] == want
    assert path.read_text() == want
    assert np.array_equal(got["track_points"], golden("candidates_csv_small.npz")[name + "_tracks"])


def test_search_file_matches_live_reference(device, reference, tmp_path):
    """A third sequence (seven movers, a fixed threshold of S/N 4) against the
    reference's own search and file."""
    sim = dict(width=112, height=96, nframes=14, nstars=80, nmovers=7, seed=33)
    kw = dict(fwhm_px=2.5, threshold_snr=4.0)
    frames, mjd, exp = reference.simulate(**sim)
    ref = reference.prepare(frames, mjd, exp, **kw).search(csv_path=str(tmp_path / "ref.csv"), backend="cpu", **kw)
    got = device.search(frames, mjd, exp, **kw)
    assert len(ref["candidates"]) > 0
    assert got["candidates_csv"] == ref["candidates_csv"]
    assert np.array_equal(got["track_points"], ref["track_points"])


def test_unwritable_path_is_an_error(device, tmp_path):
    name, *_ = csv_cases()[1]
    setup = _setup(name)
    g = golden("search_small.npz")
    with pytest.raises(RuntimeError, match="cannot write"):
        device.search(g["raw"], g["mjd"], g["exptime"], csv_path=tmp_path / "missing" / "c.csv",
                      **dict(setup["search"], fwhm_px=2.5))
