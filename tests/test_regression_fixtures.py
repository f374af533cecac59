"""The reference's real-data regression cases (tests/regression/*-cut.case) as
fixtures, checked without a GPU: the threshold the reference's search gives
equals its committed baseline's (baselines/<case>.csv, written to 3 decimals),
and, where the reference build is present, its search of the rebuilt frames
today equals the fixture bit for bit."""
import numpy as np
import pytest

from regression_cases import CASES, load_case, same_search


@pytest.mark.parametrize("case", CASES)
def test_fixture_threshold_equals_baseline(case):
    g = load_case(case)
    assert g["method"] == "null-fit gauss"
    assert round(g["threshold"], 3) == g["baseline_threshold"]
    assert g["frames"].shape[0] >= 11 and np.isfinite(g["frames"]).any()


@pytest.mark.parametrize("case", CASES)
def test_reference_search_equals_fixture(reference, case):
    g = load_case(case)
    prep = reference.prepare(g["frames"], g["mjd"], g["exptime"], reg_dx=g["reg_dx"], reg_dy=g["reg_dy"],
                             **g["params"])
    res = prep.search(backend="cpu", **g["params"])
    res["fwhm"] = prep.fwhm
    same_search(res, g)
