"""Pin the CPU oracle against the reference's golden vectors and against OpenCV.

Mirrors test/opencv.jl and the fixture cases of test/peak.jl: ZNCC surfaces within 1e-4 of
OpenCV with identical peaks, low-contrast windows recovered at the centre, pyrUp steps within
1e-6 and cascades within 1e-4, and the peak fixtures exactly.
"""

import os
from pathlib import Path

import numpy as np
import pytest

# The reference checkout, when present (its full fixture tree): AUTORIFT_REFERENCE names it.
_REF_ENV = os.environ.get("AUTORIFT_REFERENCE")
REFERENCE = Path(_REF_ENV) if _REF_ENV else None


def _zncc_cases(g):
    return [c for c in g.cases("matchtemplate__zncc") if "lowcontrast" not in c]


def test_zncc_surfaces_match_reference_fixtures(O, ref_golden):
    cases = _zncc_cases(ref_golden)
    assert len(cases) >= 20
    worst = 0.0
    for case in cases:
        a = ref_golden[case]
        r = ref_golden.meta[case]["search_radius"]
        s, deg = O.correlate(a["search"], a["chip"], r)
        assert not deg
        assert s.shape == a["expected"].shape
        worst = max(worst, float(np.abs(s.astype(np.float64) - a["expected"]).max()))
        assert O.peak_index(s) == O.peak_index(a["expected"]), case
    assert worst < 1e-4


def test_lowcontrast_recovered_where_opencv_gives_up(O, ref_golden):
    cases = ref_golden.cases("matchtemplate__zncc")
    cases = [c for c in cases if "lowcontrast" in c]
    assert cases
    bound = 1.0 + 2048 * np.finfo(np.float32).eps
    for case in cases:
        a = ref_golden[case]
        r = ref_golden.meta[case]["search_radius"]
        assert np.all(a["expected"] == 0)  # OpenCV declined to answer
        s, _ = O.correlate(a["search"], a["chip"], r)
        assert O.peak_index(s) == (r, r)
        assert abs(float(s.max()) - 1.0) <= 1e-3
        assert np.all(np.isfinite(s)) and np.all(np.abs(s) <= bound)


def test_dc_offset_cancels(O, ref_golden):
    plain = ref_golden["matchtemplate__zncc_c32_r25_float32_plain"]
    off = ref_golden["matchtemplate__zncc_c32_r25_float32_dc_offset"]
    s1, _ = O.correlate(plain["search"], plain["chip"], 25)
    s2, _ = O.correlate(off["search"], off["chip"], 25)
    assert O.peak_index(s1) == O.peak_index(s2)
    assert np.abs(s1 - s2).max() < 1e-4


def test_pyrup_steps_and_cascades(O, ref_golden):
    worst_step = 0.0
    for case in ref_golden.cases("pyrup__"):
        a = ref_golden[case]
        params = ref_golden.meta[case]
        cur = a["src"]
        # A step fixture is one pyrUp of a source at that level; a cascade runs log2(factor).
        for _ in range(1 if params["single_step"] else params["steps"]):
            cur = O.pyrup(cur)
        err = float(np.abs(cur - a["expected"]).max())
        if params["single_step"]:
            worst_step = max(worst_step, err)
        else:
            assert err < 1e-4, case
    assert worst_step < 1e-6


def test_peak_fixtures(O, ref_golden):
    for case in ref_golden.cases("peak__"):
        a = ref_golden[case]
        params = ref_golden.meta[case]
        i, j = O.peak_index(a["surface"])
        assert (i, j) == tuple(params["row_col_0based"])
        assert a["surface"][i, j] == np.float32(params["maxval"])


def test_opencv_golden(O, cv_golden):
    for case in cv_golden.meta["cases"]:
        a = cv_golden[case["name"]]
        s, deg = O.correlate(a["search"], a["chip"], (case["rx"], case["ry"]))
        assert not deg
        assert np.abs(s - a["expected"]).max() < 1e-4, case["name"]
        assert O.peak_index(s) == O.peak_index(a["expected"]), case["name"]
        assert O.peak_index(s) == tuple(case["shift_rc"])
    for k in range(3):
        a = cv_golden[f"pyrup_cascade_{k}"]
        cur = a["src"]
        for _ in range(4):
            cur = O.pyrup(cur)
        assert np.abs(cur - a["expected"]).max() < 1e-4


@pytest.mark.skipif(REFERENCE is None or not (REFERENCE / "test" / "fixtures").is_dir(),
                    reason="reference checkout not present")
def test_all_27_reference_surfaces(O):
    """The full fixture matrix of test/opencv.jl:22-67, read from the reference tree."""
    import json

    root = REFERENCE / "test" / "fixtures" / "matchtemplate"
    n = 0
    worst = 0.0
    for cs in (32, 64, 128):
        for r in (6, 10, 25):
            for dt in ("uint8", "float32"):
                for var in ("plain", "dc_offset"):
                    d = root / f"zncc_c{cs}_r{r}_{dt}_{var}"
                    if not d.is_dir():
                        continue
                    meta = json.loads((d / "meta.json").read_text())
                    arr = {k: np.fromfile(d / f"{k}.bin", dtype=v["dtype"]).reshape(v["shape"])
                           for k, v in meta["arrays"].items()}
                    s, _ = O.correlate(arr["search"], arr["chip"], r)
                    worst = max(worst, float(np.abs(s - arr["expected"]).max()))
                    assert O.peak_index(s) == O.peak_index(arr["expected"])
                    n += 1
    assert n == 27
    assert worst < 1e-4
