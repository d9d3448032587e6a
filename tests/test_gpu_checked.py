"""The checked build (-DVFR_CHECKED): every id a kernel reads from memory is
range-checked.  On a valid mesh it renders what the product build renders;
an id overwritten on the device past the upload's validation comes back as
VFR_DEV_RANGE, not as an out-of-range access, and the context stays usable.
Each case runs in a process of its own (tests/checked_case.py), so the
checked library is the only one loaded there."""
import json
import os
import subprocess
import sys

import pytest

from tests.conftest import ROOT

pytestmark = pytest.mark.gpu

VFR_DEV_RANGE = 4


def run_case(case):
    p = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "checked_case.py"), case],
                       cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-3000:]
    return json.loads(p.stdout.strip().splitlines()[-1])


def assert_clean(c):
    assert c["ref_steps_equal"] and c["comp_steps_equal"], c
    assert c["ref_rgb_maxdiff"] <= 2 and c["comp_rgb_maxdiff"] <= 2, c
    assert c["status"] == [0, 0], c


def test_checked_build_renders_like_the_product():
    out = run_case("clean")
    assert out["loaded"] == "libvfray_b200_checked.so"
    assert_clean(out)


@pytest.mark.parametrize("case", ["walk", "tet", "extf"])
def test_bad_id_is_reported_not_followed(case):
    out = run_case(case)
    assert out["error"] and "range=4" in out["error"], out
    assert out["status"] & VFR_DEV_RANGE, out
    assert_clean(out["after"])
