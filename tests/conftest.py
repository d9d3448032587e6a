import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = ["convex6_rot", "carved10_rot", "convex5_axis", "single_tet", "cfg0_convex24"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU test")


def has_reference_sources():
    import oracle

    return os.path.isdir(oracle.REF_SOURCES)


def load_golden(name):
    """A golden case with its inputs (regenerated from seeds where the
    fixture stores only a checksum) and the reference outputs."""
    import vfray_b200 as vb
    from tests.golden.make_golden import checksum, make_inputs

    d = dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))
    d["name"] = name
    d["W"], d["H"], d["n_ext"] = int(d["W"]), int(d["H"]), int(d["n_ext"])
    d["psi"] = vb.psi_table()
    assert checksum(d["psi"]) == str(d["psi_sha256"]), "generated psi table drifted"
    if "vert" not in d:
        vert, tet, tf = make_inputs(name)
        p = vb.prepare(vert, tet)
        d.update(vert=p["vert"], tet=p["tet"], con=p["con"], extf=p["extf"], tf=tf)
        assert np.array_equal(p["lmt"], d["lmt"])
    assert checksum(d["vert"], d["tet"], d["con"], d["extf"], d["tf"]) == str(d["input_sha256"])
    return d


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle

    return oracle.Oracle()


@pytest.fixture(scope="session")
def renderer():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import vfray_b200 as vb

    r = vb.Renderer(0)
    yield r
    r.close()
