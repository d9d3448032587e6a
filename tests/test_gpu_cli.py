"""The drop-in driver: `vfRay <volume>` reads <dir>/<volume>.off, computes and
writes the missing .con .tf .extf .lmt next to it (as vfRay.cu:745-842 does),
renders 512x512 and writes <volume>_gpu_img.ppm.  A second run reads the
files back (six-digit .lmt/.tf, as the reference's later runs do); its image
is checked against the oracle rendered from the same read-back files."""
import os
import subprocess

import numpy as np
import pytest

import vfray_b200 as vb
from vfray_b200 import synth
from tests.conftest import ROOT

pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "vfray_b200", "bin", "vfRay")


def read_ppm(path):
    data = open(path, "rb").read()
    assert data.startswith(b"P6\n")
    parts = data.split(b"\n", 3)
    w, h = map(int, parts[1].split())
    assert parts[2] == b"255"
    return np.frombuffer(parts[3], np.uint8).reshape(h, w, 3)


def test_cli_renders_like_the_oracle(tmp_path, oracle_lib):
    if not os.path.exists(CLI):
        pytest.skip("driver not built")
    ds = tmp_path / "tet_offs"
    ds.mkdir()
    vert, tet = synth.make_mesh(9, carved=True, view_seed=5)
    vb.write_off(str(ds / "blob.off"), vert, tet)
    vb.write_tf(str(ds / "blob.tf"), synth.transfer_function(2))
    for run in range(2):
        out = subprocess.run([CLI, "--dir", str(ds), "blob"], cwd=tmp_path, capture_output=True,
                             text=True, timeout=300)
        assert out.returncode == 0, out.stdout + out.stderr
        assert "# VisFaces" in out.stdout
    for ext in ("con", "extf", "lmt"):
        assert (ds / f"blob.{ext}").exists()
    img = read_ppm(tmp_path / "blob_gpu_img.ppm")
    # the files as written, read back
    v, t = vb.read_off(str(ds / "blob.off"))
    v = vb.normalize(v)
    con, n_ext = vb.read_con(str(ds / "blob.con"))
    extf = vb.read_extf(str(ds / "blob.extf"))
    lmt = vb.read_lmt(str(ds / "blob.lmt"))
    tf = vb.read_tf(str(ds / "blob.tf"))
    p = vb.prepare(vert, tet)
    assert np.array_equal(con, p["con"]) and extf.shape[0] == n_ext
    m = oracle_lib.mesh(v, t, con, extf, tf, vb.psi_table(), lmt[0])
    o = oracle_lib.render_ref(m, 512, 512)
    diff = np.abs(img.astype(int) - o["rgb8"].astype(int))
    assert diff.max() <= 2
    assert (img.sum(-1) > 0).sum() > 1000


def test_cli_binary_cache(tmp_path):
    """--cache writes <volume>.vfrb after the text files and reads it on the
    next run; both runs give the same image."""
    if not os.path.exists(CLI):
        pytest.skip("driver not built")
    ds = tmp_path / "tet_offs"
    ds.mkdir()
    vert, tet = synth.make_mesh(8, carved=True, view_seed=3)
    vb.write_off(str(ds / "blob.off"), vert, tet)
    imgs = []
    for run in range(2):
        out = subprocess.run([CLI, "--cache", "--dir", str(ds), "--out", f"r{run}.ppm", "blob"],
                             cwd=tmp_path, capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stdout + out.stderr
        assert ("Writing" if run == 0 else "Reading") in out.stdout and "binary cache" in out.stdout
        imgs.append(read_ppm(tmp_path / f"r{run}.ppm"))
    assert (ds / "blob.vfrb").exists()
    assert np.array_equal(imgs[0], imgs[1]) and (imgs[0].sum(-1) > 0).sum() > 1000


def test_cli_usage_and_missing_file(tmp_path):
    if not os.path.exists(CLI):
        pytest.skip("driver not built")
    out = subprocess.run([CLI], capture_output=True, text=True, timeout=60)
    assert out.returncode == 1 and "use:" in out.stdout
    out = subprocess.run([CLI, "--dir", str(tmp_path), "nothing"], capture_output=True, text=True,
                         timeout=60)
    assert out.returncode == 1 and "Cannot read" in out.stdout
