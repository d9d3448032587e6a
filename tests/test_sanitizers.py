"""The library's host code (precomputation, file readers and writers, mesh
validation and walk records) built with AddressSanitizer and
UndefinedBehaviorSanitizer and run over a carved mesh whose .off file is
large enough for the chunk-parallel reader, with the hashed adjacency
build on all threads.  The reference's own host code had exactly these bug
classes (a stack overflow in its face cache, a new[]/free mismatch), so
this build has to show it has none."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from vfray_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "vfray_b200", "csrc")


@pytest.mark.slow
def test_host_code_under_asan_ubsan(tmp_path):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no g++")
    exe = str(tmp_path / "sanitize_host")
    subprocess.run([cxx, "-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer",
                    "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
                    "-I", os.path.join(ROOT, "include"), "-I", CSRC,
                    os.path.join(ROOT, "tests", "native", "sanitize_host.cc"),
                    os.path.join(CSRC, "precomp.cc"), os.path.join(CSRC, "vfr_validate.cc"),
                    "-o", exe, "-lpthread", "-ldl"], check=True, timeout=600)
    vert, tet = synth.make_mesh(84, carved=True, view_seed=None)
    off = str(tmp_path / "mesh.off")
    synth.write_off(off, vert, tet)
    assert os.path.getsize(off) > (64 << 20)  # the reader's chunk-parallel path
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    r = subprocess.run([exe, off, str(tmp_path)], capture_output=True, text=True, timeout=900,
                       env=env)
    assert r.returncode == 0, r.stderr[-4000:]
    assert r.stdout.startswith("ok"), r.stdout
