"""vfr_find_visible_static: stage (a) for callers that cannot let the library
allocate device memory (an application that owns the GPU's memory as a fixed
pool, or a frame loop where cudaMalloc's possible device synchronisation is
not allowed).  Its scratch is a fixed device array inside the library; the
test passes it device buffers it allocated itself and checks the result
against the allocating entry point, vfr_find_visible, on two calls in a row.
Collected last (file name) so that a run stopping at the first failure has
run every other test first."""
import ctypes as C

import numpy as np
import pytest

import vfray_b200 as vb
from vfray_b200 import _lib, synth
from tests.conftest import load_golden

pytestmark = pytest.mark.gpu


def _static_call(lib, vert_d, tet_d, extf_d, n_ext, vis_d, nvis_d, stream):
    return lib.vfr_find_visible_static(
        C.c_void_p(vert_d.data_ptr()), vert_d.shape[0], C.c_void_p(tet_d.data_ptr()),
        tet_d.shape[0], C.c_void_p(extf_d.data_ptr()), n_ext, C.c_void_p(vis_d.data_ptr()),
        C.c_void_p(nvis_d.data_ptr()), C.c_void_p(stream))


def _cases():
    d = load_golden("cfg0_convex24")
    yield "cfg0_convex24", d["vert"], d["tet"], d["con"], d["extf"], d["lmt"]
    d = load_golden("carved10_rot")
    yield "carved10_rot", d["vert"], d["tet"], d["con"], d["extf"], d["lmt"]
    vert, tet = synth.make_mesh(48, carved=True, view_seed=6)
    p = vb.prepare(vert, tet)
    yield "carved48", p["vert"], p["tet"], p["con"], p["extf"], p["lmt"]


def test_static_scratch_matches_allocating_entry_point():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = vb.load()
    with vb.Renderer(0) as r:
        r.upload_tables(synth.transfer_function(2))
        stream = torch.cuda.current_stream().cuda_stream
        for name, vert, tet, con, extf, lmt in _cases():
            mid = r.upload_mesh(vert, tet, con, extf, lmt)
            want, _ = r.find_visible(mid, extf.shape[0])
            r.release_mesh(mid)
            vert_d = torch.from_numpy(np.ascontiguousarray(vert, np.float32)).cuda()
            tet_d = torch.from_numpy(np.ascontiguousarray(tet, np.uint32).view(np.int32)).cuda()
            extf_d = torch.from_numpy(np.ascontiguousarray(extf, np.uint32).view(np.int32)).cuda()
            n_ext = extf.shape[0]
            for call in range(2):  # the scratch keeps the previous call's contents
                vis_d = torch.full((max(n_ext, 1),), -7, dtype=torch.int32, device="cuda")
                nvis_d = torch.full((1,), -7, dtype=torch.int32, device="cuda")
                rc = _static_call(lib, vert_d, tet_d, extf_d, n_ext, vis_d, nvis_d, stream)
                assert rc == _lib.VFR_OK, (name, call, rc)
                torch.cuda.synchronize()
                n = int(nvis_d.item())
                got = vis_d[:n].cpu().numpy().view(np.uint32)
                assert n == len(want), (name, call, n, len(want))
                assert np.array_equal(got, want), (name, call)


def test_static_rejects_oversize_and_bad_arguments():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = vb.load()
    too_many = _lib.load().vfr_find_visible_static
    buf = torch.zeros(16, dtype=torch.int32, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    # more external faces than the fixed scratch holds: refused before any GPU work
    assert too_many(p, 4, p, 1, p, (1 << 18) + 1, p, p, None) == _lib.VFR_ERR_BUDGET
    # missing buffers
    assert lib.vfr_find_visible_static(None, 4, p, 1, p, 4, p, p, None) == _lib.VFR_ERR_INVALID
    # misaligned vertex buffer
    bad = C.c_void_p(buf.data_ptr() + 4)
    assert lib.vfr_find_visible_static(bad, 4, p, 1, p, 4, p, p, None) == _lib.VFR_ERR_INVALID
    # misaligned outputs (written with 4-byte stores): refused on the host
    odd = C.c_void_p(buf.data_ptr() + 2)
    assert lib.vfr_find_visible_static(p, 4, p, 1, p, 4, odd, p, None) == _lib.VFR_ERR_INVALID
    assert lib.vfr_find_visible_static(p, 4, p, 1, p, 4, p, odd, None) == _lib.VFR_ERR_INVALID
