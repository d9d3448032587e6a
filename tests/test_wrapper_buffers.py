"""Buffer lifetimes in the Python wrappers of the served and batched forms,
without a GPU.

* Server: the image buffer of a request must stay referenced while the
  request is in flight.  vfr_server_wait returns VFR_ERR_TIMEOUT while the
  request is still queued or rendering (the server writes its image later),
  and the request's own status once it is done and forgotten.  The C server
  is replaced by a fake whose wait answers are scripted.
* Batch jobs: the output tensors whose addresses a job records stay alive as
  long as the job."""
import gc
import weakref

import numpy as np
import pytest

from vfray_b200 import _lib
from vfray_b200.serve import Server


class FakeLib:
    def __init__(self, answers):
        self.answers = list(answers)

    def vfr_server_wait(self, h, ticket, timeout_ms, info_ref):
        return self.answers.pop(0)

    def vfr_server_destroy(self, h):
        pass


def _server(answers):
    s = Server.__new__(Server)  # no renderer or C server behind it
    s.lib = FakeLib(answers)
    s.h = None
    s._outs = {}
    return s


def test_buffer_kept_across_a_timed_out_wait():
    s = _server([_lib.VFR_ERR_TIMEOUT, _lib.VFR_OK])
    out = np.empty((4, 4, 3), np.uint8)
    ref = weakref.ref(out)
    s._outs[7] = out
    del out
    with pytest.raises(_lib.VfrError) as e:
        s.wait(7, timeout_ms=1)
    assert e.value.status == _lib.VFR_ERR_TIMEOUT
    gc.collect()
    assert ref() is not None and 7 in s._outs  # still the server's to write
    img, _ = s.wait(7)
    assert img is ref() and 7 not in s._outs


def test_buffer_released_with_the_request_status():
    s = _server([_lib.VFR_ERR_BUDGET])
    s._outs[3] = np.empty((2, 2, 3), np.uint8)
    with pytest.raises(_lib.VfrError) as e:
        s.wait(3)
    assert e.value.status == _lib.VFR_ERR_BUDGET and 3 not in s._outs


def test_batch_job_keeps_its_output_tensors():
    """A batch job records raw device addresses of its outputs (a captured
    graph writes through them on every run); the job holds the tensors so
    that a caller's temporaries are not freed under it."""
    torch = pytest.importorskip("torch")
    from vfray_b200.batch import job

    t = torch.empty(2 * 2 * 3, dtype=torch.uint8)
    ref = weakref.ref(t)
    j = job(0, 2, 2, rgb8=t)
    assert j.rgb8_dev == t.data_ptr()
    del t
    gc.collect()
    assert ref() is not None
    del j
    gc.collect()
    assert ref() is None
