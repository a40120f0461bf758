"""Failure detection on the GPU without a GPU fault.

The plane kernel's wait for its bulk-copied plane is bounded.  With the limit
set to zero polls (edus_set_wait_limit) the waits run out: the kernel sets the
handle's status word, lets its copies land and returns; the next synchronising
call reports EDUS_ERR_TIMEOUT and clears the word; the handle, given its state
again, propagates correctly afterwards.  Nothing faults, traps or hangs.
"""
import numpy as np
import pytest

from test_gpu_parity import make_pair, model_input, rel

pytestmark = pytest.mark.gpu


def test_plane_wait_timeout_is_reported_and_handle_recovers(pkg, po, tmp_path):
    E = pkg.edus
    # 13 bands (169 planes: the persistent plane kernel, not the many-CTA path)
    # on 72 x 64 (4608 points: planes arrive by bulk copies)
    inp = model_input(pkg, tmp_path, "timeout", (72, 64, 1), nb=13, dt=0.01, envelope="gauss")
    cfg, o, s = make_pair(pkg, po, inp)
    rho0 = o.get("rho")
    s.set_wait_limit(0)
    with pytest.raises(E.EdusError) as ei:
        s.step(2)
        s.synchronize()
    assert ei.value.code == 3  # EDUS_ERR_TIMEOUT
    assert "bounded wait" in str(ei.value)
    s.synchronize()  # the status word was cleared once reported
    s.set_wait_limit(-1)
    s.set_state(rho0)
    s.time = 0.0
    s.step(5)
    o.step(5)
    assert rel(s.get_state(), o.get("rho")) < 1e-10
