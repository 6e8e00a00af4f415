"""Failure detection without a fault: the bounded in-kernel wait that the copy pipelines use
gives up on a barrier that nothing completes, records MMN_ERR_TIMEOUT in the workspace's
status word, and returns; the host reads the status, and the same context then runs a
backprojection that matches the one taken before the timeout.  The completed-barrier case
leaves the status clear.  The copy pipelines give up after one second of %globaltimer; the
probe takes its own limit, and the measured wait must last at least that long."""
import numpy as np
import pytest

from mmnorm_b200 import scenes

pytestmark = pytest.mark.gpu


def _probe(ws, limit_us, arrive):
    import torch
    from mmnorm_b200 import _lib, ops
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.current_stream(ws.device)
    start.record(stream)
    rc = _lib.load().mmn_wait_timeout_probe(limit_us, arrive, ops._vp(ws), stream.cuda_stream)
    end.record(stream)
    _lib.check(rc, "mmn_wait_timeout_probe")
    status = ops.read_status(ws)
    return status, start.elapsed_time(end)


def test_bounded_wait_times_out_and_context_survives(cuda_dev):
    import torch
    from mmnorm_b200 import _lib, ops
    sc = scenes.sphere_scene(seed=4, n_ap=8, nf=32, n_vox=8, n_pts=16)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=cuda_dev)
    args = (t(sc.x_locs), t(sc.y_locs), t(sc.z_locs), t(sc.antenna_locs),
            t(np.zeros((1, 3), np.float32)), t(sc.meas), sc.wavelength, sc.slope)
    i0, v0 = ops.backproject(*args)
    torch.cuda.synchronize()

    ws = torch.zeros(64, dtype=torch.uint8, device=cuda_dev)
    st_done, ms_done = _probe(ws, 1000000, 1)
    assert st_done == _lib.MMN_OK and ms_done < 100.0
    st_small, ms_small = _probe(ws, 2000, 0)
    st_large, ms_large = _probe(ws, 50000, 0)
    print("bounded wait: completed %.3f ms, 2 ms limit %.3f ms, 50 ms limit %.3f ms"
          % (ms_done, ms_small, ms_large))
    assert st_small == _lib.MMN_ERR_TIMEOUT and st_large == _lib.MMN_ERR_TIMEOUT
    assert ops.read_status(ws) == _lib.MMN_OK  # read_status cleared the word
    assert 1.99 <= ms_small < 100.0 and 49.9 <= ms_large < 250.0
    assert _lib.load().mmn_wait_timeout_probe(20000000, 0, ops._vp(ws), None) == \
        _lib.MMN_ERR_INVALID_ARGUMENT

    i1, v1 = ops.backproject(*args)
    torch.cuda.synchronize()
    assert torch.equal(i0, i1) and torch.equal(v0, v1)
