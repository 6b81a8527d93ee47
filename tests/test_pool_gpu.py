"""Handles take their device memory from the library's per-device pool and
give it back in the order of their stream, without waiting for the device
(icar_adv_destroy).  A handle destroyed while its steps are still queued
must let them finish on its memory, and handles created right after, which
may receive that memory, must compute exactly what they would on fresh
memory."""
import numpy as np
import pytest

from hicar_b200 import synth
from hicar_b200.advection import Domain, Options, adv_init, advect

pytestmark = pytest.mark.gpu


def _run(case, nsteps, path=0, keep=True):
    d = Domain.from_case(case)
    opts = Options()
    adv_init(d, opts)
    d.set_path(path)
    for _ in range(nsteps):
        advect(d, opts, case.dt)
    if not keep:
        d.close()          # steps still queued: destroy does not wait for them
        return None
    out = {k: d.fetch(k).copy() for k in case.species}
    d.close()
    return out


@pytest.mark.parametrize("path", [0, 3])
def test_destroy_with_queued_work_then_reuse(oracle_lib, path):
    case = synth.config2(seed=21, nx=130, ny=90, nz=20)
    want = _run(case, 3, path)
    if path == 0:
        ref = oracle_lib.run_steps(case, oracle_lib.make_opts(), case.dt, 3)
        for k in ref:
            assert np.array_equal(want[k], ref[k]), k
    for _ in range(4):
        _run(case, 6, path, keep=False)     # destroyed with six steps in flight
        got = _run(case, 3, path)           # may reuse that memory
        for k in want:
            assert np.array_equal(got[k], want[k]), k


def test_destroy_on_caller_stream_then_reuse(oracle_lib):
    """The same on a caller's stream (icar_adv_set_stream), switched to
    while the handle's own stream still has its upload queued."""
    import ctypes as C

    import torch

    from hicar_b200 import _lib as L
    case = synth.config2(seed=22, nx=100, ny=70, nz=16)
    ref = oracle_lib.run_steps(case, oracle_lib.make_opts(), case.dt, 3)
    lib = L.load()
    st = torch.cuda.Stream()
    for _ in range(3):
        d = Domain.from_case(case)
        opts = Options()
        adv_init(d, opts)
        L.check(lib.icar_adv_set_stream(d.handle, C.c_void_p(st.cuda_stream)), d.handle)
        for _ in range(5):
            advect(d, opts, case.dt)
        d.close()                       # five steps queued on the caller's stream
        got = _run(case, 3)
        for k in ref:
            assert np.array_equal(got[k], ref[k]), k
    st.synchronize()
