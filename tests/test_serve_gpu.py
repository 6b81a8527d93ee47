"""Served form: continuous batching under a memory budget.  Every request's
result must be the same alone and in the mix."""
import numpy as np
import pytest

from hicar_b200 import synth
from hicar_b200.advection import Domain, Options, step
from hicar_b200.serve import Request, Server, footprint

pytestmark = pytest.mark.gpu


def alone(req: Request, path: int = 0) -> dict:
    import torch
    fields, dt = synth.device_member(req.nx, req.ny, req.nz, req.seed, species=req.species)
    d = Domain.create_on_device(fields, req.nx, req.ny, req.nz, 4000.0, Options(), forcing=True)
    d.set_path(path)
    for _ in range(req.steps):
        step(d, Options(), dt)
    out = {}
    for k in req.species:
        t = torch.empty(req.ny * req.nz * req.nx, dtype=torch.float32, device="cuda")
        d.fetch_device(k, t)
        d.sync()
        out[k] = t.cpu().numpy().reshape(req.ny, req.nz, req.nx)
    d.close()
    return out


def test_results_are_the_same_alone_and_in_the_mix():
    sp = ("qv", "qc", "nr", "theta")
    reqs = [Request(0, 48, 40, 10, 6, 101, 0.00, sp), Request(1, 70, 33, 14, 9, 102, 0.00, sp),
            Request(2, 35, 61, 8, 4, 103, 0.02, sp), Request(3, 90, 50, 12, 7, 104, 0.04, sp),
            Request(4, 40, 40, 20, 5, 105, 0.05, sp), Request(5, 64, 64, 9, 8, 106, 0.06, sp)]
    # a budget for about three requests at a time: later arrivals queue, then
    # join the running batch as earlier ones finish
    budget = sorted(footprint(r, Options()) for r in reqs)[-3:]
    srv = Server(budget_bytes=sum(budget) + 1)
    for r in reqs:
        srv.submit(r)
    srv.run(max_wall=120)
    rep = srv.report()
    assert rep["requests"] == len(reqs)
    assert srv.peak_used <= srv.budget
    assert srv.peak_live >= 2                 # work of different requests overlapped
    assert rep["queueing_share"] >= 0
    for r in reqs:
        ref = alone(r)
        for k in sp:
            assert np.array_equal(r.result[k], ref[k]), (r.rid, k)
    srv.close()


def test_request_over_budget_is_refused():
    srv = Server(budget_bytes=1e6)
    with pytest.raises(ValueError):
        srv.submit(Request(0, 64, 64, 20, 3, 1))
    srv.close()


def test_single_pass_fast_results_are_the_same_alone_and_in_the_mix():
    """The server on the single-pass fast kernel: a request's result in the
    mix equals the same request run alone on that kernel (the batched and
    single-domain launches compute every tile the same way)."""
    sp = ("qv", "qc", "nr", "theta")
    reqs = [Request(0, 80, 70, 12, 5, 201, 0.00, sp), Request(1, 130, 60, 9, 7, 202, 0.00, sp),
            Request(2, 57, 90, 14, 4, 203, 0.03, sp)]
    srv = Server(path=3)
    for r in reqs:
        srv.submit(r)
    srv.run(max_wall=120)
    assert srv.report()["requests"] == len(reqs)
    for r in reqs:
        ref = alone(r, path=3)
        for k in sp:
            assert np.array_equal(r.result[k], ref[k]), (r.rid, k)
    srv.close()


def test_failed_requests_leave_the_batch_and_the_others_are_unaffected():
    """Failures injected on the host: request 1 fails while it is set up,
    request 2 after its third step (between steps, none of its work in
    flight).  Both are reported with their errors and leave the batch; the
    other requests finish with results identical to running them alone."""
    from hicar_b200.serve import InjectedFault
    sp = ("qv", "qc", "nr", "theta")
    reqs = [Request(0, 48, 40, 10, 6, 301, 0.00, sp), Request(1, 70, 33, 14, 5, 302, 0.00, sp),
            Request(2, 35, 61, 8, 7, 303, 0.00, sp), Request(3, 64, 52, 11, 8, 304, 0.01, sp)]

    def hook(req, stage, steps_done):
        if req.rid == 1 and stage == "setup":
            raise InjectedFault("injected set-up failure")
        if req.rid == 2 and stage == "step" and steps_done == 3:
            raise InjectedFault("injected failure between steps")

    srv = Server(fault_hook=hook)
    for r in reqs:
        srv.submit(r)
    srv.run(max_wall=120)
    rep = srv.report()
    assert rep["requests"] == 2 and rep["failed"] == 2
    assert reqs[1].error and "set-up failed" in reqs[1].error and reqs[1].result is None
    assert reqs[2].error and "after 3 steps" in reqs[2].error and reqs[2].result is None
    assert not srv.batch.members or all(m is not None for m in srv.batch.members)
    for r in (reqs[0], reqs[3]):
        assert r.error is None
        ref = alone(r)
        for k in sp:
            assert np.array_equal(r.result[k], ref[k]), (r.rid, k)
    srv.close()
