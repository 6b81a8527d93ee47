"""Host side of the served form, without a GPU: the Poisson request stream
of the served workload (20 requests/s for 120 s, lognormal area with a
median of 256^2, sides clipped to 64..1024, nz ~ U[20, 60], steps ~
U[50, 500]) and the admission footprint the server charges each request."""
import numpy as np

from hicar_b200.advection import Options
from hicar_b200.serve import Request, footprint, poisson_requests


def test_request_stream_has_the_workload_distribution():
    reqs = poisson_requests(20.0, 120.0, seed=3)
    n = len(reqs)
    assert abs(n - 2400) < 4 * np.sqrt(2400)                     # Poisson count, 4 sigma
    t = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(t) > 0) and t[-1] <= 120.0
    assert [r.rid for r in reqs] == list(range(n))
    sides = np.array([(r.nx, r.ny) for r in reqs])
    assert sides.min() >= 64 and sides.max() <= 1024
    area = sides[:, 0] * sides[:, 1]
    assert abs(np.median(area) / 256 ** 2 - 1.0) < 0.1
    nz = np.array([r.nz for r in reqs])
    steps = np.array([r.steps for r in reqs])
    assert nz.min() >= 20 and nz.max() <= 60 and steps.min() >= 50 and steps.max() <= 500
    assert len({r.seed for r in reqs}) == n                      # every request its own inputs
    again = poisson_requests(20.0, 120.0, seed=3)
    assert [(r.arrival, r.nx, r.ny, r.nz, r.steps) for r in again] == \
        [(r.arrival, r.nx, r.ny, r.nz, r.steps) for r in reqs]


def test_footprint_grows_with_the_request(cuda_lib):
    opts = Options()
    base = footprint(Request(0, 128, 96, 20, 50, 0), opts)
    assert base > 4 * 128 * 96 * 20 * 12 * 2                     # at least two copies of every species
    assert footprint(Request(0, 256, 96, 20, 50, 0), opts) > base
    assert footprint(Request(0, 128, 192, 20, 50, 0), opts) > base
    assert footprint(Request(0, 128, 96, 40, 50, 0), opts) > base
    assert footprint(Request(0, 128, 96, 20, 50, 0, species=("qv", "theta")), opts) < base
    assert footprint(Request(0, 128, 96, 20, 500, 0), opts) == base  # steps cost time, not memory
