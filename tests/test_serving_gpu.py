"""Continuous batching on the device: a stream of runs of different grids and
lengths, admitted by free device memory while others are in flight, each
finishing with exactly the state it reaches alone (FP32 form, zero ULP: no
arithmetic couples runs that share a launch)."""
import numpy as np
import pytest

from nimbus_b200 import cuda
from nimbus_b200.ensemble import Request
from nimbus_b200.initial import Case, initial_state
from nimbus_b200.run import PROGNOSTIC, EngineRun
from nimbus_b200.serve import Server, serve_one_by_one, summarize

pytestmark = pytest.mark.gpu


def _requests():
    shapes = [(24, 24, 12), (40, 36, 16), (16, 20, 10), (32, 32, 14), (20, 28, 12), (36, 18, 16)]
    steps = [5, 3, 6, 2, 4, 3]
    arrivals = [0.0, 0.0, 0.02, 0.05, 0.05, 0.12]
    out = []
    for r, (shape, n, t) in enumerate(zip(shapes, steps, arrivals)):
        case = Case(*shape, 500.0, 500.0, 20000.0 / shape[2] / 4, 3.0, noise_amp=0.2, seed=9, member=r,
                    bubble_rh=4000.0)
        out.append(Request(r, case, n, t))
    return out


@pytest.fixture(scope="module")
def ctx():
    c = cuda.Context(0)
    yield c
    c.close()


def test_each_served_result_equals_the_run_alone(ctx):
    import torch
    reqs = _requests()
    prepared = {r.rid: initial_state(r.case) for r in reqs}
    # Leave room for about three of these runs at a time so admission queues.
    free, _ = torch.cuda.mem_get_info()
    probe = cuda.Engine(ctx)
    st0, base0 = prepared[1]
    d = cuda.member_desc(reqs[1].case.shape, (500.0, 500.0, reqs[1].case.dz), 3.0, 4, reqs[1].case.bc, base0)
    per = probe.member_bytes(d)
    probe.close()
    server = Server(ctx, reserve_bytes=max(0, free - int(3.2 * per)), keep_results=True)
    done, makespan = server.serve(reqs, prepared)
    server.close()
    assert sorted(c.rid for c in done) == [r.rid for r in reqs]
    assert all(c.status == 0 and c.latency_s > 0 for c in done)
    s = summarize(done, makespan)
    assert s["p99_s"] >= s["p50_s"] > 0 and s["cell_updates_per_s"] > 0
    for c in done:
        r = reqs[c.rid]
        alone = EngineRun(ctx, cuda.PRECISION_FP32)
        mid = alone.admit(r.case, *prepared[r.rid])
        alone.step(r.steps)
        want = alone.read(mid)
        alone.close()
        for k in PROGNOSTIC:
            a, b = c.state[k], want[k]
            assert np.count_nonzero(a.view(np.uint32) != b.view(np.uint32)) == 0, (c.rid, k)
    # The one-by-one plain path reaches the same states.
    plain, _ = serve_one_by_one(ctx, reqs[:3], prepared=prepared, keep_results=True)
    served = {c.rid: c for c in done}
    for c in plain:
        for k in PROGNOSTIC:
            assert np.array_equal(c.state[k].view(np.uint32), served[c.rid].state[k].view(np.uint32)), (c.rid, k)
