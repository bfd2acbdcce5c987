"""Served queries with continuous batching: requests that arrive while others are on the device are
admitted as memory frees, and every result equals the same request solved alone (bit for bit)."""
import numpy as np
import pytest

from exaca_b200 import serve


def test_request_stream_seeded():
    a = serve.request_stream(50, rate=200.0, seed=4)
    assert a == serve.request_stream(50, rate=200.0, seed=4)
    t = np.array([x[0] for x in a])
    assert t[0] == 0.0 and np.all(np.diff(t) >= 0)
    # Poisson: mean gap near 1/rate
    assert 0.5 / 200 < np.diff(t).mean() < 2.0 / 200
    assert all(48 <= p[k] <= 256 for _, p in a for k in ("nx", "ny", "nz"))


@pytest.mark.gpu
def test_each_result_same_alone_and_in_the_mix(lib):
    reqs = serve.request_stream(8, rate=400.0, seed=21, side=(10, 24))
    alone = serve.sequential_plain(reqs)
    # a budget that holds only part of the stream at once forces admission as memory frees
    from exaca_b200 import batch
    sizes = [p.slot_bytes() for p in batch.build_problems([prm for _, prm in reqs])]
    mixed = serve.serve(reqs, budget_bytes=3 * max(sizes), chunk_cycles=200, keep_results=True,
                        list_capacity=1 << 22)
    for k in range(len(reqs)):
        g, c, cyc = mixed["results"][k]
        ga, ca, cyca = alone["results"][k]
        assert cyc == cyca, f"request {k}: cycle {cyc} vs {cyca} alone"
        assert np.array_equal(g, ga) and np.array_equal(c, ca), f"request {k} differs from its solve alone"
    assert all(x is not None and x > 0 for x in mixed["latency"])
