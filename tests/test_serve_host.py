"""Host logic of the request server (gmpt.serve.serve) with a fake runner:
which requests become one call, and how the results of a merged call are
handed back per request.  No GPU: the runner only records what it is asked."""
import numpy as np

from gmpt import serve as S


class FakeRunner:
    def __init__(self):
        self.calls = []

    def build(self, run):
        return sum(r.n for r in run), 0, 0

    def features(self, run, n, kb, vb):
        return np.zeros(8, np.float32)

    def put(self, run, k, n, kb, vb):
        self.calls.append(("put", [r.i for r in run], k))

    def get(self, n, kb):
        self.calls.append(("get", n))
        return np.arange(n, dtype=np.int32)

    def mixed(self, run, k, n, kb, vb):
        self.calls.append(("mixed", [r.i for r in run], k))
        # read results in read order: request i's keys answer 1000 * i + j
        return np.concatenate([1000 * r.i + np.arange(r.n, dtype=np.int32) for r in run if r.kind == "get"])


def stream(kinds, tenants=None):
    tenants = tenants or [0] * len(kinds)
    return [S.Request(i, k, t, 3 + i, 0.5, 0.5, i) for i, (k, t) in enumerate(zip(kinds, tenants))]


def test_mixed_window_is_one_call_in_request_order():
    reqs = stream(["put", "get", "put", "get", "get"])
    for r in reqs:
        r.arrival = 0.0  # all queued at once: one drained window
    fr = FakeRunner()
    res = S.serve(fr, reqs, lambda *a: 3, batching=True, mixed=True)
    assert fr.calls == [("mixed", [0, 1, 2, 3, 4], 3)]
    assert res.groups == 1
    for r, got in zip(reqs, res.get_sizes):
        if r.kind == "put":
            assert got is None
        else:
            assert np.array_equal(got, 1000 * r.i + np.arange(r.n))


def test_single_kind_window_and_per_kind_merging():
    reqs = stream(["get", "get", "get"])
    for r in reqs:
        r.arrival = 0.0
    fr = FakeRunner()
    res = S.serve(fr, reqs, lambda *a: 0, batching=True, mixed=True)
    assert fr.calls == [("get", sum(r.n for r in reqs))]  # no mixed call without a put
    assert [len(x) for x in res.get_sizes] == [r.n for r in reqs]
    # without mixed, a put/get window splits into same-kind runs per tenant
    reqs = stream(["put", "get", "put", "get"], tenants=[0, 1, 1, 0])
    for r in reqs:
        r.arrival = 0.0
    fr = FakeRunner()
    res = S.serve(fr, reqs, lambda *a: 2, batching=True, mixed=False)
    # tenant 0: put 0, get 3; tenant 1: get 1, put 2 -> put [0]; gets 1 and 3; put [2]
    assert fr.calls == [("put", [0], 2), ("get", reqs[1].n + reqs[3].n), ("put", [2], 2)]
    assert np.array_equal(res.get_sizes[1], np.arange(reqs[1].n))
    assert np.array_equal(res.get_sizes[3], reqs[1].n + np.arange(reqs[3].n))


def test_one_at_a_time_server_never_merges():
    reqs = stream(["put", "get", "put"])
    for r in reqs:
        r.arrival = 0.0
    fr = FakeRunner()
    res = S.serve(fr, reqs, lambda *a: 1, batching=False, mixed=True)
    assert [c[0] for c in fr.calls] == ["put", "get", "put"]
    assert res.groups == 3
