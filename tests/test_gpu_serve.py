"""Request loop over a forest of tenant tries: results never depend on the
schedule (configuration, merging of queued requests), and equal the
oracle's; the learned selector trains on measured times and picks
configurations; device-generated batches have the promised shape."""
import numpy as np
import pytest

import oracle as O
from gmpt import serve as S
from gmpt import tuner as TU
from gmpt import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev(gpu_lib):
    import torch

    return torch.device("cuda", 0)


def _oracle_roots(record, tenants):
    ts = {t.tid: O.OracleTrie(O.MODE_REF) for t in tenants}
    for batch, tids in record:
        for t in sorted(set(tids.tolist())):
            sel = np.nonzero(tids == t)[0]
            sub = batch.subset(sel)
            ts[t].puts(sub.keys_hexs, sub.keys_indexs, sub.values, sub.values_indexs)
    out = []
    for t in tenants:
        ts[t.tid].hash()
        out.append(ts[t.tid].root())
    return out


def test_served_stream_matches_oracle_under_every_schedule(gpu_lib, dev):
    tenants = S.make_tenants([0, 1500, 6000])
    reqs = S.make_stream(7, 40, tenants, 0.4, 50, 3000, load_frac=0.2)
    S.poisson_arrivals(reqs, 5000.0)  # dense arrivals: the batched server merges
    rng = np.random.default_rng(0)
    runs = []
    for batching, mixed in ((False, False), (True, False), (True, True)):
        r = S.Runner(gpu_lib, tenants, 0, dev, record=True)
        picks = []

        def policy(runner, run, n, kb, vb):
            k = int(rng.integers(len(TU.CONFIGS)))
            picks.append(k)
            return k

        res = S.serve(r, reqs, policy, batching, mixed=mixed)
        runs.append((r.roots(), res, r.record, picks))
        r.close()
    (roots_a, res_a, rec_a, picks_a), (roots_b, res_b, rec_b, _), (roots_c, res_c, rec_c, _) = runs
    assert roots_a == roots_b == roots_c
    assert roots_a == _oracle_roots(rec_a, tenants)
    assert roots_c == _oracle_roots(rec_c, tenants)
    assert len(set(picks_a)) > 3  # many configurations exercised
    assert res_b.groups < res_a.groups  # merging happened
    assert res_c.groups < res_b.groups  # mixed windows became single calls
    # lookups answer the same whichever way they were grouped
    for x, y, z in zip(res_a.get_sizes, res_b.get_sizes, res_c.get_sizes):
        assert (x is None) == (y is None) == (z is None)
        assert x is None or (np.array_equal(x, y) and np.array_equal(x, z))


def test_time_matrix_replicas_agree_and_selector_trains(gpu_lib, dev):
    tenants = S.make_tenants([0, 4000, 20000])
    reqs = S.make_stream(11, 30, tenants, 0.2, 100, 20000, load_frac=0.25)
    reps = [S.Runner(gpu_lib, tenants, 0, dev) for _ in TU.CONFIGS]
    T, G, F = S.time_matrix(reps, reqs)  # raises if any configuration changes a root
    roots = [r.roots() for r in reps]
    assert all(x == roots[0] for x in roots)
    puts = np.array([r.kind == "put" for r in reqs])
    assert np.all(np.isfinite(T[puts])) and np.all(np.isnan(T[~puts]))
    assert np.all(np.isfinite(G[~puts]))
    sel = TU.Selector(gpu_lib.Net(len(TU.FEATURES), 32, len(TU.CONFIGS), seed=3), TU.Autotuner())
    loss = sel.fit(F[puts], T[puts], max_epochs=200)
    assert np.isfinite(loss) and loss > 0
    v = sel.validation
    assert v["held_out"] > 0 and v["use_net"] == (v["net_regret"] <= v["rule_regret"])
    for f in F[puts]:
        assert 0 <= sel.choose(f) < len(TU.CONFIGS)
        assert sel._net_choice(f) in sel.cols
    # the rule's per-bucket choice is the measured fastest configuration there
    assert TU.regret(T[puts], [sel.rule.choose(f) for f in F[puts]]) <= TU.regret(
        T[puts], [TU.FIXED_PHASENU] * int(puts.sum()))
    for r in reps:
        r.close()


def test_generated_ids_keys_and_values(gpu_lib, dev):
    import torch

    n = 50000
    ids = torch.empty(n, dtype=torch.int64, device=dev)
    nn = gpu_lib.gen_ids(5, n, 1000, 1000, 0.3, 0.99, ids.data_ptr())
    h = ids.cpu().numpy()
    fresh = h >= 1000
    assert nn == fresh.sum() and abs(nn / n - 0.3) < 0.02
    assert np.array_equal(np.sort(h[fresh]), np.arange(1000, 1000 + nn))  # dense fresh ids
    old = h[~fresh]
    assert old.min() >= 0 and old.max() < 1000
    cnt = np.bincount(old, minlength=1000)
    assert cnt.max() > 20 * np.median(cnt[cnt > 0])  # skewed
    # same seed, same ids
    ids2 = torch.empty(n, dtype=torch.int64, device=dev)
    gpu_lib.gen_ids(5, n, 1000, 1000, 0.3, 0.99, ids2.data_ptr())
    assert torch.equal(ids, ids2)
    keys = torch.empty(n * 41 + 64, dtype=torch.uint8, device=dev)
    kidx = torch.empty(2 * n, dtype=torch.int32, device=dev)
    gpu_lib.gen_keys(9, ids.data_ptr(), n, 20, keys.data_ptr(), kidx.data_ptr())
    k = keys[: n * 41].cpu().numpy().reshape(n, 41)
    assert np.all(k[:, 40] == 16) and k[:, :40].max() <= 15
    # equal ids give equal keys
    for a in np.nonzero(~fresh)[0][:200]:
        b = np.nonzero(h == h[a])[0]
        assert all(np.array_equal(k[a], k[j]) for j in b[:5])
    assert np.array_equal(kidx.cpu().numpy()[0::2], np.arange(n) * 41)
    vals = torch.empty(n * 7 + 64, dtype=torch.uint8, device=dev)
    vidx = torch.empty(2 * n, dtype=torch.int64, device=dev)
    gpu_lib.gen_values(3, n, 7, vals.data_ptr(), vidx.data_ptr())
    assert np.array_equal(vidx.cpu().numpy()[1::2], np.arange(n) * 7 + 6)


def test_device_feature_sampler_matches_host_restatement(gpu_lib, dev):
    import torch

    from conftest import make_batch, nib

    rng = np.random.default_rng(3)
    for n in (1, 5, 64, 65, 1000):
        words = [bytes(rng.integers(0, 4, size=rng.integers(1, 9)).astype(np.uint8)) for _ in range(max(n // 3, 1))]
        keys = [nib(words[int(rng.integers(len(words)))] + bytes(rng.integers(0, 256, size=2).astype(np.uint8)))
                for _ in range(n)]
        b = make_batch(keys, [b"v"] * n)
        dk = torch.from_numpy(b.keys_hexs).to(dev)
        di = torch.from_numpy(b.keys_indexs).to(dev)
        got = gpu_lib.batch_features_device(dk.data_ptr(), di.data_ptr(), n, len(b.keys_hexs))
        want = TU.sample_stats(b.keys_hexs, b.keys_indexs)
        assert np.allclose(got, want, rtol=1e-5, atol=1e-5), (n, got, want)


def test_trained_selector_gains_over_fixed_schedules(gpu_lib, dev):
    """Train the selector on times measured for one stream; on a second
    stream's times, the library's selector (the network when its held-out
    regret is no worse than the rule's, else the rule) must cost less than
    running every put with the fixed LockNU schedule (what the reference
    does) or the fixed PhaseNU one, and the network alone less than fixed
    PhaseNU.  The network alone is not held to beat fixed LockNU on the
    unseen stream: trained on ~150 puts it can misjudge a batch unlike its
    training ones (its regret there is printed), which is what the
    held-out gate in front of it is for."""
    def matrix(seed, count):
        tenants = S.make_tenants([0, 20000, 100000])
        reqs = S.make_stream(seed, count, tenants, 0.1, 500, 200000, load_frac=0.25)
        reps = [S.Runner(gpu_lib, tenants, 0, dev) for _ in TU.CONFIGS]
        for r in reps:
            r.reserve_for(reqs)
        T, _, F = S.time_matrix(reps, reqs)
        for r in reps:
            r.close()
        puts = np.array([r.kind == "put" for r in reqs])
        return F[puts], T[puts]

    Ftr, Ttr = matrix(0x7E57, 160)
    Fev, Tev = matrix(0x7E58, 100)
    sel = TU.Selector(gpu_lib.Net(len(TU.FEATURES), 32, len(TU.CONFIGS), seed=2), TU.Autotuner())
    sel.fit(Ftr, Ttr, max_epochs=400)
    net = TU.regret(Tev, [sel._net_choice(f) for f in Fev])
    chosen = TU.regret(Tev, [sel.choose(f) for f in Fev])
    locknu = TU.regret(Tev, [TU.FIXED_LOCKNU] * len(Fev))
    phasenu = TU.regret(Tev, [TU.FIXED_PHASENU] * len(Fev))
    rule = TU.regret(Tev, [sel.rule.choose(f) for f in Fev])
    print(f"regret on unseen stream: network {net:.3f} selector {chosen:.3f} rule {rule:.3f} "
          f"fixed LockNU {locknu:.3f} fixed PhaseNU {phasenu:.3f}; validation {sel.validation}")
    assert chosen < locknu and chosen < phasenu
    assert net < phasenu
