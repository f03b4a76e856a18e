"""Schedule selection inside the library: every schedule gives the oracle's
trie, gmpt_puts_auto picks schedules that vary with the batch and still
reaches the oracle's roots, the reference ABI does the same under
GMPT_SCHEDULE=auto, and a trained selector makes the same choices in the
library (C++ rule, CUDA network inference) as in Python."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O
from gmpt import tuner as TU
from gmpt import workloads as W

pytestmark = pytest.mark.gpu


def oracle_roots(batches):
    o = O.OracleTrie()
    out = []
    for b in batches:
        o.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        o.hash()
        out.append(o.root())
    return out


@pytest.fixture(scope="module")
def three_batches():
    n = 1 << 16
    load = W.ycsb_load(n, seed=0x5EED0002)
    small = W.ycsb_zipf_updates(n, 1000, seed=0x5EED0005)
    fresh = W.random_keys(1 << 17, 32, 40, seed=0x5EED0006)
    return [load, small, fresh]


@pytest.mark.parametrize("k", range(len(TU.CONFIGS)))
def test_every_schedule_reaches_the_oracle_roots(gpu_lib, three_batches, k):
    want = oracle_roots(three_batches)
    t = gpu_lib.MPT()
    for b, r in zip(three_batches, want):
        t.puts_schedule(k, b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        t.hash_onepass_v2()
        assert t.get_root_hash() == r, TU.CONFIGS[k]["name"]
    t.close()


def test_puts_auto_varies_the_schedule_and_matches_the_oracle(gpu_lib, three_batches):
    want = oracle_roots(three_batches)
    t = gpu_lib.MPT()
    chosen = []
    for b, r in zip(three_batches, want):
        chosen.append(t.puts_auto(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs))
        t.hash_onepass_v2()
        assert t.get_root_hash() == r
    t.close()
    # the built-in rule: empty trie -> PhaseNU, 1000 keys -> persistent launch,
    # 128K keys into a 64K-key trie -> LockNU
    assert chosen[0] == TU.FIXED_PHASENU
    assert TU.CONFIGS[chosen[1]].get("persistent")
    assert chosen[2] == TU.FIXED_LOCKNU
    assert len(set(chosen)) == 3


def test_device_batches_through_puts_auto(gpu_lib, three_batches):
    import torch

    dev = torch.device("cuda", 0)
    want = oracle_roots(three_batches)
    t = gpu_lib.MPT()
    for b, r in zip(three_batches, want):
        d = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
             for a in (b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)]
        torch.cuda.synchronize()
        t.puts_auto_device(*[x.data_ptr() for x in d], b.n, b.key_bytes(), b.value_bytes())
        t.hash_onepass_v2()
        assert t.get_root_hash() == r
    t.close()


def test_reference_abi_with_schedule_auto(gpu_lib, three_batches):
    L = gpu_lib.lib()
    want = oracle_roots(three_batches)
    os.environ["GMPT_SCHEDULE"] = "auto"
    try:
        h = L.init_mpt()
        assert h
        P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        for b, r in zip(three_batches, want):
            ki = np.ascontiguousarray(b.keys_indexs, np.int32)
            vi = np.ascontiguousarray(b.values_indexs, np.int64)
            out = L.insert_mpt_olc(h, P(b.keys_hexs), P(ki), P(b.values), P(vi), None, b.n)
            assert out, L.gmpt_last_error_message()
            assert ctypes.string_at(out, 32) == r
            L.gmpt_free_buffer(out)
        L.free_mpt(h)
    finally:
        del os.environ["GMPT_SCHEDULE"]


def test_host_features_equal_the_python_restatement(gpu_lib, three_batches):
    t = gpu_lib.MPT()
    for b in three_batches:
        f = t.features(b.keys_hexs, b.keys_indexs, b.values_indexs)
        st = TU.sample_stats(b.keys_hexs, b.keys_indexs)
        want = TU.features_from_stats(b.n, b.key_bytes(), st, b.value_bytes() / b.n,
                                      t.stats()["n_value"], 1)
        np.testing.assert_allclose(f, want, rtol=1e-5, atol=1e-5)
        t.puts_2phase_with_valuehp(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        t.hash_onepass_v2()
    t.close()


def test_trained_selector_chooses_the_same_in_the_library(gpu_lib, tmp_path):
    rng = np.random.default_rng(8)
    n = 600
    F = np.zeros((n, len(TU.FEATURES)), np.float32)
    F[:, 0] = rng.uniform(10, 24, n)
    F[:, 1] = rng.uniform(0.3, 3.0, n)
    F[:, 3] = rng.uniform(0, 0.8, n)
    F[:, 4] = rng.uniform(0, 26, n)
    F[:, 5] = rng.uniform(4, 8, n)
    # synthetic times with structure the network can learn
    base = np.exp(0.7 * F[:, :1] - 6.0)
    T = base * (1.0 + 0.3 * rng.uniform(size=(n, len(TU.CONFIGS))))
    T[:, TU.FIXED_PHASENU] *= np.where(F[:, 4] < 1, 0.4, 2.0)
    T[:, 6] *= np.where(F[:, 0] < 14, 0.3, 3.0)
    sel = TU.Selector(gpu_lib.Net(len(TU.FEATURES), 32, len(TU.CONFIGS), seed=4), TU.Autotuner())
    sel.fit(F, T, max_epochs=200, lr=3e-3)
    sel.use_net = True  # exercise the network path whatever the hold-out said
    cs = sel.to_library(0, tmp_path / "trained.gmpt-selector")
    probe = F[rng.permutation(n)[:200]].copy()
    probe[:20, 0] = 40.0  # far outside the training range: the rule decides
    agree = 0
    for f in probe:
        k_py = sel.choose(f)
        k_lib, used_net = cs.choose(f)
        assert used_net == sel.in_range(f)
        if used_net:
            # same network, same inputs: fp32 forward on the device both ways
            agree += k_lib == k_py
        else:
            assert k_lib == k_py
    assert agree >= 0.97 * sum(sel.in_range(f) for f in probe)
    assert cs.counts()[1] >= 20


def test_gets_with_device_results_match_host_results(gpu_lib, three_batches):
    import torch

    dev = torch.device("cuda", 0)
    b = three_batches[0]
    t = gpu_lib.MPT()
    hp = np.arange(1, b.n + 1, dtype=np.uint64) * 16
    t.puts_2phase_with_valuehp(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs, values_hps=hp)
    probe = W.random_keys(1000, 32, 4, seed=77)  # absent keys mixed in
    q = W.Batch(np.concatenate([b.keys_hexs, probe.keys_hexs]),
                np.concatenate([b.keys_indexs, probe.keys_indexs + len(b.keys_hexs)]).astype(np.int32),
                b.values, b.values_indexs)
    dk = torch.from_numpy(q.keys_hexs).to(dev)
    di = torch.from_numpy(q.keys_indexs).to(dev)
    n = len(q.keys_indexs) // 2
    ohp = torch.zeros(n, dtype=torch.int64, device=dev)
    olen = torch.zeros(n, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    t.gets_device(dk.data_ptr(), di.data_ptr(), n, len(q.keys_hexs), ohp.data_ptr(), olen.data_ptr())
    want_hp, want_len = t.gets_forest_device(dk.data_ptr(), di.data_ptr(), 0, n, len(q.keys_hexs))
    assert np.array_equal(ohp.cpu().numpy().view(np.uint64), want_hp)
    assert np.array_equal(olen.cpu().numpy(), want_len)
    assert np.array_equal(want_hp[: b.n], hp) and not want_hp[b.n:].any()
    t.close()
