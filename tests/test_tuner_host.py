"""The schedule selector's host side (no GPU): the Python configuration
table equals the library's schedule table, and a rule-only selector file
written by gmpt.tuner gives the same choices inside the library (C++ rule)
as in Python."""
import numpy as np

import gmpt
from gmpt import tuner as TU


def test_python_configs_are_the_library_schedules():
    lib = gmpt.schedules()
    assert len(lib) == len(TU.CONFIGS)
    for k, s in enumerate(lib):
        assert s == TU.config_knobs(k), k


def test_rule_file_round_trip_gives_the_same_choices(tmp_path):
    rng = np.random.default_rng(4)
    n = 400
    F = np.zeros((n, len(TU.FEATURES)), np.float32)
    F[:, 0] = rng.uniform(8, 26, n)          # log2 n
    F[:, 3] = rng.choice([0.0, 0.1, 0.6], n)  # repeated-key share
    F[:, 4] = rng.choice([0.0, 0.5, 10.0, 20.0, 25.0], n)
    T = rng.uniform(1, 10, (n, len(TU.CONFIGS)))
    T[rng.uniform(size=T.shape) < 0.2] = np.nan
    sel = TU.Selector(net=None, rule=TU.Autotuner().fit(F[: n // 2], T[: n // 2]))
    path = tmp_path / "rule.gmpt-selector"
    sel.save(path)
    cs = gmpt.CSelector(0, str(path))  # rule only: no device work
    for f in F:
        k, used_net = cs.choose(f)
        assert not used_net
        assert k == sel.rule.choose(f)
    assert cs.counts() == (n, n)


def test_builtin_rule_without_a_file():
    cs = gmpt.CSelector(0, None)
    f = np.zeros(8, np.float32)
    f[0] = 20.0  # 1M keys into an empty trie: PhaseNU bulk load
    assert cs.choose(f)[0] == TU.FIXED_PHASENU
    f[4] = 20.0  # into a 1M-key trie: LockNU
    assert cs.choose(f)[0] == TU.FIXED_LOCKNU
    f[0] = 12.0  # a small batch: one persistent launch
    assert TU.CONFIGS[cs.choose(f)[0]].get("persistent")


def test_selector_file_errors_are_reported(tmp_path):
    bad = tmp_path / "bad.gmpt-selector"
    bad.write_text("gmpt-selector 1\nschedules 3\n")
    try:
        gmpt.CSelector(0, str(bad))
        raise AssertionError("expected an error")
    except gmpt.GmptError as e:
        assert "schedules" in str(e)


def test_network_candidates_are_the_near_best_configurations():
    # configuration 0 is best everywhere, 1 within 5 % on a quarter of the
    # batches, 2 close on a single batch (under the 2 % share), 3 never
    # close, 4 never measured
    rng = np.random.default_rng(3)
    t = np.full((200, 5), np.nan)
    t[:, 0] = rng.uniform(1.0, 2.0, 200)
    t[:, 1] = t[:, 0] * 1.5
    t[:50, 1] = t[:50, 0] * 1.03
    t[:, 2] = t[:, 0] * 3.0
    t[0, 2] = t[0, 0]
    t[:, 3] = t[:, 0] * 10.0
    assert TU.candidates(t) == [0, 1]
    assert TU.candidates(t, share=0.0) == [0, 1, 2]
    # nothing near the best anywhere but the best itself
    assert TU.candidates(t[:, [3, 4]]) == [0]
