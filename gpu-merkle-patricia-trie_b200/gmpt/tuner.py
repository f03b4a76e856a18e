"""Schedule selection for put batches.

A put batch can run as PhaseNU (sort + level build, gmpt_puts_2phase) or
LockNU (CAS insert, gmpt_puts_latching), each with launch-shape knobs.
Results are bit-identical whichever runs (the tests check it), so choosing
one only changes time.  Three pieces:

* ``CONFIGS``           the schedule space (strategy + knobs);
* ``Autotuner`` rule    a table from coarse batch buckets (size, trie size,
                        duplicate share) to the configuration that measured
                        fastest there -- the plain autotuned rule;
* ``Selector``          an MLP (hand-written CUDA training / inference
                        kernels, gmpt.Net) that predicts log(ms) of every
                        configuration from the batch features and picks the
                        smallest; the rule is its fallback for inputs outside
                        the range it was trained on.

The reference fixes the strategy (LockNU in libgmpt.cu:107-111, 192-196,
299-303) and fits its cost model offline (experiments.cu:3250-3348).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# The library's schedule table (csrc/schedule.cu kSchedules, gmpt.schedules()),
# index for index; tests/test_tuner_host.py checks that the two agree.
CONFIGS = [
    {"name": "phasenu", "two_phase": True, "local_build": 1, "local_sort": 1},
    {"name": "phasenu-global-build", "two_phase": True, "local_build": 0, "local_sort": 1},
    {"name": "locknu-4", "two_phase": False, "latch_ways": 4},
    {"name": "locknu-2", "two_phase": False, "latch_ways": 2},
    {"name": "locknu-1", "two_phase": False, "latch_ways": 1},
    # LockNU insert + PhaseHC + root read in one graph-replayed persistent
    # launch (gmpt_block_update with every key in stage 0), with two or one
    # co-resident CTAs per SM (block_grid 0 = the device's maximum)
    {"name": "persistent-2cta", "two_phase": False, "persistent": True, "block_grid": 0},
    {"name": "persistent-1cta", "two_phase": False, "persistent": True, "block_grid": 148},
    # LockNU without the repeated-key drop (latch_dedup 0)
    {"name": "locknu-4-nodedup", "two_phase": False, "latch_ways": 4, "latch_dedup": 0},
    # PhaseNU with every sort pass device-wide
    {"name": "phasenu-global-sort", "two_phase": True, "local_build": 1, "local_sort": 0},
    # PhaseNU, and PhaseHC hashes levels of up to 64K branches one warp each
    {"name": "phasenu-warp-hash", "two_phase": True, "local_build": 1, "local_sort": 1, "warp_full_max": 65536},
]
FIXED_PHASENU = 0
FIXED_LOCKNU = 2  # the reference's fixed choice

FEATURES = ["log2_n", "key_nibbles", "key_nibbles_std", "dup_frac", "log2_trie_keys", "log2_value_bytes",
            "lcp_frac", "log2_tries"]


def apply_config(mpt, k: int) -> bool:
    """Set every knob of configuration k on the trie (as the library's
    apply_schedule does); returns two_phase."""
    c = CONFIGS[k]
    mpt.set_option("local_build", c.get("local_build", 1))
    mpt.set_option("local_sort", c.get("local_sort", 1))
    mpt.set_option("latch_ways", c.get("latch_ways", 4))
    mpt.set_option("latch_dedup", c.get("latch_dedup", 1))
    mpt.set_option("warp_full_max", c.get("warp_full_max", 4096))
    if c.get("persistent"):
        mpt.set_option("block_grid", c.get("block_grid", 0))
    return bool(c["two_phase"])


def config_knobs(k: int) -> dict:
    """Configuration k with every knob explicit (the library's defaults filled in)."""
    c = CONFIGS[k]
    return {"name": c["name"], "two_phase": bool(c["two_phase"]), "persistent": bool(c.get("persistent", False)),
            "local_build": c.get("local_build", 1), "local_sort": c.get("local_sort", 1),
            "latch_ways": c.get("latch_ways", 4), "latch_dedup": c.get("latch_dedup", 1),
            "block_grid": c.get("block_grid", 0), "warp_full_max": c.get("warp_full_max", 4096)}


def sample_stats(keys_hexs: np.ndarray, keys_indexs: np.ndarray, samples: int = 64) -> np.ndarray:
    """Host restatement of gmpt_batch_features_device (k_sample_features):
    over `samples` evenly spaced keys (j * n // s), mean and spread of key
    length in nibbles, share of samples equal to an earlier sample, and the
    mean longest common prefix of a sample with any other sample (= with
    its neighbours in sorted order) over the mean length."""
    ki = np.asarray(keys_indexs).reshape(-1, 2)
    n = len(ki)
    s = min(n, samples)
    if s == 0:
        return np.zeros(4, dtype=np.float32)
    pos = (np.arange(s, dtype=np.int64) * n) // s
    keys = [bytes(keys_hexs[ki[i, 0]: ki[i, 1] + 1]) for i in pos]
    lens = np.array([len(k) for k in keys], dtype=np.float64)
    seen, dup = set(), 0
    for k in keys:
        dup += k in seen
        seen.add(k)
    order = sorted(range(s), key=lambda j: keys[j])
    best = np.zeros(s)

    def lcp(a, b):
        m = min(len(a), len(b))
        i = 0
        while i < m and a[i] == b[i]:
            i += 1
        return i

    for r in range(1, s):
        a, b = order[r - 1], order[r]
        v = lcp(keys[a], keys[b])
        best[a] = max(best[a], v)
        best[b] = max(best[b], v)
    mean = lens.mean()
    return np.array([mean, lens.std(), dup / s, best.mean() / mean if mean > 0 else 0.0], dtype=np.float32)


def features_from_stats(n: int, key_bytes_total: int, stats, value_bytes: float, trie_keys: int,
                        n_tries: int = 1) -> np.ndarray:
    """Selector features of a put batch: exact size and key bytes, sampled
    key statistics (sample_stats / gmpt_batch_features_device), the mean
    value size, the key count of the tries it touches and how many."""
    st = np.asarray(stats, dtype=np.float64)
    return np.array([math.log2(n + 1), key_bytes_total / max(n, 1) / 64.0, st[1] / 64.0, st[2],
                     math.log2(trie_keys + 1), math.log2(value_bytes + 1), st[3], math.log2(max(n_tries, 1))],
                    dtype=np.float32)


# -- the plain autotuned rule --------------------------------------------------

def bucket(f) -> tuple:
    log2_n, log2_trie, dup = float(f[0]), float(f[4]), float(f[3])
    bn = int(min(max(log2_n, 10), 24) // 2)
    bt = 0 if log2_trie < 1 else 1 + min(3, int(log2_trie // 6))
    bd = 0 if dup < 0.05 else (1 if dup < 0.3 else 2)
    return bn, bt, bd


@dataclass
class Autotuner:
    """Measured fastest configuration per bucket (the plain rule)."""

    table: dict = field(default_factory=dict)
    default: int = FIXED_LOCKNU

    def fit(self, feats: np.ndarray, times_ms: np.ndarray):
        """feats [N, F]; times_ms [N, K] measured times (nan = not measured)."""
        acc = {}
        for f, t in zip(feats, times_ms):
            b = bucket(f)
            s, c = acc.setdefault(b, (np.zeros(len(CONFIGS)), np.zeros(len(CONFIGS))))
            ok = ~np.isnan(t)
            s[ok] += np.log(t[ok])
            c[ok] += 1
        self.table = {}
        for b, (s, c) in acc.items():
            mean = np.where(c > 0, s / np.maximum(c, 1), np.inf)
            self.table[b] = int(np.argmin(mean))
        return self

    def choose(self, f) -> int:
        if not self.table:
            return self.default
        b = bucket(f)
        if b in self.table:
            return self.table[b]
        near = min(self.table, key=lambda x: sum(abs(p - q) for p, q in zip(x, b)))
        return self.table[near]


# -- the MLP selector ----------------------------------------------------------

def regret(times_ms: np.ndarray, choice) -> float:
    """Total time of the chosen configurations over the per-batch best, - 1."""
    t = np.asarray(times_ms, dtype=np.float64)
    best = np.nanmin(t, 1)
    got = t[np.arange(len(t)), np.asarray(choice)]
    return float(np.nansum(got) / np.nansum(best) - 1.0)


def candidates(times_ms: np.ndarray, near: float = 1.05, share: float = 0.02) -> list:
    """Configurations the network may pick: those within `near` of the
    per-batch best on at least `share` of the measured batches (and at
    least one).  A configuration that never came close in training has only
    extrapolated predictions, and one low guess for it (a PhaseNU rebuild of
    a large trie, say) costs several times the batch; leaving it out bounds
    what a wrong pick can cost."""
    t = np.asarray(times_ms, dtype=np.float64)
    best = np.nanmin(t, 1, keepdims=True)
    close = np.where(np.isnan(t), False, t <= near * best)
    need = max(1, int(np.ceil(share * len(t))))
    cols = [k for k in range(t.shape[1]) if close[:, k].sum() >= need]
    if not cols:  # every configuration measured somewhere is a candidate
        cols = [k for k in range(t.shape[1]) if np.any(~np.isnan(t[:, k]))]
    return cols


@dataclass
class Selector:
    """MLP schedule selector with the autotuned rule as fallback and yardstick:
    fit() holds out a quarter of the measured batches, and the network is
    used only if its regret there is no worse than the rule's (fit on the
    same three quarters); either way both are then refit on all batches."""

    net: object                 # gmpt.Net(len(FEATURES), hidden, len(CONFIGS))
    rule: Autotuner
    mean: np.ndarray | None = None
    std: np.ndarray | None = None
    lo: np.ndarray | None = None
    hi: np.ndarray | None = None
    cols: list | None = None    # configurations with measurements
    ood_margin: float = 0.5     # fallback outside [lo - m*range, hi + m*range]
    use_net: bool = False
    validation: dict = field(default_factory=dict)
    fallbacks: int = 0
    choices: int = 0

    def _train(self, feats, times_ms, epochs, lr, seed, batch):
        x = np.asarray(feats, dtype=np.float64)
        self.mean = x.mean(0)
        self.std = np.where(x.std(0) > 1e-6, x.std(0), 1.0)
        self.lo, self.hi = x.min(0), x.max(0)
        z = ((x - self.mean) / self.std).astype(np.float32)
        t = np.asarray(times_ms, dtype=np.float64)
        self.cols = candidates(t)
        tgt, m = self._targets(t)
        return self.net.train(z, tgt, m, epochs=epochs, batch=batch, lr=lr, seed=seed)

    def fit(self, feats: np.ndarray, times_ms: np.ndarray, max_epochs: int = 600, lr: float = 3e-3, seed: int = 17,
            batch: int = 64, holdout: float = 0.25, step: int = 50) -> float:
        """Train on measured times (target log(ms) per configuration, masked
        where a configuration was not measured) with the GPU kernels.  The
        epoch count is the one with the least regret on the held-out
        quarter (checked every `step` epochs); the network is enabled only
        if that regret is no worse than the rule's."""
        feats = np.asarray(feats, dtype=np.float64)
        times_ms = np.asarray(times_ms, dtype=np.float64)
        n = len(feats)
        init = self.net.params()
        epochs = max_epochs
        if n >= 8:
            hold = np.zeros(n, dtype=bool)
            hold[np.random.default_rng(seed).permutation(n)[: max(2, int(n * holdout))]] = True
            rule = Autotuner().fit(feats[~hold], times_ms[~hold])
            rule_r = regret(times_ms[hold], [rule.choose(f) for f in feats[hold]])
            self._train(feats[~hold], times_ms[~hold], step, lr, seed, batch)
            curve = []
            for e in range(step, max_epochs + 1, step):
                if e > step:
                    self.net.train(((feats[~hold] - self.mean) / self.std).astype(np.float32),
                                   *self._targets(times_ms[~hold]), epochs=step, batch=batch, lr=lr, seed=seed + e)
                curve.append((regret(times_ms[hold], [self._net_choice(f) for f in feats[hold]]), e))
            net_r, epochs = min(curve)
            self.use_net = net_r <= rule_r
            self.validation = {"held_out": int(hold.sum()), "net_regret": round(net_r, 4), "epochs": epochs,
                               "rule_regret": round(rule_r, 4), "use_net": self.use_net}
            self.net.set_params(init)
        else:
            self.use_net = True
        self.rule.fit(feats, times_ms)
        return self._train(feats, times_ms, epochs, lr, seed, batch)

    def _targets(self, times_ms):
        t = np.asarray(times_ms, dtype=np.float64)
        m = (~np.isnan(t)).astype(np.float32)
        tgt = np.where(np.isnan(t), 0.0, np.log(np.maximum(np.nan_to_num(t, nan=1.0), 1e-6))).astype(np.float32)
        return tgt, m

    def predict(self, feats) -> np.ndarray:
        z = ((np.atleast_2d(feats) - self.mean) / self.std).astype(np.float32)
        return self.net.forward(z)

    def _net_choice(self, f) -> int:
        y = self.predict(f)[0]
        return int(self.cols[int(np.argmin(y[self.cols]))])

    def in_range(self, f) -> bool:
        span = np.maximum(self.hi - self.lo, 1e-6)
        return bool(np.all(f >= self.lo - self.ood_margin * span) and np.all(f <= self.hi + self.ood_margin * span))

    def choose(self, f) -> int:
        self.choices += 1
        if self.mean is None or not self.use_net or not self.in_range(f):
            self.fallbacks += 1
            return self.rule.choose(f)
        return self._net_choice(f)

    def save(self, path) -> None:
        """Write the selector for the library's C++ selector
        (gmpt_selector_create): rule table, network, normalisation.  The
        format is documented at Selector::load in csrc/schedule.cu."""
        lines = ["gmpt-selector 1", f"schedules {len(CONFIGS)}", f"default {int(self.rule.default)}",
                 f"rules {len(self.rule.table)}"]
        for b, k in self.rule.table.items():
            lines.append(f"{b[0]} {b[1]} {b[2]} {int(k)}")
        if self.mean is None:
            lines.append("net 0 0 0 0")
        else:
            p = self.net.params()
            n_in, n_hidden, n_out = self.net.dims
            lines.append(f"net {1 if self.use_net else 0} {n_in} {n_hidden} {n_out}")
            lines.append(f"margin {self.ood_margin!r}")
            for name, v in (("mean", self.mean), ("std", self.std), ("lo", self.lo), ("hi", self.hi)):
                lines.append(name + " " + " ".join(repr(float(np.float32(x))) for x in v))
            lines.append(f"cols {len(self.cols)} " + " ".join(str(int(c)) for c in self.cols))
            lines.append(f"params {len(p)} " + " ".join(repr(float(x)) for x in p))
        with open(path, "w") as f:
            f.write("\n".join(lines) + "\n")

    def to_library(self, device: int = 0, path=None):
        """The same selector inside the library (gmpt.CSelector): choices are
        then made by the C++ rule and the network's CUDA inference kernel."""
        import os
        import tempfile

        from . import CSelector

        if path is None:
            fd, path = tempfile.mkstemp(suffix=".gmpt-selector")
            os.close(fd)
        self.save(path)
        return CSelector(device, path)
