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

CONFIGS = [
    {"name": "phasenu", "two_phase": True, "local_build": 1, "local_sort": 1},
    {"name": "phasenu-global-build", "two_phase": True, "local_build": 0, "local_sort": 1},
    {"name": "phasenu-global-sort", "two_phase": True, "local_build": 1, "local_sort": 0},
    {"name": "locknu-4", "two_phase": False, "latch_ways": 4},
    {"name": "locknu-2", "two_phase": False, "latch_ways": 2},
    {"name": "locknu-1", "two_phase": False, "latch_ways": 1},
]
FIXED_PHASENU = 0
FIXED_LOCKNU = 3  # the reference's fixed choice

FEATURES = ["log2_n", "key_nibbles", "key_nibbles_std", "dup_frac", "log2_trie_keys", "log2_value_bytes",
            "lcp_frac", "new_frac_hint"]


def apply_config(mpt, k: int) -> bool:
    """Set every knob of configuration k on the trie; returns two_phase."""
    c = CONFIGS[k]
    mpt.set_option("local_build", c.get("local_build", 1))
    mpt.set_option("local_sort", c.get("local_sort", 1))
    mpt.set_option("latch_ways", c.get("latch_ways", 4))
    return bool(c["two_phase"])


def batch_features(n: int, sample_keys: list, value_bytes: float, trie_keys: int, new_frac_hint: float = 0.0):
    """Features of a put batch from a sample of its keys (bytes objects, hex
    nibble form) and the trie's current key count."""
    s = max(len(sample_keys), 1)
    lens = np.array([len(k) for k in sample_keys] or [0], dtype=np.float64)
    distinct = len(set(sample_keys))
    dup = 1.0 - distinct / s
    ks = sorted(set(sample_keys))
    lcp = 0.0
    if len(ks) > 1:
        tot = 0
        for a, b in zip(ks, ks[1:]):
            m = min(len(a), len(b))
            j = 0
            while j < m and a[j] == b[j]:
                j += 1
            tot += j
        lcp = tot / (len(ks) - 1) / max(lens.mean(), 1.0)
    return np.array([math.log2(n + 1), lens.mean() / 64.0, lens.std() / 64.0, dup, math.log2(trie_keys + 1),
                     math.log2(value_bytes + 1), lcp, new_frac_hint], dtype=np.float32)


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

@dataclass
class Selector:
    net: object                 # gmpt.Net(len(FEATURES), hidden, len(CONFIGS))
    rule: Autotuner
    mean: np.ndarray | None = None
    std: np.ndarray | None = None
    lo: np.ndarray | None = None
    hi: np.ndarray | None = None
    ood_margin: float = 0.5     # fallback outside [lo - m*range, hi + m*range]
    fallbacks: int = 0
    choices: int = 0

    def fit(self, feats: np.ndarray, times_ms: np.ndarray, epochs: int = 300, lr: float = 3e-3, seed: int = 17,
            batch: int = 64) -> float:
        """Train on measured times: target log(ms) per configuration, masked
        where a configuration was not measured.  Uses the GPU kernels."""
        x = np.asarray(feats, dtype=np.float64)
        self.mean = x.mean(0)
        self.std = np.where(x.std(0) > 1e-6, x.std(0), 1.0)
        self.lo, self.hi = x.min(0), x.max(0)
        z = ((x - self.mean) / self.std).astype(np.float32)
        t = np.asarray(times_ms, dtype=np.float64)
        m = (~np.isnan(t)).astype(np.float32)
        tgt = np.where(np.isnan(t), 0.0, np.log(np.maximum(t, 1e-6))).astype(np.float32)
        return self.net.train(z, tgt, m, epochs=epochs, batch=batch, lr=lr, seed=seed)

    def predict(self, feats) -> np.ndarray:
        z = ((np.atleast_2d(feats) - self.mean) / self.std).astype(np.float32)
        return self.net.forward(z)

    def in_range(self, f) -> bool:
        span = np.maximum(self.hi - self.lo, 1e-6)
        return bool(np.all(f >= self.lo - self.ood_margin * span) and np.all(f <= self.hi + self.ood_margin * span))

    def choose(self, f) -> int:
        self.choices += 1
        if self.mean is None or not self.in_range(f):
            self.fallbacks += 1
            return self.rule.choose(f)
        return int(np.argmin(self.predict(f)[0]))
