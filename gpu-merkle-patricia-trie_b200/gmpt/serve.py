"""Request loop over a forest of tenant tries: put and get batches arriving
as a Poisson stream, served one at a time or drained and merged.

* A tenant is one trie of a forest (gmpt.MPT with max_tries), with a fixed
  key length (20..96 bytes) and value length; its keys are ids 0..count-1
  expanded on the device (gmpt.gen_keys), so replicas regenerate identical
  batches without host copies.
* A put request inserts n keys: fresh ids with probability p_new, else
  zipf(theta) over the tenant's existing ids (updates).  A get request
  looks up n zipf(theta) existing ids.
* ``Runner`` applies requests to one forest replica: a run of same-kind
  requests (several tenants) becomes one forest put + PhaseHC + root read,
  or one forest lookup, under a schedule configuration (gmpt.tuner).
* ``time_matrix`` runs every put under every configuration on its own
  replica (all replicas stay logically identical: results do not depend on
  the configuration), giving per-request times for the fixed strategies,
  the autotuned rule, the selector and the per-request best.
* ``serve`` runs a live server (one request at a time, or draining the queue
  and merging same-kind runs) on a virtual clock: start = max(free, arrival),
  latency = completion - arrival, service times measured on the device.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import tuner as TU
from . import workloads as W


@dataclass
class Tenant:
    tid: int
    key_bytes: int
    value_bytes: int
    initial: int          # keys loaded before the stream


@dataclass
class Request:
    i: int
    kind: str             # "put" | "get"
    tenant: int
    n: int
    theta: float
    p_new: float
    seed: int
    arrival: float = 0.0  # seconds


def make_tenants(sizes, seed: int = 0x5EED0C50):
    rng = W.Xoshiro256ss(seed, lanes=64)
    kb = 20 + (rng.words(len(sizes)) % np.uint64(77)).astype(int)        # 20..96 B keys
    vb = 16 + (rng.words(len(sizes)) % np.uint64(113)).astype(int)       # 16..128 B values
    return [Tenant(t, int(kb[t]), int(vb[t]), int(s)) for t, s in enumerate(sizes)]


def make_stream(seed: int, count: int, n_tenants: int, read_ratio: float, n_min: int, n_max: int,
                theta_max: float = 1.2):
    rng = W.Xoshiro256ss(seed, lanes=256)
    u = rng.uniform(5 * count).reshape(count, 5)
    reqs = []
    for i in range(count):
        n = int(round(math.exp(math.log(n_min) + u[i, 0] * (math.log(n_max) - math.log(n_min)))))
        kind = "get" if u[i, 1] < read_ratio else "put"
        reqs.append(Request(i, kind, int(u[i, 2] * n_tenants) % n_tenants, max(n, 1), float(u[i, 3] * theta_max),
                            float(u[i, 4]), int(rng.words(1)[0])))
    return reqs


def poisson_arrivals(reqs, rate_per_s: float, seed: int = 0x5EED0C51):
    rng = W.Xoshiro256ss(seed, lanes=256)
    gaps = -np.log(np.maximum(rng.uniform(len(reqs)), 1e-300)) / rate_per_s
    t = np.cumsum(gaps)
    for r, a in zip(reqs, t):
        r.arrival = float(a)


KEY_SEED = 0x6B65795EED000000
VALUE_SEED = 0x76616CEED0000000


class Stage:
    """Device buffers for one merged batch (grown as needed)."""

    def __init__(self, dev):
        import torch

        self.torch = torch
        self.dev = dev
        self.cap = 0
        self.kcap = 0
        self.vcap = 0

    def ensure(self, n, kb, vb):
        t = self.torch
        if n > self.cap:
            self.cap = int(n * 1.25) + 1024
            self.ids = t.empty(self.cap, dtype=t.int64, device=self.dev)
            self.kidx = t.empty(2 * self.cap, dtype=t.int32, device=self.dev)
            self.vidx = t.empty(2 * self.cap, dtype=t.int64, device=self.dev)
            self.tids = t.empty(self.cap, dtype=t.int32, device=self.dev)
        if kb > self.kcap:
            self.kcap = int(kb * 1.25) + 4096
            self.keys = t.empty(self.kcap + 64, dtype=t.uint8, device=self.dev)
        if vb > self.vcap:
            self.vcap = int(vb * 1.25) + 4096
            self.vals = t.empty(self.vcap + 64, dtype=t.uint8, device=self.dev)


class Runner:
    """One forest replica holding every tenant, plus its id counters."""

    def __init__(self, gmpt, tenants, device: int, dev, mode: int = 0, chunk: int = 1 << 22, record: bool = False):
        self.g = gmpt
        self.tenants = tenants
        self.mpt = gmpt.MPT(device=device, mode=mode, max_tries=len(tenants))
        self.stage = Stage(dev)
        self.count = {t.tid: 0 for t in tenants}
        self.stream = self.mpt.stream_ptr()
        self.record = [] if record else None  # host copies of every applied put (tests)
        for t in tenants:  # initial contents, PhaseNU bulk loads
            left = t.initial
            while left > 0:
                n = min(chunk, left)
                self._load_fresh(t, n)
                left -= n
        self.mpt.hash_onepass_v2()

    def _load_fresh(self, t, n):
        s = self.stage
        s.ensure(n, n * (2 * t.key_bytes + 1), n * t.value_bytes)
        torch = s.torch
        s.ids[:n] = torch.arange(self.count[t.tid], self.count[t.tid] + n, device=s.dev)
        self.g.gen_keys(KEY_SEED ^ t.tid, s.ids.data_ptr(), n, t.key_bytes, s.keys.data_ptr(), s.kidx.data_ptr())
        self.g.gen_values(VALUE_SEED ^ (t.tid << 40) ^ self.count[t.tid], n, t.value_bytes, s.vals.data_ptr(),
                          s.vidx.data_ptr())
        s.tids[:n] = t.tid
        torch.cuda.synchronize(s.dev)
        if self.record is not None:
            self.record.append(self.snapshot(n, n * (2 * t.key_bytes + 1), n * t.value_bytes))
        self.mpt.puts_forest_device(True, s.keys.data_ptr(), s.kidx.data_ptr(), s.vals.data_ptr(), s.vidx.data_ptr(),
                                    s.tids.data_ptr(), n, n * (2 * t.key_bytes + 1), n * t.value_bytes)
        self.count[t.tid] += n

    def build(self, reqs):
        """Generate the merged batch of same-kind requests into the stage."""
        s = self.stage
        torch = s.torch
        n = sum(r.n for r in reqs)
        kb = sum(r.n * (2 * self.tenants[r.tenant].key_bytes + 1) for r in reqs)
        vb = sum(r.n * self.tenants[r.tenant].value_bytes for r in reqs) if reqs[0].kind == "put" else 0
        s.ensure(n, kb, max(vb, 1))
        off = koff = voff = 0
        for r in reqs:
            t = self.tenants[r.tenant]
            cnt = self.count[t.tid]
            ids = s.ids[off: off + r.n]
            if r.kind == "put":
                nn = self.g.gen_ids(r.seed, r.n, cnt, cnt, r.p_new, r.theta, ids.data_ptr())
                self.count[t.tid] = cnt + nn
            else:
                self.g.gen_ids(r.seed, r.n, cnt, cnt, 0.0, r.theta, ids.data_ptr())
            w = 2 * t.key_bytes + 1
            self.g.gen_keys(KEY_SEED ^ t.tid, ids.data_ptr(), r.n, t.key_bytes, s.keys.data_ptr() + koff,
                            s.kidx.data_ptr() + 8 * off)
            if koff:
                s.kidx[2 * off: 2 * (off + r.n)] += koff
            if r.kind == "put":
                self.g.gen_values(VALUE_SEED ^ r.seed, r.n, t.value_bytes, s.vals.data_ptr() + voff,
                                  s.vidx.data_ptr() + 16 * off)
                if voff:
                    s.vidx[2 * off: 2 * (off + r.n)] += voff
                voff += r.n * t.value_bytes
            s.tids[off: off + r.n] = t.tid
            off += r.n
            koff += r.n * w
        torch.cuda.synchronize(s.dev)
        return n, kb, voff

    def features(self, reqs, n, kb, vb, sample: int = 512, probe: int = 256):
        """Selector features from a sample of the staged batch (keys copied
        to the host) and a lookup of a few sampled keys (new-key share)."""
        s = self.stage
        torch = s.torch
        rng = np.random.default_rng(reqs[0].seed & 0xFFFFFFFF)
        pos = np.sort(rng.choice(n, size=min(n, sample), replace=False)) if n > sample else np.arange(n)
        dpos = torch.from_numpy(pos).to(s.dev)
        kid = s.kidx[: 2 * n].view(-1, 2)[dpos].long()
        lens = kid[:, 1] - kid[:, 0] + 1
        starts = torch.repeat_interleave(kid[:, 0], lens)
        within = torch.arange(int(lens.sum().item()), device=s.dev) - torch.repeat_interleave(
            torch.cumsum(lens, 0) - lens, lens)
        flat = s.keys[starts + within].cpu().numpy()
        lh = lens.cpu().numpy()
        keys, at = [], 0
        for ln in lh.tolist():
            keys.append(flat[at: at + ln].tobytes())
            at += ln
        # new-key share of a few sampled keys (lookups on the live forest)
        pk = min(len(pos), probe)
        pidx = np.zeros(2 * pk, np.int32)
        buf = b"".join(keys[:pk])
        at = 0
        for j in range(pk):
            pidx[2 * j], pidx[2 * j + 1] = at, at + len(keys[j]) - 1
            at += len(keys[j])
        tids = s.tids[: n][torch.from_numpy(pos[:pk]).to(s.dev)].cpu().numpy().astype(np.int32)
        _, sizes = self.mpt.gets_forest(np.frombuffer(buf, np.uint8), pidx, tids)
        new_frac = float(np.mean(sizes == 0)) if pk else 0.0
        trie_keys = sum(self.count[t] for t in set(r.tenant for r in reqs))
        return TU.batch_features(n, keys, vb / max(n, 1), trie_keys, new_frac)

    def snapshot(self, n, kb, vb):
        """Host copy of the staged batch (keys, values, trie ids)."""
        s = self.stage
        return W.Batch(s.keys[:kb].cpu().numpy(), s.kidx[: 2 * n].cpu().numpy(), s.vals[:vb].cpu().numpy(),
                       s.vidx[: 2 * n].cpu().numpy()), s.tids[:n].cpu().numpy()

    def put(self, reqs, k: int, n, kb, vb):
        if self.record is not None:
            self.record.append(self.snapshot(n, kb, vb))
        two = TU.apply_config(self.mpt, k)
        s = self.stage
        self.mpt.puts_forest_device(two, s.keys.data_ptr(), s.kidx.data_ptr(), s.vals.data_ptr(), s.vidx.data_ptr(),
                                    s.tids.data_ptr(), n, kb, vb)
        self.mpt.hash_onepass_v2()
        return self.mpt.get_roots(sorted(set(r.tenant for r in reqs)))

    def get(self, n, kb):
        s = self.stage
        _, sizes = self.mpt.gets_forest_device(s.keys.data_ptr(), s.kidx.data_ptr(), s.tids.data_ptr(), n, kb)
        return sizes

    def roots(self):
        return self.mpt.get_roots(n=len(self.tenants))

    def close(self):
        self.mpt.close()


def _timed(fn):
    t0 = time.perf_counter()
    out = fn()
    return out, (time.perf_counter() - t0) * 1e3


def time_matrix(replicas, reqs, with_features=True):
    """Every put under every configuration (replica k runs configuration k).
    Returns times [N, K] (ms; nan for gets), get times [N] (nan for puts),
    features [N, F] of the puts (zeros for gets)."""
    K = len(replicas)
    T = np.full((len(reqs), K), np.nan)
    G = np.full(len(reqs), np.nan)
    F = np.zeros((len(reqs), len(TU.FEATURES)), dtype=np.float32)
    for i, r in enumerate(reqs):
        if r.kind == "put":
            roots = None
            for k, rep in enumerate(replicas):
                n, kb, vb = rep.build([r])
                if k == 0 and with_features:
                    F[i] = rep.features([r], n, kb, vb)
                out, ms = _timed(lambda: rep.put([r], k, n, kb, vb))
                T[i, k] = ms
                if roots is None:
                    roots = out
                elif out != roots:
                    raise AssertionError(f"configuration {k} changed the root at request {i}")
        else:
            # lookups leave the id counters alone: one replica answers
            n, kb, _ = replicas[0].build([r])
            _, ms = _timed(lambda: replicas[0].get(n, kb))
            G[i] = ms
    return T, G, F


def fifo_latency(reqs, service_ms):
    """Latencies (ms) of a one-at-a-time FIFO server with the given service times."""
    free = 0.0
    lat = np.zeros(len(reqs))
    for j, (r, s) in enumerate(zip(reqs, service_ms)):
        start = max(free, r.arrival)
        free = start + s / 1e3
        lat[j] = (free - r.arrival) * 1e3
    return lat


@dataclass
class ServeResult:
    latency_ms: np.ndarray
    busy_ms: float
    keys: int
    launches: int
    groups: int
    choices: dict = field(default_factory=dict)
    get_sizes: list = field(default_factory=list)


def serve(runner, reqs, policy, batching: bool, max_keys: int = 1 << 23) -> ServeResult:
    """Live server on a virtual clock.  policy(runner, reqs, n, kb, vb) ->
    configuration index (its own time is part of the service time)."""
    lat = np.zeros(len(reqs))
    free = 0.0
    busy = 0.0
    groups = 0
    choices = {}
    gets = []
    i = 0
    while i < len(reqs):
        start = max(free, reqs[i].arrival)
        j = i + 1
        if batching:
            tot = reqs[i].n
            while j < len(reqs) and reqs[j].arrival <= start and tot + reqs[j].n <= max_keys:
                tot += reqs[j].n
                j += 1
        # runs of same-kind requests, in arrival order
        a = i
        t = start
        while a < j:
            b = a + 1
            while b < j and reqs[b].kind == reqs[a].kind:
                b += 1
            run = reqs[a:b]
            n, kb, vb = runner.build(run)
            t0 = time.perf_counter()
            if run[0].kind == "put":
                k = policy(runner, run, n, kb, vb)
                choices[k] = choices.get(k, 0) + 1
                runner.put(run, k, n, kb, vb)
            else:
                gets.append(runner.get(n, kb))
            ms = (time.perf_counter() - t0) * 1e3
            busy += ms
            t += ms / 1e3
            groups += 1
            for r in run:
                lat[r.i - reqs[0].i] = (t - r.arrival) * 1e3
            a = b
        free = t
        i = j
    return ServeResult(lat, busy, sum(r.n for r in reqs), 0, groups, choices, gets)
