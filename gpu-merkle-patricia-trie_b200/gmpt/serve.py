"""Request loop over a forest of tenant tries: put and get batches arriving
as a Poisson stream, served one at a time or drained and merged.

* A tenant is one trie of a forest (gmpt.MPT with max_tries), with a fixed
  key length (20..96 bytes) and value length; its keys are ids 0..count-1
  expanded on the device (gmpt.gen_keys), so replicas regenerate identical
  batches without host copies.
* A put request inserts n keys: fresh ids with probability p_new, else
  zipf(theta) over the tenant's existing ids (updates).  A load request
  fills a tenant trie created for it (empty, all keys fresh).  A get request
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
    kind: str             # "put" | "get" (a load is a put with p_new 1 into a new tenant)
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


def make_stream(seed: int, count: int, tenants: list, read_ratio: float, n_min: int, n_max: int,
                theta_max: float = 1.2, load_frac: float = 0.0):
    """count requests; a put is a load into a new tenant (appended to
    `tenants`, empty) with probability load_frac.  Requests target tenants
    that exist by then; gets only non-empty ones."""
    rng = W.Xoshiro256ss(seed, lanes=256)
    u = rng.uniform(7 * count).reshape(count, 7)
    live = [t.tid for t in tenants]
    filled = {t.tid for t in tenants if t.initial > 0}
    reqs = []
    for i in range(count):
        n = max(1, int(round(math.exp(math.log(n_min) + u[i, 0] * (math.log(n_max) - math.log(n_min))))))
        seed_i = int(rng.words(1)[0])
        if u[i, 1] < read_ratio and filled:
            pool = sorted(filled)
            reqs.append(Request(i, "get", pool[int(u[i, 2] * len(pool)) % len(pool)], n,
                                float(u[i, 3] * theta_max), 0.0, seed_i))
        elif u[i, 5] < load_frac:
            t = make_tenants([0], seed=seed_i)[0]
            t.tid = len(tenants)
            tenants.append(t)
            live.append(t.tid)
            filled.add(t.tid)
            reqs.append(Request(i, "put", t.tid, n, 0.0, 1.0, seed_i))
        else:
            tid = live[int(u[i, 2] * len(live)) % len(live)]
            filled.add(tid)
            reqs.append(Request(i, "put", tid, n, float(u[i, 3] * theta_max), float(u[i, 4]), seed_i))
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
            self.rw = t.empty(self.cap, dtype=t.uint8, device=self.dev)        # mixed batches
            self.out_hp = t.empty(self.cap, dtype=t.int64, device=self.dev)
            self.out_len = t.empty(self.cap, dtype=t.int32, device=self.dev)
        if kb > self.kcap:
            self.kcap = int(kb * 1.25) + 4096
            self.keys = t.empty(self.kcap + 64, dtype=t.uint8, device=self.dev)
        if vb > self.vcap:
            self.vcap = int(vb * 1.25) + 4096
            self.vals = t.empty(self.vcap + 64, dtype=t.uint8, device=self.dev)


class Runner:
    """One forest replica holding every tenant, plus its id counters."""

    def __init__(self, gmpt, tenants, device: int, dev, mode: int = 0, chunk: int = 1 << 22, record: bool = False,
                 max_tries: int = 0):
        self.g = gmpt
        self.mpt = gmpt.MPT(device=device, mode=mode, max_tries=max(max_tries, len(tenants)))
        self.stage = Stage(dev)
        self.stream = self.mpt.stream_ptr()
        self.record = [] if record else None  # host copies of every applied put (tests)
        self.get_cap = 0
        self.chunk = chunk
        self._fill(tenants)

    def _fill(self, tenants):
        self.tenants = tenants
        self.tenant_of = {t.tid: t for t in tenants}
        self.count = {t.tid: 0 for t in tenants}
        for t in tenants:  # initial contents, PhaseNU bulk loads
            left = t.initial
            while left > 0:
                n = min(self.chunk, left)
                self._load_fresh(t, n)
                left -= n
        self.mpt.hash_onepass_v2()

    def reset(self, tenants):
        """Empty the forest (capacity kept) and load a new tenant set."""
        if len(tenants) > self.mpt_max_tries():
            raise ValueError("more tenants than the forest holds")
        self.mpt.reset()
        self._fill(tenants)

    def mpt_max_tries(self) -> int:
        return int(self.mpt._L.gmpt_max_tries(self.mpt._h))

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

    def reserve_for(self, reqs, merged_keys: int = 0):
        """Grow pools, arenas and block buffers now for every put of the
        stream (no growth, no graph capture inside a timed request)."""
        kmax = max(2 * t.key_bytes + 1 for t in self.tenants)
        vmax = max(t.value_bytes for t in self.tenants)
        puts = [r for r in reqs if r.kind == "put"]
        total = sum(r.n for r in puts)
        big = max([r.n for r in reqs] + [merged_keys, 1])
        total += 2 * big  # the warm-up puts
        kbytes = sum(r.n * (2 * self.tenant_of[r.tenant].key_bytes + 1 + 8) for r in puts) + 2 * big * (kmax + 8)
        vbytes = sum(r.n * self.tenant_of[r.tenant].value_bytes for r in puts) + 2 * big * 16
        # growth of the stream (a new key adds about one short node and a
        # fraction of a branch) plus the per-batch headroom the inserts check
        # for (PhaseNU: 2 branches and 4 short nodes per key of the batch)
        self.mpt.reserve_nodes(total // 2 + 2 * big, total + total // 4 + 4 * big, total + big, total + big,
                               kbytes + big * kmax, vbytes + big * vmax)
        self.warm(big)
        gets = [r for r in reqs if r.kind == "get"]
        if gets:  # grow the lookup workspaces and result buffers now (read only)
            g = max(gets, key=lambda r: r.n)
            warm = Request(-1, "get", g.tenant, max(g.n, merged_keys if merged_keys else 0), 0.0, 0.0, 1)
            n, kb, _ = self.build([warm])
            self.get(n, kb)
        for c in TU.CONFIGS:  # capture the block graph of every persistent grid
            if c.get("persistent"):
                self.mpt.set_option("block_grid", c.get("block_grid", 0))
                self.mpt.reserve_block(big, big * kmax, big * vmax, len(self.tenants))
        self.stage.ensure(big, big * kmax, big * vmax)

    def warm(self, n: int):
        """Grow every insert workspace for batches of up to n keys: one put of
        n fresh keys under each strategy into a scratch trie (the forest's
        last id, outside the tenants), so no timed request pays for growth."""
        tid = self.mpt_max_tries() - 1
        if tid in self.tenant_of or n <= 0:
            return
        kmax = max(t.key_bytes for t in self.tenants)
        scratch = Tenant(tid, kmax, 16, 0)
        self.tenant_of[tid] = scratch
        self.count[tid] = 0
        for k in (TU.FIXED_PHASENU, TU.FIXED_LOCKNU):
            r = Request(-1, "put", tid, n, 0.0, 1.0, 0x5C7A7C4 + k)
            nn, kb, vb = self.build([r])
            TU.apply_config(self.mpt, k)
            s = self.stage
            self.mpt.puts_forest_device(TU.CONFIGS[k]["two_phase"], s.keys.data_ptr(), s.kidx.data_ptr(),
                                        s.vals.data_ptr(), s.vidx.data_ptr(), s.tids.data_ptr(), nn, kb, vb)
            self.mpt.hash_onepass_v2()
        # and the read/write resolution of a mixed batch of that size
        rec, self.record = self.record, None
        run = [Request(-1, "put", tid, n // 2 + 1, 0.5, 0.5, 0x5C7A7C7), Request(-1, "get", tid, n // 2 + 1, 0.5,
                                                                                0.0, 0x5C7A7C8)]
        nn, kb, vb = self.build(run)
        self.mixed(run, TU.FIXED_LOCKNU, nn, kb, vb)
        self.record = rec
        del self.tenant_of[tid]
        del self.count[tid]

    def build(self, reqs):
        """Generate the merged batch of the requests into the stage, in
        request order; in a mixed batch get keys have empty values and
        stage.rw flags every key (1 put, 0 get)."""
        s = self.stage
        torch = s.torch
        n = sum(r.n for r in reqs)
        kb = sum(r.n * (2 * self.tenant_of[r.tenant].key_bytes + 1) for r in reqs)
        vb = sum(r.n * self.tenant_of[r.tenant].value_bytes for r in reqs if r.kind == "put")
        mixed = len(set(r.kind for r in reqs)) > 1
        s.ensure(n, kb, max(vb, 1))
        off = koff = voff = 0
        for r in reqs:
            t = self.tenant_of[r.tenant]
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
            elif mixed:
                s.vidx[2 * off: 2 * (off + r.n): 2] = voff
                s.vidx[2 * off + 1: 2 * (off + r.n): 2] = voff - 1
            if mixed:
                s.rw[off: off + r.n] = 1 if r.kind == "put" else 0
            s.tids[off: off + r.n] = t.tid
            off += r.n
            koff += r.n * w
        torch.cuda.synchronize(s.dev)
        return n, kb, voff

    def features(self, reqs, n, kb, vb):
        """Selector features from the library (gmpt_batch_features_trie_device:
        exact totals plus one sampling kernel over the staged keys), with the
        touched tenants' key count and number."""
        s = self.stage
        touched = set(r.tenant for r in reqs)
        trie_keys = sum(self.count[t] for t in touched)
        return self.mpt.features_device(s.keys.data_ptr(), s.kidx.data_ptr(), n, kb, vb, len(touched), trie_keys)

    def snapshot(self, n, kb, vb):
        """Host copy of the staged batch (keys, values, trie ids)."""
        s = self.stage
        return W.Batch(s.keys[:kb].cpu().numpy(), s.kidx[: 2 * n].cpu().numpy(), s.vals[:vb].cpu().numpy(),
                       s.vidx[: 2 * n].cpu().numpy()), s.tids[:n].cpu().numpy()

    def put(self, reqs, k: int, n, kb, vb):
        if self.record is not None:
            self.record.append(self.snapshot(n, kb, vb))
        s = self.stage
        touched = sorted(set(r.tenant for r in reqs))
        # the library runs schedule k (a persistent schedule hashes in the
        # same launch, and the hash call then has nothing left to do)
        self.mpt.puts_schedule_device(k, s.keys.data_ptr(), s.kidx.data_ptr(), s.vals.data_ptr(), s.vidx.data_ptr(),
                                      n, kb, vb, d_tids=s.tids.data_ptr())
        self.mpt.hash_onepass_v2()
        return self.mpt.get_roots(touched)

    def mixed(self, reqs, k: int, n, kb, vb):
        """A built mixed batch in one gmpt_puts_with_read_device call (as if
        applied in request order) + PhaseHC + roots of the written tries;
        returns the read sizes in read order.  A persistent configuration
        (no read support) runs as LockNU with its latch ways."""
        s = self.stage
        if self.record is not None:
            b, tids = self.snapshot(n, kb, vb)
            sel = np.nonzero(s.rw[:n].cpu().numpy() == 1)[0]
            self.record.append((b.subset(sel), tids[sel]))
        two = TU.apply_config(self.mpt, k) and not TU.CONFIGS[k].get("persistent")
        cnt = self.mpt.puts_with_read_device(two, s.keys.data_ptr(), s.kidx.data_ptr(), s.rw.data_ptr(),
                                             s.vals.data_ptr(), s.vidx.data_ptr(), n, kb, vb,
                                             s.out_hp.data_ptr(), s.out_len.data_ptr(), d_tids=s.tids.data_ptr())
        self.mpt.hash_onepass_v2()
        self.mpt.get_roots(sorted(set(r.tenant for r in reqs if r.kind == "put")))
        return s.out_len[:cnt].cpu().numpy()

    def get(self, n, kb):
        s = self.stage
        if n > self.get_cap:  # pinned result buffers, reused
            torch = s.torch
            self.get_cap = int(n * 1.25) + 1024
            self.h_hps = torch.empty(self.get_cap, dtype=torch.int64).pin_memory().numpy().view(np.uint64)
            self.h_sizes = torch.empty(self.get_cap, dtype=torch.int32).pin_memory().numpy()
        _, sizes = self.mpt.gets_forest_device(s.keys.data_ptr(), s.kidx.data_ptr(), s.tids.data_ptr(), n, kb,
                                               self.h_hps, self.h_sizes)
        return sizes.copy()

    def roots(self):
        return self.mpt.get_roots(n=len(self.tenants))

    def close(self):
        self.mpt.close()


def _timed(fn):
    t0 = time.perf_counter()
    out = fn()
    return out, (time.perf_counter() - t0) * 1e3


def time_matrix(replicas, reqs, with_features=True, configs=None):
    """Every put under every configuration (replica j runs configuration
    configs[j], default j).  Returns times [N, len(CONFIGS)] (ms; nan for
    gets and for configurations not run), get times [N] (nan for puts),
    features [N, F] of the puts (zeros for gets)."""
    configs = list(range(len(replicas))) if configs is None else list(configs)
    T = np.full((len(reqs), len(TU.CONFIGS)), np.nan)
    G = np.full(len(reqs), np.nan)
    F = np.zeros((len(reqs), len(TU.FEATURES)), dtype=np.float32)
    for i, r in enumerate(reqs):
        if r.kind == "put":
            roots = None
            for j, rep in enumerate(replicas):
                k = configs[j]
                n, kb, vb = rep.build([r])
                if j == 0 and with_features:
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
    service_ms: np.ndarray | None = None  # per request (one-at-a-time server)
    slowest: list = field(default_factory=list)  # (ms, kinds, keys) of the slowest calls


def _groups(window):
    """Merge a drained window into forest calls: tenants are independent tries,
    so requests of different tenants commute; each tenant's requests keep
    their order.  Repeatedly, every tenant whose next request is of the kind
    of the oldest pending head contributes its leading run of that kind."""
    queues = {}
    for r in window:
        queues.setdefault(r.tenant, []).append(r)
    out = []
    while queues:
        heads = [q[0] for q in queues.values()]
        kind = min(heads, key=lambda r: r.i).kind
        run = []
        for t in list(queues):
            q = queues[t]
            k = 0
            while k < len(q) and q[k].kind == kind:
                k += 1
            run.extend(q[:k])
            if k == len(q):
                del queues[t]
            else:
                queues[t] = q[k:]
        out.append(sorted(run, key=lambda r: r.i))
    return out


def serve(runner, reqs, policy, batching: bool, max_keys: int = 1 << 23, mixed: bool = False) -> ServeResult:
    """Live server on a virtual clock.  policy(runner, reqs, n, kb, vb) ->
    configuration index (its own time is part of the service time).  With
    batching, the requests that arrived while the server was busy are drained
    and merged by _groups; with mixed as well, a drained window holding puts
    and gets is one mixed read/write call instead (the batch acts as if
    applied in request order, so results are unchanged).  get_sizes holds
    each get request's result sizes (None for puts), in request order."""
    lat = np.zeros(len(reqs))
    svc = np.zeros(len(reqs))
    free = 0.0
    busy = 0.0
    groups = 0
    choices = {}
    gets = [None] * len(reqs)
    calls = []
    base = reqs[0].i if reqs else 0
    i = 0
    while i < len(reqs):
        start = max(free, reqs[i].arrival)
        j = i + 1
        if batching:
            tot = reqs[i].n
            while j < len(reqs) and reqs[j].arrival <= start and tot + reqs[j].n <= max_keys:
                tot += reqs[j].n
                j += 1
        t = start
        window = reqs[i:j]
        if not batching:
            runs = [[reqs[i]]]
        elif mixed and len(set(r.kind for r in window)) > 1:
            runs = [window]
        else:
            runs = _groups(window)
        for run in runs:
            n, kb, vb = runner.build(run)
            t0 = time.perf_counter()
            if len(set(r.kind for r in run)) > 1:
                k = policy(runner, run, n, kb, vb)
                choices[k] = choices.get(k, 0) + 1
                sizes = runner.mixed(run, k, n, kb, vb)
                at = 0
                for r in run:
                    if r.kind == "get":
                        gets[r.i - base] = sizes[at: at + r.n]
                        at += r.n
            elif run[0].kind == "put":
                k = policy(runner, run, n, kb, vb)
                choices[k] = choices.get(k, 0) + 1
                runner.put(run, k, n, kb, vb)
            else:
                sizes = runner.get(n, kb)
                at = 0
                for r in run:
                    gets[r.i - base] = sizes[at: at + r.n]
                    at += r.n
            ms = (time.perf_counter() - t0) * 1e3
            calls.append((round(ms, 3), "".join(sorted(set(r.kind[0] for r in run))), n))
            busy += ms
            t += ms / 1e3
            groups += 1
            for r in run:
                lat[r.i - base] = (t - r.arrival) * 1e3
                svc[r.i - base] = ms / len(run)
        free = t
        i = j
    return ServeResult(lat, busy, sum(r.n for r in reqs), 0, groups, choices, gets, svc,
                       sorted(calls, reverse=True)[:3])
