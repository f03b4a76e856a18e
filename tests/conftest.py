"""Shared test setup: import paths, the `gpu` marker and golden fixtures."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO / "oracle"))
sys.path.insert(0, str(REPO / "gpu-merkle-patricia-trie_b200"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200 / sm_100a)")


def make_batch(keys_nibbles, values):
    """Flat reference layout from python lists of nibble lists / bytes."""
    from gmpt import workloads as W

    kh, ki, pos = [], [], 0
    for k in keys_nibbles:
        kh += list(k)
        ki += [pos, pos + len(k) - 1]
        pos += len(k)
    vb, vi, pos = b"", [], 0
    for v in values:
        vb += v
        vi += [pos, pos + len(v) - 1]
        pos += len(v)
    return W.Batch(np.array(kh, np.uint8), np.array(ki, np.int32), np.frombuffer(vb, np.uint8).copy(),
                   np.array(vi, np.int64))


def nib(key: bytes):
    return [b for x in key for b in (x >> 4, x & 15)] + [16]


@pytest.fixture(scope="session")
def golden():
    data = json.loads((REPO / "tests" / "golden" / "golden_cases.json").read_text())
    cases = []
    for c in data["cases"]:
        batches = [make_batch([list(bytes.fromhex(k)) for k in b["keys"]],
                              [bytes.fromhex(v) for v in b["values"]]) for b in c["batches"]]
        probes = make_batch([list(bytes.fromhex(p)) for p in c["probes"]], [b"x"] * len(c["probes"]))
        cases.append({"name": c["name"], "batches": batches, "roots": [bytes.fromhex(r) for r in c["roots"]],
                      "probes": probes,
                      "probe_values": [None if v is None else bytes.fromhex(v) for v in c["probe_values"]]})
    return cases


@pytest.fixture(scope="session")
def config_roots():
    """Oracle roots of the benchmark configurations at full size
    (tests/golden/make_config_roots.py)."""
    return json.loads((REPO / "tests" / "golden" / "config_roots.json").read_text())["cases"]


def last_occurrence(batch, idx):
    """For sampled key positions idx, the batch position of the last
    occurrence of the same key (keys of any length): a 64-bit hash of every
    key groups the candidates, whose bytes are then compared."""
    ki = batch.keys_indexs.reshape(-1, 2).astype(np.int64)
    lens = ki[:, 1] - ki[:, 0] + 1
    n = len(ki)
    kh = batch.keys_hexs.astype(np.uint64)
    total = int(lens.sum())
    starts = np.zeros(n, dtype=np.int64)
    np.cumsum(lens[:-1], out=starts[1:])
    if total != len(kh) or np.any(ki[:, 0] != starts):
        raise ValueError("keys must tile the stream")
    pos = np.arange(total, dtype=np.uint64) - np.repeat(starts, lens).astype(np.uint64)
    with np.errstate(over="ignore"):
        w = (pos + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
        w ^= w >> np.uint64(29)
        h = np.add.reduceat((kh + np.uint64(1)) * w, starts) ^ (lens.astype(np.uint64) * np.uint64(0xC2B2AE3D27D4EB4F))
    order = np.argsort(h, kind="stable")
    hs = h[order]
    out = []
    for i in np.asarray(idx, dtype=np.int64):
        a = np.searchsorted(hs, h[i], side="left")
        z = np.searchsorted(hs, h[i], side="right")
        best = -1
        for j in order[a:z]:
            if batch.key(int(j)) == batch.key(int(i)):
                best = max(best, int(j))
        out.append(best)
    return np.array(out, dtype=np.int64)


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library; GPU tests fail loudly if it is missing."""
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import gmpt

    gmpt.lib()
    return gmpt
