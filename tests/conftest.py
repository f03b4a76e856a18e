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
def gpu_lib():
    """The CUDA library; GPU tests fail loudly if it is missing."""
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import gmpt

    gmpt.lib()
    return gmpt
