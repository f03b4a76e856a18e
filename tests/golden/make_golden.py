"""Generate tests/golden/golden_cases.json from the REFERENCE's own CPU MPT.

Runs the reference's CpuMPT::Compress::MPT (puts_baseline + hashs_dirty_flag +
gets_baseline, compiled from its unmodified sources into
oracle/_ref/libgmpt_ref.so by oracle/Makefile) on small seeded batches and
records the root after every batch and the value of sampled keys.  The CPU
restatement in oracle/ is checked against the same numbers while writing, and
the tests check both the restatement and the GPU path against this file.

Usage (where oracle/_ref is built):  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO / "oracle"))
sys.path.insert(0, str(REPO / "gpu-merkle-patricia-trie_b200"))

import oracle as O  # noqa: E402
from gmpt import workloads as W  # noqa: E402


def batch_from(keys_nibbles, values):
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


def run_case(name, batches, probes):
    ref = O.RefTrie()
    orc = O.OracleTrie(O.MODE_REF)
    roots = []
    for b in batches:
        ref.puts_baseline(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        ref.hash()
        orc.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        orc.hash()
        r = ref.root()
        assert r == orc.root(), name
        roots.append(r.hex())
    pb = batch_from(probes, [b"x"] * len(probes))
    got = ref.gets(pb.keys_hexs, pb.keys_indexs)
    assert got == orc.gets(pb.keys_hexs, pb.keys_indexs), name
    ref.close()
    return {
        "name": name,
        "batches": [{"keys": [bytes(b.key(i)).hex() for i in range(b.n)],
                     "values": [b.value(i).hex() for i in range(b.n)]} for b in batches],
        "roots": roots,
        "probes": [bytes(p).hex() for p in probes],
        "probe_values": [None if g is None else g.hex() for g in got],
    }


def main():
    rng = W.Xoshiro256ss(0x601D)
    cases = []

    # the reference tests' three-key fixture (test/trie.cu:153-199)
    keys = [nib(b"doe"), nib(b"dog"), nib(b"dogglesworth")]
    cases.append(run_case("doe_dog_dogglesworth", [batch_from(keys, [b"reindeer", b"puppy", b"cat"])],
                          keys + [nib(b"do"), nib(b"dogs")]))
    # small nodes everywhere: 1-2 byte keys over a 4-letter alphabet, short values, duplicates
    for nk, vmax, tag in ((60, 4, "tiny"), (300, 12, "small")):
        ks = [nib(bytes(int(x) % 4 for x in rng.words(1 + int(rng.words(1)[0] % 2)))) for _ in range(nk)]
        vs = [rng.bytes(1 + int(rng.words(1)[0] % vmax)).tobytes() for _ in range(nk)]
        cases.append(run_case(f"{tag}_alphabet4", [batch_from(ks, vs)], ks[:40] + [nib(b"\x03\x03\x03")]))
    # one key; one-byte values below 0x80 (encoded as themselves).  Empty
    # values are left out: the reference asserts on them (node.cuh:253).
    cases.append(run_case("single_key", [batch_from([nib(b"k")], [b"\x01"])], [nib(b"k"), nib(b"j")]))
    cases.append(run_case("one_byte_values", [batch_from([nib(b"ab"), nib(b"ac")], [b"\x00", b"\x7f"])],
                          [nib(b"ab"), nib(b"ac")]))
    # random 32-byte keys / 64-byte values (bulk-load shape), two batches with overlap
    b1 = W.random_keys(200, seed=0xA1)
    b2 = W.random_keys(200, seed=0xA2)
    over = b1.subset(np.arange(0, 200, 3))  # updates of existing keys
    mix = W.Batch(*_concat(b2, over))
    cases.append(run_case("random32_two_batches", [b1, mix],
                          [list(b1.key(i)) for i in range(0, 200, 17)] + [list(b2.key(i)) for i in range(0, 200, 19)]))
    # YCSB-shaped keys with zipf duplicates
    ld = W.ycsb_load(300, seed=0xB1)
    up = W.ycsb_zipf_updates(300, 400, seed=0xB2)
    cases.append(run_case("ycsb_load_update", [ld, up], [list(ld.key(i)) for i in range(0, 300, 15)]))
    # variable-length vocabulary keys, long shared prefixes, multi-block values
    vk = W.vocab_keys(100, seed=0xC1, vmin=32, vmax=400, vmu=5.0)
    vk2 = W.vocab_keys(100, seed=0xC2, vmin=1, vmax=200, vmu=4.0)
    cases.append(run_case("vocab_two_batches", [vk, vk2], [list(vk.key(i)) for i in range(0, 100, 7)]))
    # odd-length nibble keys without byte alignment (hex keys given directly)
    ks = [[int(x) % 16 for x in rng.words(1 + int(rng.words(1)[0] % 7))] + [16] for _ in range(120)]
    vs = [rng.bytes(20 + int(rng.words(1)[0] % 40)).tobytes() for _ in range(120)]
    cases.append(run_case("odd_nibble_keys", [batch_from(ks, vs)], ks[:30]))

    out = REPO / "tests" / "golden" / "golden_cases.json"
    out.write_text(json.dumps({"generator": "tests/golden/make_golden.py",
                               "source": "reference CpuMPT (mpt-with-compress/include/mpt/cpu_mpt.cuh) via oracle/_ref",
                               "cases": cases}, indent=0))
    print(f"wrote {out} ({out.stat().st_size} bytes, {len(cases)} cases)")


def _concat(a: W.Batch, b: W.Batch):
    kh = np.concatenate([a.keys_hexs, b.keys_hexs])
    ki = np.concatenate([a.keys_indexs, b.keys_indexs + (a.keys_indexs[-1] + 1)]).astype(np.int32)
    vb = np.concatenate([a.values, b.values])
    vi = np.concatenate([a.values_indexs, b.values_indexs + (a.values_indexs[-1] + 1)])
    return kh, ki, vb, vi


if __name__ == "__main__":
    main()
