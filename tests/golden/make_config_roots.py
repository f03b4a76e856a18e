"""Roots of the benchmark configurations at their full sizes, from the oracle.

Writes tests/golden/config_roots.json.  Every input is regenerated from the
seeded generators in gmpt.workloads / gmpt.eth (the GPU tests and bench.py
rebuild the same bytes), inserted into the C restatement of the reference
CPU MPT (oracle/mpt_oracle.c, single thread, sequential puts in index order
with the last write winning, cpu_mpt.cuh:232-505) and hashed; the roots are
recorded.  The 1M-key cases are also run through the reference's own CpuMPT
built from its sources (oracle/_ref) when that library exists here, and the
script stops if the two disagree.

Cases (keys are hex-nibble keys as everywhere else):
  c1_random_1m   2^20 random 32 B keys, 64 B values, one batch (REF mode)
  c2_ycsb_16m    16M YCSB-shaped loads (23 B keys, 100 B values), then 16M
                 zipf(0.99) updates over them: the root after each (REF)
  c2_ycsb_1m     the same at 2^20 keys (also checked on the reference build)
  c3_vocab_1m    2^20 vocabulary keys of 8-96 B, values 128 B - 4 KB (REF)
  c3_vocab_8m    the same at 8M keys (REF)
  c4_eth_1m      Ethereum-shaped forest in go-ethereum encoding: a state trie
                 of 2^20 accounts, then 16 blocks of U[150, 400] account
                 updates with power-law storage tries (alpha 1.5, <= 5000
                 slots); per block the state root and a Keccak-256 over the
                 concatenated roots (state root, then each touched storage
                 trie's root zero-padded to 32 bytes, in out_ids order)

Run from the repository root (about 10 minutes and 40 GB of host memory for
the 16M and 8M cases; --quick skips them):
    python tests/golden/make_config_roots.py [--quick]
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO / "oracle"))
sys.path.insert(0, str(REPO / "gpu-merkle-patricia-trie_b200"))

import oracle as O  # noqa: E402
from gmpt import eth  # noqa: E402
from gmpt import workloads as W  # noqa: E402

OUT = Path(__file__).resolve().parent / "config_roots.json"

ETH_ACCOUNTS = 1 << 20
ETH_BLOCKS = 16


def oracle_roots(batches, mode=O.MODE_REF):
    t = O.OracleTrie(mode)
    roots = []
    for b in batches:
        t.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        t.hash()
        roots.append(t.root())
    t.close()
    return roots


def reference_roots(batches):
    """The reference's own CpuMPT (puts_baseline + hashs_dirty_flag), or None."""
    if O.ref_lib(big=True) is None:
        return None
    t = O.RefTrie(big=True, threads=1)
    roots = []
    for b in batches:
        t.puts_baseline(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        t.hash()
        roots.append(t.root())
    t.close()
    return roots


def block_digest(roots):
    return O.keccak256(b"".join(r[:32].ljust(32, b"\0") for r in roots))


def eth_case(accounts, blocks):
    state = eth.make_state(accounts, O.keccak256_rows)
    t_state = O.OracleTrie(O.MODE_GETH)
    b = state.batch
    t_state.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    t_state.hash()
    out = {"state_root": t_state.root().hex(), "blocks": []}
    storage = {}
    gen = eth.EthBlocks(state, O.keccak256_rows)
    for _ in range(blocks):
        blk = gen.next()
        bb = blk.batch
        sroots = {}
        for j, sid in enumerate(blk.storage_ids.tolist()):
            sub = bb.subset(np.arange(blk.spans[j], blk.spans[j + 1]))
            t = storage.setdefault(sid, O.OracleTrie(O.MODE_GETH))
            t.puts(sub.keys_hexs, sub.keys_indexs, sub.values, sub.values_indexs)
            t.hash()
            sroots[sid] = t.root()
        vb = eth.patched_values(blk, sroots)
        acc = W.Batch(bb.keys_hexs, bb.keys_indexs, vb, bb.values_indexs).subset(np.arange(blk.n0, blk.n))
        t_state.puts(acc.keys_hexs, acc.keys_indexs, acc.values, acc.values_indexs)
        t_state.hash()
        roots = [t_state.root()] + [sroots[s] for s in blk.storage_ids.tolist()]
        out["blocks"].append({"keys": int(blk.n), "tries": int(len(roots)), "state_root": roots[0].hex(),
                              "roots_digest": block_digest(roots).hex()})
    for t in storage.values():
        t.close()
    t_state.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true", help="skip the 16M and 8M cases")
    args = ap.parse_args()
    data = json.loads(OUT.read_text()) if OUT.exists() else {}
    data["generator"] = "tests/golden/make_config_roots.py (oracle/mpt_oracle.c restatement)"
    cases = data.setdefault("cases", {})

    def record(name, batches, mode=O.MODE_REF, pin_reference=False, **meta):
        t0 = time.time()
        roots = oracle_roots(batches, mode)
        entry = {"roots": [r.hex() for r in roots], "mode": "geth" if mode == O.MODE_GETH else "ref",
                 "keys": [int(b.n) for b in batches], **meta}
        if pin_reference:
            ref = reference_roots(batches)
            if ref is not None:
                if ref != roots:
                    raise SystemExit(f"{name}: the oracle and the reference build disagree")
                entry["reference_build_agrees"] = True
        cases[name] = entry
        print(f"{name}: {[r.hex()[:16] for r in roots]} ({time.time() - t0:.1f} s)", flush=True)
        OUT.write_text(json.dumps(data, indent=1) + "\n")

    record("c1_random_1m", [W.random_keys(1 << 20)], pin_reference=True,
           workload="random_keys(2^20), seed 0x5EED0001")
    n = 1 << 20
    record("c2_ycsb_1m", [W.ycsb_load(n, seed=0x5EED0002), W.ycsb_zipf_updates(n, n, seed=0x5EED0003)],
           pin_reference=True, workload="ycsb_load(2^20) then ycsb_zipf_updates(2^20, 2^20)")
    record("c3_vocab_1m", [W.vocab_keys(1 << 20)], pin_reference=True, workload="vocab_keys(2^20), defaults")
    t0 = time.time()
    cases["c4_eth_1m"] = dict(eth_case(ETH_ACCOUNTS, ETH_BLOCKS), accounts=ETH_ACCOUNTS,
                              workload=f"eth.make_state({ETH_ACCOUNTS}) + {ETH_BLOCKS} EthBlocks, geth encoding")
    print(f"c4_eth_1m: {cases['c4_eth_1m']['state_root'][:16]} ({time.time() - t0:.1f} s)", flush=True)
    OUT.write_text(json.dumps(data, indent=1) + "\n")
    if not args.quick:
        n = 1 << 24
        record("c2_ycsb_16m", [W.ycsb_load(n, seed=0x5EED0002), W.ycsb_zipf_updates(n, n, seed=0x5EED0003)],
               workload="ycsb_load(2^24) then ycsb_zipf_updates(2^24, 2^24)")
        record("c3_vocab_8m", [W.vocab_keys(8 << 20)], workload="vocab_keys(8 * 2^20), defaults")


if __name__ == "__main__":
    main()
