"""Benchmark of the batched MPT put + root-hash path (one JSON line on rank 0).

Workload (default): YCSB-shaped bulk load + update on one trie per GPU --
16M inserts of 'user' + 19-digit keys (23 B) with 100 B values into an empty
trie, root hash, then 16M zipf(0.99) updates over the loaded keys, root hash.
One step = both batches (32M keys) on a fresh trie; metric = keys / second.

  value  inputs already in HBM when the timed region starts (device API)
  e2e    the same through the host C ABI from pinned host buffers, H2D of the
         step's inputs and D2H of both roots inside the timed region
Multi-GPU: replicas only (each rank runs the same independent step on its own
GPU); value = keys of all ranks / max over ranks of the step time.
`--impl reference` times the reference's own CPU MPT (oracle/_ref, compiled
from the reference sources) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "gpu-merkle-patricia-trie_b200"))

from gmpt import workloads as W  # noqa: E402

PEAKS_FILE = REPO / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--n", type=int, default=1 << 24, help="keys per batch")
    p.add_argument("--strategy", default="auto", help="auto | 2phase | latching | 2phase,latching")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--cpu-sample", type=int, default=1 << 20)
    return p.parse_args()


# --------------------------------------------------------------------------


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def peaks():
    if PEAKS_FILE.exists():
        d = json.loads(PEAKS_FILE.read_text())
        return float(d.get("hbm_gbs", FALLBACK_HBM_GBS)), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------


def make_workload(n):
    load = W.ycsb_load(n, seed=0x5EED0002)
    upd = W.ycsb_zipf_updates(n, n, seed=0x5EED0003)
    return [load, upd]


def choose(strategy, k):
    if strategy == "auto":
        # bulk load into the empty trie: sort-based build; update batch: in-place CAS
        return "2phase" if k == 0 else "latching"
    parts = strategy.split(",")
    return parts[min(k, len(parts) - 1)]


def run_reference(args, world, rank):
    if rank != 0:
        return
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as O

    threads = os.cpu_count() or 1
    n = min(args.cpu_sample, args.n)
    batches = make_workload(args.n)
    sample = [b.subset(np.arange(n)) for b in batches]
    kind = "reference" if O.ref_lib(big=True) is not None else "port"
    times = []
    for it in range(args.warmup + args.steps):
        if kind == "reference":
            t = O.RefTrie(big=True, threads=threads)
            t0 = time.perf_counter()
            for b in sample:
                t.puts_lock_and_hash(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
            root = t.root(parallel=True)
            dt = time.perf_counter() - t0
            t.close()
        else:
            t = O.OracleTrie()
            t0 = time.perf_counter()
            for b in sample:
                t.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
                t.hash()
            root = t.root()
            dt = time.perf_counter() - t0
        if it >= args.warmup:
            times.append(dt)
    keys = 2 * n
    v = keys / statistics.median(times) / 1e6
    line = {
        "metric": "put+root-hash Mkeys/s", "value": round(v, 4), "unit": "Mkeys/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(statistics.median(times) * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": f"ycsb load {args.n} + zipf0.99 updates {args.n}, 23 B keys / 100 B values",
                   "sample_keys_per_batch": n},
        "cpu_baseline": {"value": round(v, 4), "unit": "Mkeys/s", "cores": threads if kind == "reference" else 1,
                         "kind": kind,
                         "sample": f"first {n} keys of each batch (load, update); reference CpuMPT "
                                   "puts_lock + hashs_onepass on std::thread parallel_for"},
        "e2e": {"value": round(v, 4), "unit": "Mkeys/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "root": root.hex(),
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(args, batches):
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as O

    n = min(args.cpu_sample, args.n)
    sample = [b.subset(np.arange(n)) for b in batches]
    threads = os.cpu_count() or 1
    if O.ref_lib(big=True) is not None:
        t = O.RefTrie(big=True, threads=threads)
        t0 = time.perf_counter()
        for b in sample:
            t.puts_lock_and_hash(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
        dt = time.perf_counter() - t0
        t.close()
        kind, cores = "reference", threads
        desc = "reference CpuMPT puts_lock + hashs_onepass (std::thread parallel_for)"
    else:
        t = O.OracleTrie()
        t0 = time.perf_counter()
        for b in sample:
            t.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
            t.hash()
        dt = time.perf_counter() - t0
        kind, cores, desc = "port", 1, "C restatement of the reference CPU MPT, one thread"
    return {"value": round(2 * n / dt / 1e6, 4), "unit": "Mkeys/s", "cores": cores, "kind": kind,
            "sample": f"first {n} keys of the load and of the update batch; {desc}"}


def run_ours(args, world, rank, local):
    import torch

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", device_id=dev)
    import gmpt

    batches = make_workload(args.n)
    dbat = []
    for b in batches:
        dbat.append(dict(
            k=torch.from_numpy(b.keys_hexs).to(dev), ki=torch.from_numpy(b.keys_indexs).to(dev),
            v=torch.from_numpy(b.values).to(dev), vi=torch.from_numpy(b.values_indexs).to(dev),
            n=b.n, kb=b.key_bytes(), vb=b.value_bytes()))
    t = gmpt.MPT(device=local)
    stream = torch.cuda.ExternalStream(t.stream_ptr(), device=dev)
    keys_per_step = sum(b.n for b in batches)

    def step_device(timing=False):
        t.reset()
        roots = []
        info = []
        for k, d in enumerate(dbat):
            s = choose(args.strategy, k)
            t.puts_device(s == "2phase", d["k"].data_ptr(), d["ki"].data_ptr(), d["v"].data_ptr(),
                          d["vi"].data_ptr(), d["n"], d["kb"], d["vb"])
            t.hash_onepass_v2()
            roots.append(t.get_root_hash())
            if timing:
                info.append(t.stats())
        return roots, info

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    t.set_timing(False)
    for _ in range(args.warmup):
        roots, _ = step_device()
    # timed region (device-resident inputs)
    t.set_timing(True)
    sampler = ClockSampler(local)
    ev = []
    stats_all = []
    barrier()
    launches0 = gmpt.launch_count()
    sampler.start()
    for _ in range(args.steps):
        a = torch.cuda.Event(enable_timing=True)
        z = torch.cuda.Event(enable_timing=True)
        # reset is not part of the step: a fresh trie per step
        t.reset()
        a.record(stream)
        roots_s = []
        info = []
        for k, d in enumerate(dbat):
            s = choose(args.strategy, k)
            t.puts_device(s == "2phase", d["k"].data_ptr(), d["ki"].data_ptr(), d["v"].data_ptr(),
                          d["vi"].data_ptr(), d["n"], d["kb"], d["vb"])
            st_put = t.stats()
            t.hash_onepass_v2()
            roots_s.append(t.get_root_hash())
            info.append((st_put, t.stats()))
        z.record(stream)
        ev.append((a, z))
        stats_all.append(info)
    barrier()
    clocks = sampler.stop()
    launches_per_step = (gmpt.launch_count() - launches0) / args.steps
    step_ms = [a.elapsed_time(z) for a, z in ev]
    ms = statistics.mean(step_ms)
    if world > 1:
        import torch.distributed as dist

        x = torch.tensor([ms], device=dev)
        dist.all_reduce(x, op=dist.ReduceOp.MAX)
        ms = float(x.item())
    value = keys_per_step * world / (ms / 1e3) / 1e6

    # dominant kernel: the fused encode + Keccak level kernels of PhaseHC
    hk_ms = [h["t_hash_kernels_ms"] for info in stats_all for (_, h) in info]
    hk_launch = [h["hash_launches"] for info in stats_all for (_, h) in info]
    enc = [h["last_enc_bytes"] + 32 * h["last_hashed"] for info in stats_all for (_, h) in info]
    perms = [h["last_keccak_blocks"] for info in stats_all for (_, h) in info]
    hash_ms_step = sum(hk_ms) / len(stats_all)
    alg_bytes_per_launch = sum(enc) / sum(hk_launch)
    avg_launch_s = (sum(hk_ms) / 1e3) / sum(hk_launch)
    hbm_peak, peak_kind = peaks()
    kpeak = gmpt.keccak_peak(local)
    achieved = alg_bytes_per_launch / avg_launch_s / 1e9
    phase = {}
    for key in ("t_stage_ms", "t_sort_ms", "t_walk_ms", "t_build_ms"):
        phase[key] = [round(statistics.mean(info[k][0][key] for info in stats_all), 3) for k in range(len(dbat))]
    phase["t_hash_ms"] = [round(statistics.mean(info[k][1]["t_hash_ms"] for info in stats_all), 3)
                          for k in range(len(dbat))]
    phase["hash_kernels_ms"] = [round(statistics.mean(info[k][1]["t_hash_kernels_ms"] for info in stats_all), 3)
                                for k in range(len(dbat))]
    last = stats_all[-1]

    # e2e: host C ABI from pinned buffers
    e2e = None
    if not args.no_e2e:
        pinned = []
        h2d = 0
        for b in batches:
            arrs = [torch.from_numpy(a).pin_memory() for a in (b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)]
            pinned.append(arrs)
            h2d += sum(a.numel() * a.element_size() for a in arrs)
        L = gmpt.lib()
        import ctypes

        def step_host():
            t.reset()
            out = []
            for k, (arrs, b) in enumerate(zip(pinned, batches)):
                s = choose(args.strategy, k)
                f = L.gmpt_puts_2phase if s == "2phase" else L.gmpt_puts_latching
                rc = f(t._h, *[ctypes.c_void_p(a.data_ptr()) for a in arrs], None, b.n)
                if rc:
                    raise RuntimeError(L.gmpt_last_error_message().decode())
                t.hash_onepass_v2()
                out.append(t.get_root_hash())
            return out

        t.set_timing(False)
        step_host()
        e2e_ms = []
        barrier()
        for _ in range(args.steps):
            t.reset()
            torch.cuda.synchronize(dev)
            a = torch.cuda.Event(enable_timing=True)
            z = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            r2 = step_host()
            z.record(stream)
            z.synchronize()
            e2e_ms.append(a.elapsed_time(z))
            assert r2 == roots_s, "host and device paths disagree"
        barrier()
        ems = statistics.mean(e2e_ms)
        if world > 1:
            import torch.distributed as dist

            x = torch.tensor([ems], device=dev)
            dist.all_reduce(x, op=dist.ReduceOp.MAX)
            ems = float(x.item())
        e2e = {"value": round(keys_per_step * world / (ems / 1e3) / 1e6, 3), "unit": "Mkeys/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": 32 * len(batches),
               "ms_per_step": round(ems, 3)}

    line = {
        "metric": "put+root-hash Mkeys/s", "value": round(value, 3), "unit": "Mkeys/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": f"ycsb-shaped load {args.n} + zipf(0.99) updates {args.n}; 23 B keys, 100 B values;"
                               " fresh trie per step",
                   "keys_per_step": keys_per_step, "strategy": [choose(args.strategy, k) for k in range(len(dbat))],
                   "l2": "inputs (> 5 GB per step) larger than the 126 MB L2; no flush needed",
                   "parallelism": f"replicas x{world}"},
        "gpu_launches": int(round(launches_per_step)),
        "roots": [r.hex() for r in roots_s],
        "phases_ms": phase,
        "roofline": {"bound": "hbm", "kernel": "k_hash_level (fused RLP encode + Keccak-256)",
                     "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                     "frac": round(achieved / hbm_peak, 4), "traffic": None, "peak_kind": peak_kind,
                     "alg_bytes_per_launch": int(alg_bytes_per_launch),
                     "avg_launch_us": round(avg_launch_s * 1e6, 2)},
        "keccak": {"permutations_per_step": int(sum(perms) / len(stats_all)),
                   "perm_per_s": round(sum(perms) / (sum(hk_ms) / 1e3), 1),
                   "peak_perm_per_s": round(kpeak, 1),
                   "frac": round(sum(perms) / (sum(hk_ms) / 1e3) / kpeak, 4),
                   "peak_kind": "measured live: register-only Keccak-f[1600] loop (gmpt_keccak_peak)",
                   "hash_kernels_ms_per_step": round(hash_ms_step, 3)},
        "clocks": clocks,
        "e2e": e2e,
        "trie": {k: last[-1][1][k] for k in ("n_full", "n_short", "n_value", "last_dirty", "last_hashed")},
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(args, batches)
    if rank == 0:
        print(json.dumps(line), flush=True)
    t.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
