"""Failure bounds, exercised without faulting or hanging the GPU: each is a
limit set by the host (a CAS retry budget of 1, a grid-barrier wait of 1 ns,
a branch-pool cap) that the kernels run into and report through the error
word, after which the library stays usable.  The reference instead spins
without bound on its node locks (util/lock.cuh:17-21,
gpu_mpt_kernels.cuh:978) and asserts on arena overflow
(util/allocator.cuh:115-118)."""
import numpy as np
import pytest

import oracle as O
from gmpt import workloads as W

pytestmark = pytest.mark.gpu

E_CAPACITY, E_RETRY_LIMIT, E_INTERNAL = 3, 4, 6


def oracle_root(*batches):
    o = O.OracleTrie()
    for b in batches:
        o.puts(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    o.hash()
    return o.root()


def test_locknu_retry_limit_reports_and_the_batch_can_be_completed(gpu_lib):
    b = W.random_keys(1 << 16, 32, 40, seed=0x5EED0F01)
    t = gpu_lib.MPT()
    t.set_option("latch_dedup", 0)
    t.set_option("retry_limit", 1)  # every key races for the empty root slot
    with pytest.raises(gpu_lib.GmptError) as ei:
        t.puts_latching_with_valuehp_v2(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    assert ei.value.code == E_RETRY_LIMIT and "retry" in str(ei.value)
    # keys that gave up linked nothing; putting the batch again completes it
    t.set_option("retry_limit", 1 << 20)
    t.puts_latching_with_valuehp_v2(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    t.hash_onepass_v2()
    assert t.get_root_hash() == oracle_root(b)
    t.close()


def test_block_barrier_wait_gives_up_and_the_trie_is_reloaded(gpu_lib):
    b = W.random_keys(1 << 15, 32, 40, seed=0x5EED0F02)
    t = gpu_lib.MPT()
    t.set_option("block_grid", 0)
    t.set_option("block_barrier_ns", 1)  # any wait at a grid barrier runs out
    tid = np.zeros(b.n, np.int32)
    with pytest.raises(gpu_lib.GmptError) as ei:
        t.block_update(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs, tid, b.n, [0])
    assert ei.value.code == E_INTERNAL and "barrier" in str(ei.value)
    # the block is partly applied: reset, restore the wait, load again
    t.reset()
    t.set_option("block_barrier_ns", 2_000_000_000)
    roots = t.block_update(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs, tid, b.n, [0])
    assert roots[0] == oracle_root(b)
    t.close()


@pytest.mark.parametrize("strategy", ["2phase", "latching"])
def test_branch_pool_cap_reports_capacity_from_the_kernel(gpu_lib, strategy):
    b = W.random_keys(1 << 16, 32, 40, seed=0x5EED0F03)
    t = gpu_lib.MPT()
    t.set_option("max_branch_nodes", 2048)  # a 64K-key trie needs ~4.4K branches
    put = t.puts_2phase_with_valuehp if strategy == "2phase" else t.puts_latching_with_valuehp_v2
    with pytest.raises(gpu_lib.GmptError) as ei:
        put(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    assert ei.value.code == E_CAPACITY
    t.reset()
    t.set_option("max_branch_nodes", 0)
    put(b.keys_hexs, b.keys_indexs, b.values, b.values_indexs)
    t.hash_onepass_v2()
    assert t.get_root_hash() == oracle_root(b)
    t.close()


def test_failure_options_reject_bad_values(gpu_lib):
    t = gpu_lib.MPT()
    for name, v in (("retry_limit", 0), ("block_barrier_ns", 0), ("max_branch_nodes", -1)):
        with pytest.raises(gpu_lib.GmptError):
            t.set_option(name, v)
    t.close()
