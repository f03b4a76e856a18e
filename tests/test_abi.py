"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import re
from pathlib import Path

import gmpt

REPO = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in sorted((REPO / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name in ("if", "defined", "sizeof", "extern"):
                continue
            # function declarations end with ');' at top level
            rest = text[m.end():]
            depth, i = 1, 0
            while depth and i < len(rest):
                depth += {"(": 1, ")": -1}.get(rest[i], 0)
                i += 1
            if rest[i:].lstrip().startswith(";"):
                names.add(name)
    return names


def test_library_builds_and_loads():
    if not gmpt.LIB_PATH.exists():
        gmpt.build()
    L = gmpt.lib()
    assert L.gmpt_version() == 1


def test_every_declared_symbol_is_exported():
    gmpt.lib()
    so = ctypes.CDLL(str(gmpt.LIB_PATH))
    names = declared_functions()
    assert {"build_mpt_2phase", "build_mpt_olc", "preprocess", "get_all_nodes", "init_mpt",
            "insert_mpt_2phase", "insert_mpt_olc", "free_mpt"} <= names
    missing = [n for n in sorted(names) if not hasattr(so, n)]
    assert not missing, missing
    assert set(gmpt.EXPORTS) >= names


def test_reference_abi_types_match():
    # struct nodeset and enum TrieType keep the reference layout (lib/libgmpt.h:7-18)
    assert ctypes.sizeof(gmpt.NodeSet) == 32
    text = (REPO / "include" / "libgmpt.h").read_text()
    assert "STATE_TRIE = 0" in text and "TRANSACTION_TRIE = 1" in text and "RECEIPT_TRIE = 2" in text


def test_cpp_facade_compiles_against_the_headers(tmp_path):
    import subprocess

    exe = tmp_path / "facade_example"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(REPO / "include"),
                        str(REPO / "tests" / "cpp" / "facade_example.cpp"),
                        "-L", str(gmpt.LIB_PATH.parent), "-lgmpt_b200", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_entry_points_reject_a_null_trie_without_touching_the_device():
    # argument checks run before any CUDA call, so they hold on a GPU-less host
    L = gmpt.lib()
    E_ARG = 5
    null = None
    n = ctypes.c_int(0)
    assert L.gmpt_deletes(null, null, null, null, 1) == E_ARG
    assert L.gmpt_deletes_device(null, null, null, null, 1, 16) == E_ARG
    assert L.gmpt_puts_raw(null, 0, null, null, null, null, null, null, 1) == E_ARG
    assert L.gmpt_puts_raw_device(null, 1, null, null, null, null, null, null, 1, 8, 8) == E_ARG
    assert L.gmpt_puts_with_read_forest(null, 0, null, null, null, null, null, null, null, 1, null, null,
                                        ctypes.byref(n)) == E_ARG
    assert L.gmpt_puts_latching_with_read(null, null, null, ctypes.byref(n), null, null, null, null, 1, null,
                                          null) == E_ARG
    assert L.gmpt_puts_pipeline_raw(null, 1, null, null, null, null, null, null, null, null, null) == E_ARG
    assert b"null" in L.gmpt_last_error_message()


def test_keccak_batches_reject_an_end_index_that_would_overflow():
    # an end index near INT64_MAX must fail the argument check (before any
    # CUDA call), not wrap to a small byte count in `end + 1`
    L = gmpt.lib()
    E_ARG = 5
    data = (ctypes.c_uint8 * 16)()
    out = (ctypes.c_uint8 * 32)()
    for end in (2 ** 63 - 1, 2 ** 63 - 2, 2 ** 63 - 60):
        idx = (ctypes.c_int64 * 2)(0, end)
        assert L.gmpt_keccak256_batch(data, idx, 1, out) == E_ARG
        assert L.gmpt_keccak256_batch_noalloc(data, idx, 1, out) == E_ARG
    # the no-alloc limit is checked per pair, before any device work
    idx = (ctypes.c_int64 * 2)(0, 2 << 20)
    assert L.gmpt_keccak256_batch_noalloc(data, idx, 1, out) == E_ARG
    assert b"limit" in L.gmpt_last_error_message()
