"""CPU tests of the C-ABI boundary: the library loads, exports every declared symbol, and fails
loudly (no fallback) when no GPU is present."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

import csm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def ensure_built():
    if not os.path.exists(csm.LIB_PATH) or not os.path.exists(csm.CSMG_PATH):
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "gcsm-bu_b200")], check=True)


def declared_symbols(headers=("csm.h", "csm_server.h")):
    found = set()
    for h in headers:
        text = open(os.path.join(ROOT, "include", h)).read()
        found |= set(re.findall(r"\b(csm_[a-z_]+)\s*\(", text))
    return sorted(found)


def test_header_matches_python_binding():
    assert declared_symbols(("csm.h",)) == sorted(csm.EXPORTED)
    assert declared_symbols(("csm_server.h",)) == sorted(csm.SERVER_EXPORTED)


def test_library_exports_every_declared_symbol():
    ensure_built()
    lib = ctypes.CDLL(csm.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", csm.LIB_PATH], capture_output=True, text=True).stdout
    exported = sorted(set(re.findall(r" T (csm_\w+)", out)))
    assert exported == declared_symbols()


def test_version_and_default_config():
    ensure_built()
    assert "sm_100a" in csm.version()
    cfg = csm.default_config()
    assert cfg.algorithm == 0 and cfg.matching_order == 2 and cfg.search_strategy == 2
    assert cfg.local_index == 1 and cfg.cartesian_product == 1


def test_create_fails_loudly_without_gpu():
    ensure_built()
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(csm.CsmError) as ei:
        csm.Engine()
    assert ei.value.code in (-8, -2)


def test_struct_layouts():
    assert ctypes.sizeof(csm.CsmConfig) == 4 * 8 + 8 * 4 + 4 * 8 + 4 * 2 + 8
    assert ctypes.sizeof(csm.CsmBatchResult) == 64
    assert ctypes.sizeof(csm.CsmStats) == 20 * 8
    assert ctypes.sizeof(csm.CsmServerConfig) == 4 + 4 + 8 + 8 + 4 + 7 * 4
    assert ctypes.sizeof(csm.CsmRequestInfo) == 8 + 7 * 8
    assert ctypes.sizeof(csm.CsmServerStats) == 12 * 8


def test_server_create_fails_loudly_without_gpu():
    ensure_built()
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(csm.CsmError) as ei:
        csm.Server()
    assert ei.value.code == -8


def test_binary_formats_round_trip(tmp_path):
    from csm import gen, textio
    w = gen.make_workload("c1", gen.scaled("c1", 0.05))
    df, uf = str(tmp_path / "d.bin"), str(tmp_path / "u.bin")
    textio.write_binary_data(df, w.data)
    textio.write_binary_updates(uf, w.batches)
    vl, s, d, l = textio.read_binary_data(df)
    assert (vl == w.data.vlabels).all() and (s == w.data.src).all() and (d == w.data.dst).all()
    assert (l == w.data.elabels).all()
    us, ud, ul, udl = textio.read_binary_updates(uf)
    assert len(us) == sum(len(b.src) for b in w.batches)
    assert (us[: len(w.batches[0].src)] == w.batches[0].src).all()


def test_csmg_fails_loudly_without_gpu(tmp_path):
    ensure_built()
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from csm import gen, textio
    w = gen.make_workload("c1", gen.scaled("c1", 0.05))
    qf, df, uf = (str(tmp_path / x) for x in ("q.graph", "d.graph", "u.graph"))
    textio.write_query(qf, w.queries[0])
    textio.write_data(df, w.data)
    textio.write_updates(uf, w.batches)
    p = subprocess.run([csm.CSMG_PATH, "--query", qf, "--data", df, "--update", uf, "--batch_size", "100"],
                       capture_output=True, text=True, timeout=60)
    assert p.returncode != 0
    assert "Read Graphs from Files" in p.stdout  # parsing ran, then the engine refused
    assert "no CUDA device" in p.stdout + p.stderr


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_ctypes_layouts_match_the_c_headers(tmp_path):
    # Field offsets and struct sizes of the Python binding equal the C compiler's for every
    # struct of include/csm.h and include/csm_server.h.
    exe = str(tmp_path / "abi_layout")
    subprocess.run(["gcc", "-std=c11", "-Wall", "-o", exe, os.path.join(ROOT, "tests", "native", "abi_layout.c"),
                    "-I", os.path.join(ROOT, "include")], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    types = {"csm_config": csm.CsmConfig, "csm_batch_result": csm.CsmBatchResult, "csm_stats": csm.CsmStats,
             "csm_server_config": csm.CsmServerConfig, "csm_request_info": csm.CsmRequestInfo,
             "csm_server_stats": csm.CsmServerStats}
    checked = 0
    for line in out:
        if not line.strip():
            continue
        name, off = line.split()
        a, b = name.split(".")
        if a == "sizeof":
            assert ctypes.sizeof(types[b]) == int(off), name
        else:
            assert getattr(types[a], b).offset == int(off), name
        checked += 1
    assert checked > 60
