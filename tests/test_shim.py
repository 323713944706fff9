"""The C++ drop-in layer (triton-vm-prover_b200/cpp): it compiles against the
reference's own headers, and its self-check program -- every public function of
NTT, LDE, LDETable, RandomizedLDE, Tip5, MerkleTree and hash_row, compared with
the oracle -- passes on the GPU."""
import os
import subprocess

import pytest

from conftest import ROOT
from oracle import REF_DIR

REF_INCLUDE = os.path.join(REF_DIR, "include")
BIN = os.path.join(ROOT, "tests", "cpp", "_bin", "shim_selftest")


@pytest.mark.skipif(not os.path.isdir(REF_INCLUDE), reason="reference headers not present")
def test_shim_compiles_against_reference_headers():
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "triton-vm-prover_b200", "cpp"), "check",
                        f"REF={REF_DIR}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


def test_selftest_binary_links_the_library():
    if not os.path.exists(BIN):
        pytest.skip("self-check not built (needs the reference headers)")
    out = subprocess.run(["ldd", BIN], capture_output=True, text=True).stdout
    assert "libtvmc.so" in out and "not found" not in out, out


@pytest.mark.gpu
def test_shim_selftest_on_gpu():
    assert os.path.exists(BIN), "tests/cpp/_bin/shim_selftest missing: run __graft_entry__.build()"
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert " 0 failed" in r.stdout, r.stdout[-2000:]


TC_BIN = os.path.join(ROOT, "tests", "cpp", "_bin", "table_commitment_check")


def test_table_commitment_check_links_the_library():
    if not os.path.exists(TC_BIN):
        pytest.skip("TableCommitment check not built (needs the reference sources)")
    out = subprocess.run(["ldd", TC_BIN], capture_output=True, text=True).stdout
    assert "libtvmc.so" in out and "not found" not in out, out


@pytest.mark.gpu
def test_reference_table_commitment_over_the_drop_in():
    """src/table/table_commitment.cpp, compiled unchanged, over the drop-in
    layer: the per-column LDE of MasterMainTable::low_degree_extend, row
    hashes, TableCommitment roots, paths, structures and verify vs the oracle."""
    assert os.path.exists(TC_BIN), "tests/cpp/_bin/table_commitment_check missing: run __graft_entry__.build()"
    r = subprocess.run([TC_BIN], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert " 0 failed" in r.stdout, r.stdout[-2000:]


@pytest.mark.gpu
def test_per_column_drop_in_lde_equals_batched():
    assert os.path.exists(TC_BIN)
    r = subprocess.run([TC_BIN, "time", "12", "16"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert '"equal": true' in r.stdout
