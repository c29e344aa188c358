"""The C ABI from a C host: tests/c_host/commit_host.c is compiled with plain
gcc against include/starkgpu.h and libstarkgpu.so (no Python, no torch) and,
on a GPU, its commitment root, authentication paths and grinding nonce are
checked against the oracle."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_host", "commit_host.c")
LIBDIR = os.path.join(ROOT, "lambda_vm_b200")
P = (1 << 64) - (1 << 32) + 1


def _build(tmp_path):
    exe = str(tmp_path / "commit_host")
    r = subprocess.run(["gcc", "-O2", "-std=c11", "-I" + os.path.join(ROOT, "include"), SRC, "-L" + LIBDIR,
                        "-lstarkgpu", "-Wl,-rpath," + LIBDIR, "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_host_compiles_and_links(tmp_path):
    assert os.path.exists(os.path.join(LIBDIR, "libstarkgpu.so"))
    _build(tmp_path)


def _trace(n, m):
    x = 0x9E3779B97F4A7C15
    out = np.empty(n * m, np.uint64)
    M = (1 << 64) - 1
    for i in range(n * m):
        x ^= (x << 13) & M
        x ^= x >> 7
        x ^= (x << 17) & M
        out[i] = x % P
    return out.reshape(n, m)


@pytest.mark.gpu
def test_c_host_matches_oracle(tmp_path):
    n, m, B = 1024, 20, 4
    exe = _build(tmp_path)
    r = subprocess.run([exe, str(n), str(m)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    root_hex, sib0, sib1, nonce = r.stdout.split()
    tr = _trace(n, m)
    w = O.canon_array(O.coset_weights(n, 3))
    lde = O.canon_array(O.coset_lde_row_major(tr, B, w))
    nodes = O.merkle_nodes(O.leaves_row_major(lde, 2, False))
    assert nodes[0].tobytes().hex() == root_hex
    L = (n * B) // 2
    assert bytes(O.merkle_path(nodes, 0)[0]).hex() == sib0
    assert bytes(O.merkle_path(nodes, L - 1)[0]).hex() == sib1
    root = bytes.fromhex(root_hex)
    nonce = int(nonce)
    assert O.grind_is_valid(root, nonce, 12)
    assert not any(O.grind_is_valid(root, k, 12) for k in range(nonce))
