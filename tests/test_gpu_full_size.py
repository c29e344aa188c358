"""Oracle parity at the sizes the benchmark and the proofs actually run.

The smaller parity tests (test_gpu_commit.py) reach 2^17-row traces, whose
four-step passes are 2^6..2^9 points. These cases run the kernel plans of the
full-size workloads and compare every output value with the CPU oracle
(crypto/math/src/polynomial.rs:527-608 restated in oracle/oracle.c):

* the benchmark's default workload exactly: a 2^20 x 256 trace, blowup 4
  (2^10-point passes over 16-column tiles), one-row little-endian leaves and
  the Keccak tree over 2^22 leaves, through the device-resident calls the
  timed step makes and through the host-trace commit (32-column chunks);
* 2^22-row traces (2^11-point passes, the plan of the largest proof tables),
  with the prover's row-pair big-endian leaves;
* one large table proved end to end and accepted by the independent verifier.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from lambda_vm_b200 import math_cuda as mc
from lambda_vm_b200 import native
from lambda_vm_b200.device import DeviceBuffer

pytestmark = [pytest.mark.gpu, pytest.mark.slow]
P = O.P


def rand_field(rng, shape):
    x = rng.integers(0, 2**64, size=shape, dtype=np.uint64)
    return np.where(x >= np.uint64(P), x - np.uint64(P), x)


def device_commit(be, trace, blowup, rows_per_leaf, little_endian):
    """The timed step of bench.py: sg_coset_lde, sg_keccak_leaves and
    sg_merkle_build on device-resident buffers. Returns (LDE, nodes)."""
    L = native.lib()
    n, m = trace.shape
    N = n * blowup
    nl = N // rows_per_leaf
    w = O.coset_weights(n, 3)
    dt = DeviceBuffer.from_host(trace, be)
    dw = DeviceBuffer.from_host(w, be)
    dout = DeviceBuffer(N * m * 8, be)
    dnodes = DeviceBuffer((2 * nl - 1) * 32, be)
    lay = native.LeafLayout(rows_per_leaf, 1 if little_endian else 0, 0, 0)
    root = (C.c_uint8 * 32)()
    native.check(L.sg_coset_lde(be.h, None, dt.ptr, n, m, blowup, dw.ptr, dout.ptr))
    native.check(L.sg_keccak_leaves(be.h, None, dout.ptr, N, m, C.byref(lay), dnodes.ptr + (nl - 1) * 32))
    native.check(L.sg_merkle_build(be.h, None, dnodes.ptr + (nl - 1) * 32, nl, dnodes.ptr, root))
    lde = dout.download(np.uint64).reshape(N, m)
    nodes = dnodes.download(np.uint8).reshape(-1, 32)
    for b in (dt, dw, dout, dnodes):
        b.close()
    assert bytes(root) == nodes[0].tobytes()
    return lde, nodes


def canon_inplace(a, rows=1 << 18):
    """Canonical representatives, in place, a block of rows at a time (the
    full-size LDE is 8 GiB; no second copy of it is made)."""
    for i in range(0, a.shape[0], rows):
        blk = a[i:i + rows]
        np.subtract(blk, np.uint64(P), out=blk, where=blk >= np.uint64(P))
    return a


def test_benchmark_workload_2pow20x256_blowup4_matches_oracle(be):
    """Every LDE value and the root of the default bench workload."""
    rng = np.random.default_rng(20_256_4)
    n, m, B = 1 << 20, 256, 4
    t = rand_field(rng, (n, m))
    lde, nodes = device_commit(be, t, B, 1, True)
    want = canon_inplace(O.coset_lde_row_major(t, B, O.coset_weights(n, 3)))
    assert lde.shape == want.shape
    assert np.array_equal(lde, want)
    del lde
    leaves = O.leaves_row_major(want, 1, True)
    del want
    root = O.merkle_root(leaves)
    assert nodes[0].tobytes() == root
    # the same commitment through the host-trace path (chunked upload, windowed leaves)
    h, _ = mc.lde_commit(t, n, m, B, O.coset_weights(n, 3), 1, True, None, False, be)
    assert h.root == root
    h.free()


@pytest.mark.parametrize("m,blowup", [(16, 2), (9, 2), (8, 4)])
def test_2pow22_row_lde_matches_oracle(be, m, blowup):
    """2^22-row traces run 2^11-point passes (8- or 4-column tiles): values and
    the prover's row-pair big-endian root."""
    rng = np.random.default_rng(22 * 100 + m)
    n = 1 << 22
    t = rng.integers(0, 2**64, size=(n, m), dtype=np.uint64)  # non-canonical inputs too
    lde, nodes = device_commit(be, t, blowup, 2, False)
    want = canon_inplace(O.coset_lde_row_major(t, blowup, O.coset_weights(n, 3)))
    assert np.array_equal(lde, want)
    del lde
    assert nodes[0].tobytes() == O.merkle_root(O.leaves_row_major(want, 2, False))


def test_large_table_proof_verifies(be):
    """A 2^18-row table (2^19-row LDE, 2^9-point four-step passes; LogUp aux,
    composition, DEEP and 13 FRI layers at their full sizes) proved by the
    native table driver and by the scheduler, identical, and accepted by the
    independent verifier built on the oracle."""
    from lambda_vm_b200.air import SynthTableAir
    from lambda_vm_b200.proof_io import serialize
    from lambda_vm_b200.scheduler import multi_prove_scheduled
    from lambda_vm_b200.stark import GpuBackend, Options, multi_prove
    from oracle.verifier import verify
    opts = Options(blowup=2, grinding=16, final_log_degree=5)
    airs = [SynthTableAir(18, 40, 6), SynthTableAir(12, 9, 2)]
    seeds = [4242, 4243]
    plain = multi_prove(airs, seeds, opts, GpuBackend(be))
    sched = multi_prove_scheduled(airs, seeds, opts, workers=2, be=be)
    assert serialize(plain) == serialize(sched)
    assert verify(airs, plain, opts) == (True, "ok")


def test_keccak_guest_1mib_proof_verifies(be):
    """The Keccak guest at its benchmark size (a 1 048 560-byte buffer, 1.8 M
    cycles, six tables up to 2^21 x 234 and 2^18 x 2605) proved on the GPU by
    the plain and the batched prover: the same proof, the guest's own output,
    accepted by the library verifier (GPU query phase) and by the independent
    verifier built on the oracle; a wrong output is rejected."""
    from lambda_vm_b200 import rv64
    from lambda_vm_b200 import rv64_air as RA
    from lambda_vm_b200.proof_io import serialize
    from lambda_vm_b200.scheduler import multi_prove_scheduled
    from lambda_vm_b200.stark import GpuBackend, Options, multi_prove
    from oracle.verifier import verify as oracle_verify
    opts = Options(blowup=2, grinding=20, final_log_degree=5)
    words = rv64.keccak_program(136 * 7710)
    airs, traces, pub = RA.build(words)
    assert pub["cycles"] == 1796454 and pub["output"] == rv64.keccak_reference(136 * 7710)
    proof = multi_prove(airs, traces, opts, GpuBackend(be), label=pub["label"])
    batched = multi_prove_scheduled(airs, traces, opts, workers=8, be=be, label=pub["label"])
    assert serialize(batched) == serialize(proof)
    counts, out, h = pub["counts"], pub["output"], pub["heights"]
    assert RA.verify(words, counts, out, proof, opts, device=be, heights=h) == (True, "ok")
    full = RA.airs_for(words, counts, h)
    assert oracle_verify(full, proof, opts, label=RA.statement_label(words, counts, out, h),
                         public_terms=full[0].public_terms(counts, out)) == (True, "ok")
    assert RA.verify(words, counts, out ^ (1 << 63), proof, opts, heights=h)[0] is False
