"""The RV64 front-end proved on the GPU: the Fibonacci guest's execution
(CPU table + 16-bit RANGE table) proved by the library's prover, accepted by
the library's verifier (host and GPU query phase) and by the independent
verifier built on the oracle, both given the public statement (program,
execution counts, output); a wrong output or wrong counts are rejected."""
import pytest

from lambda_vm_b200 import rv64
from lambda_vm_b200 import rv64_air as RA
from lambda_vm_b200.stark import GpuBackend, Options
from oracle.verifier import verify as oracle_verify

pytestmark = pytest.mark.gpu
OPTS = Options(blowup=2, grinding=8, final_log_degree=3, queries=12)


@pytest.mark.parametrize("n", [3, 40, 1000])
def test_fibonacci_execution_proof_verifies(be, n):
    words = rv64.fib_program(n)
    proof, pub = RA.prove(words, OPTS, GpuBackend(be))
    assert pub["output"] == rv64.fib_reference(n)
    counts, out = pub["counts"], pub["output"]
    assert RA.verify(words, counts, out, proof, OPTS) == (True, "ok")
    assert RA.verify(words, counts, out, proof, OPTS, device=be) == (True, "ok")
    airs = RA.airs_for(words, counts)
    assert oracle_verify(airs, proof, OPTS, label=RA.statement_label(words, counts, out),
                         public_terms=airs[0].public_terms(counts, out)) == (True, "ok")
    # a different output, or different counts, is not what was proved
    assert RA.verify(words, counts, (out + 1) % (1 << 64), proof, OPTS)[0] is False
    bad = list(counts)
    bad[3] += 1
    bad[0] -= 1
    assert RA.verify(words, bad, out, proof, OPTS)[0] is False
