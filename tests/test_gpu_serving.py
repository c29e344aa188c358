"""Serving on the GPU: jobs admitted concurrently under a budget produce the
same proof as each job proved alone, and every proof verifies."""
import pytest

from lambda_vm_b200.air import SynthTableAir
from lambda_vm_b200.serving import ProofServer, serve_poisson
from lambda_vm_b200.stark import GpuBackend, Options, multi_prove
from oracle.verifier import verify
from proofcmp import diff

pytestmark = pytest.mark.gpu


def _jobs():
    shapes = [
        [(10, 12, 4), (7, 8, 2)],
        [(11, 20, 6)],
        [(8, 9, 2), (9, 30, 4), (6, 6, 2)],
        [(12, 16, 4)],
        [(7, 40, 6), (10, 8, 2)],
    ]
    return [([SynthTableAir(*s) for s in js], [500 + 10 * j + i for i in range(len(js))])
            for j, js in enumerate(shapes)]


def test_jobs_in_the_mix_equal_jobs_alone(be):
    opts = Options(blowup=2, grinding=8, final_log_degree=3, queries=8)
    specs = _jobs()
    alone = [multi_prove(airs, srcs, opts, GpuBackend(be)) for airs, srcs in specs]
    with ProofServer(budget_bytes=be.budget() // 2, max_jobs=3, drivers=3, opts=opts, be=be) as srv:
        jobs, st = serve_poisson(srv, specs, rate=50.0, seed=1)
    assert st.failed == 0, [j.error for j in jobs]
    for j, ref, (airs, _) in zip(jobs, alone, specs):
        assert diff(j.proof, ref) is None, diff(j.proof, ref)
        assert verify(airs, j.proof, opts) == (True, "ok")
    assert st.p50_s is not None and st.p99_s >= st.p50_s


def test_served_fibonacci_guests_verify_against_their_statements(be):
    """Fibonacci RV64 guests served beside synthetic jobs: each served proof
    equals the guest proved alone under its own statement label, and the
    verifier accepts it for the statement (program, counts, output) with the
    public bus terms."""
    from lambda_vm_b200 import rv64
    from lambda_vm_b200 import rv64_air as RA
    from oracle.verifier import verify as oracle_verify
    opts = Options(blowup=2, grinding=8, final_log_degree=3, queries=8)
    ns = (3, 40, 200)
    guests = [RA.build(rv64.fib_program(n)) for n in ns]
    synth = _jobs()[:2]
    specs = [(airs, traces, pub["label"]) for airs, traces, pub in guests] + [s + (b"lambda_vm_b200/synthetic-multi-table",)
                                                                            for s in synth]
    alone = [multi_prove(airs, srcs, opts, GpuBackend(be), label=label) for airs, srcs, label in specs]
    with ProofServer(budget_bytes=be.budget() // 2, max_jobs=3, drivers=3, opts=opts, be=be) as srv:
        jobs, st = serve_poisson(srv, specs, rate=50.0, seed=2)
    assert st.failed == 0, [j.error for j in jobs]
    for j, ref in zip(jobs, alone):
        assert diff(j.proof, ref) is None, diff(j.proof, ref)
    for j, (airs, _, pub), n in zip(jobs, guests, ns):
        assert pub["output"] == rv64.fib_reference(n)
        ok = RA.verify(pub["words"], pub["counts"], pub["output"], j.proof, opts)
        assert ok == (True, "ok"), ok
        cpu = airs[0]
        assert oracle_verify(airs, j.proof, opts, label=pub["label"],
                             public_terms=cpu.public_terms(pub["counts"], pub["output"])) == (True, "ok")
        bad = RA.verify(pub["words"], pub["counts"], pub["output"] + 1, j.proof, opts)
        assert bad[0] is False
