"""One proof across ranks (world_size 2, gloo, CPU oracle backend): the
tables are partitioned heaviest first, the ranks exchange only the R1 roots,
and the assembled proof equals the single-process proof."""
import multiprocessing as mp
import os
import socket

import pytest

from lambda_vm_b200.air import SynthTableAir
from lambda_vm_b200.distributed import assign_tables, table_weight
from lambda_vm_b200.stark import Options, multi_prove

SHAPES = [(5, 8, 2), (6, 12, 4), (4, 6, 2), (7, 9, 6), (5, 20, 4)]
OPTS = dict(blowup=2, grinding=4, final_log_degree=2, queries=5)


def _airs():
    return [SynthTableAir(*s) for s in SHAPES]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    from lambda_vm_b200.distributed import multi_prove_distributed
    from oracle.stark_backend import OracleBackend
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        airs = _airs()
        proof = multi_prove_distributed(airs, [900 + i for i in range(len(airs))], Options(**OPTS), OracleBackend())
        if rank == 0:
            q.put(proof)
        else:
            q.put(None if proof is None else "non-zero rank returned a proof")
    finally:
        dist.destroy_process_group()


def test_assignment_is_a_balanced_partition():
    opts = Options(**OPTS)
    airs = [SynthTableAir(l, w, 2) for l, w in [(12, 8), (10, 300), (11, 50), (6, 6), (12, 100), (9, 9)]]
    for world in (1, 2, 3, 4):
        parts = assign_tables(airs, opts, world)
        assert sorted(i for p in parts for i in p) == list(range(len(airs)))
        loads = [sum(table_weight(airs[i], opts) for i in p) for p in parts]
        # LPT bound: no rank exceeds the average by more than the heaviest table
        assert max(loads) <= sum(loads) / world + max(table_weight(a, opts) for a in airs)


@pytest.mark.timeout(300)
def test_two_rank_proof_equals_single_process_proof():
    from oracle.stark_backend import OracleBackend
    from oracle.verifier import verify
    from proofcmp import diff
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=240) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    proofs = [g for g in got if isinstance(g, dict)]
    assert len(proofs) == 1 and all(g is None or isinstance(g, dict) for g in got)
    airs = _airs()
    ref = multi_prove(airs, [900 + i for i in range(len(airs))], Options(**OPTS), OracleBackend())
    assert diff(proofs[0], ref) is None, diff(proofs[0], ref)
    assert verify(airs, proofs[0], Options(**OPTS)) == (True, "ok")
