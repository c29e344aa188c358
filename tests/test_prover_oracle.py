"""The multi-table protocol on the CPU oracle backend: proofs verify, and
tampering with any committed or opened value is rejected (no GPU)."""
import copy

import pytest

from lambda_vm_b200.air import SynthTableAir
from lambda_vm_b200.stark import Options, fri_layout, multi_prove
from oracle.stark_backend import OracleBackend
from oracle.verifier import verify

OPTS = Options(blowup=2, grinding=6, final_log_degree=2, queries=6)


@pytest.fixture(scope="module")
def proof():
    airs = [SynthTableAir(4, 6, 2), SynthTableAir(5, 8, 4), SynthTableAir(6, 7, 6)]
    trs = [a.trace(i + 1) for i, a in enumerate(airs)]
    return airs, multi_prove(airs, trs, OPTS, OracleBackend())


def test_fri_layout_matches_reference_rules():
    # FriFoldLayout::new (fri/terminal.rs:45-55)
    assert fri_layout(20, 1, 7) == {"total_folds": 12, "num_committed": 11, "terminal_len": 256, "effective_k": 7}
    assert fri_layout(5, 1, 7) == {"total_folds": 0, "num_committed": 0, "terminal_len": 32, "effective_k": 4}


def test_honest_proof_verifies(proof):
    airs, pr = proof
    assert verify(airs, pr, OPTS) == (True, "ok")


@pytest.mark.parametrize("field,mutate", [
    ("parts_ood", lambda tp: tp["parts_ood"].__setitem__(0, (1, 2, 3))),
    ("trace_ood", lambda tp: tp["trace_ood"][0].__setitem__(1, (7, 0, 0))),
    ("open_main", lambda tp: tp["open_main"][0].__setitem__(0, tp["open_main"][0][0] ^ 1)),
    ("open_aux", lambda tp: tp["open_aux"][1].__setitem__(2, tp["open_aux"][1][2] ^ 1)),
    ("fri_open", lambda tp: tp["fri_open"][0][0].__setitem__(0, tp["fri_open"][0][0][0] ^ 1)),
    ("nonce", lambda tp: tp.__setitem__("nonce", tp["nonce"] + 1)),
    ("fri_final", lambda tp: tp["fri_final_coeffs"].__setitem__(0, (5, 5, 5))),
])
def test_tampering_is_rejected(proof, field, mutate):
    airs, pr = proof
    bad = copy.deepcopy(pr)
    mutate(bad["tables"][2])
    ok, why = verify(airs, bad, OPTS)
    assert not ok, field
