"""Canonical proof bytes and the product verifier (CPU, oracle-backend proofs):
serialize/deserialize round trip, the library-side verifier accepts what the
oracle verifier accepts and rejects tampered bytes and fields."""
import copy

import numpy as np
import pytest

from lambda_vm_b200.air import SynthTableAir
from lambda_vm_b200.proof_io import deserialize, serialize
from lambda_vm_b200.stark import Options, multi_prove
from lambda_vm_b200.verifier import verify, verify_bytes
from oracle.stark_backend import OracleBackend
from oracle.verifier import verify as oracle_verify
from proofcmp import diff

OPTS = Options(blowup=2, grinding=4, final_log_degree=2, queries=5)


@pytest.fixture(scope="module")
def proof():
    airs = [SynthTableAir(5, 8, 2), SynthTableAir(6, 10, 4), SynthTableAir(4, 7, 6)]
    return airs, multi_prove(airs, [40 + i for i in range(3)], OPTS, OracleBackend())


def test_round_trip_is_exact(proof):
    airs, p = proof
    blob = serialize(p)
    q = deserialize(blob)
    assert diff(p, q) is None, diff(p, q)
    assert serialize(q) == blob


def test_product_verifier_accepts(proof):
    airs, p = proof
    assert verify(airs, p, OPTS) == (True, "ok")
    assert verify_bytes(airs, serialize(p), OPTS) == (True, "ok")
    assert oracle_verify(airs, p, OPTS) == (True, "ok")


def test_rejects_truncated_and_trailing_bytes(proof):
    airs, p = proof
    blob = serialize(p)
    assert verify_bytes(airs, blob[:-1], OPTS)[0] is False
    assert verify_bytes(airs, blob + b"\0", OPTS)[0] is False
    assert verify_bytes(airs, b"XXXX" + blob[4:], OPTS)[0] is False


@pytest.mark.parametrize("where", ["main_root", "trace_ood", "fri_final_coeffs", "nonce", "open_aux", "fri_paths"])
def test_tampering_is_rejected_by_both_verifiers(proof, where):
    airs, p = proof
    q = copy.deepcopy(p)
    t = q["tables"][1]
    if where == "main_root":
        t["main_root"] = bytes([t["main_root"][0] ^ 1]) + t["main_root"][1:]
    elif where == "trace_ood":
        v = t["trace_ood"][0][0]
        t["trace_ood"][0][0] = ((v[0] + 1) % 0xFFFFFFFF00000001, v[1], v[2])
    elif where == "fri_final_coeffs":
        v = t["fri_final_coeffs"][0]
        t["fri_final_coeffs"][0] = (v[0], (v[1] + 1) % 0xFFFFFFFF00000001, v[2])
    elif where == "nonce":
        t["nonce"] = t["nonce"] + 1
    elif where == "open_aux":
        t["open_aux"] = np.array(t["open_aux"], copy=True)
        t["open_aux"][0, 0] = (int(t["open_aux"][0, 0]) + 1) % 0xFFFFFFFF00000001
    else:
        t["fri_paths"][0] = np.array(t["fri_paths"][0], copy=True)
        t["fri_paths"][0][0, 0, 0] ^= 0xFF
    assert verify(airs, q, OPTS)[0] is False
    assert oracle_verify(airs, q, OPTS)[0] is False
    assert verify_bytes(airs, serialize(q), OPTS)[0] is False


def test_a_proof_with_more_or_fewer_tables_than_the_statement_is_rejected(proof):
    """Every table of a proof is checked against an AIR of the statement: a
    proof carrying an extra table (whose bus contribution would otherwise
    go unchecked) or missing one is rejected by both verifiers."""
    airs, p = proof
    extra = copy.deepcopy(p)
    extra["tables"].append(copy.deepcopy(p["tables"][0]))
    short = copy.deepcopy(p)
    short["tables"].pop()
    for q in (extra, short):
        assert verify(airs, q, OPTS)[0] is False
        assert oracle_verify(airs, q, OPTS)[0] is False
    assert verify(airs[:2], p, OPTS)[0] is False


def test_a_malformed_proof_is_rejected_not_raised(proof):
    airs, p = proof
    q = copy.deepcopy(p)
    q["tables"][0]["trace_ood"] = [[]]
    assert verify(airs, q, OPTS)[0] is False
    q = copy.deepcopy(p)
    del q["tables"][2]["fri_roots"]
    assert verify(airs, q, OPTS)[0] is False
