"""The library's host-side Fiat-Shamir transcript and Keccak-256 (no GPU):
pinned to the reference's KATs and checked against the oracle on random
absorb/sample sequences."""
import json
import os

import numpy as np
import pytest

import oracle as O
from lambda_vm_b200 import math_cuda as mc

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))


@pytest.mark.parametrize("kat", KATS["keccak256"], ids=lambda k: repr(k["msg"][:12]))
def test_library_keccak256_kat(kat):
    assert mc.keccak256(kat["msg"].encode()).hex() == kat["digest"]


def test_library_transcript_kat():
    k = KATS["transcript"]
    t = mc.Transcript(k["label"].encode())
    assert [t.sample_base() for _ in range(5)] == k["base"]
    assert t.sample_u64(1 << k["u64_bound_log2"]) == k["u64"]
    te = mc.Transcript(k["label"].encode())
    te.append_bytes(k["ext3_phase"].encode())
    assert [int(x) for x in te.sample_ext3()] == k["ext3"]


def test_library_transcript_matches_oracle_random_sequences():
    rng = np.random.default_rng(0)
    for trial in range(20):
        label = bytes(rng.integers(0, 256, size=int(rng.integers(0, 40)), dtype=np.uint8))
        a, b = mc.Transcript(label), O.Transcript(label)
        for step in range(30):
            op = int(rng.integers(0, 7))
            if op == 0:
                d = bytes(rng.integers(0, 256, size=int(rng.integers(0, 300)), dtype=np.uint8))
                a.append_bytes(d)
                b.append_bytes(d)
            elif op == 1:
                v = int(rng.integers(0, 2**63)) * 2 + 1
                a.append_base(v)
                b.append_base(v)
            elif op == 2:
                v = rng.integers(0, 2**64, size=3, dtype=np.uint64)
                a.append_ext3(v)
                b.append_ext3(v)
            elif op == 3:
                assert a.sample_base() == b.sample_base()
            elif op == 4:
                assert list(a.sample_ext3()) == list(b.sample_ext3())
            elif op == 5:
                ub = int(rng.integers(1, 2**40))
                assert a.sample_u64(ub) == b.sample_u64(ub)
            else:
                assert a.sample() == b.sample()
            assert a.state() == b.state()
        c = a.clone()
        assert c.sample_base() == a.sample_base()


def test_sample_z_ood_avoids_domains():
    t = mc.Transcript(b"z-ood")
    z = t.sample_z_ood(1 << 10, 1 << 12, 3)
    # z^n != 1 and z^(lde) != g^(lde)
    o = O.Transcript(b"z-ood")
    z2 = o.sample_ext3()
    assert list(z) == list(z2)  # first candidate is accepted with overwhelming probability


def test_bulk_ext3_absorb_equals_one_by_one():
    rng = np.random.default_rng(11)
    vals = rng.integers(0, 2**64, size=(37, 3), dtype=np.uint64)
    vals[0] = [0xFFFFFFFF00000001, 0xFFFFFFFFFFFFFFFF, 5]  # non-canonical inputs are canonicalised
    a, b, c = mc.Transcript(b"bulk"), mc.Transcript(b"bulk"), O.Transcript(b"bulk")
    a.sample_ext3()
    b.sample_ext3()
    c.sample_ext3()
    a.append_ext3_many(vals)
    for v in vals:
        b.append_ext3(v)
        c.append_ext3(v)
    assert a.sample() == b.sample() == c.sample()
    assert [int(x) for x in a.sample_ext3()] == [int(x) for x in b.sample_ext3()] == [int(x) for x in c.sample_ext3()]
