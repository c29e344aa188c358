"""Batched verification on the GPU (sg_verify_queries): the query phase of
the verifier — openings' Merkle paths, DEEP values, FRI fold chain, terminal
polynomial — for every table of every proof in one launch, against the
host-side verifier (lambda_vm_b200/verifier.py, restating
crypto/stark/src/verifier.rs) on valid and tampered proofs: the same verdict
and the same reason."""
import copy

import numpy as np
import pytest

from lambda_vm_b200.air import SynthTableAir
from lambda_vm_b200.stark import GpuBackend, Options, multi_prove
from lambda_vm_b200.verifier import verify, verify_many

pytestmark = pytest.mark.gpu

OPTS = Options(blowup=2, grinding=6, final_log_degree=2, queries=9)


def _proof(be, shapes, seed):
    airs = [SynthTableAir(*s) for s in shapes]
    return airs, multi_prove(airs, [seed + i for i in range(len(airs))], OPTS, GpuBackend(be))


@pytest.mark.parametrize("shapes", [[(4, 6, 2), (5, 8, 4)], [(9, 16, 6), (7, 10, 4), (6, 300, 2)], [(12, 24, 4)]])
def test_gpu_verifier_accepts_valid_proofs(be, shapes):
    airs, pr = _proof(be, shapes, 50)
    assert verify(airs, pr, OPTS) == (True, "ok")
    assert verify(airs, pr, OPTS, device=be) == (True, "ok")


def _tampers(pr):
    """(label, function that changes one opened value or path byte of table 0)."""
    def arr(t, k):
        return np.array(t[k], copy=True)

    def set_field(k, idx, delta=1):
        def f(p):
            t = p["tables"][0]
            a = arr(t, k)
            a[idx] = (a[idx] + np.uint64(delta)) if a.dtype == np.uint64 else a[idx] ^ 1
            t[k] = a
        return f

    def set_layer(k, layer, idx):
        def f(p):
            t = p["tables"][0]
            lst = [np.array(x, copy=True) for x in t[k]]
            a = lst[layer]
            a[idx] = (a[idx] + np.uint64(1)) if a.dtype == np.uint64 else a[idx] ^ 1
            t[k] = lst
        return f

    out = [("main value", set_field("open_main", (3, 1))), ("aux value", set_field("open_aux", (0, 2))),
           ("parts value", set_field("open_parts", (5, 4))), ("main path", set_field("path_main", (2, 3, 7))),
           ("aux path", set_field("path_aux", (1, 0, 0))), ("parts path", set_field("path_parts", (4, 1, 31)))]
    if len(pr["tables"][0]["fri_open"]) >= 2:
        out += [("fri value 1", set_layer("fri_open", 0, (2, 1))), ("fri value 2", set_layer("fri_open", 1, (7, 0))),
                ("fri path 1", set_layer("fri_paths", 0, (0, 0, 5))), ("fri path 2", set_layer("fri_paths", 1, (8, 1, 9)))]
    return out


def test_gpu_verifier_rejects_what_the_host_verifier_rejects(be):
    airs, pr = _proof(be, [(9, 16, 6), (7, 10, 4)], 80)
    for label, tamper in _tampers(pr):
        bad = copy.deepcopy(pr)
        tamper(bad)
        host = verify(airs, bad, OPTS)
        assert host[0] is False, label
        assert verify(airs, bad, OPTS, device=be) == host, label


def test_verify_many_batches_proofs(be):
    items = [_proof(be, [(8, 12, 4), (6, 9, 2)], 10 * k) for k in range(4)]
    airs2, pr2 = items[2]
    bad = copy.deepcopy(pr2)
    t = bad["tables"][1]
    om = np.array(t["open_main"], copy=True)
    om[0, 0] += np.uint64(1)
    t["open_main"] = om
    items[2] = (airs2, bad)
    got = verify_many(items, OPTS, be)
    want = [verify(a, p, OPTS) for a, p in items]
    assert got == want
    assert [g[0] for g in got] == [True, True, False, True]
