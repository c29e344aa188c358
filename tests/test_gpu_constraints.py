"""GPU parity of the constraint interpreter and the composition split.

Random programs in the reference IR are lowered exactly like
DeviceProgram::lower (tests/irgen.py) and run through sg_eval_constraints;
the expected values come from evaluating the UNLOWERED program with the
oracle's field arithmetic (crypto/stark/tests/gpu_constraint_interp.rs shape:
flat walker == IR interpreter == kernel)."""
import numpy as np
import pytest

import oracle as O
from irgen import composition, eval_rows, lower, random_program
from lambda_vm_b200 import math_cuda as mc
from lambda_vm_b200.native import SgError

pytestmark = pytest.mark.gpu
P = O.P


def rf(rng, shape):
    x = rng.integers(0, 2**64, size=shape, dtype=np.uint64)
    return np.where(x >= np.uint64(P), x - np.uint64(P), x)


@pytest.mark.parametrize("stream", [True, False])
@pytest.mark.parametrize("seed,rows,m,a,nodes,roots,next_step", [
    (1, 16, 4, 0, 30, 3, 1), (2, 64, 6, 2, 60, 5, 2), (3, 128, 10, 3, 120, 8, 4), (4, 32, 3, 1, 200, 12, 1),
    (5, 256, 8, 2, 80, 6, 2)])
def test_constraint_matrix_matches_ir(be, seed, rows, m, a, nodes, roots, next_step, stream):
    """Both program shapes: streaming (trace operands, constraints folded as
    completed; the library's lowering) and the reference's pinned roots."""
    rng = np.random.default_rng(seed)
    prog = random_program(rng, m, a, 2, 3, n_nodes=nodes, n_roots=roots)
    if seed == 4:
        prog["roots"] = prog["roots"] + prog["roots"][:3]  # constraints that share a node
        prog["roots"].sort(key=lambda r: prog["dims"][r])
    low = lower(prog, stream)
    main = rf(rng, (rows, m))
    aux = rf(rng, (rows, 3 * a)) if a else np.zeros((rows, 0), np.uint64)
    rap, alpha, off = rf(rng, (2, 3)), rf(rng, (3, 3)), rf(rng, (3,))
    got = mc.eval_constraints_on_device(low, main, aux, rap, alpha, off, next_step, None, be)
    want = np.array(eval_rows(prog, main, aux, rap, alpha, off, next_step), np.uint64)  # rows x roots x 3
    assert (got.transpose(1, 0, 2) == want).all()


@pytest.mark.parametrize("stream", [True, False])
@pytest.mark.parametrize("seed,rows,nb", [(7, 64, 0), (8, 128, 3), (9, 256, 2)])
def test_composition_matches_evaluator(be, seed, rows, nb, stream):
    rng = np.random.default_rng(seed)
    m, a = 6, 2
    prog = random_program(rng, m, a, 2, 3, n_nodes=70, n_roots=6)
    low = lower(prog, stream)
    main = rf(rng, (rows, m))
    aux = rf(rng, (rows, 3 * a))
    rap, alpha, off = rf(rng, (2, 3)), rf(rng, (3, 3)), rf(rng, (3,))
    beta = rf(rng, (6, 3))
    z_inv = rf(rng, (rows // 4,))
    bnd = [(int(rng.integers(0, a if i % 2 else m)), bool(i % 2), rf(rng, (3,)), rf(rng, (3,))) for i in range(nb)]
    b_z_inv = rf(rng, (max(nb, 1), rows))
    comp = {"beta": beta, "z_inv": z_inv, "boundary": bnd, "b_z_inv": b_z_inv[:nb]}
    got = mc.eval_constraints_on_device(low, main, aux, rap, alpha, off, 2, comp, be)
    vals = eval_rows(prog, main, aux, rap, alpha, off, 2)
    want = composition(vals, beta, z_inv, bnd, b_z_inv, main, aux)
    assert (got == want).all()


def test_program_validation_rejects_bad_slots(be):
    rng = np.random.default_rng(11)
    prog = random_program(rng, 4, 0, 1, 1, n_nodes=20, n_roots=2)
    main = rf(rng, (8, 4))
    args = (main, np.zeros((8, 0), np.uint64), rf(rng, (1, 3)), rf(rng, (1, 3)), rf(rng, (3,)), 1, None, be)
    low = lower(prog, False)
    low["num_base_slots"] = 0  # every base slot now out of range
    with pytest.raises(SgError):
        mc.eval_constraints_on_device(low, *args)
    # streaming programs: a trace operand past the last column, a constraint
    # no instruction completes, a constraint completed twice
    low = lower(prog)
    bad = low["nodes"].copy()
    k, j = next((i, j) for i in range(bad.shape[0]) for j in (1, 2) if bad[i, 0] in (6, 7, 8) and bad[i, j] >> 29 == 7)
    bad[k, j] = (7 << 29) | 4
    with pytest.raises(SgError):
        mc.eval_constraints_on_device(dict(low, nodes=bad), *args)
    nr = low["node_roots"].copy()
    nr[nr != 0xFFFFFFFF] = 0xFFFFFFFF
    with pytest.raises(SgError):
        mc.eval_constraints_on_device(dict(low, node_roots=nr), *args)
    nr = low["node_roots"].copy()
    nr[nr == 1] = 0
    with pytest.raises(SgError):
        mc.eval_constraints_on_device(dict(low, node_roots=nr), *args)


def test_decompose_d2_matches_formula(be):
    rng = np.random.default_rng(12)
    rows = 1 << 10
    h = rf(rng, (rows, 3))
    inv2x = rf(rng, (rows // 2,))
    h0, h1 = mc.decompose_d2(h, inv2x, be)
    two_inv = (P + 1) // 2
    for i in range(0, rows // 2, 37):
        x, y = [int(v) for v in h[i]], [int(v) for v in h[i + rows // 2]]
        assert list(map(int, h0[i])) == [O.canonical(O.gl_mul(O.gl_add(x[k], y[k]), two_inv)) for k in range(3)]
        assert list(map(int, h1[i])) == [O.canonical(O.gl_mul(O.gl_sub(x[k], y[k]), int(inv2x[i]))) for k in range(3)]
