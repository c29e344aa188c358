"""Test helpers for the constraint interpreter (test infrastructure only).

* `random_program` builds a random constraint program in the reference's IR
  (crypto/stark/src/constraint_ir/ir.rs: Op nodes with Base/Ext dims);
* `lower` is the library's DeviceProgram::lower restatement (lambda_vm_b200.ir),
  checked here only through the kernel against the unlowered evaluation;
* `eval_rows` evaluates the UNLOWERED program row by row with the oracle's
  field arithmetic (constraint_ir/interp.rs semantics), plus the composition
  accumulation of constraints/evaluator.rs.
"""
import numpy as np

import oracle as O

P = O.P
OP_CONST_BASE, OP_CONST_EXT, OP_VAR, OP_RAP, OP_ALPHA, OP_OFFSET = 0, 1, 2, 3, 4, 5
OP_ADD, OP_SUB, OP_MUL, OP_NEG, OP_EMBED = 6, 7, 8, 9, 10
OPK_SHIFT = 29
OPK_BASE_SLOT, OPK_EXT_SLOT, OPK_BASE_CONST, OPK_EXT_CONST, OPK_RAP, OPK_ALPHA, OPK_OFFSET = range(7)
RES_EXT_BIT = 1 << 31
BASE, EXT = 0, 1


def rp(rng):
    return int(rng.integers(0, 2**64, dtype=np.uint64)) % P


def random_program(rng, m, a, n_rap, n_alpha, n_nodes=60, n_roots=5, max_offset=1):
    """Nodes: list of (op, x, y) with dims. Leaves: ('var', main, offset, col),
    ('cb', idx), ('ce', idx), ('rap', idx), ('alpha', idx), ('off',)."""
    nodes, dims = [], []
    base_consts = [rp(rng) for _ in range(4)]
    ext_consts = [[rp(rng), rp(rng), rp(rng)] for _ in range(3)]

    def add(node, dim):
        nodes.append(node)
        dims.append(dim)
        return len(nodes) - 1

    for _ in range(6):
        add(("var", True, int(rng.integers(0, max_offset + 1)), int(rng.integers(0, m))), BASE)
    if a:
        for _ in range(3):
            add(("var", False, int(rng.integers(0, max_offset + 1)), int(rng.integers(0, a))), EXT)
    add(("cb", int(rng.integers(0, 4))), BASE)
    add(("ce", int(rng.integers(0, 3))), EXT)
    if n_rap:
        add(("rap", int(rng.integers(0, n_rap))), EXT)
    if n_alpha:
        add(("alpha", int(rng.integers(0, n_alpha))), EXT)
    add(("off",), EXT)
    while len(nodes) < n_nodes:
        kind = int(rng.integers(0, 5))
        i = int(rng.integers(0, len(nodes)))
        j = int(rng.integers(0, len(nodes)))
        if kind <= 2:
            op = ("add", "sub", "mul")[kind]
            add((op, i, j), EXT if (dims[i] == EXT or dims[j] == EXT) else BASE)
        elif kind == 3:
            add(("neg", i), dims[i])
        else:
            if dims[i] == BASE:
                add(("embed", i), EXT)
    # roots: base-rooted prefix, then ext (num_base semantics)
    cand = list(range(len(nodes) // 2, len(nodes)))
    rng.shuffle(cand)
    roots = cand[:n_roots]
    roots.sort(key=lambda r: dims[r])  # base first
    return {"nodes": nodes, "dims": dims, "base_consts": base_consts, "ext_consts": ext_consts, "roots": roots}


from lambda_vm_b200.ir import lower  # noqa: E402,F401  (DeviceProgram::lower restatement under test)


# ---------------- reference evaluation (unlowered IR) ----------------
def _e(x):
    return [int(v) for v in x]


def f3add(a, b):
    return [O.gl_add(a[i], b[i]) for i in range(3)]


def f3sub(a, b):
    return [O.gl_sub(a[i], b[i]) for i in range(3)]


def f3mul(a, b):
    return _e(O.fp3_mul(np.array(a, np.uint64), np.array(b, np.uint64)))


def eval_rows(prog, main, aux, rap, alpha, offset, next_step):
    rows = main.shape[0]
    vals_all = []
    for row in range(rows):
        v = []
        for nd in prog["nodes"]:
            k = nd[0]
            if k == "var":
                _, is_main, off, col = nd
                r = (row + off * next_step) % rows
                v.append([int(main[r, col]), 0, 0] if is_main else _e(aux[r, 3 * col:3 * col + 3]))
            elif k == "cb":
                v.append([prog["base_consts"][nd[1]], 0, 0])
            elif k == "ce":
                v.append(list(prog["ext_consts"][nd[1]]))
            elif k == "rap":
                v.append(_e(rap[nd[1]]))
            elif k == "alpha":
                v.append(_e(alpha[nd[1]]))
            elif k == "off":
                v.append(_e(offset))
            elif k == "add":
                v.append(f3add(v[nd[1]], v[nd[2]]))
            elif k == "sub":
                v.append(f3sub(v[nd[1]], v[nd[2]]))
            elif k == "mul":
                v.append(f3mul(v[nd[1]], v[nd[2]]))
            elif k == "neg":
                v.append([O.gl_neg(x) for x in v[nd[1]]])
            else:
                v.append(list(v[nd[1]]))
        vals_all.append([[O.canonical(x) for x in v[r]] for r in prog["roots"]])
    return vals_all  # rows x roots x 3


def composition(vals, beta, z_inv, bnd, b_z_inv, main, aux):
    """evaluator.rs accumulation: H = z_inv * sum beta_c C_c + sum_b z_b_inv beta_b (cell - value)."""
    rows = len(vals)
    out = []
    for row in range(rows):
        s = [0, 0, 0]
        for c, cv in enumerate(vals[row]):
            s = f3add(s, f3mul(_e(beta[c]), cv))
        zi = int(z_inv[row % len(z_inv)])
        h = [O.gl_mul(x, zi) for x in s]
        for b, (col, is_aux, value, bb) in enumerate(bnd):
            cell = _e(aux[row, 3 * col:3 * col + 3]) if is_aux else [int(main[row, col]), 0, 0]
            zb = [O.gl_mul(x, int(b_z_inv[b, row])) for x in _e(bb)]
            h = f3add(h, f3mul(zb, f3sub(cell, _e(value))))
        out.append([O.canonical(x) for x in h])
    return np.array(out, np.uint64)
