"""Test helpers for the constraint interpreter (test infrastructure only).

* `random_program` builds a random constraint program in the reference's IR
  (crypto/stark/src/constraint_ir/ir.rs: Op nodes with Base/Ext dims);
* `lower` restates DeviceProgram::lower (constraint_ir/device.rs:160-330):
  uniform-leaf propagation, liveness slot reuse per dim class, pinned roots;
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


def _operands(node):
    if node[0] in ("add", "sub", "mul"):
        return [node[1], node[2]]
    if node[0] in ("neg", "embed"):
        return [node[1]]
    return []


def _uniform(node):
    return node[0] in ("cb", "ce", "rap", "alpha", "off")


def lower(prog):
    """DeviceProgram::lower restated: returns dict of numpy arrays."""
    nodes, dims, roots = prog["nodes"], prog["dims"], prog["roots"]
    n = len(nodes)
    used = [False] * n
    last = [0] * n
    for i, nd in enumerate(nodes):
        for o in _operands(nd):
            used[o] = True
            last[o] = i
    is_root = [False] * n
    for r in roots:
        is_root[r] = True
        used[r] = True
    emitted = [used[i] and (not _uniform(nodes[i]) or is_root[i]) for i in range(n)]

    def enc_uniform(nd):
        k = nd[0]
        if k == "cb":
            return (OPK_BASE_CONST << OPK_SHIFT) | nd[1]
        if k == "ce":
            return (OPK_EXT_CONST << OPK_SHIFT) | nd[1]
        if k == "rap":
            return (OPK_RAP << OPK_SHIFT) | nd[1]
        if k == "alpha":
            return (OPK_ALPHA << OPK_SHIFT) | nd[1]
        return OPK_OFFSET << OPK_SHIFT

    slot_of = [None] * n
    free = {BASE: [], EXT: []}
    count = {BASE: 0, EXT: 0}
    out = []
    for i in range(n):
        if not emitted[i]:
            continue
        nd = nodes[i]

        def enc(j):
            if not emitted[j]:
                return enc_uniform(nodes[j])
            kind = OPK_BASE_SLOT if dims[j] == BASE else OPK_EXT_SLOT
            return (kind << OPK_SHIFT) | slot_of[j]

        k = nd[0]
        if k == "cb":
            t = (OP_CONST_BASE, nd[1], 0)
        elif k == "ce":
            t = (OP_CONST_EXT, nd[1], 0)
        elif k == "var":
            _, main, off, col = nd
            t = (OP_VAR, col, (int(main) << 16) | (off << 8))
        elif k == "rap":
            t = (OP_RAP, nd[1], 0)
        elif k == "alpha":
            t = (OP_ALPHA, nd[1], 0)
        elif k == "off":
            t = (OP_OFFSET, 0, 0)
        elif k in ("add", "sub", "mul"):
            t = ({"add": OP_ADD, "sub": OP_SUB, "mul": OP_MUL}[k], enc(nd[1]), enc(nd[2]))
        elif k == "neg":
            t = (OP_NEG, enc(nd[1]), 0)
        else:
            t = (OP_EMBED, enc(nd[1]), 0)
        for o in _operands(nd):
            if emitted[o] and not is_root[o] and last[o] == i and slot_of[o] is not None:
                free[dims[o]].append(slot_of[o])
                slot_of[o] = None
        d = dims[i]
        if free[d]:
            s = free[d].pop()
        else:
            s = count[d]
            count[d] += 1
        slot_of[i] = s
        out.append((t[0], t[1], t[2], s | (RES_EXT_BIT if d == EXT else 0)))
    root_enc = [slot_of[r] | (RES_EXT_BIT if dims[r] == EXT else 0) for r in roots]
    return {"nodes": np.array(out, np.uint32).reshape(-1, 4), "roots": np.array(root_enc, np.uint32),
            "base_consts": np.array(prog["base_consts"], np.uint64),
            "ext_consts": np.array(prog["ext_consts"], np.uint64).reshape(-1, 3),
            "num_base_slots": count[BASE], "num_ext_slots": count[EXT]}


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
