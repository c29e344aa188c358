"""Constraint IR capture and device lowering.

`Builder` captures constraints in the reference's flat IR
(crypto/stark/src/constraint_ir/ir.rs: topologically ordered Op nodes, each
with a Base/Ext dim, constants in side tables, per-constraint roots with the
base-rooted constraints first), hash-consing identical nodes like
constraint_ir/builder.rs. `lower` turns a program into the device blob of
constraint_ir/device.rs (DeviceProgram::lower): uniform leaves propagated into
operands, dim-split value slots reused at each operand's last use, roots pinned.
"""
import numpy as np

OP_CONST_BASE, OP_CONST_EXT, OP_VAR, OP_RAP, OP_ALPHA, OP_OFFSET = 0, 1, 2, 3, 4, 5
OP_ADD, OP_SUB, OP_MUL, OP_NEG, OP_EMBED = 6, 7, 8, 9, 10
OPK_SHIFT = 29
OPK_BASE_SLOT, OPK_EXT_SLOT, OPK_BASE_CONST, OPK_EXT_CONST, OPK_RAP, OPK_ALPHA, OPK_OFFSET = range(7)
RES_EXT_BIT = 1 << 31
BASE, EXT = 0, 1


class Builder:
    def __init__(self):
        self.nodes, self.dims = [], []
        self.base_consts, self.ext_consts = [], []
        self._memo = {}
        self.roots = []
        self.num_base = 0

    def _node(self, node, dim):
        key = (node, dim)
        if key in self._memo:
            return self._memo[key]
        self.nodes.append(node)
        self.dims.append(dim)
        self._memo[key] = len(self.nodes) - 1
        return self._memo[key]

    # leaves
    def main(self, offset, col):
        return self._node(("var", True, offset, col), BASE)

    def aux(self, offset, col):
        return self._node(("var", False, offset, col), EXT)

    def const_base(self, v):
        v = int(v)
        if v not in self.base_consts:
            self.base_consts.append(v)
        return self._node(("cb", self.base_consts.index(v)), BASE)

    def challenge(self, idx):
        return self._node(("rap", idx), EXT)

    def alpha_pow(self, idx):
        return self._node(("alpha", idx), EXT)

    def table_offset(self):
        return self._node(("off",), EXT)

    # arithmetic
    def _bin(self, op, a, b):
        return self._node((op, a, b), EXT if (self.dims[a] == EXT or self.dims[b] == EXT) else BASE)

    def add(self, a, b):
        return self._bin("add", a, b)

    def sub(self, a, b):
        return self._bin("sub", a, b)

    def mul(self, a, b):
        return self._bin("mul", a, b)

    def neg(self, a):
        return self._node(("neg", a), self.dims[a])

    def emit(self, root):
        self.roots.append(root)

    def program(self):
        base = [r for r in self.roots if self.dims[r] == BASE]
        ext = [r for r in self.roots if self.dims[r] == EXT]
        return {"nodes": list(self.nodes), "dims": list(self.dims), "base_consts": list(self.base_consts),
                "ext_consts": list(self.ext_consts), "roots": base + ext, "num_base": len(base)}


def _operands(node):
    if node[0] in ("add", "sub", "mul"):
        return [node[1], node[2]]
    if node[0] in ("neg", "embed"):
        return [node[1]]
    return []


def _uniform(node):
    return node[0] in ("cb", "ce", "rap", "alpha", "off")


def lower(prog):
    """DeviceProgram::lower (constraint_ir/device.rs:160-330)."""
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
            _, is_main, off, col = nd
            t = (OP_VAR, col, (int(is_main) << 16) | (off << 8))
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
        s = free[d].pop() if free[d] else count[d]
        if s == count[d]:
            count[d] += 1
        slot_of[i] = s
        out.append((t[0], t[1], t[2], s | (RES_EXT_BIT if d == EXT else 0)))
    root_enc = [slot_of[r] | (RES_EXT_BIT if dims[r] == EXT else 0) for r in roots]
    return {"nodes": np.array(out, np.uint32).reshape(-1, 4), "roots": np.array(root_enc, np.uint32),
            "base_consts": np.array(prog["base_consts"], np.uint64),
            "ext_consts": np.array(prog["ext_consts"], np.uint64).reshape(-1, 3),
            "num_base_slots": count[BASE], "num_ext_slots": count[EXT]}
