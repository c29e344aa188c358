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


OPK_VAR = 7                    # trace operand: payload = aux << 28 | frame offset << 20 | column
VAR_AUX_BIT, VAR_OFF_SHIFT, VAR_COL_MASK = 1 << 28, 20, (1 << 20) - 1
NO_ROOT = 0xFFFFFFFF


def lower(prog, stream=True):
    """DeviceProgram::lower (constraint_ir/device.rs:160-330).

    stream=False gives the reference's program shape: every trace read is an
    OP_VAR node with a slot of its own and every constraint's value stays
    pinned in its slot until the walk ends, when the roots are combined. That
    costs a slot for every constraint and every live trace value: a wide AIR
    (thousands of constraints) needs thousands of slots per row.

    stream=True (the default) lowers for the streaming walker: trace reads
    become OPK_VAR operands read where they are used, and `node_roots` names
    the constraint each instruction completes (NO_ROOT otherwise), so the
    kernel folds the constraint into the composition as soon as it is computed
    and its slot is free for reuse; a node that several constraints share gets
    one extra copy instruction per further constraint. Only intermediate
    values occupy slots, so the slot file stays small whatever the width."""
    nodes, dims, roots = prog["nodes"], prog["dims"], prog["roots"]
    # a device program may name its constraints' indices in a larger program
    # (prog["num_roots"] constraints) whose first constraints a hand-written
    # kernel evaluates (prog["hand"]) and whose LogUp constraints the library
    # evaluates from the table's descriptor (prog["logup"] = (first index,
    # descriptor))
    index = prog.get("root_index", list(range(len(roots))))
    n = len(nodes)
    base_consts = list(prog["base_consts"])
    used = [False] * n
    last = [0] * n
    for i, nd in enumerate(nodes):
        for o in _operands(nd):
            used[o] = True
            last[o] = i
    is_root = [False] * n
    root_ids = [[] for _ in range(n)]
    for c, r in enumerate(roots):
        is_root[r] = True
        used[r] = True
        root_ids[r].append(index[c])
    leaf = [_uniform(nodes[i]) or (stream and nodes[i][0] == "var") for i in range(n)]
    emitted = [used[i] and (not leaf[i] or is_root[i]) for i in range(n)]
    if stream:
        if 0 not in base_consts:
            base_consts.append(0)
        zero_enc = (OPK_BASE_CONST << OPK_SHIFT) | base_consts.index(0)

    def enc_leaf(nd):
        k = nd[0]
        if k == "var":
            _, is_main, off, col = nd
            assert off < 256 and col <= VAR_COL_MASK
            return (OPK_VAR << OPK_SHIFT) | (0 if is_main else VAR_AUX_BIT) | (off << VAR_OFF_SHIFT) | col
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
    out, node_roots = [], []

    def take(d):
        s_ = free[d].pop() if free[d] else count[d]
        if s_ == count[d]:
            count[d] += 1
        return s_

    def enc(j):
        if not emitted[j]:
            return enc_leaf(nodes[j])
        kind = OPK_BASE_SLOT if dims[j] == BASE else OPK_EXT_SLOT
        return (kind << OPK_SHIFT) | slot_of[j]

    for i in range(n):
        if not emitted[i]:
            continue
        nd = nodes[i]
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
        pinned = (lambda o: is_root[o]) if not stream else (lambda o: False)
        for o in _operands(nd):
            if emitted[o] and not pinned(o) and last[o] == i and slot_of[o] is not None:
                free[dims[o]].append(slot_of[o])
                slot_of[o] = None
        d = dims[i]
        slot_of[i] = take(d)
        ext = RES_EXT_BIT if d == EXT else 0
        out.append((t[0], t[1], t[2], slot_of[i] | ext))
        if stream:
            ids = root_ids[i]
            node_roots.append(ids[0] if ids else NO_ROOT)
            for c in ids[1:]:  # a node several constraints share: one copy per further constraint
                sc = take(d)
                out.append((OP_ADD, enc(i), zero_enc, sc | ext))
                node_roots.append(c)
                free[d].append(sc)
            if not last[i] > i:  # no later use: the slot is free again
                free[d].append(slot_of[i])
                slot_of[i] = None
    if stream:
        root_enc = [0] * len(roots)
    else:
        root_enc = [slot_of[r] | (RES_EXT_BIT if dims[r] == EXT else 0) for r in roots]
    low = {"nodes": np.array(out, np.uint32).reshape(-1, 4), "roots": np.array(root_enc, np.uint32),
           "base_consts": np.array(base_consts, np.uint64),
           "ext_consts": np.array(prog["ext_consts"], np.uint64).reshape(-1, 3),
           "num_base_slots": count[BASE], "num_ext_slots": count[EXT]}
    if stream:
        low["node_roots"] = np.array(node_roots, np.uint32)
    if "hand" in prog:
        assert stream, "a hand kernel's program is a streaming program"
        low["hand_kernel"], low["hand_roots"] = prog["hand"]
        low["num_roots"] = prog["hand"][1] + len(roots)
    if "logup" in prog:
        # the table's LogUp constraints, evaluated by the library from its descriptor
        assert stream, "LogUp constraints from a descriptor need a streaming program"
        low["logup_root"], low["logup_desc"] = prog["logup"]
    if "num_roots" in prog:
        low["num_roots"] = prog["num_roots"]
    return low


def restrict(prog, keep):
    """The program of the nodes the roots `keep` (indices into prog["roots"])
    depend on, renumbered in their order, with those roots in that order."""
    nodes, dims = prog["nodes"], prog["dims"]
    need = [False] * len(nodes)
    stack = [prog["roots"][c] for c in keep]
    while stack:
        i = stack.pop()
        if not need[i]:
            need[i] = True
            stack.extend(_operands(nodes[i]))
    new_id, out, out_dims = {}, [], []
    for i, nd in enumerate(nodes):
        if not need[i]:
            continue
        new_id[i] = len(out)
        if nd[0] in ("add", "sub", "mul"):
            nd = (nd[0], new_id[nd[1]], new_id[nd[2]])
        elif nd[0] in ("neg", "embed"):
            nd = (nd[0], new_id[nd[1]])
        out.append(nd)
        out_dims.append(dims[i])
    roots = [new_id[prog["roots"][c]] for c in keep]
    return {"nodes": out, "dims": out_dims, "base_consts": list(prog["base_consts"]),
            "ext_consts": list(prog["ext_consts"]), "roots": roots,
            "num_base": sum(1 for r in roots if out_dims[r] == BASE)}


def lowered(prog):
    """lower(prog), computed once per program (kept in the program dict: a
    table's program does not change, and a wide AIR takes a while to lower)."""
    low = prog.get("_lowered")
    if low is None:
        low = prog["_lowered"] = lower(prog)
    return low


def device_program(air):
    """The program the GPU prover runs for `air`: its device_program when it
    has one (a program some of whose constraints the library's own kernels
    evaluate: a hand-written table kernel, the LogUp constraints from the
    table's descriptor), else its constraint program."""
    return getattr(air, "device_program", None) or air.program
