"""AIRs of the RV64 front-end: the CPU table and the 16-bit range table.

One CPU row per executed instruction (rv64.execute). The register file is
carried in the row (x1..x31 as two 32-bit limbs each; x0 is zero and has no
column), so register reads are one-hot dot products and writes are one-hot
updates of the next row: no memory argument is needed for this ISA subset
(ADD, SUB, ADDI, LUI, BEQ, BNE, ECALL). Every value written is range-checked
limb by limb (four 16-bit pieces looked up in the RANGE table), so every
register limb is below 2^32 and the 64-bit additions with boolean carries are
exact integer identities in the field.

The prover's transition constraints are cyclic (they also link the last row
to row 0). A STEP flag column marks the one row whose successor is not its
next instruction: that row must be the halting ECALL (pc = the program's halt
pc) and the row after it (cyclically: row 0) must hold the initial state
(pc 0, every register zero). Its multiplicity (1 - STEP) on the END bus, which
the verifier balances against one public (a0) tuple, makes it exactly one
row. So the trace is one execution from the initial state to the halt, whose
a0 is the claimed output.

Buses (LogUp, lookup.rs conventions: fingerprint z - (bus + sum alpha^(i+1)
v_i), senders +m, receivers -m): ROM (bus 1): each CPU row sends its
instruction tuple (pc, opcode id, rd, rs1, rs2, imm low and high 32-bit limbs,
imm as a field element); the verifier receives every instruction of the
public program with its execution count. RANGE (bus 2): CPU rows send the four
16-bit pieces of the written value, the RANGE table receives 0..2^16-1 with
multiplicities. END (bus 3): see above. The public program, counts and output
are absorbed into the transcript label before any challenge is drawn.
"""
import numpy as np

from . import field as F
from .air import split_interactions
from .ir import Builder
from .rv64 import MASK64, OP_ID, OPS, decode, execute

P = F.P
NEG_ONE = P - 1
BUS_ROM, BUS_RANGE, BUS_END = 1, 2, 3


class BusAir:
    """LogUp plumbing shared by the front-end tables. An interaction is
    {"bus", "elems": [lin], "mult": lin, "sender"} with lin = (const, [(coef,
    col)]) a linear form over the row's main columns."""

    def _logup_setup(self, interactions):
        self.interactions = interactions
        self.num_committed, self.num_absorbed = split_interactions(len(interactions))
        self.aux_width = self.num_committed + 1
        self.acc_col = self.num_committed
        self.max_alpha = 1 + max(len(it["elems"]) for it in interactions)
        self.boundary = [(self.acc_col, True, 0)]
        self.num_parts = 2

    @staticmethod
    def _lin(b, lin, offset=0):
        const, terms = lin
        e = b.const_base(const % P) if const else None
        for coef, col in terms:
            t = b.main(offset, col)
            if coef % P != 1:
                t = b.mul(b.const_base(coef % P), t)
            e = t if e is None else b.add(e, t)
        return e if e is not None else b.const_base(0)

    def _fp(self, b, it):
        fp = b.neg(b.sub(b.const_base(it["bus"]), b.challenge(0)))  # z - bus
        for i, lin in enumerate(it["elems"]):
            fp = b.sub(fp, b.mul(b.alpha_pow(i + 1), self._lin(b, lin)))
        return fp

    def _signed_m(self, b, it):
        m = self._lin(b, it["mult"])
        return m if it["sender"] else b.neg(m)

    def _emit_logup(self, b):
        """Batched committed pairs and the accumulated column
        (crypto/stark/src/lookup.rs:2185-2290)."""
        its = self.interactions
        for p in range(self.num_committed):
            ia, ib = its[2 * p], its[2 * p + 1]
            fa, fb = self._fp(b, ia), self._fp(b, ib)
            main = b.mul(b.mul(b.aux(0, p), fa), fb)
            b.emit(b.sub(b.sub(main, b.mul(self._signed_m(b, ia), fb)), b.mul(self._signed_m(b, ib), fa)))
        delta = b.sub(b.aux(1, self.acc_col), b.aux(0, self.acc_col))
        for p in range(self.num_committed):
            delta = b.sub(delta, b.aux(0, p))
        delta = b.add(delta, b.table_offset())
        ab = its[2 * self.num_committed:]
        if len(ab) == 1:
            b.emit(b.neg(b.sub(self._signed_m(b, ab[0]), b.mul(delta, self._fp(b, ab[0])))))
        else:
            f1, f2 = self._fp(b, ab[0]), self._fp(b, ab[1])
            root = b.mul(b.mul(delta, f1), f2)
            root = b.sub(root, b.mul(self._signed_m(b, ab[0]), f2))
            root = b.sub(root, b.mul(self._signed_m(b, ab[1]), f1))
            b.emit(root)

    def logup_descriptor(self):
        """CSR descriptor (crypto/math-cuda/src/logup.rs:26-44) of the interactions."""
        K = len(self.interactions)
        eo, ea, ec, to, tc, tl = [0], [], [], [0], [], []
        mc, mo, mk, ml = [], [0], [], []
        for it in self.interactions:
            for i, (const, terms) in enumerate(it["elems"]):
                ea.append(i + 1)
                ec.append(const % P)
                for coef, col in terms:
                    tc.append(coef % P)
                    tl.append(col)
                to.append(len(tc))
            eo.append(len(ea))
            const, terms = it["mult"]
            sg = 1 if it["sender"] else NEG_ONE
            mc.append(const * sg % P)
            for coef, col in terms:
                mk.append(coef * sg % P)
                ml.append(col)
            mo.append(len(mk))
        oo, oi = [0], []
        for c in range(self.num_committed):
            oi += [2 * c, 2 * c + 1]
            oo.append(len(oi))
        oi += list(range(2 * self.num_committed, K))
        oo.append(len(oi))
        u32 = lambda x: np.array(x, np.uint32)
        u64 = lambda x: np.array(x, np.uint64)
        return {"num_interactions": K, "bus_ids": u64([it["bus"] for it in self.interactions]),
                "elem_offsets": u32(eo), "elem_alpha_idx": u32(ea), "elem_consts": u64(ec), "term_offsets": u32(to),
                "term_coefs": u64(tc), "term_cols": u32(tl), "num_out_cols": self.num_committed + 1,
                "out_col_offsets": u32(oo), "out_col_interactions": u32(oi), "mult_consts": u64(mc),
                "mult_term_offsets": u32(mo), "mult_term_coefs": u64(mk), "mult_term_cols": u32(ml),
                "num_committed": self.num_committed}


# ---------------------------------------------------------------- CPU table columns
PC, STEP = 0, 1
SEL = {op: 2 + i for i, op in enumerate(OPS)}   # one-hot opcode selectors
RD0 = 2 + len(OPS)                                # rd one-hot, 32 columns
RS10 = RD0 + 32                                   # rs1 one-hot
RS20 = RS10 + 32                                  # rs2 one-hot
IMM_LO, IMM_HI, IMM_F = RS20 + 32, RS20 + 33, RS20 + 34
A_LO, A_HI, B_LO, B_HI = IMM_F + 1, IMM_F + 2, IMM_F + 3, IMM_F + 4
R_LO, R_HI = B_HI + 1, B_HI + 2
R16 = R_HI + 1                                    # four 16-bit pieces of the written value
C0, C1 = R16 + 4, R16 + 5
INV_LO, INV_HI, E_LO, E_HI, NE, BR = C1 + 1, C1 + 2, C1 + 3, C1 + 4, C1 + 5, C1 + 6
X0 = BR + 1                                       # x1..x31: lo at X0 + 2(k-1), hi next
CPU_WIDTH = X0 + 62
TWO16, TWO32 = 1 << 16, 1 << 32


def _batch_inverse(vals):
    """Inverses mod p of a list of ints (0 -> 0) with one exponentiation
    (prefix products, Montgomery's trick)."""
    nz = [v for v in vals if v]
    pre, acc = [], 1
    for v in nz:
        pre.append(acc)
        acc = acc * v % P
    inv = pow(acc, P - 2, P) if nz else 1
    out_nz = [0] * len(nz)
    for i in range(len(nz) - 1, -1, -1):
        out_nz[i] = inv * pre[i] % P
        inv = inv * nz[i] % P
    it = iter(out_nz)
    return [next(it) if v else 0 for v in vals]


def xlo(k):
    return X0 + 2 * (k - 1)


def xhi(k):
    return X0 + 2 * (k - 1) + 1


def rom_tuple(pc, op, rd, rs1, rs2, imm):
    """The instruction tuple both sides of the ROM bus agree on."""
    u = imm & MASK64
    return (pc, OP_ID[op], rd, rs1, rs2, u & 0xFFFFFFFF, u >> 32, imm % P)


class CpuAir(BusAir):
    def __init__(self, words, log_n):
        self.words = list(words)
        self.prog = [decode(w) for w in self.words]
        self.halt_pc = 4 * next(i for i, ins in enumerate(self.prog) if ins[0] == "ecall")
        self.log_n, self.n, self.width = log_n, 1 << log_n, CPU_WIDTH
        self._logup_setup([
            {"bus": BUS_ROM, "sender": True, "mult": (1, []),
             "elems": [(0, [(1, PC)]), (0, [(OP_ID[o], SEL[o]) for o in OPS]), (0, [(k, RD0 + k) for k in range(1, 32)]),
                       (0, [(k, RS10 + k) for k in range(1, 32)]), (0, [(k, RS20 + k) for k in range(1, 32)]),
                       (0, [(1, IMM_LO)]), (0, [(1, IMM_HI)]), (0, [(1, IMM_F)])]},
        ] + [{"bus": BUS_RANGE, "sender": True, "mult": (1, []), "elems": [(0, [(1, R16 + i)])]} for i in range(4)] + [
            {"bus": BUS_END, "sender": True, "mult": (1, [(NEG_ONE, STEP)]),
             "elems": [(0, [(1, xlo(10))]), (0, [(1, xhi(10))])]},
        ])
        self.program = self._build_program()

    def _build_program(self):
        b = Builder()
        M = lambda c: b.main(0, c)
        N = lambda c: b.main(1, c)
        one = b.const_base(1)
        k32 = b.const_base(TWO32)
        sel = {o: M(c) for o, c in SEL.items()}
        step = M(STEP)
        nstep = b.sub(one, step)

        def boolean(e):
            b.emit(b.mul(e, b.sub(e, one)))

        def total(cols):
            s = M(cols[0])
            for c in cols[1:]:
                s = b.add(s, M(c))
            return s

        # one-hot selections and booleans
        for c in [STEP, C0, C1] + list(SEL.values()) + [RD0 + k for k in range(32)] + \
                [RS10 + k for k in range(32)] + [RS20 + k for k in range(32)]:
            boolean(M(c))
        for group in (list(SEL.values()), [RD0 + k for k in range(32)], [RS10 + k for k in range(32)],
                      [RS20 + k for k in range(32)]):
            b.emit(b.sub(total(group), one))

        # operand reads: a = x[rs1], b = x[rs2] (x0 = 0 has no column)
        def read(base, limb):
            s = None
            for k in range(1, 32):
                t = b.mul(M(base + k), M(xlo(k) if limb == 0 else xhi(k)))
                s = t if s is None else b.add(s, t)
            return s
        b.emit(b.sub(M(A_LO), read(RS10, 0)))
        b.emit(b.sub(M(A_HI), read(RS10, 1)))
        b.emit(b.sub(M(B_LO), read(RS20, 0)))
        b.emit(b.sub(M(B_HI), read(RS20, 1)))
        # written value in 16-bit pieces (each one looked up in the RANGE table)
        k16 = b.const_base(TWO16)
        b.emit(b.sub(M(R_LO), b.add(M(R16), b.mul(k16, M(R16 + 1)))))
        b.emit(b.sub(M(R_HI), b.add(M(R16 + 2), b.mul(k16, M(R16 + 3)))))
        # results per opcode, with 32-bit carries
        rl, rh, al, ah, bl, bh, c0, c1 = (M(c) for c in (R_LO, R_HI, A_LO, A_HI, B_LO, B_HI, C0, C1))
        il, ih = M(IMM_LO), M(IMM_HI)
        # add / addi: r + c*2^32 = a + b (limb by limb, carry c0 into the high limb)
        for s, ol, oh in ((sel["add"], bl, bh), (sel["addi"], il, ih)):
            b.emit(b.mul(s, b.sub(b.add(rl, b.mul(c0, k32)), b.add(al, ol))))
            b.emit(b.mul(s, b.sub(b.add(rh, b.mul(c1, k32)), b.add(b.add(ah, oh), c0))))
        # sub: r + b = a + c*2^32 (borrows)
        b.emit(b.mul(sel["sub"], b.sub(b.add(rl, bl), b.add(al, b.mul(c0, k32)))))
        b.emit(b.mul(sel["sub"], b.sub(b.add(b.add(rh, bh), c0), b.add(ah, b.mul(c1, k32)))))
        # lui: r = imm
        b.emit(b.mul(sel["lui"], b.sub(rl, il)))
        b.emit(b.mul(sel["lui"], b.sub(rh, ih)))
        # no value for branches and ecall; no carries where none is used
        nores = b.add(b.add(sel["beq"], sel["bne"]), sel["ecall"])
        b.emit(b.mul(nores, rl))
        b.emit(b.mul(nores, rh))
        nocarry = b.add(nores, sel["lui"])
        b.emit(b.mul(nocarry, c0))
        b.emit(b.mul(nocarry, c1))
        # on branch rows, a != b: e = d * inv, d (1 - e) = 0 per limb; ne = e_lo
        # OR e_hi; branch taken. Elsewhere e, ne and the branch flag are 0.
        branch = b.add(sel["beq"], sel["bne"])
        for d, inv, e in ((b.sub(al, bl), INV_LO, E_LO), (b.sub(ah, bh), INV_HI, E_HI)):
            b.emit(b.mul(branch, b.sub(M(e), b.mul(d, M(inv)))))
            b.emit(b.mul(branch, b.mul(d, b.sub(one, M(e)))))
            b.emit(b.mul(b.sub(one, branch), M(e)))
        el, eh, ne = M(E_LO), M(E_HI), M(NE)
        b.emit(b.sub(ne, b.sub(b.add(el, eh), b.mul(el, eh))))
        b.emit(b.sub(M(BR), b.add(b.mul(sel["beq"], b.sub(one, ne)), b.mul(sel["bne"], ne))))
        # transitions (rows with STEP = 1): next pc and the register file
        four = b.const_base(4)
        adv = b.add(b.mul(four, b.sub(one, sel["ecall"])), b.mul(M(BR), b.sub(M(IMM_F), four)))
        b.emit(b.mul(step, b.sub(N(PC), b.add(M(PC), adv))))
        for k in range(1, 32):
            for col, r in ((xlo(k), rl), (xhi(k), rh)):
                upd = b.mul(M(RD0 + k), b.sub(r, M(col)))
                b.emit(b.mul(step, b.sub(N(col), b.add(M(col), upd))))
        # the END row (STEP = 0): the halting ECALL, followed by the initial state
        b.emit(b.mul(nstep, b.sub(M(PC), b.const_base(self.halt_pc))))
        b.emit(b.mul(nstep, b.sub(one, sel["ecall"])))
        b.emit(b.mul(nstep, N(PC)))
        for k in range(1, 32):
            b.emit(b.mul(nstep, N(xlo(k))))
            b.emit(b.mul(nstep, N(xhi(k))))
        self._emit_logup(b)
        return b.program()

    # ---------------------------------------------------------- trace
    def trace(self, rows):
        """CPU table of an execution (rv64.execute rows), padded to n rows by
        repeating the halting ECALL; the last row is the END row. Built column
        by column with numpy."""
        n, T = self.n, len(rows)
        assert 1 <= T <= n, "the execution does not fit the table"
        cols = list(zip(*rows))
        ext = lambda c: np.concatenate([c, np.full(n - T, c[-1], dtype=c.dtype)])
        pc, rd, rs1, rs2 = (ext(np.array(cols[i], dtype=np.uint64)) for i in (0, 2, 3, 4))
        imm_i = ext(np.array(cols[5], dtype=np.int64))
        imm_u = imm_i.view(np.uint64)
        a, bv, r = (ext(np.array(cols[i], dtype=np.uint64)) for i in (6, 7, 8))
        op_of = {o: OP_ID[o] for o in OPS}
        op = ext(np.array([op_of[o] for o in cols[1]], dtype=np.int64))
        m32, s32 = np.uint64(0xFFFFFFFF), np.uint64(32)
        t = np.zeros((CPU_WIDTH, n), dtype=np.uint64)  # column-major while filling
        t[PC] = pc
        t[STEP] = 1
        t[STEP, n - 1] = 0
        opcol = 2 + op - 1  # SEL columns follow OPS order, ids start at 1
        idx = np.arange(n)
        t[opcol, idx] = 1
        t[RD0 + rd.astype(np.int64), idx] = 1
        t[RS10 + rs1.astype(np.int64), idx] = 1
        t[RS20 + rs2.astype(np.int64), idx] = 1
        t[IMM_LO], t[IMM_HI] = imm_u & m32, imm_u >> s32
        t[IMM_F] = np.where(imm_i < 0, np.uint64(P) - (-imm_i).astype(np.uint64), imm_u)
        t[A_LO], t[A_HI] = a & m32, a >> s32
        t[B_LO], t[B_HI] = bv & m32, bv >> s32
        t[R_LO], t[R_HI] = r & m32, r >> s32
        for j in range(4):
            t[R16 + j] = (r >> np.uint64(16 * j)) & np.uint64(0xFFFF)
        is_add = (op == OP_ID["add"]) | (op == OP_ID["addi"])
        o = np.where(op == OP_ID["add"], bv, imm_u)
        c0 = ((a & m32) + (o & m32)) >> s32
        c1 = ((a >> s32) + (o >> s32) + c0) >> s32
        sb = op == OP_ID["sub"]
        b0 = ((a & m32) < (bv & m32)).astype(np.uint64)
        b1 = ((a >> s32) < (bv >> s32) + b0).astype(np.uint64)
        t[C0] = np.where(is_add, c0, np.where(sb, b0, 0))
        t[C1] = np.where(is_add, c1, np.where(sb, b1, 0))
        # branch rows: per-limb difference, its inverse, the flags
        br_rows = np.nonzero((op == OP_ID["beq"]) | (op == OP_ID["bne"]))[0]
        for ac, bc, ic, ec in ((A_LO, B_LO, INV_LO, E_LO), (A_HI, B_HI, INV_HI, E_HI)):
            d = [(x - y) % P for x, y in zip(t[ac, br_rows].tolist(), t[bc, br_rows].tolist())]
            t[ic, br_rows] = np.array(_batch_inverse(d), dtype=np.uint64)
            t[ec, br_rows] = np.array([1 if x else 0 for x in d], dtype=np.uint64)
        ne = t[E_LO] | t[E_HI]
        t[NE] = ne
        t[BR] = np.where(op == OP_ID["bne"], ne, np.where(op == OP_ID["beq"], 1 - ne, 0))
        # register file before each row: the last value written below it
        writes = np.isin(op, [OP_ID[x] for x in ("add", "sub", "addi", "lui")]) & (rd != 0) & (idx < T)
        for k in range(1, 32):
            wk = np.where(writes & (rd == k), idx, -1)
            last = np.maximum.accumulate(wk)
            before = np.concatenate(([-1], last[:-1]))
            val = np.where(before >= 0, r[np.maximum(before, 0)], np.uint64(0))
            t[xlo(k)], t[xhi(k)] = val & m32, val >> s32
        return np.ascontiguousarray(t.T)

    def counts(self, rows):
        """Execution count of every program instruction over the n table rows."""
        pcs = np.array([r[0] for r in rows], dtype=np.int64) // 4
        c = np.bincount(pcs, minlength=len(self.prog))
        c[pcs[-1]] += self.n - len(rows)  # the repeated halting row
        return [int(v) for v in c]

    def public_terms(self, counts, output):
        """The verifier's side of the ROM and END buses: (bus, tuple, signed
        multiplicity), receivers negative."""
        terms = []
        for i, (op, rd, rs1, rs2, imm) in enumerate(self.prog):
            if counts[i]:
                terms.append((BUS_ROM, rom_tuple(4 * i, op, rd, rs1, rs2, imm), -counts[i]))
        terms.append((BUS_END, (output & 0xFFFFFFFF, output >> 32), -1))
        return terms


class RangeAir(BusAir):
    """The values 0..2^16-1, one per row, each with its multiplicity: V(next)
    = V + 1 - 2^16 W with W boolean and W (V - (2^16 - 1)) = 0. Around the
    cycle of 2^16 rows the V increments sum to zero, so W is 1 on exactly one
    row, where V = 2^16 - 1: V takes every value of 0..2^16-1 once."""

    def __init__(self):
        self.log_n, self.n, self.width = 16, 1 << 16, 3
        self.V, self.W, self.M = 0, 1, 2
        self._logup_setup([{"bus": BUS_RANGE, "sender": False, "mult": (0, [(1, self.M)]),
                            "elems": [(0, [(1, self.V)])]}])
        self.program = self._build_program()

    def _build_program(self):
        b = Builder()
        v, w, vn = b.main(0, self.V), b.main(0, self.W), b.main(1, self.V)
        one = b.const_base(1)
        b.emit(b.mul(w, b.sub(w, one)))
        b.emit(b.sub(vn, b.sub(b.add(v, one), b.mul(b.const_base(TWO16), w))))
        b.emit(b.mul(w, b.sub(v, b.const_base(TWO16 - 1))))
        self._emit_logup(b)
        return b.program()

    def trace(self, cpu_trace):
        t = np.zeros((self.n, 3), np.uint64)
        t[:, self.V] = np.arange(self.n, dtype=np.uint64)
        t[self.n - 1, self.W] = 1
        vals = cpu_trace[:, R16:R16 + 4].reshape(-1).astype(np.int64)
        t[:, self.M] = np.bincount(vals, minlength=self.n).astype(np.uint64)
        return t


def statement_label(words, counts, output):
    """Transcript label binding the public statement (program words, counts,
    output) before any challenge is drawn."""
    from .math_cuda import keccak256
    blob = b"".join(int(w).to_bytes(4, "little") for w in words)
    blob += b"".join(int(c).to_bytes(8, "little") for c in counts)
    blob += int(output).to_bytes(8, "little")
    return b"lambda_vm_b200/rv64/" + keccak256(blob)


def native_trace(words, max_steps=1 << 32):
    """Execute and build the CPU table in the library (sg_rv64_trace, C++):
    (table, counts, a0, cycles)."""
    import ctypes as C
    from . import native
    L = native.lib()
    w = np.ascontiguousarray(np.asarray(words, dtype=np.uint32))
    a0, cyc = C.c_uint64(), C.c_uint64()
    native.check(L.sg_rv64_trace(w.ctypes.data, len(w), max_steps, 0, None, None, C.byref(a0), C.byref(cyc)))
    n = 1 << max(1, (cyc.value - 1).bit_length())
    t = np.empty((n, CPU_WIDTH), np.uint64)
    counts = np.zeros(len(w), np.uint64)
    native.check(L.sg_rv64_trace(w.ctypes.data, len(w), max_steps, n, t.ctypes.data, counts.ctypes.data,
                                 C.byref(a0), C.byref(cyc)))
    return t, [int(c) for c in counts], a0.value, cyc.value


def build(words):
    """Execute a program and build its tables (the CPU table by the library's
    native executor): (airs, traces, public) with public = {"words", "counts",
    "output", "cycles", "label", "terms"}."""
    ct, counts, out, cycles = native_trace(words)
    cpu = CpuAir(words, ct.shape[0].bit_length() - 1)
    rng = RangeAir()
    rt = rng.trace(ct)
    pub = {"words": list(words), "counts": counts, "output": out, "cycles": cycles,
           "label": statement_label(words, counts, out), "terms": cpu.public_terms(counts, out)}
    return [cpu, rng], [ct, rt], pub


def airs_for(words, counts):
    """The verifier's tables of a statement (it never executes the program):
    the CPU table has one row per counted instruction execution."""
    n = sum(int(c) for c in counts)
    assert n >= 2 and n & (n - 1) == 0, "the counts must cover a power-of-two table"
    return [CpuAir(words, n.bit_length() - 1), RangeAir()]


def prove(words, opts, bk):
    """Execute `words` and prove the execution on backend `bk` (stark.multi_prove,
    the plain per-table form): (proof, public statement)."""
    from .stark import multi_prove
    airs, traces, pub = build(words)
    proof = multi_prove(airs, traces, opts, bk, label=pub["label"])
    return proof, pub


def verify(words, counts, output, proof, opts, device=None):
    """Verify that `words` run from the initial state halts with a0 = output,
    having executed each instruction counts[i] times: (ok, reason)."""
    from . import verifier
    airs = airs_for(words, counts)
    cpu = airs[0]
    return verifier.verify(airs, proof, opts, label=statement_label(words, counts, output), device=device,
                           public_terms=cpu.public_terms(counts, output))
