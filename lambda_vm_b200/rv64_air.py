"""AIRs of the RV64 front-end: the CPU table and the chips beside it.

Tables (a chip is present in a proof only when the execution uses it):

* CPU: one row per executed instruction (rv64.run). The register file is
  carried in the row (x1..x31 as two 32-bit limbs each; x0 is zero and has no
  column), so register reads are one-hot dot products and writes are one-hot
  updates of the next row. Every value written to a register is range-checked
  limb by limb (four 16-bit pieces looked up in the RANGE table), so every
  register limb is below 2^32 and 64-bit additions with boolean carries are
  exact integer identities in the field.
* RANGE: the values 0..2^16-1 with multiplicities.
* BITWISE: every pair of bytes (x, y) with x XOR y, x OR y, x AND y; the CPU
  looks up the eight byte triples of a bitwise instruction.
* SHIFT: one row per executed shift (SLLI, SRLI): the operand's 64 bits and
  the result of shifting them in two stages (by k mod 8 bits, then by k div 8
  bytes).
* MEMORY: one row per data-memory cell the run touches, sorted by address:
  the cell's initial zero and its final value and timestamp. Offline memory
  checking: every access receives the cell's (address, value, timestamp) as
  the access before it left it and sends its own; a range check keeps each
  previous timestamp below the access's.
* KECCAK: 24 rows per keccak-f[1600] ecall, one per round, with the bits of
  theta's column parities and output; it reads the 25 lanes from memory on
  its first row and writes them back on its last.

The prover's transition constraints are cyclic (they also link the last row
to row 0). A STEP flag column in the CPU table marks the one row whose
successor is not its next instruction: that row must be an exit ECALL
(a7 = 93, so the machine halts there) and the row after it (cyclically: row 0) must
hold the initial state (pc 0, every register zero, timestamp 1). Its
multiplicity (1 - STEP) on the END bus, which the verifier balances against
one public (a0) tuple, makes it exactly one row. So the CPU table is one
execution from the initial state to the halt, whose a0 is the claimed output.

Buses (LogUp, lookup.rs conventions: fingerprint z - (bus + sum alpha^(i+1)
v_i), senders +m, receivers -m): ROM (1): each CPU row sends its instruction
tuple (pc, opcode id, rd, rs1, rs2, imm low and high 32-bit limbs, imm as a
field element); the verifier receives every instruction of the public
program with its execution count. RANGE (2), END (3), BITWISE (4): (kind,
x, y, result), SHIFT (5): (direction, a low, a high, amount, r low, r high),
MEM (6): (address, value low, value high, timestamp), KECCAK (7): (timestamp,
state address), WRAP (8): the one row of the MEMORY table whose successor is
not the next address. The public program, counts, output and table heights
are absorbed into the transcript label before any challenge is drawn.
"""
import numpy as np

from . import field as F
from .air import split_interactions
from .ir import Builder, restrict
from .rv64 import EXIT, KECCAK, KECCAK_RC, KECCAK_ROT, MASK64, OP_ID, OPS, decode, run

P = F.P
NEG_ONE = P - 1
BUS_ROM, BUS_RANGE, BUS_END, BUS_BITWISE, BUS_SHIFT, BUS_MEM, BUS_KECCAK, BUS_WRAP = 1, 2, 3, 4, 5, 6, 7, 8
TWO16, TWO32 = 1 << 16, 1 << 32
MIN_LOG_N = 6
CHIPS = ("bitwise", "shift", "memory", "keccak")
_PROGRAMS = {}  # constraint programs by (table, parameters): a table's program depends on neither its height nor its trace


def _hand_program(air, key, kernel):
    """The GPU prover's program for a table whose base constraints a
    hand-written library kernel evaluates (SG_AIR_* `kernel`): no nodes; the
    library also evaluates the LogUp constraints, which follow the base
    constraints in the table's whole program, from the table's descriptor."""
    if key not in _PROGRAMS:
        nb = air.program["num_base"]
        prog = Builder().program()
        assert nb + air.num_committed + 1 == len(air.program["roots"])
        prog["root_index"] = []
        prog["hand"] = (kernel, nb)
        prog["logup"] = (nb, air.logup_descriptor())
        prog["num_roots"] = len(air.program["roots"])
        _PROGRAMS[key] = prog
    return _PROGRAMS[key]


def _logup_program(air, key):
    """The GPU prover's program for a table without a hand-written kernel:
    its base constraints walked, its LogUp constraints (which follow them in
    the table's whole program) evaluated by the library from its descriptor."""
    if key not in _PROGRAMS:
        full = air.program
        nb = full["num_base"]
        assert nb + air.num_committed + 1 == len(full["roots"])
        prog = restrict(full, range(nb))
        prog["logup"] = (nb, air.logup_descriptor())
        prog["num_roots"] = len(full["roots"])
        _PROGRAMS[key] = prog
    return _PROGRAMS[key]


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

    def _program(self, key):
        if key not in _PROGRAMS:
            _PROGRAMS[key] = self._build_program()
        return _PROGRAMS[key]

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


def _col(c, coef=1):
    return (0, [(coef, c)])


def _sum_of(cols, coefs=None):
    return (0, [(1 if coefs is None else coefs[i], c) for i, c in enumerate(cols)])


class _Expr:
    """Helpers over a Builder: sums, scaling, booleans, XOR of bits."""

    def __init__(self, b):
        self.b = b
        self.one = b.const_base(1)
        self.zero = b.const_base(0)

    def total(self, es):
        s = None
        for e in es:
            s = e if s is None else self.b.add(s, e)
        return s if s is not None else self.zero

    def scaled(self, k, e):
        return e if k % P == 1 else self.b.mul(self.b.const_base(k % P), e)

    def boolean(self, e):
        self.b.emit(self.b.mul(e, self.b.sub(e, self.one)))

    def xor2(self, x, y):
        b = self.b
        return b.sub(b.add(x, y), self.scaled(2, b.mul(x, y)))

    def xor3(self, x, y, z):
        """x ^ y ^ z of bits: x + y + z - 2(xy + yz + xz) + 4xyz."""
        b = self.b
        pairs = b.add(b.add(b.mul(x, y), b.mul(y, z)), b.mul(x, z))
        return b.add(b.sub(b.add(b.add(x, y), z), self.scaled(2, pairs)), self.scaled(4, b.mul(b.mul(x, y), z)))


# ---------------------------------------------------------------- CPU table columns
CPU_OPS = OPS + ("keccak",)   # the keccak ecall has a selector of its own; its ROM opcode is ECALL's
PC, STEP, CLK = 0, 1, 2
SEL = {op: 3 + i for i, op in enumerate(CPU_OPS)}  # one-hot opcode selectors
RD0 = 3 + len(CPU_OPS)                            # rd one-hot, 32 columns
RS10 = RD0 + 32                                   # rs1 one-hot
RS20 = RS10 + 32                                  # rs2 one-hot
IMM_LO, IMM_HI, IMM_F = RS20 + 32, RS20 + 33, RS20 + 34
A_LO, A_HI, B_LO, B_HI = IMM_F + 1, IMM_F + 2, IMM_F + 3, IMM_F + 4
R_LO, R_HI = B_HI + 1, B_HI + 2
R16 = R_HI + 1                                    # four 16-bit pieces of the written value
C0, C1 = R16 + 4, R16 + 5
INV_LO, INV_HI, E_LO, E_HI, NE, BR = C1 + 1, C1 + 2, C1 + 3, C1 + 4, C1 + 5, C1 + 6
X0 = BR + 1                                       # x1..x31: lo at X0 + 2(k-1), hi next
CPU_CORE_WIDTH = X0 + 62                          # the table of a run that needs no chip ends here
AB0 = CPU_CORE_WIDTH                              # bytes of a, of the second operand, of the result
BB0 = AB0 + 8
RB0 = BB0 + 8
MA = RB0 + 8                                      # memory address (ld / sd / keccak state)
MW0, MW1 = MA + 1, MA + 2                         # MA = 8 MW0 + 2^19 MW1
MV_LO, MV_HI, MT = MA + 3, MA + 4, MA + 5         # the cell's value and timestamp before the access
MD0, MD1 = MA + 6, MA + 7                         # CLK - MT - 1 in 16-bit pieces
NV_LO, NV_HI = MA + 8, MA + 9                     # the value the access leaves
CPU_WIDTH = NV_HI + 1
KECCAK_OP = len(OPS) + 1                          # the keccak ecall's op in a row record
REG_CHUNK = 64                                    # register snapshots every REG_CHUNK rows
WRITES = ("add", "sub", "addi", "lui", "xor", "or", "and", "xori", "ori", "andi", "slli", "srli", "ld")
BIT_REG, BIT_IMM = ("xor", "or", "and"), ("xori", "ori", "andi")
BIT_KIND = {"xor": 1, "xori": 1, "or": 2, "ori": 2, "and": 3, "andi": 3}
NEEDS = {"xor": "bitwise", "or": "bitwise", "and": "bitwise", "xori": "bitwise", "ori": "bitwise",
         "andi": "bitwise", "slli": "shift", "srli": "shift", "ld": "memory", "sd": "memory"}


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


def _log2_rows(k):
    return max(MIN_LOG_N, (max(k, 1) - 1).bit_length())


class CpuAir(BusAir):
    """The CPU table. `chips` names the chips the proof carries; the CPU's
    lookups into a chip are part of the table only when the chip is, and an
    instruction whose chip is absent cannot occur."""

    def __init__(self, words, log_n, chips=()):
        self.words = list(words)
        self.prog = [decode(w) for w in self.words]
        assert any(ins[0] == "ecall" for ins in self.prog), "a program halts by an ecall"
        self.chips = tuple(c for c in CHIPS if c in chips)
        self.log_n, self.n = log_n, 1 << log_n
        self.width = CPU_WIDTH if self.chips else CPU_CORE_WIDTH
        rom_op = [(OP_ID["ecall" if o == "keccak" else o], SEL[o]) for o in CPU_OPS]
        its = [
            {"bus": BUS_ROM, "sender": True, "mult": (1, []),
             "elems": [_col(PC), (0, rom_op), (0, [(k, RD0 + k) for k in range(1, 32)]),
                       (0, [(k, RS10 + k) for k in range(1, 32)]), (0, [(k, RS20 + k) for k in range(1, 32)]),
                       _col(IMM_LO), _col(IMM_HI), _col(IMM_F)]},
        ] + [{"bus": BUS_RANGE, "sender": True, "mult": (1, []), "elems": [_col(R16 + i)]} for i in range(4)] + [
            {"bus": BUS_END, "sender": True, "mult": (1, [(NEG_ONE, STEP)]),
             "elems": [_col(xlo(10)), _col(xhi(10))]},
        ]
        if "bitwise" in self.chips:
            kind = (0, [(BIT_KIND[o], SEL[o]) for o in BIT_REG + BIT_IMM])
            mult = _sum_of([SEL[o] for o in BIT_REG + BIT_IMM])
            its += [{"bus": BUS_BITWISE, "sender": True, "mult": mult,
                     "elems": [kind, _col(AB0 + i), _col(BB0 + i), _col(RB0 + i)]} for i in range(8)]
        if "shift" in self.chips:
            its.append({"bus": BUS_SHIFT, "sender": True, "mult": _sum_of([SEL["slli"], SEL["srli"]]),
                        "elems": [_col(SEL["srli"]), _col(A_LO), _col(A_HI), _col(IMM_LO), _col(R_LO),
                                  _col(R_HI)]})
        if "memory" in self.chips:
            smem = _sum_of([SEL["ld"], SEL["sd"]])
            saddr = _sum_of([SEL["ld"], SEL["sd"], SEL["keccak"]])
            its += [
                {"bus": BUS_MEM, "sender": False, "mult": smem,
                 "elems": [_col(MA), _col(MV_LO), _col(MV_HI), _col(MT)]},
                {"bus": BUS_MEM, "sender": True, "mult": smem,
                 "elems": [_col(MA), _col(NV_LO), _col(NV_HI), _col(CLK)]},
                {"bus": BUS_RANGE, "sender": True, "mult": saddr, "elems": [_col(MW0)]},
                {"bus": BUS_RANGE, "sender": True, "mult": saddr, "elems": [_col(MW1, 8)]},
                {"bus": BUS_RANGE, "sender": True, "mult": smem, "elems": [_col(MD0)]},
                {"bus": BUS_RANGE, "sender": True, "mult": smem, "elems": [_col(MD1)]},
            ]
        if "keccak" in self.chips:
            its.append({"bus": BUS_KECCAK, "sender": True, "mult": _col(SEL["keccak"]),
                        "elems": [_col(CLK), _col(MA)]})
        self._logup_setup(its)
        self.program = self._program(("cpu", self.chips))
        mask = sum(1 << i for i, c in enumerate(CHIPS) if c in self.chips)
        self.device_program = _hand_program(self, ("cpu-device", self.chips), 2 | (mask << 8))

    def _build_program(self):
        b = Builder()
        x = _Expr(b)
        M = lambda c: b.main(0, c)
        N = lambda c: b.main(1, c)
        one = x.one
        k32 = b.const_base(TWO32)
        k16 = b.const_base(TWO16)
        sel = {o: M(c) for o, c in SEL.items()}
        sel_sum = lambda ops: x.total([sel[o] for o in ops])
        step = M(STEP)
        nstep = b.sub(one, step)
        has = lambda chip: chip in self.chips

        # one-hot selections and booleans
        for c in [STEP, C0, C1] + list(SEL.values()) + [RD0 + k for k in range(32)] + \
                [RS10 + k for k in range(32)] + [RS20 + k for k in range(32)]:
            x.boolean(M(c))
        for group in (list(SEL.values()), [RD0 + k for k in range(32)], [RS10 + k for k in range(32)],
                      [RS20 + k for k in range(32)]):
            b.emit(b.sub(x.total([M(c) for c in group]), one))
        # an instruction whose chip the proof does not carry cannot occur
        for o, chip in list(NEEDS.items()) + [("keccak", "keccak")]:
            if not has(chip) or (o == "keccak" and not has("memory")):
                b.emit(sel[o])

        # operand reads: a = x[rs1], b = x[rs2] (x0 = 0 has no column)
        def read(base, limb):
            return x.total([b.mul(M(base + k), M(xlo(k) if limb == 0 else xhi(k))) for k in range(1, 32)])
        b.emit(b.sub(M(A_LO), read(RS10, 0)))
        b.emit(b.sub(M(A_HI), read(RS10, 1)))
        b.emit(b.sub(M(B_LO), read(RS20, 0)))
        b.emit(b.sub(M(B_HI), read(RS20, 1)))
        # written value in 16-bit pieces (each one looked up in the RANGE table)
        b.emit(b.sub(M(R_LO), b.add(M(R16), b.mul(k16, M(R16 + 1)))))
        b.emit(b.sub(M(R_HI), b.add(M(R16 + 2), b.mul(k16, M(R16 + 3)))))
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
        # no value for branches, ecalls and stores; carries only where an addition uses them
        nores = sel_sum(("beq", "bne", "ecall", "keccak", "sd"))
        b.emit(b.mul(nores, rl))
        b.emit(b.mul(nores, rh))
        nocarry = b.sub(one, sel_sum(("add", "addi", "sub", "ld", "sd")))
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
        # ecalls: exit with a7 = 93, keccak with a7 = 2^64 - 2
        b.emit(b.mul(sel["ecall"], b.sub(M(xlo(17)), b.const_base(EXIT))))
        b.emit(b.mul(sel["ecall"], M(xhi(17))))
        b.emit(b.mul(sel["keccak"], b.sub(M(xlo(17)), b.const_base(KECCAK & 0xFFFFFFFF))))
        b.emit(b.mul(sel["keccak"], b.sub(M(xhi(17)), b.const_base(KECCAK >> 32))))

        if has("bitwise"):
            # the operands and the result as bytes (each triple looked up in BITWISE)
            def bytes_of(first, lo):
                return x.total([x.scaled(1 << (8 * i), M(first + i + (0 if lo else 4))) for i in range(4)])
            sreg, simm = sel_sum(BIT_REG), sel_sum(BIT_IMM)
            sbit = b.add(sreg, simm)
            for lo, (a_, b_, i_, r_) in ((True, (al, bl, il, rl)), (False, (ah, bh, ih, rh))):
                b.emit(b.mul(sbit, b.sub(a_, bytes_of(AB0, lo))))
                ob = bytes_of(BB0, lo)
                b.emit(b.add(b.mul(sreg, b.sub(b_, ob)), b.mul(simm, b.sub(i_, ob))))
                b.emit(b.mul(sbit, b.sub(r_, bytes_of(RB0, lo))))
        if has("memory"):
            smem = b.add(sel["ld"], sel["sd"])
            saddr = b.add(smem, sel["keccak"])
            ma = M(MA)
            # ld / sd: address = a + imm below 2^32 (the high limbs' sum is 0 or 2^32)
            b.emit(b.mul(smem, b.sub(b.add(ma, b.mul(c0, k32)), b.add(al, il))))
            b.emit(b.mul(smem, b.sub(b.mul(c1, k32), b.add(b.add(ah, ih), c0))))
            # keccak: the state address is a0, below 2^32
            b.emit(b.mul(sel["keccak"], b.sub(ma, M(xlo(10)))))
            b.emit(b.mul(sel["keccak"], M(xhi(10))))
            # 8-byte aligned, below 2^32: MA = 8 MW0 + 2^19 MW1, MW0 and 8 MW1 in RANGE
            b.emit(b.mul(saddr, b.sub(ma, b.add(x.scaled(8, M(MW0)), x.scaled(1 << 19, M(MW1))))))
            # the previous access is earlier: CLK - MT - 1 = MD0 + 2^16 MD1
            gap = b.sub(b.sub(M(CLK), M(MT)), one)
            b.emit(b.mul(smem, b.sub(gap, b.add(M(MD0), b.mul(k16, M(MD1))))))
            for nv, mv, bv, r_ in ((NV_LO, MV_LO, B_LO, rl), (NV_HI, MV_HI, B_HI, rh)):
                b.emit(b.mul(sel["ld"], b.sub(M(nv), M(mv))))
                b.emit(b.mul(sel["sd"], b.sub(M(nv), M(bv))))
                b.emit(b.mul(sel["ld"], b.sub(r_, M(mv))))

        # transitions (rows with STEP = 1): next pc, timestamp and register file
        four = b.const_base(4)
        adv = b.add(b.mul(four, b.sub(one, sel["ecall"])), b.mul(M(BR), b.sub(M(IMM_F), four)))
        b.emit(b.mul(step, b.sub(N(PC), b.add(M(PC), adv))))
        b.emit(b.mul(step, b.sub(N(CLK), b.add(M(CLK), one))))
        for k in range(1, 32):
            for col, r in ((xlo(k), rl), (xhi(k), rh)):
                upd = b.mul(M(RD0 + k), b.sub(r, M(col)))
                b.emit(b.mul(step, b.sub(N(col), b.add(M(col), upd))))
        # the END row (STEP = 0): an exit ECALL (a7 = 93, above), followed by the initial state
        b.emit(b.mul(nstep, b.sub(one, sel["ecall"])))
        b.emit(b.mul(nstep, N(PC)))
        b.emit(b.mul(nstep, b.sub(N(CLK), one)))
        for k in range(1, 32):
            b.emit(b.mul(nstep, N(xlo(k))))
            b.emit(b.mul(nstep, N(xhi(k))))
        self._emit_logup(b)
        return b.program()

    # ---------------------------------------------------------- trace
    def trace(self, records):
        """CPU table of an execution from its row records (T x 8 u64, the
        layout sg_rv64_run writes: pc | op << 32 | rd << 40 | rs1 << 48 |
        rs2 << 56, imm, a, b, r, memory address, the cell's previous value and
        timestamp), padded to n rows by repeating the halting ECALL; the last
        row is the END row. Built column by column with numpy."""
        rec = np.asarray(records, np.uint64).reshape(-1, 8)
        n, T = self.n, rec.shape[0]
        assert 1 <= T <= n, "the execution does not fit the table"
        rec = np.concatenate([rec, np.repeat(rec[-1:], n - T, axis=0)])
        w0 = rec[:, 0]
        pc = w0 & np.uint64(0xFFFFFFFF)
        op = ((w0 >> np.uint64(32)) & np.uint64(0xFF)).astype(np.int64)
        rd, rs1, rs2 = (((w0 >> np.uint64(s_)) & np.uint64(0xFF)).astype(np.int64) for s_ in (40, 48, 56))
        imm_u, a, bv, r, ma, mv, mt = (rec[:, i] for i in range(1, 8))
        imm_i = imm_u.view(np.int64)
        is_op = lambda *names: np.isin(op, [KECCAK_OP if o == "keccak" else OP_ID[o] for o in names])
        m32, s32 = np.uint64(0xFFFFFFFF), np.uint64(32)
        idx = np.arange(n)
        t = np.zeros((self.width, n), dtype=np.uint64)  # column-major while filling
        t[PC] = pc
        t[STEP] = 1
        t[STEP, n - 1] = 0
        t[CLK] = idx + 1
        t[SEL["add"] + op - 1, idx] = 1
        t[RD0 + rd, idx] = 1
        t[RS10 + rs1, idx] = 1
        t[RS20 + rs2, idx] = 1
        t[IMM_LO], t[IMM_HI] = imm_u & m32, imm_u >> s32
        t[IMM_F] = np.where(imm_i < 0, np.uint64(P) - (-imm_i).astype(np.uint64), imm_u)
        t[A_LO], t[A_HI] = a & m32, a >> s32
        t[B_LO], t[B_HI] = bv & m32, bv >> s32
        t[R_LO], t[R_HI] = r & m32, r >> s32
        for j in range(4):
            t[R16 + j] = (r >> np.uint64(16 * j)) & np.uint64(0xFFFF)
        # carries of the additions: add / addi / ld / sd (a + operand), sub's borrows
        is_add = is_op("add", "addi", "ld", "sd")
        o = np.where(op == OP_ID["add"], bv, imm_u)
        c0 = ((a & m32) + (o & m32)) >> s32
        c1 = ((a >> s32) + (o >> s32) + c0) >> s32
        sb = op == OP_ID["sub"]
        b0 = ((a & m32) < (bv & m32)).astype(np.uint64)
        b1 = ((a >> s32) < (bv >> s32) + b0).astype(np.uint64)
        t[C0] = np.where(is_add, c0, np.where(sb, b0, 0))
        t[C1] = np.where(is_add, c1, np.where(sb, b1, 0))
        # branch rows: per-limb difference, its inverse, the flags
        br_rows = np.nonzero(is_op("beq", "bne"))[0]
        for ac, bc, ic, ec in ((A_LO, B_LO, INV_LO, E_LO), (A_HI, B_HI, INV_HI, E_HI)):
            d = [(x_ - y_) % P for x_, y_ in zip(t[ac, br_rows].tolist(), t[bc, br_rows].tolist())]
            t[ic, br_rows] = np.array(_batch_inverse(d), dtype=np.uint64)
            t[ec, br_rows] = np.array([1 if v else 0 for v in d], dtype=np.uint64)
        ne = t[E_LO] | t[E_HI]
        t[NE] = ne
        t[BR] = np.where(op == OP_ID["bne"], ne, np.where(op == OP_ID["beq"], 1 - ne, 0))
        # register file before each row: the last value written below it
        writes = is_op(*WRITES) & (rd != 0) & (idx < T)
        for k in range(1, 32):
            wk = np.where(writes & (rd == k), idx, -1)
            last = np.maximum.accumulate(wk)
            before = np.concatenate(([-1], last[:-1]))
            val = np.where(before >= 0, r[np.maximum(before, 0)], np.uint64(0))
            t[xlo(k)], t[xhi(k)] = val & m32, val >> s32
        if self.width == CPU_WIDTH:
            # bitwise rows: bytes of a, of the second operand, of the result
            bit = is_op(*BIT_REG, *BIT_IMM)
            second = np.where(is_op(*BIT_REG), bv, imm_u)
            for first, v in ((AB0, a), (BB0, second), (RB0, r)):
                for i in range(8):
                    t[first + i] = np.where(bit, (v >> np.uint64(8 * i)) & np.uint64(0xFF), 0)
            # memory rows
            mem = is_op("ld", "sd")
            addr = mem | is_op("keccak")
            t[MA] = np.where(addr, ma, 0)
            t[MW0] = np.where(addr, (ma >> np.uint64(3)) & np.uint64(0xFFFF), 0)
            t[MW1] = np.where(addr, ma >> np.uint64(19), 0)
            t[MV_LO], t[MV_HI] = np.where(mem, mv & m32, 0), np.where(mem, mv >> s32, 0)
            t[MT] = np.where(mem, mt, 0)
            gap = np.where(mem, (idx + 1).astype(np.uint64) - mt - np.uint64(1), np.uint64(0))
            t[MD0], t[MD1] = gap & np.uint64(0xFFFF), gap >> np.uint64(16)
            nv = np.where(op == OP_ID["ld"], mv, np.where(op == OP_ID["sd"], bv, 0))
            t[NV_LO], t[NV_HI] = nv & m32, nv >> s32
        else:
            assert not is_op(*NEEDS, "keccak").any(), "a chip instruction in a table without the chips' columns"
        return np.ascontiguousarray(t.T)

    def counts(self, records):
        """Execution count of every program instruction over the n table rows."""
        rec = np.asarray(records, np.uint64).reshape(-1, 8)
        pcs = ((rec[:, 0] & np.uint64(0xFFFFFFFF)) // np.uint64(4)).astype(np.int64)
        c = np.bincount(pcs, minlength=len(self.prog))
        c[pcs[-1]] += self.n - rec.shape[0]  # the repeated halting row
        return [int(v) for v in c]

    def public_terms(self, counts, output):
        """The verifier's side of the ROM and END buses (and of WRAP with the
        memory chip): (bus, tuple, signed multiplicity), receivers negative."""
        terms = []
        for i, (op, rd, rs1, rs2, imm) in enumerate(self.prog):
            if counts[i]:
                terms.append((BUS_ROM, rom_tuple(4 * i, op, rd, rs1, rs2, imm), -counts[i]))
        terms.append((BUS_END, (output & 0xFFFFFFFF, output >> 32), -1))
        if "memory" in self.chips:
            terms.append((BUS_WRAP, (1,), -1))
        return terms


class RangeAir(BusAir):
    """The values 0..2^16-1, one per row, each with its multiplicity: V(next)
    = V + 1 - 2^16 W with W boolean and W (V - (2^16 - 1)) = 0. Around the
    cycle of 2^16 rows the V increments sum to zero, so W is 1 on exactly one
    row, where V = 2^16 - 1: V takes every value of 0..2^16-1 once."""

    V, W, M = 0, 1, 2

    def __init__(self):
        self.log_n, self.n, self.width = 16, 1 << 16, 3
        self._logup_setup([{"bus": BUS_RANGE, "sender": False, "mult": _col(self.M), "elems": [_col(self.V)]}])
        self.program = self._program(("range",))
        self.device_program = _logup_program(self, ("range-device",))

    def _build_program(self):
        b = Builder()
        v, w, vn = b.main(0, self.V), b.main(0, self.W), b.main(1, self.V)
        one = b.const_base(1)
        b.emit(b.mul(w, b.sub(w, one)))
        b.emit(b.sub(vn, b.sub(b.add(v, one), b.mul(b.const_base(TWO16), w))))
        b.emit(b.mul(w, b.sub(v, b.const_base(TWO16 - 1))))
        self._emit_logup(b)
        return b.program()

    def trace(self, lookups, counts=None):
        """lookups: arrays of the 16-bit values looked up (with repetition),
        added to counts (per value) if given."""
        t = np.zeros((self.n, 3), np.uint64)
        t[:, self.V] = np.arange(self.n, dtype=np.uint64)
        t[self.n - 1, self.W] = 1
        m = np.zeros(self.n, np.int64) if counts is None else np.asarray(counts, np.uint64).astype(np.int64)
        for v in lookups:
            v = np.asarray(v).reshape(-1).astype(np.int64)
            assert v.size == 0 or (v.min() >= 0 and v.max() < self.n), "a range lookup outside 0..2^16-1"
            m += np.bincount(v, minlength=self.n)
        t[:, self.M] = m.astype(np.uint64)
        return t


class BitwiseAir(BusAir):
    """Every pair of bytes (x, y) with x XOR y, x OR y and x AND y, each with
    a multiplicity: x and y are sums of boolean bit columns, so the table holds
    bytes only, and each result is the bitwise identity over those bits."""

    XB, YB, XOR, OR, AND, MX, MO, MAN = 0, 8, 16, 17, 18, 19, 20, 21

    def __init__(self):
        self.log_n, self.n, self.width = 16, 1 << 16, 22
        xs = _sum_of([self.XB + i for i in range(8)], [1 << i for i in range(8)])
        ys = _sum_of([self.YB + i for i in range(8)], [1 << i for i in range(8)])
        self._logup_setup([{"bus": BUS_BITWISE, "sender": False, "mult": _col(m), "elems": [(k, []), xs, ys, _col(r)]}
                           for k, r, m in ((1, self.XOR, self.MX), (2, self.OR, self.MO), (3, self.AND, self.MAN))])
        self.program = self._program(("bitwise",))
        self.device_program = _logup_program(self, ("bitwise-device",))

    def _build_program(self):
        b = Builder()
        x = _Expr(b)
        M = lambda c: b.main(0, c)
        xb = [M(self.XB + i) for i in range(8)]
        yb = [M(self.YB + i) for i in range(8)]
        for e in xb + yb:
            x.boolean(e)
        both = [b.mul(xb[i], yb[i]) for i in range(8)]
        b.emit(b.sub(M(self.AND), x.total([x.scaled(1 << i, both[i]) for i in range(8)])))
        b.emit(b.sub(M(self.XOR), x.total([x.scaled(1 << i, b.sub(b.add(xb[i], yb[i]), x.scaled(2, both[i])))
                                           for i in range(8)])))
        b.emit(b.sub(M(self.OR), x.total([x.scaled(1 << i, b.sub(b.add(xb[i], yb[i]), both[i]))
                                          for i in range(8)])))
        self._emit_logup(b)
        return b.program()

    _fixed_columns = None

    @classmethod
    def _fixed(cls):
        """The table with zero multiplicities (the bit and result columns do
        not depend on the run), built once a process."""
        if cls._fixed_columns is None:
            n = 1 << 16
            t = np.zeros((n, 22), np.uint64)
            v = np.arange(n, dtype=np.uint64)
            xv, yv = v >> np.uint64(8), v & np.uint64(0xFF)
            for i in range(8):
                t[:, cls.XB + i] = (xv >> np.uint64(i)) & np.uint64(1)
                t[:, cls.YB + i] = (yv >> np.uint64(i)) & np.uint64(1)
            t[:, cls.XOR], t[:, cls.OR], t[:, cls.AND] = xv ^ yv, xv | yv, xv & yv
            t.setflags(write=False)
            cls._fixed_columns = t
        return cls._fixed_columns

    def trace(self, records, counts=None):
        """The table with the multiplicities of the byte triples the CPU's
        bitwise rows (row records, as CpuAir.trace) look up, or with the
        executor's counts (3 x 2^16: XOR, OR, AND)."""
        t = self._fixed().copy()
        if counts is not None:
            cnt = np.asarray(counts, np.uint64).reshape(3, self.n)
            t[:, self.MX], t[:, self.MO], t[:, self.MAN] = cnt[0], cnt[1], cnt[2]
            return t
        rec = np.asarray(records, np.uint64).reshape(-1, 8)
        op = ((rec[:, 0] >> np.uint64(32)) & np.uint64(0xFF)).astype(np.int64)
        sh = np.arange(0, 64, 8, dtype=np.uint64)
        for k, mcol in ((1, self.MX), (2, self.MO), (3, self.MAN)):
            reg = np.isin(op, [OP_ID[o] for o in BIT_REG if BIT_KIND[o] == k])
            imm = np.isin(op, [OP_ID[o] for o in BIT_IMM if BIT_KIND[o] == k])
            rows = reg | imm
            a = rec[rows, 2]
            second = np.where(reg[rows], rec[rows, 3], rec[rows, 1])
            keys = (((a[:, None] >> sh) & np.uint64(0xFF)) << np.uint64(8)) | ((second[:, None] >> sh) & np.uint64(0xFF))
            t[:, mcol] = np.bincount(keys.reshape(-1).astype(np.int64), minlength=self.n).astype(np.uint64)
        return t


class ShiftAir(BusAir):
    """One row per executed shift: DIR (0 left, 1 right), the operand's 64
    bits, the amount k = s + 8q as one-hot s (0..7) and q (0..7), the operand
    shifted by s bits (TB), and the result's limbs: TB_j = sum_s S_s a_(j-+s),
    r_i = sum_q Q_q TB_(i-+8q), bits shifted in are zero."""

    DIR, AB, S, Q, TB, R_LO, R_HI, M = 0, 1, 65, 73, 81, 145, 146, 147

    def __init__(self, log_n):
        self.log_n, self.n, self.width = log_n, 1 << log_n, 148
        k = (0, [(s, self.S + s) for s in range(1, 8)] + [(8 * q, self.Q + q) for q in range(1, 8)])
        alo = _sum_of([self.AB + i for i in range(32)], [1 << i for i in range(32)])
        ahi = _sum_of([self.AB + 32 + i for i in range(32)], [1 << i for i in range(32)])
        self._logup_setup([{"bus": BUS_SHIFT, "sender": False, "mult": _col(self.M),
                            "elems": [_col(self.DIR), alo, ahi, k, _col(self.R_LO), _col(self.R_HI)]}])
        self.program = self._program(("shift",))
        self.device_program = _hand_program(self, ("shift-device",), 3)

    def _build_program(self):
        b = Builder()
        x = _Expr(b)
        M = lambda c: b.main(0, c)
        d = M(self.DIR)
        nd = b.sub(x.one, d)
        a = [M(self.AB + i) for i in range(64)]
        s = [M(self.S + i) for i in range(8)]
        q = [M(self.Q + i) for i in range(8)]
        tb = [M(self.TB + i) for i in range(64)]
        for e in [d] + a + s + q:
            x.boolean(e)
        b.emit(b.sub(x.total(s), x.one))
        b.emit(b.sub(x.total(q), x.one))

        def shifted(src, j, k_, size=64):
            """Element j of src (size elements) shifted by k_ in the row's
            direction (None: zero either way)."""
            parts = []
            if j - k_ >= 0:
                parts.append(b.mul(nd, src[j - k_]))
            if j + k_ < size:
                parts.append(b.mul(d, src[j + k_]))
            return x.total(parts) if parts else None

        for j in range(64):
            terms = [b.mul(s[k_], e) for k_ in range(8) if (e := shifted(a, j, k_)) is not None]
            b.emit(b.sub(tb[j], x.total(terms)))
        # the second stage moves whole bytes: with TB's bytes tB[i] = sum_j 2^j
        # TB_(8i+j), r's byte k is sum_q Q_q tB[k -+ q] (the same polynomial as
        # the bit-by-bit sum, with 16 products a limb instead of 256)
        tB = [x.total([x.scaled(1 << j, tb[8 * i + j]) for j in range(8)]) for i in range(8)]
        for limb, col in ((0, self.R_LO), (1, self.R_HI)):
            acc = []
            for k in range(4 * limb, 4 * limb + 4):
                terms = [b.mul(q[k_], e) for k_ in range(8) if (e := shifted(tB, k, k_, 8)) is not None]
                acc.append(x.scaled(1 << (8 * (k - 4 * limb)), x.total(terms)))
            b.emit(b.sub(M(col), x.total(acc)))
        self._emit_logup(b)
        return b.program()

    def trace(self, shifts):
        """shifts: (dir, a, k) per executed shift."""
        n = self.n
        assert len(shifts) <= n, "the shifts do not fit the table"
        t = np.zeros((n, self.width), np.uint64)
        t[:, self.S] = 1
        t[:, self.Q] = 1
        if len(shifts) == 0:
            return t
        sh = np.asarray(shifts, dtype=np.uint64).reshape(-1, 3)
        dr, av, kv = sh[:, 0], sh[:, 1], sh[:, 2]
        m = sh.shape[0]
        rows = np.arange(m)
        t[:m, self.DIR] = dr
        for i in range(64):
            t[:m, self.AB + i] = (av >> np.uint64(i)) & np.uint64(1)
        sv, qv = kv & np.uint64(7), kv >> np.uint64(3)
        t[:m, self.S] = 0
        t[:m, self.Q] = 0
        t[rows, self.S + sv.astype(np.int64)] = 1
        t[rows, self.Q + qv.astype(np.int64)] = 1
        tv = np.where(dr == 1, av >> sv, av << sv)
        for j in range(64):
            t[:m, self.TB + j] = (tv >> np.uint64(j)) & np.uint64(1)
        rv = np.where(dr == 1, av >> kv, av << kv)
        t[:m, self.R_LO], t[:m, self.R_HI] = rv & np.uint64(0xFFFFFFFF), rv >> np.uint64(32)
        t[:m, self.M] = 1
        return t


class MemoryAir(BusAir):
    """One row per data-memory cell touched, addresses strictly increasing
    down the table (ADDR(next) = ADDR + 8 + 8 (D0 + 2^16 D1), D0 and D1 in
    RANGE) except on the one row where NW = 0 (the WRAP bus holds exactly one
    such row against the verifier's public tuple), so no address has two rows.
    Active rows send the cell's initial (address, 0, 0, timestamp 0) and
    receive its final (address, value, timestamp); padding rows (ACT = 0)
    continue the addresses."""

    ADDR, V_LO, V_HI, T, ACT, NW, D0, D1 = range(8)

    def __init__(self, log_n):
        self.log_n, self.n, self.width = log_n, 1 << log_n, 8
        self._logup_setup([
            {"bus": BUS_MEM, "sender": True, "mult": _col(self.ACT),
             "elems": [_col(self.ADDR), (0, []), (0, []), (0, [])]},
            {"bus": BUS_MEM, "sender": False, "mult": _col(self.ACT),
             "elems": [_col(self.ADDR), _col(self.V_LO), _col(self.V_HI), _col(self.T)]},
            {"bus": BUS_RANGE, "sender": True, "mult": (1, []), "elems": [_col(self.D0)]},
            {"bus": BUS_RANGE, "sender": True, "mult": (1, []), "elems": [_col(self.D1)]},
            {"bus": BUS_WRAP, "sender": True, "mult": (1, [(NEG_ONE, self.NW)]), "elems": [(1, [])]},
        ])
        self.program = self._program(("memory",))
        self.device_program = _logup_program(self, ("memory-device",))

    def _build_program(self):
        b = Builder()
        x = _Expr(b)
        M = lambda c: b.main(0, c)
        x.boolean(M(self.ACT))
        x.boolean(M(self.NW))
        step = b.add(b.const_base(8), b.add(x.scaled(8, M(self.D0)), x.scaled(8 << 16, M(self.D1))))
        b.emit(b.mul(M(self.NW), b.sub(b.main(1, self.ADDR), b.add(M(self.ADDR), step))))
        self._emit_logup(b)
        return b.program()

    def trace(self, addrs, values, stamps):
        """The touched cells, sorted by address, with final values and timestamps."""
        n = self.n
        addrs = np.asarray(addrs, np.uint64)
        k = addrs.size
        assert 1 <= k <= n, "the memory cells do not fit the table"
        t = np.zeros((n, self.width), np.uint64)
        col = np.concatenate([addrs, addrs[-1] + np.uint64(8) * np.arange(1, n - k + 1, dtype=np.uint64)])
        t[:, self.ADDR] = col
        vals = np.asarray(values, np.uint64)
        t[:k, self.V_LO], t[:k, self.V_HI] = vals & np.uint64(0xFFFFFFFF), vals >> np.uint64(32)
        t[:k, self.T] = np.asarray(stamps, np.uint64)
        t[:k, self.ACT] = 1
        t[:n - 1, self.NW] = 1
        d = (col[1:] - col[:-1] - np.uint64(8)) >> np.uint64(3)
        t[:n - 1, self.D0], t[:n - 1, self.D1] = d & np.uint64(0xFFFF), d >> np.uint64(16)
        return t


# ---------------------------------------------------------------- KECCAK table columns
def _lane(x, y):
    return x + 5 * y


KR = 0                  # round flags R_0..R_23
KA = KR + 24            # the round's input lanes, 4 x 16-bit limbs each
KC = KA + 100           # bits of theta's column parities C[x][z]
KCP = KC + 320          # bits of C'[x][z] = C[x] ^ C[x-1] ^ rot(C[x+1], 1)
KAP = KCP + 320         # bits of theta's output A'[x + 5y][z]
KOUT = KAP + 1600       # the round's output lanes as limbs (lane 0 after iota)
KB00 = KOUT + 100       # bits of lane 0 after chi, before iota
KBASE = KB00 + 64       # state address
KCLK = KBASE + 1        # the ecall's timestamp
KTOLD = KCLK + 1        # previous timestamps of the 25 cells (first row)
KTD = KTOLD + 25        # KCLK - KTOLD_i - 1 in 16-bit pieces (first row)
KECCAK_WIDTH = KTD + 50


class KeccakAir(BusAir):
    """keccak-f[1600], one round per row, 24 rows per ecall (FIPS 202
    theta, rho, pi, chi, iota on lanes A[x + 5y]).

    Constraints: A's limbs are the bits A' ^ C ^ C'; for every (x, z) the
    five A'[x][y][z] and C'[x][z] have even parity, so C is A's column parity
    and A' = theta(A); OUT's limbs are chi of rho-pi of A' (lane 0: the stored
    bits, then XOR the round constant selected by the flags); a row that is
    not a permutation's last passes OUT on as the next row's A. The first row
    of a permutation (R_0) takes (timestamp, address) from the CPU's ecall and
    reads the 25 lanes from memory at earlier timestamps; the last (R_23)
    writes them back at the ecall's timestamp. Rows outside permutations hold
    the all-zero state with no flag set (every constraint holds on them)."""

    def __init__(self, log_n):
        self.log_n, self.n, self.width = log_n, 1 << log_n, KECCAK_WIDTH
        lo = lambda base, i: (0, [(1, base + 4 * i), (TWO16, base + 4 * i + 1)])
        hi = lambda base, i: (0, [(1, base + 4 * i + 2), (TWO16, base + 4 * i + 3)])
        its = [{"bus": BUS_KECCAK, "sender": False, "mult": _col(KR), "elems": [_col(KCLK), _col(KBASE)]}]
        for i in range(25):
            addr = (8 * i, [(1, KBASE)])
            its.append({"bus": BUS_MEM, "sender": False, "mult": _col(KR),
                        "elems": [addr, lo(KA, i), hi(KA, i), _col(KTOLD + i)]})
            its.append({"bus": BUS_MEM, "sender": True, "mult": _col(KR + 23),
                        "elems": [addr, lo(KOUT, i), hi(KOUT, i), _col(KCLK)]})
        for j in range(50):
            its.append({"bus": BUS_RANGE, "sender": True, "mult": _col(KR), "elems": [_col(KTD + j)]})
        self._logup_setup(its)
        self.program = self._program(("keccak",))
        self.device_program = _hand_program(self, ("keccak-device",), 1)

    def _build_program(self):
        b = Builder()
        e = _Expr(b)
        M = lambda c: b.main(0, c)
        N = lambda c: b.main(1, c)
        one = e.one
        r = [M(KR + i) for i in range(24)]
        for f in r:
            e.boolean(f)
        e.boolean(e.total(r))
        C = [[M(KC + 64 * x + z) for z in range(64)] for x in range(5)]
        CP = [[M(KCP + 64 * x + z) for z in range(64)] for x in range(5)]
        AP = [[[M(KAP + 64 * _lane(x, y) + z) for z in range(64)] for y in range(5)] for x in range(5)]
        B00 = [M(KB00 + z) for z in range(64)]
        for x in range(5):
            for z in range(64):
                e.boolean(C[x][z])
                e.boolean(CP[x][z])
                for y in range(5):
                    e.boolean(AP[x][y][z])
        for z in range(64):
            e.boolean(B00[z])
        # theta
        two, four = b.const_base(2), b.const_base(4)
        for x in range(5):
            for z in range(64):
                b.emit(b.sub(CP[x][z], e.xor3(C[x][z], C[(x - 1) % 5][z], C[(x + 1) % 5][(z - 1) % 64])))
                t = b.sub(e.total([AP[x][y][z] for y in range(5)]), CP[x][z])
                b.emit(b.mul(b.mul(t, b.sub(t, two)), b.sub(t, four)))
        for x in range(5):  # the five lanes of a column share C[x][z] * C'[x][z]: y innermost
            for l in range(4):
                for y in range(5):
                    bits = [e.xor3(AP[x][y][z], C[x][z], CP[x][z]) for z in range(16 * l, 16 * l + 16)]
                    b.emit(b.sub(M(KA + 4 * _lane(x, y) + l), e.total([e.scaled(1 << i, v) for i, v in enumerate(bits)])))
        # rho and pi: Bm[y][2x + 3y] = rot(A'[x][y], r[x][y])
        Bm = [[None] * 5 for _ in range(5)]
        for x in range(5):
            for y in range(5):
                rr = KECCAK_ROT[x][y]
                Bm[y][(2 * x + 3 * y) % 5] = [AP[x][y][(z - rr) % 64] for z in range(64)]

        def chi(x, y, z):
            b0, b1, b2 = Bm[x][y][z], Bm[(x + 1) % 5][y][z], Bm[(x + 2) % 5][y][z]
            return e.xor2(b0, b.mul(b.sub(one, b1), b2))
        for x in range(5):
            for y in range(5):
                if (x, y) == (0, 0):
                    continue
                for l in range(4):
                    v = e.total([e.scaled(1 << i, chi(x, y, z)) for i, z in enumerate(range(16 * l, 16 * l + 16))])
                    b.emit(b.sub(M(KOUT + 4 * _lane(x, y) + l), v))
        for z in range(64):
            b.emit(b.sub(B00[z], chi(0, 0, z)))
        # iota on lane 0: the round constant's bit z is the sum of the flags whose constant has it
        for l in range(4):
            acc = []
            for i, z in enumerate(range(16 * l, 16 * l + 16)):
                fl = [r[ir] for ir in range(24) if (KECCAK_RC[ir] >> z) & 1]
                acc.append(e.scaled(1 << i, e.xor2(B00[z], e.total(fl)) if fl else B00[z]))
            b.emit(b.sub(M(KOUT + l), e.total(acc)))
        # transitions inside a permutation
        for i in range(23):
            b.emit(b.sub(N(KR + i + 1), r[i]))
        g = e.total(r[:23])
        for c in range(100):
            b.emit(b.mul(g, b.sub(N(KA + c), M(KOUT + c))))
        b.emit(b.mul(g, b.sub(N(KBASE), M(KBASE))))
        b.emit(b.mul(g, b.sub(N(KCLK), M(KCLK))))
        # reads are of earlier timestamps: KCLK - KTOLD_i - 1 = KTD_2i + 2^16 KTD_2i+1
        for i in range(25):
            gap = b.sub(b.sub(M(KCLK), M(KTOLD + i)), one)
            v = b.add(M(KTD + 2 * i), e.scaled(TWO16, M(KTD + 2 * i + 1)))
            b.emit(b.mul(r[0], b.sub(gap, v)))
        self._emit_logup(b)
        return b.program()

    def trace(self, clocks, bases, lanes, told):
        """One permutation per ecall: its timestamp, state address, the 25
        input lanes and the cells' previous timestamps (arrays, one row per
        ecall)."""
        n = self.n
        clk = np.asarray(clocks, np.uint64).reshape(-1)
        Pn = clk.size
        assert 24 * Pn <= n, "the permutations do not fit the table"
        t = np.zeros((n, KECCAK_WIDTH), np.uint64)
        if not Pn:
            return t
        sh = np.arange(64, dtype=np.uint64)
        bits = lambda v: (v[..., None] >> sh) & np.uint64(1)

        def rotl(v, k):
            k %= 64
            return v if k == 0 else (v << np.uint64(k)) | (v >> np.uint64(64 - k))

        a = np.asarray(lanes, np.uint64).reshape(Pn, 25)
        base = np.asarray(bases, np.uint64).reshape(-1)
        told = np.asarray(told, np.uint64).reshape(Pn, 25)
        rows0 = 24 * np.arange(Pn)
        for ir in range(24):
            rows = rows0 + ir
            t[rows, KR + ir] = 1
            t[rows, KBASE] = base
            t[rows, KCLK] = clk
            for l in range(4):
                t[rows, KA + l:KA + 100:4] = (a >> np.uint64(16 * l)) & np.uint64(0xFFFF)
            c = a[:, 0:5] ^ a[:, 5:10] ^ a[:, 10:15] ^ a[:, 15:20] ^ a[:, 20:25]
            d = np.stack([c[:, (x - 1) % 5] ^ rotl(c[:, (x + 1) % 5], 1) for x in range(5)], axis=1)
            ap = a ^ np.tile(d, (1, 5))
            t[rows, KC:KC + 320] = bits(c).reshape(Pn, 320)
            t[rows, KCP:KCP + 320] = bits(c ^ d).reshape(Pn, 320)
            t[rows, KAP:KAP + 1600] = bits(ap).reshape(Pn, 1600)
            bm = np.zeros_like(a)
            for x in range(5):
                for y in range(5):
                    bm[:, _lane(y, (2 * x + 3 * y) % 5)] = rotl(ap[:, _lane(x, y)], KECCAK_ROT[x][y])
            out = np.zeros_like(a)
            for x in range(5):
                for y in range(5):
                    out[:, _lane(x, y)] = bm[:, _lane(x, y)] ^ (~bm[:, _lane((x + 1) % 5, y)] &
                                                               bm[:, _lane((x + 2) % 5, y)])
            t[rows, KB00:KB00 + 64] = bits(out[:, 0])
            out[:, 0] ^= np.uint64(KECCAK_RC[ir])
            for l in range(4):
                t[rows, KOUT + l:KOUT + 100:4] = (out >> np.uint64(16 * l)) & np.uint64(0xFFFF)
            a = out
        t[rows0, KTOLD:KTOLD + 25] = told
        gap = clk[:, None] - told - np.uint64(1)
        t[rows0, KTD:KTD + 50:2] = gap & np.uint64(0xFFFF)
        t[rows0, KTD + 1:KTD + 50:2] = gap >> np.uint64(16)
        return t


# ---------------------------------------------------------------- statements
def statement_label(words, counts, output, heights=None):
    """Transcript label binding the public statement (program words, counts,
    output and, with chips beside the CPU table, the chips' heights) before
    any challenge is drawn."""
    from .math_cuda import keccak256
    blob = b"".join(int(w).to_bytes(4, "little") for w in words)
    blob += b"".join(int(c).to_bytes(8, "little") for c in counts)
    blob += int(output).to_bytes(8, "little")
    if heights and any(c in heights for c in CHIPS):
        blob += bytes(int(heights.get(c, 0)) for c in CHIPS)
    return b"lambda_vm_b200/rv64/" + keccak256(blob)


def chips_of(heights):
    return tuple(c for c in CHIPS if c in (heights or {}))


def airs_for(words, counts, heights=None):
    """The verifier's tables of a statement (it never executes the program):
    the CPU table has one row per counted instruction execution; the chips'
    heights (log2 rows) are part of the statement."""
    heights = heights or {}
    n = sum(int(c) for c in counts)
    assert n >= 2 and n & (n - 1) == 0, "the counts must cover a power-of-two table"
    chips = chips_of(heights)
    airs = [CpuAir(words, n.bit_length() - 1, chips), RangeAir()]
    if "bitwise" in chips:
        airs.append(BitwiseAir())
    if "shift" in chips:
        airs.append(ShiftAir(heights["shift"]))
    if "memory" in chips:
        airs.append(MemoryAir(heights["memory"]))
    if "keccak" in chips:
        airs.append(KeccakAir(heights["keccak"]))
    return airs


class Events:
    """What the tables need from a run, as arrays: row records (T x 8, as
    CpuAir.trace takes them), register snapshots (32 registers before every
    REG_CHUNK-th row of the CPU table), counts, a0, cycles, the chips used;
    shifts (dir, a, k); the touched cells (sorted addresses, final values,
    final timestamps); Keccak ecalls (timestamps, addresses, input lanes,
    previous timestamps)."""

    def __init__(self, records, regs, counts, output, cycles, chips, shifts, cells, keccak, range_counts=None,
                 bitwise_counts=None):
        self.records, self.regs, self.counts, self.output, self.cycles = records, regs, counts, output, cycles
        self.chips, self.shifts, self.cells, self.keccak = chips, shifts, cells, keccak
        # lookup multiplicities counted by the executor: the CPU and KECCAK
        # tables' RANGE lookups, the CPU table's BITWISE lookups (None: count
        # them from the records)
        self.range_counts, self.bitwise_counts = range_counts, bitwise_counts


def _chips_used(ops):
    used = {NEEDS[o] for o in ops if o in NEEDS}
    if "keccak" in ops:
        used |= {"keccak", "memory"}
    return tuple(c for c in CHIPS if c in used)


def python_events(words, max_steps=1 << 26):
    """Events of a run of the Python executor (rv64.run)."""
    ex = run(words, max_steps)
    rows = ex.rows
    T = len(rows)
    n = 1 << max(1, (T - 1).bit_length())
    kecc = {k[0] for k in ex.keccak}
    ops = [("keccak" if i in kecc else r_[1]) for i, r_ in enumerate(rows)]
    rec = np.zeros((T, 8), np.uint64)
    opid = np.array([KECCAK_OP if o == "keccak" else OP_ID[o] for o in ops], np.uint64)
    f = lambda i: np.array([r_[i] for r_ in rows], np.uint64)
    rec[:, 0] = f(0) | (opid << np.uint64(32)) | (f(2) << np.uint64(40)) | (f(3) << np.uint64(48)) | \
        (f(4) << np.uint64(56))
    rec[:, 1] = np.array([r_[5] for r_ in rows], np.int64).view(np.uint64)
    for i in range(2, 8):
        rec[:, i] = f(i + 4)
    # register snapshots: replay the writes
    regs = np.zeros(((n + REG_CHUNK - 1) // REG_CHUNK, 32), np.uint64)
    x = [0] * 32
    for t, r_ in enumerate(rows):
        if t % REG_CHUNK == 0:
            regs[t // REG_CHUNK] = x
        if r_[2] and ops[t] in WRITES:
            x[r_[2]] = r_[8]
    for c in range((T + REG_CHUNK - 1) // REG_CHUNK, regs.shape[0]):
        regs[c] = x
    pcs = f(0).astype(np.int64) // 4
    counts = np.bincount(pcs, minlength=len(words))
    counts[pcs[-1]] += n - T
    shifts = np.array([(1 if r_[1] == "srli" else 0, r_[6], r_[5]) for r_ in rows if r_[1] in ("slli", "srli")],
                      np.uint64).reshape(-1, 3)
    addrs = sorted(ex.memory)
    cells = (np.array(addrs, np.uint64), np.array([ex.memory[a_][0] for a_ in addrs], np.uint64),
             np.array([ex.memory[a_][1] for a_ in addrs], np.uint64))
    kc = (np.array([k[0] + 1 for k in ex.keccak], np.uint64), np.array([k[1] for k in ex.keccak], np.uint64),
          np.array([k[2] for k in ex.keccak], np.uint64).reshape(-1, 25),
          np.array([k[3] for k in ex.keccak], np.uint64).reshape(-1, 25))
    return Events(rec, regs, [int(c) for c in counts], ex.regs[10], T, _chips_used(set(ops)), shifts, cells, kc)


class CpuSource:
    """The CPU table of a run's row records and register snapshots: written
    on the device by the GPU backend (sg_rv64_cpu_table), built with numpy
    otherwise."""

    def __init__(self, records, regs):
        self.records = np.ascontiguousarray(records, np.uint64)
        self.regs = np.ascontiguousarray(regs, np.uint64)

    def host_trace(self, air):
        return air.trace(self.records)

    def device_trace(self, bk, air):
        from . import native
        m = bk._alloc(air.n, air.width)
        native.check(bk.L.sg_rv64_cpu_table(bk.be.h, bk.st, self.records.ctypes.data, self.records.shape[0],
                                            self.regs.ctypes.data, air.n, air.width, m.ptr))
        return m


class ShiftSource:
    """The SHIFT table of a run's shift events (dir, a, k): written on the
    device by the GPU backend (sg_rv64_shift_table), built with numpy
    otherwise."""

    def __init__(self, shifts):
        self.shifts = np.ascontiguousarray(np.asarray(shifts, np.uint64).reshape(-1, 3))

    def host_trace(self, air):
        return air.trace(self.shifts)

    def device_trace(self, bk, air):
        from . import native
        m = bk._alloc(air.n, air.width)
        native.check(bk.L.sg_rv64_shift_table(bk.be.h, bk.st, self.shifts.ctypes.data if self.shifts.size else None,
                                              self.shifts.shape[0], air.n, m.ptr))
        return m


class MemorySource:
    """The MEMORY table of a run's touched cells (address, final value, final
    timestamp; ascending addresses): written on the device by the GPU backend
    (sg_rv64_memory_table), built with numpy otherwise."""

    def __init__(self, addrs, values, stamps):
        self.cells = np.ascontiguousarray(np.stack([np.asarray(addrs, np.uint64), np.asarray(values, np.uint64),
                                                    np.asarray(stamps, np.uint64)], axis=1).reshape(-1, 3))

    def host_trace(self, air):
        c = self.cells
        return air.trace(c[:, 0], c[:, 1], c[:, 2])

    def device_trace(self, bk, air):
        from . import native
        m = bk._alloc(air.n, air.width)
        native.check(bk.L.sg_rv64_memory_table(bk.be.h, bk.st, self.cells.ctypes.data, self.cells.shape[0], air.n,
                                               m.ptr))
        return m

    def range_lookups(self, n):
        """The table's RANGE lookups at n rows: the D0 and D1 pieces of every
        row's address gap (zero from the last cell on)."""
        a = self.cells[:, 0]
        d = (a[1:] - a[:-1] - np.uint64(8)) >> np.uint64(3)
        return [d & np.uint64(0xFFFF), d >> np.uint64(16), np.zeros(2 * (n - a.size + 1), np.uint64)]


class KeccakSource:
    """The KECCAK table of a run's ecalls (timestamp, address, 25 input lanes,
    25 previous timestamps): written on the device by the GPU backend
    (sg_rv64_keccak_table), built with numpy otherwise."""

    def __init__(self, clocks, bases, lanes, told):
        clk = np.asarray(clocks, np.uint64).reshape(-1, 1)
        self.calls = np.ascontiguousarray(np.hstack([clk, np.asarray(bases, np.uint64).reshape(-1, 1),
                                                     np.asarray(lanes, np.uint64).reshape(-1, 25),
                                                     np.asarray(told, np.uint64).reshape(-1, 25)]))

    def host_trace(self, air):
        c = self.calls
        return air.trace(c[:, 0], c[:, 1], c[:, 2:27], c[:, 27:52])

    def device_trace(self, bk, air):
        from . import native
        m = bk._alloc(air.n, air.width)
        native.check(bk.L.sg_rv64_keccak_table(bk.be.h, bk.st, self.calls.ctypes.data if self.calls.size else None,
                                               self.calls.shape[0], air.n, m.ptr))
        return m

    def range_lookups(self):
        """The 16-bit pieces of each read's timestamp gap (the table's RANGE lookups)."""
        gap = self.calls[:, :1] - self.calls[:, 27:52] - np.uint64(1)
        return [gap & np.uint64(0xFFFF), gap >> np.uint64(16)]


def tables_from_events(words, ev, host_tables=False):
    """(airs, traces, public) of a run's events: public = {"words", "counts",
    "output", "cycles", "heights", "label", "terms"}. The CPU, SHIFT, MEMORY
    and KECCAK entries of traces are table sources the GPU backend writes on
    the device (stark._gen_trace), or numpy tables with host_tables."""
    rec = ev.records
    T = rec.shape[0]
    heights = {"cpu": max(1, (T - 1).bit_length()), "range": 16}
    n = 1 << heights["cpu"]
    if "bitwise" in ev.chips:
        heights["bitwise"] = 16
    if "shift" in ev.chips:
        heights["shift"] = _log2_rows(len(ev.shifts))
    if "memory" in ev.chips:
        heights["memory"] = _log2_rows(len(ev.cells[0]))
    if "keccak" in ev.chips:
        heights["keccak"] = _log2_rows(24 * len(ev.keccak[0]))
    chips = chips_of(heights)
    cpu = CpuAir(words, heights["cpu"], chips)
    csrc = CpuSource(rec, ev.regs)
    airs, traces = [cpu, RangeAir()], [csrc.host_trace(cpu) if host_tables else csrc, None]
    # the CPU's RANGE lookups: the result's four 16-bit pieces on every row
    # (rows past the halt repeat its zero result), the address and timestamp
    # pieces of memory rows
    counted = ev.range_counts is not None
    if counted:
        look = []
    else:
        op = ((rec[:, 0] >> np.uint64(32)) & np.uint64(0xFF)).astype(np.int64)
        look = [(rec[:, 4, None] >> np.arange(0, 64, 16, dtype=np.uint64)) & np.uint64(0xFFFF),
                np.zeros(4 * (n - T), np.uint64)]
    if "bitwise" in chips:
        a = BitwiseAir()
        airs.append(a)
        traces.append(a.trace(rec, ev.bitwise_counts))
    if "shift" in chips:
        a = ShiftAir(heights["shift"])
        src = ShiftSource(ev.shifts)
        airs.append(a)
        traces.append(src.host_trace(a) if host_tables else src)
    if "memory" in chips:
        a = MemoryAir(heights["memory"])
        src = MemorySource(*ev.cells)
        airs.append(a)
        traces.append(src.host_trace(a) if host_tables else src)
        if not counted:
            mem = np.isin(op, [OP_ID["ld"], OP_ID["sd"]])
            addr = mem | (op == KECCAK_OP)
            ma = rec[addr, 5]
            gap = np.nonzero(mem)[0].astype(np.uint64) - rec[mem, 7]   # (row + 1) - mt - 1
            look += [(ma >> np.uint64(3)) & np.uint64(0xFFFF), np.uint64(8) * (ma >> np.uint64(19)),
                     gap & np.uint64(0xFFFF), gap >> np.uint64(16)]
        look += src.range_lookups(a.n)
    if "keccak" in chips:
        a = KeccakAir(heights["keccak"])
        src = KeccakSource(*ev.keccak)
        airs.append(a)
        traces.append(src.host_trace(a) if host_tables else src)
        if not counted:
            look += src.range_lookups()
    traces[1] = airs[1].trace(look, ev.range_counts)
    pub = {"words": list(words), "counts": ev.counts, "output": ev.output, "cycles": ev.cycles,
           "heights": heights, "label": statement_label(words, ev.counts, ev.output, heights),
           "terms": cpu.public_terms(ev.counts, ev.output)}
    return airs, traces, pub


class _NativeTrace:
    """A run's outputs held by the library (sg_rv64_exec), freed with the last
    array that views them."""

    def __init__(self, L, handle):
        self.L, self.h = L, handle

    def __del__(self):
        if self.h:
            self.L.sg_rv64_trace_free(self.h)
            self.h = None

    def part(self, part, cols):
        """The part's words in place, as a (-1, cols) uint64 array that keeps this trace alive."""
        import ctypes as C
        from . import native
        p, n = C.c_void_p(), C.c_uint64()
        native.check(self.L.sg_rv64_trace_part(self.h, part, C.byref(p), C.byref(n)))
        if not n.value:
            return np.zeros((0, cols), np.uint64)
        return np.asarray(_View(self, p.value, (n.value // cols, cols)))


class _View:
    """Library memory as a numpy array's base: the array keeps `owner` alive."""

    def __init__(self, owner, ptr, shape):
        self.owner = owner
        self.__array_interface__ = {"shape": shape, "typestr": "<u8", "data": (ptr, False), "version": 3}


def native_events(words, max_steps=1 << 32):
    """Events of a run of the library's C++ executor, in one run (sg_rv64_exec:
    the outputs grow as the machine runs and are read in place)."""
    import ctypes as C
    from . import native
    L = native.lib()
    w = np.ascontiguousarray(np.asarray(words, dtype=np.uint32))
    info = native.Rv64Info()
    h = C.c_void_p()
    native.check(L.sg_rv64_exec(w.ctypes.data, len(w), max_steps, C.byref(h), C.byref(info)))
    tr = _NativeTrace(L, h)
    rec = tr.part(0, 8)
    regs = tr.part(1, 32)
    counts = tr.part(2, 1).reshape(-1)
    shifts = tr.part(3, 3)
    cells = tr.part(4, 3)
    kc = tr.part(5, 52)
    rcount = tr.part(6, 1).reshape(-1)
    bcount = tr.part(7, 1).reshape(-1)
    chips = tuple(c for i, c in enumerate(CHIPS) if info.chips >> i & 1)
    return Events(rec, regs, [int(c) for c in counts], info.a0, info.cycles, chips, shifts,
                  (cells[:, 0].copy(), cells[:, 1].copy(), cells[:, 2].copy()),
                  (kc[:, 0].copy(), kc[:, 1].copy(), kc[:, 2:27].copy(), kc[:, 27:52].copy()), rcount, bcount)


def native_events_two_runs(words, max_steps=1 << 32):
    """The same events from the caller-buffer entry: a run without outputs to
    size them, then sg_rv64_run_counted into them."""
    import ctypes as C
    from . import native
    L = native.lib()
    w = np.ascontiguousarray(np.asarray(words, dtype=np.uint32))
    info = native.Rv64Info()
    native.check(L.sg_rv64_run(w.ctypes.data, len(w), max_steps, 0, None, None, None, None, None, None,
                               C.byref(info)))
    n = 1 << max(1, (info.cycles - 1).bit_length())
    rec = np.empty((info.cycles, 8), np.uint64)
    regs = np.empty(((n + REG_CHUNK - 1) // REG_CHUNK, 32), np.uint64)
    counts = np.zeros(len(w), np.uint64)
    shifts = np.empty((info.shifts, 3), np.uint64)
    cells = np.empty((info.cells, 3), np.uint64)
    kc = np.empty((info.keccak_calls, 52), np.uint64)
    rcount = np.empty(1 << 16, np.uint64)
    bcount = np.empty(3 << 16, np.uint64)
    ptr = lambda a: a.ctypes.data if a.size else None
    native.check(L.sg_rv64_run_counted(w.ctypes.data, len(w), max_steps, n, rec.ctypes.data, regs.ctypes.data,
                                       counts.ctypes.data, ptr(shifts), ptr(cells), ptr(kc), rcount.ctypes.data,
                                       bcount.ctypes.data, C.byref(info)))
    chips = tuple(c for i, c in enumerate(CHIPS) if info.chips >> i & 1)
    return Events(rec, regs, [int(c) for c in counts], info.a0, info.cycles, chips, shifts,
                  (cells[:, 0].copy(), cells[:, 1].copy(), cells[:, 2].copy()),
                  (kc[:, 0].copy(), kc[:, 1].copy(), kc[:, 2:27].copy(), kc[:, 27:52].copy()), rcount, bcount)


def build(words, native_exec=True, host_tables=False):
    """Execute a program and build its tables (by default with the library's
    native executor; the SHIFT and KECCAK tables as device-written sources
    unless host_tables): (airs, traces, public)."""
    ev = native_events(words) if native_exec else python_events(words)
    return tables_from_events(words, ev, host_tables)


def prove(words, opts, bk):
    """Execute `words` and prove the execution on backend `bk` (stark.multi_prove,
    the plain per-table form): (proof, public statement)."""
    from .stark import multi_prove
    airs, traces, pub = build(words)
    proof = multi_prove(airs, traces, opts, bk, label=pub["label"])
    return proof, pub


def verify(words, counts, output, proof, opts, device=None, heights=None):
    """Verify that `words` run from the initial state halts with a0 = output,
    having executed each instruction counts[i] times, with the chips'
    heights of the statement: (ok, reason)."""
    from . import verifier
    try:
        airs = airs_for(words, counts, heights)
    except (AssertionError, ValueError, StopIteration) as e:
        return False, f"malformed statement: {e}"
    cpu = airs[0]
    return verifier.verify(airs, proof, opts, label=statement_label(words, counts, output, heights), device=device,
                           public_terms=cpu.public_terms(counts, output))
