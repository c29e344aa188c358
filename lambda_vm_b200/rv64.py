"""RV64 guest programs for the VM front-end: encoding, decoding, execution.

A subset of RV64I large enough for the Fibonacci guest of the benchmark
configuration (the shape of executor/programs/asm/fib_iterative_1M.s: an
add/mv/mv/addi/bnez loop): ADD, SUB, ADDI, LUI, BEQ, BNE and ECALL, which
halts the machine (exit, a7 = 93). Instructions are real RV64 machine words
(base ISA encodings: R, I, U, B formats); the executor decodes the words and
runs them (executor/src/vm semantics for these opcodes: 64-bit two's
complement registers, x0 hard-wired to zero, branch offsets relative to the
branch's pc) and records one row per executed instruction for the AIR in
rv64_air.py.
"""
import numpy as np

MASK64 = (1 << 64) - 1
OPS = ("add", "sub", "addi", "lui", "beq", "bne", "ecall")
OP_ID = {op: i + 1 for i, op in enumerate(OPS)}  # ids in the ROM tuple; 0 is never used
REG = {f"x{i}": i for i in range(32)}
REG.update({"zero": 0, "ra": 1, "sp": 2, "gp": 3, "tp": 4, "t0": 5, "t1": 6, "t2": 7, "s0": 8, "s1": 9, "a0": 10,
            "a1": 11, "a2": 12, "a3": 13, "a4": 14, "a5": 15, "a6": 16, "a7": 17})


def _bits(x, hi, lo):
    return (x >> lo) & ((1 << (hi - lo + 1)) - 1)


def _sext(x, bits):
    x &= (1 << bits) - 1
    return x - (1 << bits) if x >> (bits - 1) else x


def encode(op, rd=0, rs1=0, rs2=0, imm=0):
    """One RV64 instruction word."""
    if op in ("add", "sub"):
        f7 = 0x20 if op == "sub" else 0
        return (f7 << 25) | (rs2 << 20) | (rs1 << 15) | (0 << 12) | (rd << 7) | 0x33
    if op == "addi":
        assert -2048 <= imm < 2048, "addi immediate out of range"
        return ((imm & 0xFFF) << 20) | (rs1 << 15) | (0 << 12) | (rd << 7) | 0x13
    if op == "lui":
        assert -(1 << 19) <= imm < (1 << 19), "lui immediate out of range"
        return ((imm & 0xFFFFF) << 12) | (rd << 7) | 0x37
    if op in ("beq", "bne"):
        assert -4096 <= imm < 4096 and imm % 2 == 0, "branch offset out of range"
        u = imm & 0x1FFF
        f3 = 1 if op == "bne" else 0
        return ((_bits(u, 12, 12) << 31) | (_bits(u, 10, 5) << 25) | (rs2 << 20) | (rs1 << 15) | (f3 << 12) |
                (_bits(u, 4, 1) << 8) | (_bits(u, 11, 11) << 7) | 0x63)
    if op == "ecall":
        return 0x00000073
    raise ValueError(f"unsupported instruction {op}")


def decode(word):
    """(op, rd, rs1, rs2, imm) of a word of the supported subset; imm is the
    signed immediate (for lui: the sign-extended value imm20 << 12)."""
    opc, rd, f3, rs1, rs2, f7 = word & 0x7F, _bits(word, 11, 7), _bits(word, 14, 12), _bits(word, 19, 15), \
        _bits(word, 24, 20), _bits(word, 31, 25)
    if opc == 0x33 and f3 == 0 and f7 in (0, 0x20):
        return ("sub" if f7 else "add", rd, rs1, rs2, 0)
    if opc == 0x13 and f3 == 0:
        return ("addi", rd, rs1, 0, _sext(word >> 20, 12))
    if opc == 0x37:
        return ("lui", rd, 0, 0, _sext(word >> 12, 20) << 12)
    if opc == 0x63 and f3 in (0, 1):
        imm = (_bits(word, 31, 31) << 12) | (_bits(word, 7, 7) << 11) | (_bits(word, 30, 25) << 5) | \
            (_bits(word, 11, 8) << 1)
        return ("bne" if f3 else "beq", 0, rs1, rs2, _sext(imm, 13))
    if word == 0x00000073:
        return ("ecall", 0, 0, 0, 0)
    raise ValueError(f"unsupported instruction word {word:#010x}")


def assemble(lines):
    """Two-pass assembler over (op, operands...) tuples and "label:" strings;
    "li rd, imm" expands to addi or lui + addi, "mv rd, rs" to addi rd, rs, 0,
    "bnez rs, label" to bne rs, x0, label. Returns the instruction words."""
    items, labels = [], {}
    for ln in lines:
        if isinstance(ln, str) and ln.endswith(":"):
            labels[ln[:-1]] = 4 * len(items)
            continue
        op, *a = ln
        if op == "li":
            rd, v = REG[a[0]], a[1]
            if -2048 <= v < 2048:
                items.append(("addi", rd, 0, v))
            else:
                hi = (v + 0x800) >> 12
                items.append(("lui", rd, hi))
                items.append(("addi", rd, rd, v - (hi << 12)))
        elif op == "mv":
            items.append(("addi", REG[a[0]], REG[a[1]], 0))
        elif op == "bnez":
            items.append(("bne", REG[a[0]], 0, a[1]))
        elif op in ("add", "sub"):
            items.append((op, REG[a[0]], REG[a[1]], REG[a[2]]))
        elif op == "addi":
            items.append((op, REG[a[0]], REG[a[1]], a[2]))
        elif op in ("beq", "bne"):
            items.append((op, REG[a[0]], REG[a[1]], a[2]))
        elif op == "ecall":
            items.append(("ecall",))
        else:
            raise ValueError(f"unsupported mnemonic {op}")
    words = []
    for i, it in enumerate(items):
        op = it[0]
        if op in ("add", "sub"):
            words.append(encode(op, rd=it[1], rs1=it[2], rs2=it[3]))
        elif op == "addi":
            words.append(encode(op, rd=it[1], rs1=it[2], imm=it[3]))
        elif op == "lui":
            words.append(encode(op, rd=it[1], imm=it[2]))
        elif op in ("beq", "bne"):
            target = labels[it[3]] if isinstance(it[3], str) else it[3]
            words.append(encode(op, rs1=it[1], rs2=it[2], imm=target - 4 * i))
        else:
            words.append(encode("ecall"))
    return words


def fib_program(n):
    """The Fibonacci guest: fib(n+1) mod 2^64 by n >= 1 loop iterations of
    add / mv / mv / addi / bnez, left in a0, then exit (a7 = 93)."""
    assert n >= 1, "the loop runs at least once"
    return assemble([
        ("li", "t0", 0), ("li", "t1", 1), ("li", "a0", n),
        "loop:",
        ("add", "t2", "t0", "t1"), ("mv", "t0", "t1"), ("mv", "t1", "t2"), ("addi", "a0", "a0", -1),
        ("bnez", "a0", "loop"),
        ("mv", "a0", "t1"), ("li", "a7", 93), ("ecall",),
    ])


def fib_reference(n):
    a, b = 0, 1
    for _ in range(n):
        a, b = b, (a + b) & MASK64
    return b


def execute(words, max_steps=1 << 26):
    """Run from pc 0 until ECALL with a7 = 93. Returns (rows, regs): one row
    per executed instruction, (pc, op, rd, rs1, rs2, imm, a, b, r), a and b the
    source values, r the value written (0 when nothing is written)."""
    prog = [decode(w) for w in words]
    x = [0] * 32
    pc = 0
    rows = []
    for _ in range(max_steps):
        if pc % 4 or not 0 <= pc // 4 < len(prog):
            raise ValueError(f"pc {pc:#x} outside the program")
        op, rd, rs1, rs2, imm = prog[pc // 4]
        a, b = x[rs1], x[rs2]
        r, npc = 0, pc + 4
        if op == "add":
            r = (a + b) & MASK64
        elif op == "sub":
            r = (a - b) & MASK64
        elif op == "addi":
            r = (a + imm) & MASK64
        elif op == "lui":
            r = imm & MASK64
        elif op == "beq":
            npc = pc + imm if a == b else pc + 4
        elif op == "bne":
            npc = pc + imm if a != b else pc + 4
        elif op == "ecall":
            if x[17] != 93:
                raise ValueError("only the exit ecall (a7 = 93) is supported")
            rows.append((pc, op, rd, rs1, rs2, imm, a, b, 0))
            return rows, x
        rows.append((pc, op, rd, rs1, rs2, imm, a, b, r))
        if rd and op in ("add", "sub", "addi", "lui"):
            x[rd] = r
        pc = npc
    raise ValueError("the program did not halt")
