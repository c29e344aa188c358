"""RV64 guest programs for the VM front-end: encoding, decoding, execution.

A subset of RV64I large enough for the two benchmark guests: the Fibonacci
guest (the shape of executor/programs/asm/fib_iterative_1M.s: an
add/mv/mv/addi/bnez loop) and the Keccak guest (a buffer filled by a
xorshift64 generator, hashed block by block through the Keccak ecall, the
digests XOR-folded with load/store loops). Instructions: ADD, SUB, XOR, OR,
AND, ADDI, XORI, ORI, ANDI, SLLI, SRLI, LUI, LD, SD, BEQ, BNE and ECALL. ECALL
with a7 = 93 halts the machine (exit); with a7 = 2^64 - 2 it applies
keccak-f[1600] to the 25 little-endian 64-bit lanes at address a0
(executor/src/vm/instruction/execution.rs:649-670, KECCAK_SYSCALL_NUMBER at
:53). Instructions are real RV64 machine words (base ISA encodings: R, I, S,
U, B formats); the executor decodes the words and runs them (executor/src/vm
semantics for these opcodes: 64-bit two's complement registers, x0
hard-wired to zero, branch offsets relative to the branch's pc, doubleword
loads and stores at 8-byte-aligned addresses) and records one row per
executed instruction for the AIRs in rv64_air.py. Data memory starts zeroed;
the data space is the low 4 GiB.
"""
import numpy as np

MASK64 = (1 << 64) - 1
OPS = ("add", "sub", "addi", "lui", "beq", "bne", "ecall", "xor", "or", "and", "xori", "ori", "andi", "slli",
       "srli", "ld", "sd")
OP_ID = {op: i + 1 for i, op in enumerate(OPS)}  # ids in the ROM tuple; 0 is never used
EXIT, KECCAK = 93, MASK64 - 1                     # ecall numbers (a7)
REG = {f"x{i}": i for i in range(32)}
REG.update({"zero": 0, "ra": 1, "sp": 2, "gp": 3, "tp": 4, "t0": 5, "t1": 6, "t2": 7, "s0": 8, "s1": 9, "a0": 10,
            "a1": 11, "a2": 12, "a3": 13, "a4": 14, "a5": 15, "a6": 16, "a7": 17, "s2": 18, "s3": 19, "s4": 20,
            "s5": 21, "s6": 22, "s7": 23, "s8": 24, "s9": 25, "s10": 26, "s11": 27, "t3": 28, "t4": 29, "t5": 30,
            "t6": 31})
R_F3 = {"add": (0, 0), "sub": (0, 0x20), "xor": (4, 0), "or": (6, 0), "and": (7, 0)}
I_F3 = {"addi": 0, "xori": 4, "ori": 6, "andi": 7}


def _bits(x, hi, lo):
    return (x >> lo) & ((1 << (hi - lo + 1)) - 1)


def _sext(x, bits):
    x &= (1 << bits) - 1
    return x - (1 << bits) if x >> (bits - 1) else x


def encode(op, rd=0, rs1=0, rs2=0, imm=0):
    """One RV64 instruction word (for lui, imm is the 20-bit upper immediate;
    for slli / srli the shift amount)."""
    if op in R_F3:
        f3, f7 = R_F3[op]
        return (f7 << 25) | (rs2 << 20) | (rs1 << 15) | (f3 << 12) | (rd << 7) | 0x33
    if op in I_F3:
        assert -2048 <= imm < 2048, f"{op} immediate out of range"
        return ((imm & 0xFFF) << 20) | (rs1 << 15) | (I_F3[op] << 12) | (rd << 7) | 0x13
    if op in ("slli", "srli"):
        assert 0 <= imm < 64, "shift amount out of range"
        return (imm << 20) | (rs1 << 15) | ((1 if op == "slli" else 5) << 12) | (rd << 7) | 0x13
    if op == "ld":
        assert -2048 <= imm < 2048, "load offset out of range"
        return ((imm & 0xFFF) << 20) | (rs1 << 15) | (3 << 12) | (rd << 7) | 0x03
    if op == "sd":
        assert -2048 <= imm < 2048, "store offset out of range"
        u = imm & 0xFFF
        return (_bits(u, 11, 5) << 25) | (rs2 << 20) | (rs1 << 15) | (3 << 12) | (_bits(u, 4, 0) << 7) | 0x23
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
    signed immediate (for lui: the sign-extended value imm20 << 12; for the
    shifts: the shift amount). Fields an instruction does not use are 0."""
    opc, rd, f3, rs1, rs2, f7 = word & 0x7F, _bits(word, 11, 7), _bits(word, 14, 12), _bits(word, 19, 15), \
        _bits(word, 24, 20), _bits(word, 31, 25)
    if opc == 0x33:
        for op, (g3, g7) in R_F3.items():
            if (f3, f7) == (g3, g7):
                return (op, rd, rs1, rs2, 0)
    elif opc == 0x13:
        if f3 in (1, 5):
            if _bits(word, 31, 26) == 0:
                return ("slli" if f3 == 1 else "srli", rd, rs1, 0, _bits(word, 25, 20))
        else:
            for op, g3 in I_F3.items():
                if f3 == g3:
                    return (op, rd, rs1, 0, _sext(word >> 20, 12))
    elif opc == 0x03 and f3 == 3:
        return ("ld", rd, rs1, 0, _sext(word >> 20, 12))
    elif opc == 0x23 and f3 == 3:
        return ("sd", 0, rs1, rs2, _sext((f7 << 5) | rd, 12))
    elif opc == 0x37:
        return ("lui", rd, 0, 0, _sext(word >> 12, 20) << 12)
    elif opc == 0x63 and f3 in (0, 1):
        imm = (_bits(word, 31, 31) << 12) | (_bits(word, 7, 7) << 11) | (_bits(word, 30, 25) << 5) | \
            (_bits(word, 11, 8) << 1)
        return ("bne" if f3 else "beq", 0, rs1, rs2, _sext(imm, 13))
    elif word == 0x00000073:
        return ("ecall", 0, 0, 0, 0)
    raise ValueError(f"unsupported instruction word {word:#010x}")


def assemble(lines):
    """Two-pass assembler over (op, operands...) tuples and "label:" strings.
    Pseudo-instructions: "li rd, imm" (addi, or lui + addi, for 32-bit
    values), "mv rd, rs" (addi rd, rs, 0), "bnez rs, label" (bne rs, x0).
    Loads and stores take (rd|rs2, offset, base). Returns the words."""
    items, labels = [], {}
    for ln in lines:
        if isinstance(ln, str) and ln.endswith(":"):
            labels[ln[:-1]] = 4 * len(items)
            continue
        op, *a = ln
        if op == "li":
            rd, v = REG[a[0]], a[1]
            assert -(1 << 31) <= v < (1 << 31), "li takes a 32-bit signed value"
            if -2048 <= v < 2048:
                items.append(("addi", rd, 0, 0, v))
            else:
                hi = (v + 0x800) >> 12
                items.append(("lui", rd, 0, 0, hi))
                items.append(("addi", rd, rd, 0, v - (hi << 12)))
        elif op == "mv":
            items.append(("addi", REG[a[0]], REG[a[1]], 0, 0))
        elif op == "bnez":
            items.append(("bne", 0, REG[a[0]], 0, a[1]))
        elif op in R_F3:
            items.append((op, REG[a[0]], REG[a[1]], REG[a[2]], 0))
        elif op in I_F3 or op in ("slli", "srli"):
            items.append((op, REG[a[0]], REG[a[1]], 0, a[2]))
        elif op == "ld":
            items.append((op, REG[a[0]], REG[a[2]], 0, a[1]))
        elif op == "sd":
            items.append((op, 0, REG[a[2]], REG[a[0]], a[1]))
        elif op in ("beq", "bne"):
            items.append((op, 0, REG[a[0]], REG[a[1]], a[2]))
        elif op == "ecall":
            items.append(("ecall", 0, 0, 0, 0))
        else:
            raise ValueError(f"unsupported mnemonic {op}")
    words = []
    for i, (op, rd, rs1, rs2, imm) in enumerate(items):
        if op in ("beq", "bne"):
            imm = (labels[imm] if isinstance(imm, str) else imm) - 4 * i
        words.append(encode(op, rd=rd, rs1=rs1, rs2=rs2, imm=imm))
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


# ------------------------------------------------------------------ Keccak-f[1600]
def _keccak_constants():
    """Round constants and rotation offsets of keccak-f[1600], derived from
    their definitions in FIPS 202 (the rc(t) LFSR of x^8 + x^6 + x^5 + x^4 + 1
    for iota, the (x, y) -> (y, 2x + 3y) walk for rho)."""
    def rc_bit(t):
        if t % 255 == 0:
            return 1
        r = 1
        for _ in range(t % 255):
            r <<= 1
            if r & 0x100:
                r ^= 0x171
        return r & 1
    rcs = []
    for ir in range(24):
        c = 0
        for j in range(7):
            c |= rc_bit(j + 7 * ir) << ((1 << j) - 1)
        rcs.append(c)
    rot = [[0] * 5 for _ in range(5)]
    x, y = 1, 0
    for t in range(24):
        rot[x][y] = ((t + 1) * (t + 2) // 2) % 64
        x, y = y, (2 * x + 3 * y) % 5
    return rcs, rot


KECCAK_RC, KECCAK_ROT = _keccak_constants()


def _rotl(v, r):
    return ((v << r) | (v >> (64 - r))) & MASK64 if r else v


def keccak_round(a, ir):
    """One round on lanes a[x + 5y] (ints); returns the new lanes."""
    c = [a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20] for x in range(5)]
    d = [c[(x - 1) % 5] ^ _rotl(c[(x + 1) % 5], 1) for x in range(5)]
    ap = [a[i] ^ d[i % 5] for i in range(25)]
    bb = [0] * 25
    for x in range(5):
        for y in range(5):
            bb[y + 5 * ((2 * x + 3 * y) % 5)] = _rotl(ap[x + 5 * y], KECCAK_ROT[x][y])
    out = [bb[i] ^ (~bb[(i % 5 + 1) % 5 + 5 * (i // 5)] & bb[(i % 5 + 2) % 5 + 5 * (i // 5)] & MASK64)
           for i in range(25)]
    out[0] ^= KECCAK_RC[ir]
    return out


def keccak_f(lanes):
    a = list(lanes)
    for ir in range(24):
        a = keccak_round(a, ir)
    return a


# ------------------------------------------------------------------ execution
class Execution:
    """What a run records for the tables. rows: one per executed instruction,
    (pc, op, rd, rs1, rs2, imm, a, b, r, ma, mv, mt): a and b the source
    values, r the value written (0 when nothing is written); for ld / sd: ma
    the address, mv the value the cell held and mt the timestamp of its last
    access (0 for the initial zero); for a Keccak ecall: ma the state address.
    Row t has timestamp t + 1. keccak: per Keccak ecall (row, address, input
    lanes, previous timestamps of the 25 cells). memory: final {address:
    (value, timestamp)} of every cell touched. regs: the final registers."""

    def __init__(self):
        self.rows, self.keccak, self.memory, self.regs = [], [], {}, None


def run(words, max_steps=1 << 26):
    """Run from pc 0 until ECALL with a7 = 93: an Execution."""
    prog = [decode(w) for w in words]
    x = [0] * 32
    pc = 0
    ex = Execution()
    mem = ex.memory

    def cell(addr):
        if addr % 8 or addr >= 1 << 32:
            raise ValueError(f"address {addr:#x} unaligned or outside the data space")
        return mem.get(addr, (0, 0))

    for t in range(max_steps):
        if pc % 4 or not 0 <= pc // 4 < len(prog):
            raise ValueError(f"pc {pc:#x} outside the program")
        op, rd, rs1, rs2, imm = prog[pc // 4]
        a, b = x[rs1], x[rs2]
        r, npc, ma, mv, mt = 0, pc + 4, 0, 0, 0
        clk = t + 1
        if op == "add":
            r = (a + b) & MASK64
        elif op == "sub":
            r = (a - b) & MASK64
        elif op == "xor":
            r = a ^ b
        elif op == "or":
            r = a | b
        elif op == "and":
            r = a & b
        elif op == "addi":
            r = (a + imm) & MASK64
        elif op == "xori":
            r = a ^ (imm & MASK64)
        elif op == "ori":
            r = a | (imm & MASK64)
        elif op == "andi":
            r = a & (imm & MASK64)
        elif op == "slli":
            r = (a << imm) & MASK64
        elif op == "srli":
            r = a >> imm
        elif op == "lui":
            r = imm & MASK64
        elif op in ("ld", "sd"):
            ma = (a + imm) & MASK64
            mv, mt = cell(ma)
            if op == "ld":
                r = mv
                mem[ma] = (mv, clk)
            else:
                mem[ma] = (b, clk)
        elif op == "beq":
            npc = pc + imm if a == b else pc + 4
        elif op == "bne":
            npc = pc + imm if a != b else pc + 4
        elif op == "ecall":
            if x[17] == EXIT:
                ex.rows.append((pc, op, rd, rs1, rs2, imm, a, b, 0, 0, 0, 0))
                ex.regs = x
                return ex
            if x[17] != KECCAK:
                raise ValueError(f"unsupported ecall a7 = {x[17]:#x}")
            ma = x[10]
            cells = [cell(ma + 8 * i) for i in range(25)]
            out = keccak_f([v for v, _ in cells])
            ex.keccak.append((t, ma, [v for v, _ in cells], [ts for _, ts in cells]))
            for i in range(25):
                mem[ma + 8 * i] = (out[i], clk)
        ex.rows.append((pc, op, rd, rs1, rs2, imm, a, b, r, ma, mv, mt))
        if rd and op not in ("beq", "bne", "ecall", "sd"):
            x[rd] = r
        pc = npc
    raise ValueError("the program did not halt")


def execute(words, max_steps=1 << 26):
    """(rows, final registers) of a run (see Execution)."""
    ex = run(words, max_steps)
    return ex.rows, ex.regs


# ------------------------------------------------------------------ the Keccak guest
def keccak_program(buf_bytes, seed=0x9E3779B97F4A7C15 & 0x7FFFFFFF):
    """The Keccak guest: fill a buffer of buf_bytes (a multiple of 136) from a
    xorshift64 generator (x ^= x << 13; x ^= x >> 7; x ^= x << 17), then per
    136-byte block: zero a 25-lane state, copy the block into its first 17
    lanes, apply keccak-f[1600] through the ecall, and XOR-fold the 4-lane
    digest into an accumulator with load / xor / store; a0 = the XOR of the
    accumulator's 4 lanes. The seed is a nonzero 31-bit value."""
    assert buf_bytes > 0 and buf_bytes % 136 == 0, "the buffer is whole 136-byte blocks"
    assert 0 < seed < (1 << 31)
    BUF, STATE, ACC = 0x10000, 0x8000, 0x9000
    nwords, nblocks = buf_bytes // 8, buf_bytes // 136
    prog = [("li", "s0", BUF), ("li", "s1", nwords), ("li", "t0", seed),
            "fill:",
            ("slli", "t1", "t0", 13), ("xor", "t0", "t0", "t1"),
            ("srli", "t1", "t0", 7), ("xor", "t0", "t0", "t1"),
            ("slli", "t1", "t0", 17), ("xor", "t0", "t0", "t1"),
            ("sd", "t0", 0, "s0"), ("addi", "s0", "s0", 8), ("addi", "s1", "s1", -1), ("bnez", "s1", "fill"),
            ("li", "s0", BUF), ("li", "s1", nblocks), ("li", "s2", STATE), ("li", "s3", ACC),
            ("li", "a7", -2),
            "block:"]
    prog += [("sd", "zero", 8 * j, "s2") for j in range(17, 25)]
    for j in range(17):
        prog += [("ld", "t1", 8 * j, "s0"), ("sd", "t1", 8 * j, "s2")]
    prog += [("mv", "a0", "s2"), ("ecall",)]
    for j in range(4):
        prog += [("ld", "t1", 8 * j, "s2"), ("ld", "t2", 8 * j, "s3"), ("xor", "t1", "t1", "t2"),
                 ("sd", "t1", 8 * j, "s3")]
    prog += [("addi", "s0", "s0", 136), ("addi", "s1", "s1", -1), ("bnez", "s1", "block"),
             ("ld", "a0", 0, "s3")]
    for j in range(1, 4):
        prog += [("ld", "t1", 8 * j, "s3"), ("xor", "a0", "a0", "t1")]
    prog += [("li", "a7", 93), ("ecall",)]
    return assemble(prog)


def keccak_reference(buf_bytes, seed=0x9E3779B97F4A7C15 & 0x7FFFFFFF):
    """a0 of keccak_program, computed directly."""
    x, words = seed, []
    for _ in range(buf_bytes // 8):
        x ^= (x << 13) & MASK64
        x ^= x >> 7
        x ^= (x << 17) & MASK64
        words.append(x)
    acc = [0] * 4
    for blk in range(buf_bytes // 136):
        st = keccak_f(words[17 * blk:17 * blk + 17] + [0] * 8)
        acc = [acc[j] ^ st[j] for j in range(4)]
    return acc[0] ^ acc[1] ^ acc[2] ^ acc[3]
