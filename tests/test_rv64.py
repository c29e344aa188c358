"""The RV64 front-end on the CPU: encodings, execution of the Fibonacci and
Keccak guests (Python and the library's native executor, cell for cell), and
the AIRs of the CPU table and its chips — every constraint vanishes on the
rows of an honest trace and the buses balance with the public statement,
while a tampered trace or statement breaks a constraint or the balance."""
import numpy as np
import pytest

import oracle as O
from vm_eval import bad_constraints
from lambda_vm_b200 import rv64
from lambda_vm_b200 import rv64_air as RA
from lambda_vm_b200.verifier import public_sum

P = O.P


def test_encodings_round_trip():
    cases = [("add", 7, 5, 6, 0), ("sub", 1, 2, 3, 0), ("addi", 10, 10, 0, -1), ("addi", 5, 0, 0, 2047),
             ("lui", 10, 0, 0, -(1 << 31)), ("lui", 3, 0, 0, 0x7FFFF << 12), ("beq", 0, 1, 2, -4096),
             ("bne", 0, 10, 0, 4094), ("ecall", 0, 0, 0, 0), ("xor", 5, 6, 7, 0), ("or", 31, 1, 2, 0),
             ("and", 9, 10, 11, 0), ("xori", 5, 6, 0, -1), ("ori", 8, 9, 0, 2047), ("andi", 1, 2, 0, -2048),
             ("slli", 6, 5, 0, 13), ("slli", 6, 5, 0, 63), ("srli", 6, 5, 0, 7), ("srli", 6, 5, 0, 0),
             ("ld", 6, 8, 0, -8), ("ld", 6, 8, 0, 2040), ("sd", 0, 18, 6, -2048), ("sd", 0, 18, 6, 136)]
    for op, rd, rs1, rs2, imm in cases:
        w = rv64.encode(op, rd, rs1, rs2, imm >> 12 if op == "lui" else imm)
        assert rv64.decode(w) == (op, rd, rs1, rs2, imm)
    # standard encodings
    assert rv64.encode("addi", 10, 0, 0, 10) == 0x00A00513
    assert rv64.encode("add", 7, 5, 6) == 0x006283B3
    assert rv64.encode("ecall") == 0x00000073
    assert rv64.encode("xor", 10, 11, 12) == 0x00C5C533
    assert rv64.encode("slli", 5, 5, 0, 13) == 0x00D29293
    assert rv64.encode("srli", 5, 5, 0, 7) == 0x0072D293
    assert rv64.encode("ld", 10, 2, 0, 8) == 0x00813503
    assert rv64.encode("sd", 0, 2, 10, 8) == 0x00A13423
    with pytest.raises(ValueError):
        rv64.decode(0x4072D293)  # srai: not in the subset


@pytest.mark.parametrize("n", [1, 5, 300, 30000])
def test_fibonacci_guest_runs(n):
    rows, regs = rv64.execute(rv64.fib_program(n))
    assert regs[10] == rv64.fib_reference(n)
    assert rows[-1][1] == "ecall"
    # li, li, li (lui + addi above 2047), 5 per iteration, mv, li, ecall
    assert len(rows) == 2 + (1 if n < 2048 else 2) + 5 * n + 3


def test_keccak_f_known_answers():
    """keccak-f[1600] of the zero state (its first lane is the published
    0xF1258F7940E1DDE7), and Keccak-256 built on it as a sponge (rate 136,
    pad 0x01 .. 0x80) against the oracle's Keccak-256."""
    assert rv64.keccak_f([0] * 25)[0] == 0xF1258F7940E1DDE7
    rng = np.random.default_rng(5)
    for ln in (0, 1, 135, 136, 137, 300):
        msg = bytes(rng.integers(0, 256, ln, dtype=np.uint8))
        padded = bytearray(msg + b"\x01" + b"\0" * ((-len(msg) - 1) % 136))
        padded[-1] |= 0x80
        st = [0] * 25
        for off in range(0, len(padded), 136):
            blk = padded[off:off + 136]
            for i in range(17):
                st[i] ^= int.from_bytes(blk[8 * i:8 * i + 8], "little")
            st = rv64.keccak_f(st)
        digest = b"".join(v.to_bytes(8, "little") for v in st[:4])
        assert digest == O.keccak256(msg)


@pytest.mark.parametrize("blocks", [1, 3, 20])
def test_keccak_guest_runs(blocks):
    ex = rv64.run(rv64.keccak_program(136 * blocks))
    assert ex.regs[10] == rv64.keccak_reference(136 * blocks)
    assert len(ex.keccak) == blocks
    words = 17 * blocks
    # li buf (lui + addi), li count, li seed (lui + addi); 10 per word; li buf,
    # li count, li state, li acc (two words each but the count), li a7; 63 per
    # block; ld + 3 x (ld, xor); li a7, ecall
    assert len(ex.rows) == 5 + 10 * words + 8 + 63 * blocks + 7 + 2
    # every cell touched: the buffer, the 25 state lanes, the 4 accumulator lanes
    assert len(ex.memory) == words + 25 + 4


def test_executor_errors():
    bad_addr = rv64.assemble([("li", "t0", 4), ("ld", "t1", 0, "t0"), ("li", "a7", 93), ("ecall",)])
    with pytest.raises(ValueError, match="unaligned"):
        rv64.run(bad_addr)
    bad_call = rv64.assemble([("li", "a7", 7), ("ecall",)])
    with pytest.raises(ValueError, match="ecall"):
        rv64.run(bad_call)
    # the library's executor refuses the same programs
    for w in (bad_addr, bad_call):
        with pytest.raises(Exception):
            RA.native_events(w)


@pytest.mark.parametrize("prog", ["fib7", "fib2047", "fib5000", "keccak1", "keccak9", "wrap"])
def test_native_events_equal_the_python_events(prog):
    """sg_rv64_run (the library's C++ executor) against the Python executor:
    row records, register snapshots, counts, output, chips and every chip
    event; and the CPU table built from them. "wrap": a branch whose operands'
    low limbs are 2^32 - 1 and 0, the corner of the limb differences."""
    if prog == "wrap":
        words = rv64.assemble([("li", "t0", -1), ("srli", "t0", "t0", 32), ("li", "t1", 0),
                               ("beq", "t0", "t1", "end"), ("bne", "t0", "t1", "end"), ("li", "t1", 5),
                               "end:", ("li", "a7", 93), ("ecall",)])
    elif prog.startswith("fib"):
        words = rv64.fib_program(int(prog[3:]))
    else:
        words = rv64.keccak_program(136 * int(prog[6:]))
    pe, ne = RA.python_events(words), RA.native_events(words)
    assert np.array_equal(pe.records, ne.records)
    assert np.array_equal(pe.regs, ne.regs)
    assert (pe.counts, pe.output, pe.cycles, pe.chips) == (ne.counts, ne.output, ne.cycles, ne.chips)
    assert np.array_equal(pe.shifts, ne.shifts)
    for a, b in zip(pe.cells + pe.keccak, ne.cells + ne.keccak):
        assert np.array_equal(a, b)
    airs, traces, pub = RA.tables_from_events(words, ne, host_tables=True)
    # the executor's lookup counts give the same RANGE and BITWISE tables as
    # counting the records
    _, ptraces, ppub = RA.tables_from_events(words, pe, host_tables=True)
    assert len(traces) == len(ptraces) and all(np.array_equal(x, y) for x, y in zip(traces, ptraces))
    assert ppub["label"] == pub["label"]
    if prog == "wrap":
        bad, total = _check(airs, traces, pub)
        assert not any(bad.values()) and total == (0, 0, 0)
    else:
        assert airs[0].width == (RA.CPU_CORE_WIDTH if prog.startswith("fib") else RA.CPU_WIDTH)


@pytest.mark.parametrize("prog", ["fib1", "fib2047", "keccak1", "keccak9"])
def test_single_run_executor_equals_the_two_run_one(prog):
    """sg_rv64_exec (one run, outputs growing in library buffers read in
    place) against sg_rv64_run + sg_rv64_run_counted (a run to size the
    caller's arrays, then one to fill them): every output, word for word."""
    words = rv64.fib_program(int(prog[3:])) if prog.startswith("fib") else rv64.keccak_program(136 * int(prog[6:]))
    a, b = RA.native_events(words), RA.native_events_two_runs(words)
    assert np.array_equal(a.records, b.records) and np.array_equal(a.regs, b.regs)
    assert (a.counts, a.output, a.cycles, a.chips) == (b.counts, b.output, b.cycles, b.chips)
    assert np.array_equal(a.shifts, b.shifts)
    assert all(np.array_equal(x, y) for x, y in zip(a.cells + a.keccak, b.cells + b.keccak))
    assert np.array_equal(a.range_counts, b.range_counts) and np.array_equal(a.bitwise_counts, b.bitwise_counts)


def test_single_run_executor_errors():
    """sg_rv64_exec refuses what sg_rv64_run refuses, and an unknown part."""
    import ctypes as C
    from lambda_vm_b200 import native
    L = native.lib()
    bad = np.array(rv64.assemble([("li", "t0", 4), ("ld", "t1", 0, "t0"), ("li", "a7", 93), ("ecall",)]), np.uint32)
    info, h = native.Rv64Info(), C.c_void_p()
    assert L.sg_rv64_exec(bad.ctypes.data, len(bad), 1 << 20, C.byref(h), C.byref(info)) == native.SG_ERR_INVALID
    assert not h.value
    loop = np.array(rv64.assemble(["top:", ("beq", "zero", "zero", "top")]), np.uint32)
    assert L.sg_rv64_exec(loop.ctypes.data, len(loop), 1000, C.byref(h), C.byref(info)) == native.SG_ERR_INVALID
    ok = np.array(rv64.fib_program(3), np.uint32)
    assert L.sg_rv64_exec(ok.ctypes.data, len(ok), 1 << 20, C.byref(h), C.byref(info)) == native.SG_OK
    p, n = C.c_void_p(), C.c_uint64()
    assert L.sg_rv64_trace_part(h, 8, C.byref(p), C.byref(n)) == native.SG_ERR_INVALID
    assert L.sg_rv64_trace_part(h, 0, C.byref(p), C.byref(n)) == native.SG_OK and n.value == 8 * info.cycles
    L.sg_rv64_trace_free(h)


def _aux_and_apows(airs, z, alpha):
    apows = [(1, 0, 0)]
    for _ in range(max(a.max_alpha for a in airs) - 1):
        apows.append(tuple(int(v) for v in O.fp3_mul(np.array(apows[-1], np.uint64), np.array(alpha, np.uint64))))
    return apows


def _check(airs, traces, pub, rows_limit=256, terms=None):
    """(every table's failing (constraint, row) set, bus total with the public
    terms) under fixed challenges."""
    apows = _aux_and_apows(airs, Z, ALPHA)
    total = public_sum(pub["terms"] if terms is None else terms, Z, apows)
    bad = {}
    for air, tr in zip(airs, traces):
        aux, L = O.logup_aux(tr, air.logup_descriptor(), np.array(apows, np.uint64), np.array(Z, np.uint64))
        L = [int(v) for v in L]
        offset = [int(v) for v in O.fp3_mul(np.array(L, np.uint64), np.array([O.gl_inv(air.n), 0, 0], np.uint64))]
        rows = range(air.n) if air.n <= rows_limit else \
            list(range(rows_limit // 2)) + list(range(air.n - rows_limit // 2, air.n))
        bad[type(air).__name__] = bad_constraints(air.program, tr, aux, [Z, ALPHA], apows, offset, list(rows))
        total = tuple((total[i] + L[i]) % P for i in range(3))
    return bad, total


Z, ALPHA = (0x1234567, 0xABCDEF, 0x13579), (0x2468ACE, 0x1111, 0x777)


@pytest.mark.parametrize("prog", ["fib12", "keccak2"])
def test_honest_trace_satisfies_every_constraint_and_the_buses_balance(prog):
    words = rv64.fib_program(12) if prog == "fib12" else rv64.keccak_program(272)
    airs, traces, pub = RA.build(words, host_tables=True)
    bad, total = _check(airs, traces, pub)
    assert not any(bad.values()), {k: sorted(v)[:5] for k, v in bad.items() if v}
    assert total == (0, 0, 0)
    assert sum(pub["counts"]) == airs[0].n
    if prog == "keccak2":
        assert [type(a).__name__ for a in airs] == ["CpuAir", "RangeAir", "BitwiseAir", "ShiftAir", "MemoryAir",
                                                    "KeccakAir"]
        assert pub["output"] == rv64.keccak_reference(272)
    else:
        assert len(airs) == 2 and pub["output"] == rv64.fib_reference(12)


def _tampered(airs, traces, pub, table, fn, terms=None):
    trs = [t.copy() for t in traces]
    k = [type(a).__name__ for a in airs].index(table)
    fn(trs[k])
    bad, total = _check(airs, trs, pub, terms=terms)
    return any(bad.values()) or total != (0, 0, 0)


def test_tampering_breaks_a_constraint_or_the_balance():
    airs, traces, pub = RA.build(rv64.fib_program(6), host_tables=True)
    ct = traces[0]

    def reg(t):  # a register value changed mid-run
        t[9, RA.xlo(6)] = (int(t[9, RA.xlo(6)]) + 1) % P
    assert _tampered(airs, traces, pub, "CpuAir", reg)
    row = next(i for i in range(ct.shape[0]) if ct[i, RA.SEL["add"]] == 1)

    def add(t):  # an addition with a wrong result (range pieces adjusted)
        t[row, RA.R_LO] += 1
        t[row, RA.R16] += 1
    assert _tampered(airs, traces, pub, "CpuAir", add)

    def end(t):  # a second END row
        t[t.shape[0] // 2, RA.STEP] = 0
    assert _tampered(airs, traces, pub, "CpuAir", end)
    cpu = airs[0]
    # a different claimed output, or different execution counts
    assert _tampered(airs, traces, pub, "CpuAir", lambda t: None,
                     terms=cpu.public_terms(pub["counts"], pub["output"] + 1))
    counts = list(pub["counts"])
    counts[3] += 1
    counts[4] -= 1
    assert _tampered(airs, traces, pub, "CpuAir", lambda t: None, terms=cpu.public_terms(counts, pub["output"]))
    assert not _tampered(airs, traces, pub, "CpuAir", lambda t: None)


def test_tampered_chips_are_caught():
    """Each chip's own relation, and its link to the CPU table, is enforced:
    a flipped theta bit, a wrong Keccak output lane, a wrong shift result, a
    load returning a value that was never stored, a second row for one memory
    cell, a wrong XOR byte, a store whose previous timestamp is not earlier."""
    airs, traces, pub = RA.build(rv64.keccak_program(272), host_tables=True)
    ct = traces[0]
    assert not _tampered(airs, traces, pub, "CpuAir", lambda t: None)

    def theta(t):
        t[5, RA.KAP + 77] ^= 1
    assert _tampered(airs, traces, pub, "KeccakAir", theta)

    def out(t):
        t[23, RA.KOUT + 9] += 1
    assert _tampered(airs, traces, pub, "KeccakAir", out)

    def shift(t):
        t[0, RA.ShiftAir.R_LO] += 1
    assert _tampered(airs, traces, pub, "ShiftAir", shift)
    ld = next(i for i in range(ct.shape[0]) if ct[i, RA.SEL["ld"]] == 1 and ct[i, RA.MV_LO] < 1000)

    def load(t):  # value read, written to the register and range pieces all changed together
        for c in (RA.MV_LO, RA.NV_LO, RA.R_LO, RA.R16):
            t[ld, c] += 1
    assert _tampered(airs, traces, pub, "CpuAir", load)

    def dup(t):  # the second cell takes the first one's address
        t[1, RA.MemoryAir.ADDR] = t[0, RA.MemoryAir.ADDR]
    assert _tampered(airs, traces, pub, "MemoryAir", dup)
    xr = next(i for i in range(ct.shape[0]) if ct[i, RA.SEL["xor"]] == 1)

    def xor_byte(t):
        t[xr, RA.RB0] ^= 1
        t[xr, RA.R_LO] ^= 1
        t[xr, RA.R16] ^= 1
    assert _tampered(airs, traces, pub, "CpuAir", xor_byte)
    sd = next(i for i in range(ct.shape[0]) if ct[i, RA.SEL["sd"]] == 1 and ct[i, RA.MT] > 0)

    def stamp(t):  # claims the cell's previous access is this one's own timestamp
        t[sd, RA.MT] = t[sd, RA.CLK]
    assert _tampered(airs, traces, pub, "CpuAir", stamp)


def test_statement_binds_the_chip_heights():
    words = rv64.keccak_program(272)
    _, _, pub = RA.build(words)
    h = dict(pub["heights"])
    assert RA.statement_label(words, pub["counts"], pub["output"], h) == pub["label"]
    h["keccak"] += 1
    assert RA.statement_label(words, pub["counts"], pub["output"], h) != pub["label"]
    # the Fibonacci statement (no chips) keeps its label
    fw = rv64.fib_program(9)
    _, _, fp = RA.build(fw)
    assert fp["label"] == RA.statement_label(fw, fp["counts"], fp["output"])


def test_memory_source_range_lookups_are_the_table_gaps():
    """MemorySource.range_lookups (what RANGE counts for the MEMORY table
    when the table is written on the device) holds the values of the host
    table's D0 and D1 columns, row for row including padding."""
    ev = RA.native_events(rv64.keccak_program(136 * 3))
    src = RA.MemorySource(*ev.cells)
    for log_n in (RA._log2_rows(len(ev.cells[0])), RA._log2_rows(len(ev.cells[0])) + 2):
        air = RA.MemoryAir(log_n)
        t = src.host_trace(air)
        want = np.bincount(np.concatenate([t[:, air.D0], t[:, air.D1]]).astype(np.int64), minlength=1 << 16)
        got = np.bincount(np.concatenate(src.range_lookups(air.n)).astype(np.int64), minlength=1 << 16)
        assert np.array_equal(want, got)


def test_keccak_device_program_covers_the_logup_constraints():
    """The KECCAK table's device program: no nodes; the library's kernels
    evaluate its 3383 base constraints and, from the table's LogUp
    descriptor, its LogUp constraints, which follow them in the whole
    program (one per committed pair, then the accumulated column)."""
    from lambda_vm_b200.ir import lower
    air = RA.KeccakAir(6)
    full = air.program
    dev = lower(air.device_program)
    nb = full["num_base"]
    assert nb == 3383 and dev["hand_kernel"] == 1 and dev["hand_roots"] == nb
    assert dev["num_roots"] == len(full["roots"]) and len(dev["nodes"]) == 0
    assert dev["logup_root"] == nb and nb + air.num_committed + 1 == len(full["roots"])
    d = dev["logup_desc"]
    assert d["num_committed"] == air.num_committed and d["num_interactions"] in (2 * air.num_committed + 1,
                                                                                 2 * air.num_committed + 2)
    assert list(d["out_col_offsets"]) == [2 * c for c in range(air.num_committed + 1)] + [d["num_interactions"]]


def test_synthetic_device_program_leaves_logup_to_the_descriptor():
    """A synthetic chip table's device program walks its base constraint
    only; its LogUp constraints (indices 1..) come from its descriptor."""
    from lambda_vm_b200.air import SynthTableAir
    from lambda_vm_b200.ir import lower
    for k in (2, 4, 6):
        air = SynthTableAir(6, 12, num_interactions=k)
        dev = lower(air.device_program)
        assert dev["num_roots"] == len(air.program["roots"]) == 2 + air.num_committed
        assert sorted(int(c) for c in dev["node_roots"] if c != 0xFFFFFFFF) == [0]
        assert dev["logup_root"] == 1 and dev["logup_desc"]["num_committed"] == air.num_committed