"""The RV64 front-end on the CPU: encodings, execution of the Fibonacci guest,
and the CPU and RANGE table AIRs — every constraint vanishes on every row of
an honest trace and the buses balance with the public statement, while a
tampered trace or statement breaks a constraint or the balance."""
import numpy as np
import pytest

import oracle as O
from oracle.stark_backend import eval_program_row
from lambda_vm_b200 import rv64
from lambda_vm_b200 import rv64_air as RA
from lambda_vm_b200.verifier import public_sum

P = O.P


def test_encodings_round_trip():
    cases = [("add", 7, 5, 6, 0), ("sub", 1, 2, 3, 0), ("addi", 10, 10, 0, -1), ("addi", 5, 0, 0, 2047),
             ("lui", 10, 0, 0, -(1 << 31)), ("lui", 3, 0, 0, 0x7FFFF << 12), ("beq", 0, 1, 2, -4096),
             ("bne", 0, 10, 0, 4094), ("ecall", 0, 0, 0, 0)]
    for op, rd, rs1, rs2, imm in cases:
        w = rv64.encode(op, rd, rs1, rs2, imm >> 12 if op == "lui" else imm)
        assert rv64.decode(w) == (op, rd, rs1, rs2, imm)
    # standard encodings of the guest's first instructions
    assert rv64.encode("addi", 10, 0, 0, 10) == 0x00A00513
    assert rv64.encode("add", 7, 5, 6) == 0x006283B3
    assert rv64.encode("ecall") == 0x00000073


@pytest.mark.parametrize("n", [1, 5, 300, 30000])
def test_fibonacci_guest_runs(n):
    rows, regs = rv64.execute(rv64.fib_program(n))
    assert regs[10] == rv64.fib_reference(n)
    assert rows[-1][1] == "ecall"
    # li, li, li (lui + addi above 2047), 5 per iteration, mv, li, ecall
    assert len(rows) == 2 + (1 if n < 2048 else 2) + 5 * n + 3


@pytest.mark.parametrize("n", [1, 7, 30, 2047, 2048, 5000])
def test_native_trace_equals_the_python_table(n):
    """sg_rv64_trace (the library's C++ executor and table writer) against the
    Python executor and table builder, cell for cell."""
    words = rv64.fib_program(n)
    rows, regs = rv64.execute(words)
    ct, counts, out, cycles = RA.native_trace(words)
    cpu = RA.CpuAir(words, ct.shape[0].bit_length() - 1)
    assert cycles == len(rows) and out == regs[10]
    assert np.array_equal(ct, cpu.trace(rows))
    assert counts == cpu.counts(rows)


def _aux_and_apows(airs, z, alpha):
    apows = [(1, 0, 0)]
    for _ in range(max(a.max_alpha for a in airs) - 1):
        apows.append(tuple(int(v) for v in O.fp3_mul(np.array(apows[-1], np.uint64), np.array(alpha, np.uint64))))
    return apows


def _bad_roots(air, tr, z, alpha, apows, rows=None):
    aux, L = O.logup_aux(tr, air.logup_descriptor(), np.array(apows, np.uint64), np.array(z, np.uint64))
    L = [int(v) for v in L]
    offset = [int(v) for v in O.fp3_mul(np.array(L, np.uint64), np.array([O.gl_inv(air.n), 0, 0], np.uint64))]
    bad = set()
    for r in (range(air.n) if rows is None else rows):
        vals = eval_program_row(air.program, r, tr, aux, [z, alpha], apows, offset, 1)
        bad |= {(ci, r) for ci, v in enumerate(vals) if any(int(x) % P for x in v)}
    return bad, L


Z, ALPHA = (0x1234567, 0xABCDEF, 0x13579), (0x2468ACE, 0x1111, 0x777)


def test_honest_trace_satisfies_every_constraint_and_the_buses_balance():
    airs, traces, pub = RA.build(rv64.fib_program(12))
    apows = _aux_and_apows(airs, Z, ALPHA)
    total = public_sum(pub["terms"], Z, apows)
    for air, tr in zip(airs, traces):
        rows = None if air.n <= 128 else list(range(64)) + list(range(air.n - 64, air.n))
        bad, L = _bad_roots(air, tr, Z, ALPHA, apows, rows)
        assert not bad, (type(air).__name__, sorted(bad)[:5])
        total = tuple((total[i] + L[i]) % P for i in range(3))
    assert total == (0, 0, 0)
    assert pub["output"] == rv64.fib_reference(12)
    assert sum(pub["counts"]) == airs[0].n


def test_tampering_breaks_a_constraint_or_the_balance():
    airs, traces, pub = RA.build(rv64.fib_program(6))
    cpu, ct = airs[0], traces[0]
    apows = _aux_and_apows(airs, Z, ALPHA)
    # a register value changed mid-run
    bad_tr = ct.copy()
    bad_tr[9, RA.xlo(6)] = (int(bad_tr[9, RA.xlo(6)]) + 1) % P
    assert _bad_roots(cpu, bad_tr, Z, ALPHA, apows)[0]
    # an addition with a wrong result (and its range pieces adjusted)
    row = next(i for i in range(cpu.n) if ct[i, RA.SEL["add"]] == 1)
    bad_tr = ct.copy()
    bad_tr[row, RA.R_LO] = int(bad_tr[row, RA.R_LO]) + 1
    bad_tr[row, RA.R16] = int(bad_tr[row, RA.R16]) + 1
    assert _bad_roots(cpu, bad_tr, Z, ALPHA, apows)[0]
    # a second END row
    bad_tr = ct.copy()
    bad_tr[cpu.n // 2, RA.STEP] = 0
    assert _bad_roots(cpu, bad_tr, Z, ALPHA, apows)[0]
    # a different claimed output: the END bus no longer balances
    _, L0 = _bad_roots(cpu, ct, Z, ALPHA, apows)
    _, L1 = _bad_roots(airs[1], traces[1], Z, ALPHA, apows, rows=[0])
    for out in (pub["output"] + 1,):
        ps = public_sum(cpu.public_terms(pub["counts"], out), Z, apows)
        assert tuple((L0[i] + L1[i] + ps[i]) % P for i in range(3)) != (0, 0, 0)
    # different execution counts: the ROM bus no longer balances
    counts = list(pub["counts"])
    counts[3] += 1
    counts[4] -= 1
    ps = public_sum(cpu.public_terms(counts, pub["output"]), Z, apows)
    assert tuple((L0[i] + L1[i] + ps[i]) % P for i in range(3)) != (0, 0, 0)
