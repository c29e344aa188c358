"""The RV64 front-end proved on the GPU: the Fibonacci guest's execution
(CPU table + 16-bit RANGE table) proved by the library's prover, accepted by
the library's verifier (host and GPU query phase) and by the independent
verifier built on the oracle, both given the public statement (program,
execution counts, output); a wrong output or wrong counts are rejected."""
import pytest

from lambda_vm_b200 import rv64
from lambda_vm_b200 import rv64_air as RA
from lambda_vm_b200.stark import GpuBackend, Options
from oracle.verifier import verify as oracle_verify

pytestmark = pytest.mark.gpu
OPTS = Options(blowup=2, grinding=8, final_log_degree=3, queries=12)


@pytest.mark.parametrize("n", [3, 40, 1000])
def test_fibonacci_execution_proof_verifies(be, n):
    words = rv64.fib_program(n)
    proof, pub = RA.prove(words, OPTS, GpuBackend(be))
    assert pub["output"] == rv64.fib_reference(n)
    counts, out = pub["counts"], pub["output"]
    assert RA.verify(words, counts, out, proof, OPTS) == (True, "ok")
    assert RA.verify(words, counts, out, proof, OPTS, device=be) == (True, "ok")
    airs = RA.airs_for(words, counts)
    assert oracle_verify(airs, proof, OPTS, label=RA.statement_label(words, counts, out),
                         public_terms=airs[0].public_terms(counts, out)) == (True, "ok")
    # a different output, or different counts, is not what was proved
    assert RA.verify(words, counts, (out + 1) % (1 << 64), proof, OPTS)[0] is False
    bad = list(counts)
    bad[3] += 1
    bad[0] -= 1
    assert RA.verify(words, bad, out, proof, OPTS)[0] is False


@pytest.mark.parametrize("blocks", [1, 9])
def test_keccak_guest_proof_verifies(be, blocks):
    """The Keccak guest (xorshift buffer, keccak-f ecalls, load/store
    XOR-folds): CPU, RANGE, BITWISE, SHIFT, MEMORY and KECCAK tables proved on
    the GPU; accepted by the library's verifier (host and GPU query phase) and
    by the oracle's, given the statement with the chips' heights; a wrong
    output or a wrong height is rejected."""
    words = rv64.keccak_program(136 * blocks)
    proof, pub = RA.prove(words, OPTS, GpuBackend(be))
    assert pub["output"] == rv64.keccak_reference(136 * blocks)
    counts, out, h = pub["counts"], pub["output"], pub["heights"]
    assert set(h) == {"cpu", "range", "bitwise", "shift", "memory", "keccak"}
    assert RA.verify(words, counts, out, proof, OPTS, heights=h) == (True, "ok")
    assert RA.verify(words, counts, out, proof, OPTS, device=be, heights=h) == (True, "ok")
    airs = RA.airs_for(words, counts, h)
    assert oracle_verify(airs, proof, OPTS, label=RA.statement_label(words, counts, out, h),
                         public_terms=airs[0].public_terms(counts, out)) == (True, "ok")
    assert RA.verify(words, counts, out ^ 1, proof, OPTS, heights=h)[0] is False
    bad_h = dict(h)
    bad_h["shift"] += 1
    assert RA.verify(words, counts, out, proof, OPTS, heights=bad_h)[0] is False


def test_keccak_guest_scheduled_proof_equals_plain(be):
    """The batched prover (multi-table R1 launches, concurrent table drivers)
    gives the plain prover's proof for the six-table statement."""
    from lambda_vm_b200.scheduler import multi_prove_scheduled
    from lambda_vm_b200.stark import multi_prove
    from proofcmp import diff
    airs, traces, pub = RA.build(rv64.keccak_program(136 * 4))
    plain = multi_prove(airs, traces, OPTS, GpuBackend(be), label=pub["label"])
    sched = multi_prove_scheduled(airs, traces, OPTS, workers=4, be=be, label=pub["label"])
    assert diff(sched, plain) is None, diff(sched, plain)


def test_device_chip_tables_equal_the_host_tables(be):
    """sg_rv64_cpu_table, sg_rv64_keccak_table, sg_rv64_shift_table and
    sg_rv64_memory_table (tables written on the device from the run's events)
    against the numpy builders, cell for cell: the Keccak guest (full CPU
    width), the Fibonacci guest (core width), a branch on low limbs 2^32 - 1
    and 0, then random lanes and timestamps, every shift amount in both
    directions, and memory tables of one cell, of as many cells as rows and of
    address gaps past 2^16 cells, with padding rows."""
    import numpy as np
    bk = GpuBackend(be)

    def same(src, air, host):
        m = src.device_trace(bk, air)
        got = bk.to_host(m)
        bk.free(m)
        assert np.array_equal(got, host)

    wrap = rv64.assemble([("li", "t0", -1), ("srli", "t0", "t0", 32), ("li", "t1", 0),
                          ("beq", "t0", "t1", "end"), ("bne", "t0", "t1", "end"), ("li", "t1", 5),
                          "end:", ("li", "a7", 93), ("ecall",)])
    for words, expect in ((rv64.keccak_program(136 * 11), 4), (rv64.fib_program(3000), 1), (wrap, 2)):
        ev = RA.native_events(words)
        airs, srcs, _ = RA.tables_from_events(words, ev)
        _, host, _ = RA.tables_from_events(words, ev, host_tables=True)
        checked = 0
        for air, s, h in zip(airs, srcs, host):
            if hasattr(s, "device_trace"):
                same(s, air, h)
                checked += 1
        assert checked == expect
    rng = np.random.default_rng(3)
    P_ = 7
    lanes = rng.integers(0, 2**64, size=(P_, 25), dtype=np.uint64)
    told = rng.integers(0, 1000, size=(P_, 25), dtype=np.uint64)
    clk = np.arange(1, P_ + 1, dtype=np.uint64) * 5000
    base = np.arange(P_, dtype=np.uint64) * 200 + 4096
    src = RA.KeccakSource(clk, base, lanes, told)
    air = RA.KeccakAir(8)
    same(src, air, src.host_trace(air))
    sh = [(d, int(a), k) for d in (0, 1) for k in range(64) for a in rng.integers(0, 2**64, 2, dtype=np.uint64)]
    ssrc = RA.ShiftSource(sh)
    sair = RA.ShiftAir(9)
    same(ssrc, sair, ssrc.host_trace(sair))
    empty = RA.ShiftSource(np.zeros((0, 3), np.uint64))
    same(empty, RA.ShiftAir(6), empty.host_trace(RA.ShiftAir(6)))
    for addrs, log_n in (([8], 6), (np.arange(64) * 8 + 4096, 6),
                         (np.cumsum(rng.integers(1, 2**20, 300)) * 8, 9)):
        a = np.asarray(addrs, np.uint64)
        msrc = RA.MemorySource(a, rng.integers(0, 2**64, a.size, dtype=np.uint64),
                               rng.integers(0, 2**40, a.size, dtype=np.uint64))
        mair = RA.MemoryAir(log_n)
        same(msrc, mair, msrc.host_trace(mair))


def test_memory_table_rejects_bad_cells(be):
    """sg_rv64_memory_table refuses, before any launch, cells whose addresses
    are not ascending multiples of 8 below 2^32, and more cells than rows."""
    import ctypes as C
    import numpy as np
    from lambda_vm_b200 import native
    bk = GpuBackend(be)
    m = bk._alloc(64, RA.MemoryAir(6).width)
    for addrs in ([16, 8], [8, 8], [8, 12], [8, 1 << 32]):
        cells = np.zeros((len(addrs), 3), np.uint64)
        cells[:, 0] = addrs
        rc = bk.L.sg_rv64_memory_table(bk.be.h, bk.st, cells.ctypes.data, len(addrs), 64, m.ptr)
        assert rc == native.SG_ERR_INVALID, addrs
    cells = np.zeros((65, 3), np.uint64)
    cells[:, 0] = np.arange(65) * 8
    assert bk.L.sg_rv64_memory_table(bk.be.h, bk.st, cells.ctypes.data, 65, 64, m.ptr) == native.SG_ERR_INVALID
    assert bk.L.sg_rv64_memory_table(bk.be.h, bk.st, cells.ctypes.data, 0, 64, m.ptr) == native.SG_ERR_INVALID
    bk.free(m)


@pytest.mark.parametrize("rows,step", [(256, 2), (1024, 4)])
def test_keccak_table_kernel_equals_the_walk(be, rows, step):
    """The KECCAK table's hand-written constraint kernel (SG_AIR_KECCAK, the
    first 3383 constraints) with the walk for the LogUp constraints, against
    the walk of the table's whole program, on random field elements (not a
    valid trace: every constraint value is compared): each constraint's value
    and the composition with boundary terms, exactly."""
    import numpy as np
    from lambda_vm_b200 import math_cuda as mc
    from lambda_vm_b200.ir import lower
    P_ = 0xFFFFFFFF00000001
    rng = np.random.default_rng(rows)
    rf = lambda shape: np.where((x := rng.integers(0, 2**64, size=shape, dtype=np.uint64)) >= np.uint64(P_),
                                x - np.uint64(P_), x)
    air = RA.KeccakAir(8)
    full, dev = lower(air.program), lower(air.device_program)
    assert dev["hand_kernel"] == 1 and dev["num_roots"] == len(full["roots"]) == 3434
    main = rf((rows, air.width))
    aux = rf((rows, 3 * air.aux_width))
    rap, alpha, off = rf((2, 3)), rf((air.max_alpha, 3)), rf((3,))
    a = mc.eval_constraints_on_device(full, main, aux, rap, alpha, off, step, None, be)
    b = mc.eval_constraints_on_device(dev, main, aux, rap, alpha, off, step, None, be)
    assert a.shape == b.shape and np.array_equal(a, b)
    comp = {"beta": rf((3434, 3)), "z_inv": rf((rows // 4,)),
            "boundary": [(air.acc_col, True, rf((3,)), rf((3,)))], "b_z_inv": rf((1, rows))}
    ha = mc.eval_constraints_on_device(full, main, aux, rap, alpha, off, step, comp, be)
    hb = mc.eval_constraints_on_device(dev, main, aux, rap, alpha, off, step, comp, be)
    assert np.array_equal(ha, hb)


@pytest.mark.parametrize("chips", [(), ("bitwise", "shift", "memory", "keccak"), ("shift",), ("memory",),
                                   ("bitwise", "memory", "keccak")])
def test_cpu_table_kernel_equals_the_walk(be, chips):
    """The CPU table's hand-written constraint kernel (SG_AIR_CPU with the
    chip set) with the walk for the LogUp constraints, against the walk of
    the table's whole program, on random field elements: every constraint's
    value and the composition with its boundary term, exactly."""
    import numpy as np
    from lambda_vm_b200 import math_cuda as mc
    from lambda_vm_b200.ir import lower
    P_ = 0xFFFFFFFF00000001
    rng = np.random.default_rng(len(chips) + 7)
    rf = lambda shape: np.where((x := rng.integers(0, 2**64, size=shape, dtype=np.uint64)) >= np.uint64(P_),
                                x - np.uint64(P_), x)
    air = RA.CpuAir(rv64.keccak_program(136), 9, chips)
    full, dev = lower(air.program), lower(air.device_program)
    assert dev["hand_kernel"] & 0xFF == 2 and dev["num_roots"] == len(full["roots"])
    rows, step = 512, 2
    main = rf((rows, air.width))
    aux = rf((rows, 3 * air.aux_width))
    rap, alpha, off = rf((2, 3)), rf((air.max_alpha, 3)), rf((3,))
    a = mc.eval_constraints_on_device(full, main, aux, rap, alpha, off, step, None, be)
    b = mc.eval_constraints_on_device(dev, main, aux, rap, alpha, off, step, None, be)
    assert a.shape == b.shape and np.array_equal(a, b)
    comp = {"beta": rf((len(full["roots"]), 3)), "z_inv": rf((rows // 4,)),
            "boundary": [(air.acc_col, True, rf((3,)), rf((3,)))], "b_z_inv": rf((1, rows))}
    assert np.array_equal(mc.eval_constraints_on_device(full, main, aux, rap, alpha, off, step, comp, be),
                          mc.eval_constraints_on_device(dev, main, aux, rap, alpha, off, step, comp, be))


def test_shift_table_kernel_equals_the_walk(be):
    """The SHIFT table's hand-written constraint kernel (SG_AIR_SHIFT) against
    the walk of its whole program, on random field elements, exactly."""
    import numpy as np
    from lambda_vm_b200 import math_cuda as mc
    from lambda_vm_b200.ir import lower
    P_ = 0xFFFFFFFF00000001
    rng = np.random.default_rng(31)
    rf = lambda shape: np.where((x := rng.integers(0, 2**64, size=shape, dtype=np.uint64)) >= np.uint64(P_),
                                x - np.uint64(P_), x)
    air = RA.ShiftAir(8)
    full, dev = lower(air.program), lower(air.device_program)
    assert dev["hand_kernel"] == 3 and dev["num_roots"] == len(full["roots"])
    rows = 512
    main, aux = rf((rows, air.width)), rf((rows, 3 * air.aux_width))
    rap, alpha, off = rf((2, 3)), rf((air.max_alpha, 3)), rf((3,))
    assert np.array_equal(mc.eval_constraints_on_device(full, main, aux, rap, alpha, off, 2, None, be),
                          mc.eval_constraints_on_device(dev, main, aux, rap, alpha, off, 2, None, be))
    comp = {"beta": rf((len(full["roots"]), 3)), "z_inv": rf((rows // 4,)),
            "boundary": [(air.acc_col, True, rf((3,)), rf((3,)))], "b_z_inv": rf((1, rows))}
    assert np.array_equal(mc.eval_constraints_on_device(full, main, aux, rap, alpha, off, 2, comp, be),
                          mc.eval_constraints_on_device(dev, main, aux, rap, alpha, off, 2, comp, be))


def _tables_with_logup_programs():
    from lambda_vm_b200.air import SynthTableAir
    return [("range", RA.RangeAir()), ("bitwise", RA.BitwiseAir()), ("memory", RA.MemoryAir(9)),
            ("synth2", SynthTableAir(9, 10, num_interactions=2)), ("synth4", SynthTableAir(9, 24, num_interactions=4)),
            ("synth6", SynthTableAir(9, 40, num_interactions=6))]


@pytest.mark.parametrize("name", [n for n, _ in _tables_with_logup_programs()])
def test_logup_descriptor_constraints_equal_the_walk(be, name):
    """The tables whose device program walks only the base constraints and
    leaves the LogUp ones to the library's descriptor kernel
    (k_logup_constraints): RANGE, BITWISE, MEMORY and synthetic chip tables
    of one and two committed pairs and a two-interaction tail (the RV64
    CPU, SHIFT and KECCAK tables, with one- and two-interaction tails, are
    covered with their hand kernels above), against the walk of the whole
    program on random field elements: every constraint and the composition,
    exactly."""
    import numpy as np
    from lambda_vm_b200 import math_cuda as mc
    from lambda_vm_b200.ir import lower
    P_ = 0xFFFFFFFF00000001
    air = dict(_tables_with_logup_programs())[name]
    rng = np.random.default_rng(len(name) * 101 + air.width)
    rf = lambda shape: np.where((x := rng.integers(0, 2**64, size=shape, dtype=np.uint64)) >= np.uint64(P_),
                                x - np.uint64(P_), x)
    full, dev = lower(air.program), lower(air.device_program)
    assert dev["logup_desc"] is not None and dev["num_roots"] == len(full["roots"])
    rows = 1 << 9
    main, aux = rf((rows, air.width)), rf((rows, 3 * air.aux_width))
    rap, alpha, off = rf((2, 3)), rf((air.max_alpha, 3)), rf((3,))
    assert np.array_equal(mc.eval_constraints_on_device(full, main, aux, rap, alpha, off, 2, None, be),
                          mc.eval_constraints_on_device(dev, main, aux, rap, alpha, off, 2, None, be))
    comp = {"beta": rf((len(full["roots"]), 3)), "z_inv": rf((rows // 4,)),
            "boundary": [(air.acc_col, True, rf((3,)), rf((3,)))], "b_z_inv": rf((1, rows))}
    assert np.array_equal(mc.eval_constraints_on_device(full, main, aux, rap, alpha, off, 2, comp, be),
                          mc.eval_constraints_on_device(dev, main, aux, rap, alpha, off, 2, comp, be))


def test_logup_descriptor_is_validated(be):
    """sg_eval_constraints refuses, before any launch, a LogUp descriptor
    outside the kernel's layout or reading out of range, and LogUp indices a
    node also completes or beyond the program."""
    import copy
    import numpy as np
    from lambda_vm_b200 import math_cuda as mc, native
    from lambda_vm_b200.air import SynthTableAir
    from lambda_vm_b200.ir import lower
    air = SynthTableAir(6, 12, num_interactions=4)
    dev = lower(air.device_program)
    rows = 64
    main = np.zeros((rows, air.width), np.uint64)
    aux = np.zeros((rows, 3 * air.aux_width), np.uint64)
    rap, alpha, off = np.zeros((2, 3), np.uint64), np.zeros((air.max_alpha, 3), np.uint64), np.zeros(3, np.uint64)
    mc.eval_constraints_on_device(dev, main, aux, rap, alpha, off, 2, None, be)

    def bad(edit):
        d = copy.deepcopy({k: v for k, v in dev.items()})
        edit(d, d["logup_desc"])
        with pytest.raises(native.SgError, match="INVALID"):
            mc.eval_constraints_on_device(d, main, aux, rap, alpha, off, 2, None, be)

    bad(lambda d, g: g.__setitem__("term_cols", np.array([air.width] + list(g["term_cols"][1:]), np.uint32)))
    bad(lambda d, g: g.__setitem__("mult_term_cols", np.array([air.width + 5] * len(g["mult_term_cols"]), np.uint32)))
    bad(lambda d, g: g.__setitem__("elem_alpha_idx", np.array([air.max_alpha] * len(g["elem_alpha_idx"]), np.uint32)))
    bad(lambda d, g: g.__setitem__("out_col_interactions", np.array([1, 0, 2, 3], np.uint32)))
    bad(lambda d, g: g.__setitem__("num_committed", 0))
    bad(lambda d, g: d.__setitem__("logup_root", 0))
    bad(lambda d, g: d.__setitem__("logup_root", d["num_roots"] - 1))


def test_cpu_table_rejects_bad_records(be):
    """sg_rv64_cpu_table refuses a record with an unknown opcode or a
    register index past 31, and a chip instruction in a core-width table,
    whether the records go up directly (small) or through the staged upload
    that checks them as it copies (large, the bad record in a late piece)."""
    import numpy as np
    from lambda_vm_b200 import native
    bk = GpuBackend(be)
    for count, log_n in ((1000, 10), (150000, 18)):
        n = 1 << log_n
        rec = np.zeros((count, 8), np.uint64)
        rec[:, 0] = (np.arange(count, dtype=np.uint64) * np.uint64(4)) | (np.uint64(1) << np.uint64(32))  # add x0,x0,x0
        regs = np.zeros(((n + 63) // 64, 32), np.uint64)
        m = bk._alloc(n, RA.CPU_WIDTH)
        call = lambda r, width: bk.L.sg_rv64_cpu_table(bk.be.h, bk.st, r.ctypes.data, count, regs.ctypes.data, n,
                                                       width, m.ptr)
        assert call(rec, RA.CPU_WIDTH) == native.SG_OK
        for word in ((np.uint64(0) << np.uint64(32)),                       # op 0
                     (np.uint64(1) << np.uint64(32)) | (np.uint64(40) << np.uint64(40))):  # rd 40
            bad = rec.copy()
            bad[count - 3, 0] = word
            assert call(bad, RA.CPU_WIDTH) == native.SG_ERR_INVALID
        chip = rec.copy()
        chip[count - 2, 0] = np.uint64(RA.OP_ID["xor"]) << np.uint64(32)
        assert call(chip, RA.CPU_CORE_WIDTH) == native.SG_ERR_INVALID
        assert call(chip, RA.CPU_WIDTH) == native.SG_OK
        bk.to_host(m)  # waits for the accepted calls' kernels
        bk.free(m)


def test_shift_table_rejects_bad_events(be):
    """sg_rv64_shift_table refuses a direction past 1 or an amount past 63,
    on the direct and on the staged upload."""
    import numpy as np
    from lambda_vm_b200 import native
    bk = GpuBackend(be)
    for count, log_n in ((500, 9), (200000, 18)):
        n = 1 << log_n
        ev = np.zeros((count, 3), np.uint64)
        ev[:, 1] = np.arange(count, dtype=np.uint64)
        ev[:, 2] = np.arange(count, dtype=np.uint64) % np.uint64(64)
        m = bk._alloc(n, RA.ShiftAir(log_n).width)
        call = lambda e: bk.L.sg_rv64_shift_table(bk.be.h, bk.st, e.ctypes.data, count, n, m.ptr)
        assert call(ev) == native.SG_OK
        for col, v in ((0, 2), (2, 64)):
            bad = ev.copy()
            bad[count - 5, col] = v
            assert call(bad) == native.SG_ERR_INVALID
        bk.to_host(m)
        bk.free(m)


def test_streaming_program_roots_are_not_read(be):
    """A streaming program's `roots` array is unused (node_roots names the
    constraints): sg_eval_constraints accepts it as NULL and gives the same
    composition as with it set (it once copied num_roots entries from it)."""
    import ctypes as C
    import numpy as np
    from lambda_vm_b200 import math_cuda as mc, native
    from lambda_vm_b200.ir import lower
    air = RA.KeccakAir(6)
    dev = lower(air.device_program)
    rows = 256
    rng = np.random.default_rng(9)
    P_ = 0xFFFFFFFF00000001
    rf = lambda shape: np.where((x := rng.integers(0, 2**64, size=shape, dtype=np.uint64)) >= np.uint64(P_),
                                x - np.uint64(P_), x)
    main, aux = rf((rows, air.width)), rf((rows, 3 * air.aux_width))
    rap, alpha, off = rf((2, 3)), rf((air.max_alpha, 3)), rf((3,))
    comp = {"beta": rf((dev["num_roots"], 3)), "z_inv": rf((rows // 4,)),
            "boundary": [(air.acc_col, True, rf((3,)), rf((3,)))], "b_z_inv": rf((1, rows))}
    want = mc.eval_constraints_on_device(dev, main, aux, rap, alpha, off, 2, comp, be)
    real = mc._program_struct
    try:
        def no_roots(low, keep):
            p = real(low, keep)
            p.roots = None
            return p
        mc._program_struct = no_roots
        got = mc.eval_constraints_on_device(dev, main, aux, rap, alpha, off, 2, comp, be)
    finally:
        mc._program_struct = real
    assert np.array_equal(want, got)
