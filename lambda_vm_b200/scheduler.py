"""Table scheduler: concurrent per-table drivers under an HBM budget.

Restates the reference's scheduling (crypto/stark/src/prover.rs:620-790):
heaviest-first ordering (`heaviest_first`, :785), k concurrent table drivers
(`run_admitted`, :749-783) each admitted by a byte budget (`VramGate`,
:697-747; estimate `estimate_table_vram_bytes`, :682-695). Each driver owns a
non-blocking CUDA stream, so small tables overlap on the device instead of
running one after another behind host round trips; ctypes releases the GIL
during every C-ABI call, so drivers run concurrently on the host too.

R1 is one native call (sg_batch_commit_fused): every table's LDE passes run
in shared multi-table DFT launches (one persistent launch per pass step,
length, width and direction), then each table's leaves and tree. The protocol is unchanged: the roots
are absorbed in table order, and every table's rounds 2-4 run on its own
transcript fork, so the proof is identical to the sequential prover's.
"""
import ctypes as C
import threading
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import field as F
from . import native
from .device import backend as _backend
from .ir import device_program, lowered
from .stark import GpuBackend, Options, _gen_trace, _u64le, prove_table


class VramGate:
    def __init__(self, budget_bytes):
        self.budget = budget_bytes
        self.used = 0
        self.cv = threading.Condition()

    def acquire(self, nbytes):
        with self.cv:
            # an oversized table runs alone rather than deadlocking
            while self.used > 0 and self.used + nbytes > self.budget:
                self.cv.wait()
            self.used += nbytes

    def release(self, nbytes):
        with self.cv:
            self.used -= nbytes
            self.cv.notify_all()


def estimate_table_bytes(air, opts):
    """Device bytes a table's rounds 2-4 allocate beyond its resident main LDE."""
    N = air.n * opts.blowup
    W = air.aux_width
    per_row = 8 * (3 * W) + 8 * 6 + 24 + 24 + 24 + 24 + 24 + 48 + 24  # aux, parts, H, halves, DEEP, FRI, inv_t, inv_h
    return N * per_row + air.n * 3 * W * 8


def heaviest_first(airs, opts):
    return sorted(range(len(airs)), key=lambda i: -(airs[i].n * opts.blowup * (airs[i].width + 3 * airs[i].aux_width)))


class StreamPool:
    """k non-blocking streams, each wrapped in a GpuBackend for one table
    driver. `priority` (None: the default) is a CUDA stream priority, lower
    numbers first (sg_stream_priority_range)."""

    def __init__(self, be, k, priority=None):
        self.be = be
        L = native.lib()
        self.streams = []
        for _ in range(k):
            s = C.c_void_p()
            if priority is None:
                native.check(L.sg_stream_create(be.h, C.byref(s)))
            else:
                native.check(L.sg_stream_create_priority(be.h, int(priority), C.byref(s)))
            self.streams.append(s.value)
        self.free = [GpuBackend(be, s) for s in self.streams]
        self.lock = threading.Lock()

    def take(self):
        with self.lock:
            return self.free.pop()

    def give(self, bk):
        with self.lock:
            self.free.append(bk)

    def close(self):
        L = native.lib()
        for s in self.streams:
            L.sg_stream_sync(self.be.h, s)
            L.sg_stream_destroy(self.be.h, s)
        self.streams = []


def stream_priority_range(be):
    """(least, greatest) CUDA stream priority of the context's device."""
    lo, hi = C.c_int(), C.c_int()
    native.check(native.lib().sg_stream_priority_range(be.h, C.byref(lo), C.byref(hi)))
    return lo.value, hi.value


def multi_prove_scheduled(airs, sources, opts=None, workers=8, budget_bytes=None, be=None,
                          label=b"lambda_vm_b200/synthetic-multi-table", priority=None, fused_r1=True):
    """Same proof as stark.multi_prove, with k concurrent table drivers (on
    streams of CUDA priority `priority`, None: the default). R1 commits every
    table at once: with fused_r1 (default) through sg_batch_commit_fused, whose
    multi-table DFT launches cover all tables' passes, else sg_batch_commit's
    per-table launches over `workers` streams."""
    opts = opts or Options()
    be = be or _backend()
    B, g = opts.blowup, opts.coset_offset
    base = GpuBackend(be)
    r1_stream = None
    if priority is not None:
        s = C.c_void_p()
        native.check(native.lib().sg_stream_create_priority(be.h, int(priority), C.byref(s)))
        r1_stream = s.value
    for air in airs:  # warm the domain caches serially on the legacy stream
        base.domain(air.log_n, B, g)
    # without a pass-cost model, time the DFT tile widths now, while nothing
    # else runs, rather than inside the first concurrent pass (a no-op once
    # the context has them)
    cols, cost, cnt = (C.c_uint32 * 4)(), (C.c_float * 4)(), C.c_uint32()
    for log_len in range(8, 12) if getattr(be, "pass_model", None) is None else ():
        native.check(native.lib().sg_ctx_dft_tuning(be.h, None, log_len, cols, cost, C.byref(cnt)))
    native.check(native.lib().sg_stream_sync(be.h, None))
    pool = StreamPool(be, workers, priority)
    # R1 runs on a stream of the job's priority (its batched commit's internal
    # streams inherit it); the legacy stream when no priority is asked for
    r1b = GpuBackend(be, r1_stream) if r1_stream is not None else base
    order = heaviest_first(airs, opts)
    r1 = [None] * len(airs)

    try:
        # R1: every table's trace, then one native batched commit of all tables
        # (LDEs in multi-table DFT launches, then leaves and trees).
        tms = [_gen_trace(r1b, air, src) for air, src in zip(airs, sources)]
        committed = r1b.batch_commit(tms, B, [base.domain(a.log_n, B, g).weights for a in airs], workers,
                                     fused=fused_r1)
        for i in range(len(airs)):
            lde, tree, root, release = committed[i]
            r1[i] = (tms[i], lde, tree, root, release)
        t = base.transcript(label)
        for i in range(len(airs)):
            t.append_bytes(r1[i][3])
        challenges = [F.f3(t.sample_ext3()), F.f3(t.sample_ext3())]
        alpha = challenges[1]
        alpha_pows = [(1, 0, 0)]
        for _ in range(max(a.max_alpha for a in airs) - 1):
            alpha_pows.append(F.f3mul(alpha_pows[-1], alpha))
        forks = []
        for i in range(len(airs)):
            ti = t.clone()
            if len(airs) > 1:
                ti.append_bytes(_u64le(i))
            forks.append(ti)
        in_use, _ = be.memory()
        budget = budget_bytes if budget_bytes is not None else be.budget() - in_use
        gate = VramGate(max(budget, 1 << 30))
        proofs = [None] * len(airs)

        def rounds(i):
            est = estimate_table_bytes(airs[i], opts)
            gate.acquire(est)
            bk = pool.take()
            tm, lde, tree, root, release = r1[i]
            try:
                p = prove_table(bk, airs[i], lowered(device_program(airs[i])), tm, lde, tree, forks[i], challenges, alpha_pows,
                                opts)
                p["main_root"] = root
                proofs[i] = p
            finally:
                # The R1 buffers were allocated on other streams: finish this
                # stream's use of them before they are released.
                bk.L.sg_stream_sync(bk.be.h, bk.st)
                bk.free(tm)
                release(bk)
                pool.give(bk)
                gate.release(est)

        with ThreadPoolExecutor(workers) as ex:
            list(ex.map(rounds, order))
        return {"tables": proofs, "challenges": challenges}
    finally:
        pool.close()
        if r1_stream is not None:
            native.lib().sg_stream_sync(be.h, r1_stream)
            native.lib().sg_stream_destroy(be.h, r1_stream)
