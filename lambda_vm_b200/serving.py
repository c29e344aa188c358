"""Proof serving: continuous admission of proof jobs under an HBM budget.

A request loop in the shape of the reference's multi-table driver
(crypto/stark/src/prover.rs:697-790, `VramGate` + `run_admitted`) lifted from
tables to whole proofs: jobs (one multi-table proof each) arrive at any time,
wait in a FIFO queue, and are admitted as soon as a job slot is free and the
job's HBM estimate fits the remaining budget. Admitted jobs run concurrently
(each on its own table drivers and CUDA streams), so a small proof that
arrives behind a large one overlaps with it on the device instead of waiting
for it. Every job's proof is the same as when it runs alone: jobs share no
transcript or buffers, only the device.

Latency of a job = completion time - submit time (queueing included);
`ServeStats` reports p50/p99 beside proofs/s and proved rows/s.
"""
import threading
import time
from collections import deque

from .scheduler import VramGate, estimate_table_bytes, multi_prove_scheduled
from .stark import Options


def estimate_job_bytes(airs, opts, drivers):
    """Peak device bytes of one proof: every table's main trace, LDE and tree
    stay resident from R1 until the table's rounds finish, plus rounds 2-4 of
    `drivers` tables at once (crypto/stark/src/prover.rs:682-695)."""
    resident = 0
    for a in airs:
        N = a.n * opts.blowup
        resident += a.n * a.width * 8 + N * a.width * 8 + N * 32
    per_table = sorted((estimate_table_bytes(a, opts) for a in airs), reverse=True)
    return resident + sum(per_table[:max(1, drivers)])


def job_cells(airs):
    """Trace cells of a job (main + 3 per aux column, every table): the size
    its device time grows with."""
    return sum(a.n * (a.width + 3 * a.aux_width) for a in airs)


class Job:
    __slots__ = ("id", "airs", "sources", "label", "rows", "cells", "big", "est", "t_submit", "t_start", "t_done",
                 "proof", "error", "done")

    def __init__(self, jid, airs, sources, est, big_cells=None, label=None):
        self.id = jid
        self.airs = airs
        self.sources = sources
        self.label = label
        self.rows = sum(a.n for a in airs)
        self.cells = job_cells(airs)
        self.big = big_cells is not None and self.cells >= big_cells
        self.est = est
        self.t_submit = time.perf_counter()
        self.t_start = None
        self.t_done = None
        self.proof = None
        self.error = None
        self.done = threading.Event()

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.t_submit


class ServeStats:
    def __init__(self, jobs, t0, t1):
        lat = sorted(j.latency for j in jobs if j.latency is not None)
        self.jobs = len(jobs)
        self.failed = sum(1 for j in jobs if j.error is not None)
        self.wall_s = t1 - t0
        self.proofs_per_s = len(lat) / self.wall_s if self.wall_s > 0 else 0.0
        self.rows_per_s = sum(j.rows for j in jobs if j.error is None) / self.wall_s if self.wall_s > 0 else 0.0
        self.p50_s = _quantile(lat, 0.50)
        self.p99_s = _quantile(lat, 0.99)
        self.mean_s = sum(lat) / len(lat) if lat else None

    def as_dict(self):
        r = lambda x: None if x is None else round(x * 1e3, 1)
        return {"jobs": self.jobs, "failed": self.failed, "wall_s": round(self.wall_s, 3),
                "proofs_per_s": round(self.proofs_per_s, 3), "rows_per_s": round(self.rows_per_s, 1),
                "p50_ms": r(self.p50_s), "p99_ms": r(self.p99_s), "mean_ms": r(self.mean_s)}


def _quantile(sorted_vals, q):
    """Nearest-rank quantile."""
    if not sorted_vals:
        return None
    k = max(0, min(len(sorted_vals) - 1, int(-(-q * len(sorted_vals) // 1)) - 1))
    return sorted_vals[k]


class ProofServer:
    """Job queue with slot + HBM-budget admission.

    `max_jobs` concurrent proofs, each proved by `prove_fn(airs, sources, opts,
    drivers, budget_bytes)` (default: the scheduled multi-table prover on the
    process-wide device context). A job whose estimate exceeds the whole budget
    runs alone rather than never.

    policy "fifo": jobs start in arrival order as slots and memory allow, each
    with `drivers` table drivers.

    policy "backfill" (default): a job of at least `big_cells` trace cells is
    large. Large jobs start in arrival order and never overlap one another, so a
    large proof is never stretched by another large one (what made the FIFO
    server's tail worse than one-at-a-time at low load). Small jobs start as
    soon as a slot and memory are free, also past a large job that waits for
    the running one (backfilling): they keep one slot and the waiting job's
    memory free, so the large job still starts the moment the running large
    job ends. While a large job runs, at most `beside_big` small jobs run
    beside it, which bounds how much they can stretch it; with no large job
    running, small jobs use every slot. Large jobs get `drivers` table drivers
    on streams of the device's most urgent priority, small jobs at most
    `small_drivers` on default-priority streams, so a small proof fills gaps in
    a large one instead of lengthening it.
    """

    def __init__(self, budget_bytes, max_jobs=4, drivers=4, opts=None, prove_fn=None, be=None, policy="backfill",
                 big_cells=1 << 23, small_drivers=2, beside_big=1):
        if policy not in ("fifo", "backfill"):
            raise ValueError(f"unknown admission policy {policy!r}")
        self.opts = opts or Options()
        self.max_jobs = max_jobs
        self.drivers = drivers
        self.small_drivers = small_drivers
        self.beside_big = beside_big
        self.policy = policy
        self.big_cells = big_cells if policy == "backfill" else None
        self.gate = VramGate(budget_bytes)
        self.be = be
        self.urgent = None
        if prove_fn is None and policy == "backfill" and be is not None:
            from .scheduler import stream_priority_range
            self.urgent = stream_priority_range(be)[1]
        self.prove_fn = prove_fn or self._prove_gpu
        self.queue = deque()
        self.cv = threading.Condition()
        self.running = 0
        self.big_running = 0
        self.next_id = 0
        self.jobs = []
        self.closed = False
        self.threads = []
        self.dispatcher = threading.Thread(target=self._dispatch, daemon=True)
        self.dispatcher.start()

    def _prove_gpu(self, airs, sources, opts, drivers, budget_bytes, priority=None, label=None):
        kw = {} if label is None else {"label": label}
        return multi_prove_scheduled(airs, sources, opts, workers=drivers, budget_bytes=budget_bytes, be=self.be,
                                     priority=priority, **kw)

    def _drivers(self, job):
        return self.drivers if (self.policy == "fifo" or job.big) else max(1, min(self.small_drivers, self.drivers))

    def submit(self, airs, sources, label=None):
        """Queue one proof job: its tables and their traces (host arrays or
        synthetic-trace seeds), and its statement's transcript label."""
        with self.cv:
            if self.closed:
                raise RuntimeError("server is closed")
            probe = Job(self.next_id, airs, sources, 0, self.big_cells)
            est = estimate_job_bytes(airs, self.opts, self.drivers if self.policy == "fifo" or probe.big
                                     else max(1, min(self.small_drivers, self.drivers)))
            job = Job(self.next_id, airs, sources, est, self.big_cells, label)
            self.next_id += 1
            self.jobs.append(job)
            self.queue.append(job)
            self.cv.notify_all()
        return job

    def _fits(self, job, reserve=0):
        g = self.gate
        return g.used == 0 or g.used + job.est + reserve <= g.budget

    def _can_start(self, job, reserve=0):
        if not self._fits(job, reserve):
            return False
        if job.big:
            return not self.big_running
        return not self.big_running or self.running - self.big_running < self.beside_big

    def _pick(self):
        """The queued job to start now, or None (called with the lock held)."""
        if not self.queue or self.running >= self.max_jobs:
            return None
        if self.policy == "fifo":
            return self.queue[0] if self._fits(self.queue[0]) else None
        head = self.queue[0]
        if self._can_start(head):
            return head
        # The head waits (a large job behind the running large one, or memory):
        # a small job may pass it if it leaves the head a slot and its memory.
        if self.running >= self.max_jobs - 1:
            return None
        for j in list(self.queue)[1:]:
            if not j.big and self._can_start(j, reserve=head.est):
                return j
        return None

    def _dispatch(self):
        while True:
            with self.cv:
                job = self._pick()
                while not self.closed and job is None:
                    self.cv.wait(0.05)
                    job = self._pick()
                if self.closed and not self.queue:
                    return
                if job is None:
                    continue
                self.queue.remove(job)
                self.running += 1
                self.big_running += job.big
                job.t_start = time.perf_counter()
                self.gate.acquire(job.est)
            t = threading.Thread(target=self._run, args=(job,), daemon=True)
            self.threads.append(t)
            t.start()

    def _run(self, job):
        try:
            # rounds 2-4 of this job may use what its resident R1 state leaves of its share
            if self.prove_fn == self._prove_gpu:
                job.proof = self._prove_gpu(job.airs, job.sources, self.opts, self._drivers(job), job.est,
                                            self.urgent if job.big else None, job.label)
            else:
                job.proof = self.prove_fn(job.airs, job.sources, self.opts, self._drivers(job), job.est)
        except Exception as e:  # reported per job; the server keeps serving
            job.error = e
        finally:
            job.t_done = time.perf_counter()
            self.gate.release(job.est)
            with self.cv:
                self.running -= 1
                self.big_running -= job.big
                self.cv.notify_all()
            job.done.set()

    def drain(self):
        for j in list(self.jobs):
            j.done.wait()

    def close(self):
        self.drain()
        with self.cv:
            self.closed = True
            self.cv.notify_all()
        self.dispatcher.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def warm_context(be, job_specs, opts):
    """Start-up work a serving process does once, so no job pays for it: the
    per-domain vectors of every trace height the jobs use, and the DFT tile
    timings of every pass length."""
    import ctypes as C
    from . import native
    from .stark import GpuBackend
    bk = GpuBackend(be)
    for log_n in sorted({a.log_n for spec in job_specs for a in spec[0]}):
        bk.domain(log_n, opts.blowup, opts.coset_offset)
    cols, cost, cnt = (C.c_uint32 * 4)(), (C.c_float * 4)(), C.c_uint32()
    for log_len in range(8, 12) if getattr(be, "pass_model", None) is None else ():
        native.check(native.lib().sg_ctx_dft_tuning(be.h, None, log_len, cols, cost, C.byref(cnt)))
    native.check(native.lib().sg_stream_sync(be.h, None))


def serve_poisson(server, job_specs, rate, seed=0):
    """Submit `job_specs` [(airs, sources[, label])] with exponential inter-arrival
    times of mean 1/rate (seeded); wait for all; return (jobs, ServeStats)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=len(job_specs))
    t0 = time.perf_counter()
    due = t0
    jobs = []
    for spec, gap in zip(job_specs, gaps):
        due += gap
        now = time.perf_counter()
        if due > now:
            time.sleep(due - now)
        jobs.append(server.submit(*spec))
    for j in jobs:
        j.done.wait()
    t1 = max(j.t_done for j in jobs)
    return jobs, ServeStats(jobs, t0, t1)


def serve_sequential(job_specs, rate, prove_fn, seed=0):
    """The one-at-a-time baseline: the same arrival stream, one proof at a
    time in arrival order; latency includes the wait behind earlier jobs."""
    import numpy as np
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=len(job_specs))
    arrivals = []
    t = 0.0
    for gap in gaps:
        t += gap
        arrivals.append(t)
    t0 = time.perf_counter()
    jobs = []
    for spec, at in zip(job_specs, arrivals):
        now = time.perf_counter()
        if t0 + at > now:
            time.sleep(t0 + at - now)
        j = Job(len(jobs), spec[0], spec[1], 0)
        j.t_submit = t0 + float(at)
        j.t_start = time.perf_counter()
        try:
            j.proof = prove_fn(*spec)
        except Exception as e:
            j.error = e
        j.t_done = time.perf_counter()
        j.done.set()
        jobs.append(j)
    return jobs, ServeStats(jobs, t0, max(j.t_done for j in jobs))
