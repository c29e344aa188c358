"""Serving loop host logic on the CPU with a stand-in prover: slot and HBM
budget admission, FIFO order, per-job results and errors, latency quantiles."""
import threading
import time

import pytest

from lambda_vm_b200.air import SynthTableAir
from lambda_vm_b200.serving import ProofServer, ServeStats, _quantile, estimate_job_bytes, serve_poisson
from lambda_vm_b200.stark import Options


class Recorder:
    def __init__(self, delay=0.02, fail_ids=()):
        self.lock = threading.Lock()
        self.running = {}
        self.max_running = 0
        self.max_bytes = 0
        self.starts = []
        self.delay = delay
        self.fail_ids = set(fail_ids)

    def __call__(self, airs, sources, opts, drivers, budget):
        key = sources[0]
        with self.lock:
            self.running[key] = budget
            self.max_running = max(self.max_running, len(self.running))
            self.max_bytes = max(self.max_bytes, sum(self.running.values()))
            self.starts.append(key)
        time.sleep(self.delay)
        with self.lock:
            del self.running[key]
        if key in self.fail_ids:
            raise ValueError(f"job {key} failed")
        return {"job": key}


def _spec(i, log_n=10, width=8):
    return [SynthTableAir(log_n, width, 2)], [i]


def test_slots_fifo_and_results():
    rec = Recorder()
    with ProofServer(budget_bytes=1 << 40, max_jobs=3, drivers=2, prove_fn=rec) as srv:
        jobs = [srv.submit(*_spec(i)) for i in range(10)]
        srv.drain()
    assert rec.max_running <= 3
    assert rec.starts == list(range(10))
    assert [j.proof["job"] for j in jobs] == list(range(10))
    assert all(j.latency is not None and j.latency >= 0 for j in jobs)


def test_budget_admission_limits_concurrency():
    opts = Options()
    est = estimate_job_bytes(*_spec(0, 12, 40)[:1], opts, 2)
    rec = Recorder()
    # room for two such jobs at a time, not three
    with ProofServer(budget_bytes=2 * est + est // 2, max_jobs=8, drivers=2, prove_fn=rec, opts=opts) as srv:
        for i in range(6):
            srv.submit(*_spec(i, 12, 40))
        srv.drain()
    assert rec.max_running == 2
    assert rec.max_bytes <= 2 * est + est // 2


def test_oversized_job_runs_alone():
    rec = Recorder()
    with ProofServer(budget_bytes=1, max_jobs=4, drivers=2, prove_fn=rec) as srv:
        jobs = [srv.submit(*_spec(i)) for i in range(3)]
        srv.drain()
    assert rec.max_running == 1
    assert all(j.error is None for j in jobs)


def test_job_errors_are_per_job():
    rec = Recorder(fail_ids={1})
    with ProofServer(budget_bytes=1 << 40, max_jobs=2, drivers=2, prove_fn=rec) as srv:
        jobs = [srv.submit(*_spec(i)) for i in range(4)]
        srv.drain()
    assert isinstance(jobs[1].error, ValueError)
    assert [j.error is None for j in jobs] == [True, False, True, True]
    st = ServeStats(jobs, min(j.t_submit for j in jobs), max(j.t_done for j in jobs))
    assert st.failed == 1 and st.jobs == 4


def test_poisson_stream_and_quantiles():
    rec = Recorder(delay=0.005)
    with ProofServer(budget_bytes=1 << 40, max_jobs=2, drivers=2, prove_fn=rec) as srv:
        jobs, st = serve_poisson(srv, [_spec(i) for i in range(12)], rate=200.0, seed=3)
    assert st.jobs == 12 and st.failed == 0
    assert st.p50_s <= st.p99_s
    assert _quantile([1, 2, 3, 4], 0.5) == 2
    assert _quantile([1, 2, 3, 4], 0.99) == 4
    assert _quantile(list(range(1, 101)), 0.99) == 99
    assert _quantile([], 0.5) is None


def test_closed_server_rejects():
    srv = ProofServer(budget_bytes=1 << 30, prove_fn=Recorder())
    srv.close()
    with pytest.raises(RuntimeError):
        srv.submit(*_spec(0))


class SizedRecorder(Recorder):
    """Stand-in prover whose run time grows with the job (large jobs 0.2 s,
    small ones 0.02 s), recording when each job starts and ends."""

    def __init__(self, big_cells):
        super().__init__()
        self.big_cells = big_cells
        self.spans = {}
        self.t0 = time.perf_counter()

    def __call__(self, airs, sources, opts, drivers, budget):
        from lambda_vm_b200.serving import job_cells
        big = job_cells(airs) >= self.big_cells
        self.delay = 0.2 if big else 0.02
        start = time.perf_counter() - self.t0
        out = super().__call__(airs, sources, opts, drivers, budget)
        with self.lock:
            self.spans[sources[0]] = (start, time.perf_counter() - self.t0, big, drivers)
        return out


def test_backfill_large_jobs_never_overlap_small_jobs_pass_them():
    """Large jobs run one at a time in arrival order; small jobs that arrive
    behind a waiting large job start at once (leaving it a slot), and the
    large job starts as soon as the running large job ends."""
    big = _spec(0, 14, 300)[0]
    small = _spec(0, 10, 8)[0]
    from lambda_vm_b200.serving import job_cells
    cut = job_cells(big)
    assert job_cells(small) < cut
    rec = SizedRecorder(cut)
    with ProofServer(budget_bytes=1 << 40, max_jobs=4, drivers=4, prove_fn=rec, big_cells=cut,
                     small_drivers=2) as srv:
        srv.submit(big, [0])
        srv.submit(big, [1])
        for i in range(2, 6):
            srv.submit(small, [i])
        srv.drain()
    sp = rec.spans
    a, b = sp[0], sp[1]
    assert a[2] and b[2] and not any(sp[i][2] for i in range(2, 6))
    assert b[0] >= a[1] - 1e-3  # the two large jobs never overlap
    assert b[0] - a[1] < 0.05  # and the second starts as the first ends
    # small jobs started while the first large job ran, ahead of the second
    assert sum(1 for i in range(2, 6) if sp[i][0] < a[1]) >= 2
    # one slot stays free for the waiting large job: at most 3 ran at once
    assert rec.max_running <= 4
    assert a[3] == 4 and all(sp[i][3] == 2 for i in range(2, 6))


def test_fifo_policy_keeps_arrival_order():
    big = _spec(0, 14, 300)[0]
    from lambda_vm_b200.serving import job_cells
    rec = SizedRecorder(job_cells(big))
    with ProofServer(budget_bytes=1 << 40, max_jobs=1, drivers=3, prove_fn=rec, policy="fifo") as srv:
        srv.submit(big, [0])
        for i in range(1, 4):
            srv.submit(_spec(0, 10, 8)[0], [i])
        srv.drain()
    assert rec.starts == [0, 1, 2, 3]
    assert all(v[3] == 3 for v in rec.spans.values())
    with pytest.raises(ValueError):
        ProofServer(budget_bytes=1, prove_fn=rec, policy="lifo")


def test_at_most_beside_big_small_jobs_run_beside_a_large_one():
    big = _spec(0, 14, 300)[0]
    from lambda_vm_b200.serving import job_cells
    cut = job_cells(big)
    rec = SizedRecorder(cut)
    with ProofServer(budget_bytes=1 << 40, max_jobs=4, drivers=4, prove_fn=rec, big_cells=cut,
                     beside_big=1) as srv:
        srv.submit(big, [0])
        for i in range(1, 7):
            srv.submit(_spec(0, 10, 8)[0], [i])
        srv.drain()
    a = rec.spans[0]
    smalls = [rec.spans[i] for i in range(1, 7)]
    # while the large job ran, the small jobs beside it never overlapped one another
    during = sorted((max(s, a[0]), min(e, a[1])) for s, e, _, _ in smalls if s < a[1] and e > a[0])
    assert during and all(x[1] <= y[0] + 1e-3 for x, y in zip(during, during[1:]))
