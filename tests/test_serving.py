"""Serving loop: admission by HBM budget, cohort packing, convergence retirement, and the
alone-vs-mix equality of results.

The CPU tests drive the scheduler with a stand-in for the batch context (step counts and a
geometric residual decay, no device), so its host logic is covered without a GPU.  The GPU tests
run real cohorts through the C ABI.
"""
import math
import time

import numpy as np
import pytest

from dgm_in_rust_b200 import serving
from dgm_in_rust_b200.serving import (Request, ServingLoop, footprint_bytes, latency_summary, one_at_a_time,
                                      requests_from_stream, solve_alone)
from dgm_in_rust_b200.workloads import Instance, instance_mesh, request_stream


class FakeBatch:
    """Stand-in for solver.Batch: instance i's density residual after s steps is 2^-(s-1) times
    its first one; advance is complete after ``lag`` polls (and, for the first batch created, its
    first advance only after ``hold_first_s`` seconds)."""
    lag = 2
    live = 0
    created = 0
    hold_first_s = 0.0

    def __init__(self, meshes, order, hcr, cfls, final_times, final_steps, limiter=True, device=0, precision="fp32",
                 capacities=None):
        self.meshes = list(meshes)
        self.capacities = capacities
        self.order = order
        self.precision = precision
        self.n = len(meshes)
        self.step = [0] * self.n
        self.final = list(final_steps)
        self.polls = 0
        self.uploaded = [False] * self.n
        FakeBatch.live += 1
        FakeBatch.created += 1
        self.hold = FakeBatch.hold_first_s if FakeBatch.created == 1 else 0.0
        self.ready_at = 0.0

    def set_initial(self, i, init):
        assert init.density > 0 and init.pressure > 0
        self.uploaded[i] = True

    def advance(self, n, with_residual=False):
        assert with_residual and all(self.uploaded)
        for i in range(self.n):
            self.step[i] = min(self.final[i], self.step[i] + n)
        self.polls = self.lag
        self.ready_at = time.perf_counter() + self.hold
        self.hold = 0.0

    def query(self):
        if time.perf_counter() < self.ready_at:
            return None
        if self.polls > 0:
            self.polls -= 1
            return None
        return 0

    def device_bytes(self):
        return footprint_bytes(self.meshes, self.order, self.precision, capacities=self.capacities)

    replaced = 0

    def replace(self, i, mesh, cfl, final_time, final_step):
        assert self.polls == 0, "a slot is replaced only while the cohort is idle"
        need = serving.slot_capacity(mesh)
        assert all(n <= r for n, r in zip(need, self.capacities[i]))
        self.meshes[i] = mesh
        self.step[i] = 0
        self.final[i] = final_step
        self.uploaded[i] = False
        FakeBatch.replaced += 1

    def diagnostics(self, use_residual=False):
        out = np.zeros((self.n, 8))
        for i in range(self.n):
            out[i, 6] = (3.0 * 0.5 ** (self.step[i] - 1)) ** 2
        return out

    def enqueue_diagnostics(self, use_residual=False):
        self.enqueued = self.diagnostics(use_residual)  # the steps are already applied when enqueued

    def collected_diagnostics(self):
        return self.enqueued.copy()

    def state(self, i):
        return 1e-3 * self.step[i], self.step[i], 0, -1

    def set_instance(self, i, t, step, final_time, final_step):
        self.final[i] = final_step

    def download(self, i):
        return np.full((self.meshes[i].n_elements, 4, 1), float(self.step[i]))

    def close(self):
        FakeBatch.live -= 1


@pytest.fixture
def fake_batch(monkeypatch):
    FakeBatch.live = 0
    FakeBatch.created = 0
    FakeBatch.replaced = 0
    monkeypatch.setattr(serving, "Batch", FakeBatch)
    yield FakeBatch
    assert FakeBatch.live == 0, "every cohort context is closed"


def _reqs(specs, gap=0.0):
    return [Request(i, i * gap, Instance(ni, ni // 2, 0.5, 1.0, p)) for i, (ni, p) in enumerate(specs)]


def test_footprint_grows_with_size_and_precision():
    m1, _ = instance_mesh(Instance(16, 8, 0.5, 0.0, 1))
    m2, _ = instance_mesh(Instance(32, 16, 0.5, 0.0, 1))
    assert footprint_bytes([m1], 1, "fp64") < footprint_bytes([m2], 1, "fp64")
    assert footprint_bytes([m2], 1, "fp32") < footprint_bytes([m2], 1, "fp64")
    assert footprint_bytes([m2], 2, "fp64") < footprint_bytes([m2], 3, "fp64")
    both = footprint_bytes([m1, m2], 2, "fp32")
    assert both <= footprint_bytes([m1], 2, "fp32") + footprint_bytes([m2], 2, "fp32")


def test_retires_at_convergence_or_step_cap(fake_batch):
    # residual drop 2^-(s-1): <= 1e-6 from s = 21 on; checks at s = 1, 9, 17, 25 (chunk 8)
    res = ServingLoop(prep="process", prep_workers=2, chunk_steps=8, tol=1e-6, max_steps=1000, keep_states=True).run(
        _reqs([(16, 1), (16, 2), (24, 1)]), realtime=False)
    assert [r.rid for r in res] == [0, 1, 2]
    for r in res:
        assert r.converged and r.steps == 25 and r.status == 0
        assert math.isclose(r.residual_drop, 0.5 ** 24)
        assert float(r.state[0, 0, 0]) == 25.0
    res = ServingLoop(prep="thread", chunk_steps=8, tol=1e-6, max_steps=12).run(_reqs([(16, 1)]), realtime=False)
    assert res[0].steps == 12 and not res[0].converged


def test_cohorts_are_packed_per_order(fake_batch):
    # an idle GPU admits the first prepared request at once; the other four arrive later, within
    # one window of each other, and are packed one cohort per order (three orders among them)
    FakeBatch.hold_first_s = 3.0             # the first cohort stays busy while the rest are prepared
    reqs = _reqs([(16, 1), (16, 2), (20, 1), (20, 2), (24, 3)])
    for r in reqs[1:]:
        r.arrival_s = 0.5 + 0.01 * r.rid     # well after the first, close to one another
    try:
        loop = ServingLoop(prep="thread", chunk_steps=64, tol=1e-3, max_steps=100, window_s=1.0)
        res = loop.run(reqs, realtime=True)
    finally:
        FakeBatch.hold_first_s = 0.0
    assert len(res) == 5 and all(r.converged for r in res)
    assert loop.cohorts_formed <= 4
    assert loop.max_concurrent == 5


def test_budget_admits_first_come_first_served(fake_batch):
    reqs = _reqs([(16, 1), (40, 2), (16, 1), (16, 1)], gap=0.02)
    room = [serving._room(serving.slot_capacity(instance_mesh(r.instance)[0]), 1.5) for r in reqs]
    one = max(footprint_bytes([instance_mesh(r.instance)[0]], r.instance.order, "fp32", capacities=[c])
              for r, c in zip(reqs, room))
    FakeBatch.lag = 300
    try:
        loop = ServingLoop(prep="thread", hbm_budget_bytes=one, chunk_steps=64, tol=1e-3, max_steps=100, window_s=0.0)
        res = loop.run(reqs, realtime=True)
    finally:
        FakeBatch.lag = 2
    assert len(res) == 4 and all(r.converged for r in res)
    assert loop.peak_bytes <= one
    admitted = [r.admitted_s for r in res]
    assert admitted == sorted(admitted)
    # the large request fits only alone: it waits for request 0, and 2 and 3 wait behind it
    assert res[1].admitted_s >= res[0].finished_s
    assert min(res[2].admitted_s, res[3].admitted_s) >= res[1].finished_s


def test_oversized_request_runs_alone(fake_batch):
    loop = ServingLoop(prep="thread", hbm_budget_bytes=1, chunk_steps=4, tol=1e-3, max_steps=50)
    res = loop.run(_reqs([(16, 1), (16, 1)]), realtime=False)
    assert len(res) == 2 and loop.max_concurrent == 1


def test_realtime_arrivals_join_while_others_run(fake_batch):
    FakeBatch.lag = 200                      # each chunk stays in flight for a while
    try:
        loop = ServingLoop(prep="thread", chunk_steps=4, tol=1e-3, max_steps=100, window_s=0.0)
        res = loop.run(_reqs([(16, 1), (16, 1), (16, 2)], gap=0.01), realtime=True)
    finally:
        FakeBatch.lag = 2
    assert len(res) == 3 and all(r.converged for r in res)
    assert loop.cohorts_formed >= 2 and loop.max_concurrent >= 2
    for r in res:
        assert r.finished_s >= r.admitted_s >= r.arrival_s - 1e-9


def test_preparation_errors_reach_the_caller(fake_batch):
    with pytest.raises(RuntimeError, match="preparing request 0"):
        ServingLoop(prep="process", prep_workers=2).run([Request(0, 0.0, Instance(16, 8, 0.5, 1.0, 7))], realtime=False)


def test_latency_summary_and_stream():
    stream = request_stream(20, rate=50.0, seed=3, e_max=2e4)
    reqs = requests_from_stream(stream)
    assert [r.rid for r in reqs] == list(range(20))
    assert all(b.arrival_s > a.arrival_s for a, b in zip(reqs, reqs[1:]))
    res = [serving.Result(i, 0.0, 0.0, float(i + 1), 10, 0.0, 1.0, False, 0, 100) for i in range(100)]
    s = latency_summary(res, wall_s=2.0)
    assert s["p50_s"] == pytest.approx(50.5) and s["p99_s"] == pytest.approx(99.01)
    assert s["dof_stage_updates_per_s"] == pytest.approx(100 * 100 * 3 * 10 / 2.0)


# ---------------------------------------------------------------------------------------- GPU
MIX = [(16, 1, 0.55, 2.0), (24, 2, 0.8, 1.25), (16, 3, 0.7, -2.0), (32, 1, 0.3, 4.0), (20, 2, 0.85, 0.0),
       (24, 3, 0.6, 3.0)]


def _mix_requests(gap):
    return [Request(i, i * gap, Instance(ni, ni // 2, m, a, p)) for i, (ni, p, m, a) in enumerate(MIX)]


@pytest.mark.gpu
def test_footprint_matches_device_bytes(built):
    from dgm_in_rust_b200.solver import Batch
    meshes = [instance_mesh(Instance(ni, ni // 2, 0.5, 1.0, 2))[0] for ni in (16, 24, 40)]
    for prec in ("fp64", "fp32"):
        b = Batch(meshes, 2, 1.4, [0.1] * 3, [1.0] * 3, [10] * 3, precision=prec)
        try:
            assert b.device_bytes() == footprint_bytes(meshes, 2, prec)
        finally:
            b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_result_alone_equals_result_in_mix(built, precision):
    """Tolerance: bitwise.  Each request's state, step count, time and residual drop from the
    serving loop (mixed, with staggered arrivals and with everything at once) equal those of the
    same request solved alone on a plain context."""
    kw = dict(chunk_steps=16, tol=1e-6, max_steps=49)
    alone = {r.rid: solve_alone(r, precision, keep_state=True, **kw)[0] for r in _mix_requests(0.0)}
    for gap, realtime in ((0.0, False), (0.004, True)):
        loop = ServingLoop(prep="process" if realtime else "thread", precision=precision, keep_states=True,
                           window_s=0.0, **kw)
        mixed = loop.run(_mix_requests(gap), realtime=realtime)
        assert loop.max_concurrent >= 2
        for r in mixed:
            a = alone[r.rid]
            assert r.status == 0 and a.status == 0
            assert (r.steps, r.time, r.residual_drop) == (a.steps, a.time, a.residual_drop)
            assert np.array_equal(r.state, a.state), f"request {r.rid} differs in the mix"


@pytest.mark.gpu
def test_budget_bounds_resident_bytes(built):
    reqs = _mix_requests(0.0)
    sizes = [footprint_bytes([instance_mesh(r.instance)[0]], r.instance.order, "fp32") for r in reqs]
    budget = 2 * max(sizes)
    loop = ServingLoop(prep="thread", hbm_budget_bytes=budget, chunk_steps=16, max_steps=33, window_s=0.0)
    res = loop.run(reqs, realtime=False)
    assert len(res) == len(reqs) and all(r.status == 0 and r.steps == 33 for r in res)
    assert loop.peak_bytes <= budget


@pytest.mark.gpu
def test_one_at_a_time_fifo_latency(built):
    reqs = _mix_requests(0.05)[:3]
    res, busy, prep = one_at_a_time(reqs, precision="fp64", chunk_steps=16, max_steps=17)
    assert busy > prep > 0 and all(r.steps == 17 for r in res)
    for a, b in zip(res, res[1:]):
        assert b.admitted_s >= a.finished_s - 1e-12


def test_active_work_cap_admits_in_order(fake_batch):
    """With room for two requests' elements, the third waits until one retires; arrival order is
    kept and no more than the cap runs at once."""
    reqs = _reqs([(16, 1), (16, 1), (16, 1), (16, 1)], gap=0.01)
    ne = instance_mesh(reqs[0].instance)[0].n_elements
    FakeBatch.lag = 200
    try:
        loop = ServingLoop(prep="thread", chunk_steps=64, tol=1e-3, max_steps=100, window_s=0.0,
                           max_active_elements=2 * ne)
        res = loop.run(reqs, realtime=True)
    finally:
        FakeBatch.lag = 2
    assert len(res) == 4 and all(r.converged for r in res)
    assert loop.max_concurrent <= 2
    admitted = [r.admitted_s for r in res]
    assert admitted == sorted(admitted)
    assert min(res[2].admitted_s, res[3].admitted_s) >= min(res[0].finished_s, res[1].finished_s)


def test_freed_slots_take_waiting_requests(fake_batch):
    """With room for two requests' elements in flight, requests 2 and 3 (same order and size) wait
    and then take the slots that requests 0 and 1 free, inside the running cohorts: no new context,
    admission in arrival order, each result on its own check schedule."""
    reqs = _reqs([(16, 1), (16, 1), (16, 1), (16, 1)], gap=0.0)
    ne = instance_mesh(reqs[0].instance)[0].n_elements
    FakeBatch.lag = 200                      # chunks stay in flight while every request is prepared
    try:
        loop = ServingLoop(prep="thread", chunk_steps=8, tol=1e-6, max_steps=1000, window_s=0.0,
                           max_active_elements=2 * ne, max_cohort_elements=4 * ne)
        res = loop.run(reqs, realtime=False)
    finally:
        FakeBatch.lag = 2
    assert len(res) == 4 and all(r.converged and r.steps == 25 for r in res)
    assert loop.slot_reuses == 2 and FakeBatch.replaced == 2
    # requests 0 and 1 start one or two cohorts (as their preparation finishes); 2 and 3 start none
    assert loop.cohorts_formed == FakeBatch.created <= 2
    assert loop.max_concurrent <= 2
    # (requests still being prepared hold back none behind them, so which two ran first depends on
    # preparation; the two admitted last waited for a finish)
    first, last = sorted(res, key=lambda r: r.admitted_s)[:2], sorted(res, key=lambda r: r.admitted_s)[2:]
    assert min(r.admitted_s for r in last) >= min(r.finished_s for r in first)


def test_slot_reuse_respects_fit_and_waste():
    from dgm_in_rust_b200.serving import _fits, _room
    assert _room((100, 140, 20, 2), 1.5) == (150, 210, 30, 3)
    assert _fits((150, 200, 30, 2), (150, 210, 30, 3)) and not _fits((151, 200, 30, 2), (150, 210, 30, 3))
