"""Host-side logic that needs no GPU: the bench's closed-loop client and
stream assembly, and the argument guards in front of the native entry
points (they must reject bad operands before any kernel could read past a
buffer)."""
import dataclasses
import heapq

import pytest
import torch

import bench
from curegot_backward_b200 import _solvers
from curegot_backward_b200.synthetic import stream_specs


class FakeEngine:
    """Completes each request `service` seconds (simulated) after submission,
    with at most `lanes` requests served at once; records the in-flight
    high-water mark seen by the client."""

    def __init__(self, service=0.001, lanes=1000):
        self.t = 0.0
        self.service, self.lanes = service, lanes
        self.pending = []  # (done_time, id, tag, t_submit)
        self.next_id = 0
        self.max_in_flight = 0

    def clock(self):
        return self.t

    def submit(self, M, a, b, eta, algo, tol, tag):
        rid = self.next_id
        self.next_id += 1
        start = self.t
        if len(self.pending) >= self.lanes:
            start = max(self.t, sorted(p[0] for p in self.pending)[len(self.pending) - self.lanes])
        heapq.heappush(self.pending, (start + self.service, rid, tag, self.t))
        self.max_in_flight = max(self.max_in_flight, len(self.pending))
        return rid

    def poll(self, wait_ms=0):
        if not self.pending:
            self.t += wait_ms / 1000.0
            return []
        done_t = self.pending[0][0]
        self.t = max(self.t, min(done_t, self.t + wait_ms / 1000.0))
        out = []
        while self.pending and self.pending[0][0] <= self.t:
            d, rid, tag, ts = heapq.heappop(self.pending)
            out.append({"id": rid, "tag": tag, "t_done": d, "t_submit": ts, "t_admit": ts,
                        "status": 0, "niter": 1})
        return out


def _probs(k, seed=0, rate=None):
    return [(s, None, None, None) for s in stream_specs(k, seed=seed, rate=rate, n_hi=256)]


@pytest.mark.parametrize("window", [1, 5, 24])
def test_closed_loop_keeps_window(window):
    eng = FakeEngine()
    probs = _probs(40)
    res = bench.run_engine_step(eng, probs, False, 0.0, window)
    assert sorted(r["tag"] for r in res) == list(range(40))
    assert eng.max_in_flight == min(window, 40)
    # latency runs from each request's own submission
    assert all(abs(r["latency"] - eng.service) < 1e-12 for r in res)


def test_saturation_without_window_submits_everything():
    eng = FakeEngine()
    res = bench.run_engine_step(eng, _probs(17), False, 0.0, 0)
    assert len(res) == 17 and eng.max_in_flight == 17


def test_stream_of_concatenates_steps():
    steps = [_probs(5, seed=s, rate=200.0) for s in range(3)]
    flat = bench.stream_of(steps, 200.0)
    assert len(flat) == 15
    arr = [p[0].arrival for p in flat]
    assert arr == sorted(arr)
    # each step's offsets continue from the previous step's last arrival
    base = max(p[0].arrival for p in steps[0])
    assert flat[5][0].arrival == pytest.approx(base + steps[1][0][0].arrival)
    # saturation keeps the specs as they are
    flat0 = bench.stream_of(steps, 0.0)
    assert all(a[0] is b[0] for a, b in zip(flat0, [p for st in steps for p in st]))


def test_poisson_arrivals_are_honoured():
    eng = FakeEngine(service=1e-4)
    probs = bench.stream_of([_probs(10, seed=3, rate=500.0)], 500.0)
    res = bench.run_engine_step(eng, probs, False, 500.0)
    assert len(res) == 10
    for r in res:
        assert r["t_submit"] >= r["spec"].arrival - 1e-9


def test_device_operands_rejected_before_native_code():
    M32 = torch.zeros(4, 3, dtype=torch.float32)
    M64 = torch.zeros(4, 3, dtype=torch.float64)
    a, b = torch.full((4,), 0.25, dtype=torch.float64), torch.full((3,), 1 / 3, dtype=torch.float64)
    with pytest.raises(TypeError):
        _solvers._device_operands(M32, a, b, "fp64")  # FP32 M read as FP64: 2x overrun
    with pytest.raises(TypeError):
        _solvers._device_operands(M64, a, b, "mixed")
    with pytest.raises(ValueError):
        _solvers._device_operands(M64, a, b, "fp64")  # host tensors
    with pytest.raises(TypeError):
        _solvers._device_operands(M32, a.float(), b, "mixed")


def test_points_arguments_rejected_without_gpu():
    from curegot_backward_b200.points import _check_points
    X = torch.zeros(8, 4, dtype=torch.bfloat16)
    with pytest.raises(TypeError):
        _check_points(X.float(), X)
    with pytest.raises(ValueError):
        _check_points(X, X[:, :2])
    with pytest.raises(ValueError):
        _check_points(X, X)  # host tensors


def test_cpu_sample_full_budget_solves_everything():
    """With a budget above the whole set's cost, every request is solved
    (p = 1) and the estimate is the measured total."""
    from curegot_backward_b200.synthetic import stream_problem
    specs = stream_specs(6, seed=5, n_lo=8, n_hi=48)
    got = bench.cpu_sample(specs, lambda i: stream_problem(specs[i], device="cpu"), 1e9)
    sps, cores, desc = got
    assert desc.startswith("6 of 6 requests")
    assert sps > 0 and cores >= 1


def test_cpu_sample_estimate_is_unbiased(monkeypatch):
    """Horvitz-Thompson: with a fake oracle whose solve time equals the
    predicted cost times a per-request factor, the mean of 1/solves-rate over
    seeds converges to the true total time per request."""
    import oracle
    specs = stream_specs(40, seed=9, n_hi=4096)
    times = {id(s): 1e-9 * bench._predicted_cpu_cost(s) * (0.5 + (k % 3)) for k, s in
             enumerate(specs)}
    current = {}

    class FakeM:
        def double(self):
            return self

        def numpy(self):
            return None

    def get(i):
        current["s"] = specs[i]
        return FakeM(), FakeM(), FakeM()

    clock = {"t": 0.0}
    monkeypatch.setattr(bench.time, "perf_counter", lambda: clock["t"])

    def fake_solve(*a, **k):
        clock["t"] += times[id(current["s"])]
        return {"niter": 1}

    monkeypatch.setattr(oracle, "bcd", fake_solve)
    monkeypatch.setattr(oracle, "splr", fake_solve)
    true_total = sum(times.values())
    budget = 0.2 * true_total
    est = [len(specs) / bench.cpu_sample(specs, get, budget, seed=sd)[0] for sd in range(400)]
    import numpy as np
    assert abs(np.mean(est) - true_total) < 0.05 * true_total


def test_per_step_rates():
    res = [{"t_submit": 0.0, "t_done": 0.1 * (k + 1)} for k in range(20)]
    rates = bench.per_step_rates(res, 5)
    assert len(rates) == 4
    assert all(abs(r - 10.0) < 1e-9 for r in rates)
