#!/usr/bin/env python
"""Serving-stream benchmark: solves/s and p50/p99 latency of mixed-size
entropic-OT requests at <= 1e-8 marginal error (FP64-checked), compared with
the plain FP64 path.

Workload (one "step" = one batch of requests of the serving stream):
n, m log-uniform in [64, 8192], d in {8, 32}, costs = squared distances of
Gaussian point clouds / max, eta in {0.1, 0.05, 0.01}, 70% Sinkhorn (BCD) /
30% SPLR, tol 1e-8, uniform marginals, all requests of a step arriving at its
start (saturation) unless --rate is given (Poisson arrivals).  Seeded
synthetic data with the stream's shapes and distributions.

Arms
  ours (default)   the continuous-batching engine (FP32 cost matrix, FP64 duals,
                   FP64-confirmed stop test); `value` with inputs resident in
                   HBM, `e2e` with host inputs (H2D / D2H inside the timed
                   region); plus the plain FP64 path one request at a time on
                   the same requests.
  --impl reference the reference algorithm on the host cores (the CPU
                   restatement in oracle/, the reference ships no CPU solver)
                   on the same timed requests: a seeded probability sample of
                   them is solved and the CPU time of the whole request set is
                   estimated without bias (Horvitz-Thompson), then turned
                   into solves/s.

Multi-GPU: requests are independent, so ranks are replicas that each take
their own share of the stream (no collective on the data path); timing is
the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

# Every kernel is loaded when the CUDA context starts, not at its first
# launch: with lazy loading (the CUDA 12 default) the first launch of a
# kernel variant inside the timed region (a cuSOLVER potrf size class, a
# pass template) held every stream of the process for 0.3-1 s on a fresh
# box.  A serving process pays this once at start-up (2-5 s).  Set
# CUDA_MODULE_LOADING=LAZY to measure without it.
os.environ.setdefault("CUDA_MODULE_LOADING", "EAGER")

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "solves/s + p99 latency, mixed-size OT stream @1e-8 marginal err, vs plain FP64"
TOL = 1e-8
WORKLOAD = ("serving stream: n,m log-uniform [64,8192], d in {8,32}, Gaussian clouds/max, "
            "eta in {0.1,0.05,0.01}, 70% BCD / 30% SPLR, tol 1e-8, uniform marginals")
SPLR_WORKERS = 32
IN_FLIGHT = 24
CHUNK = 8


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=8)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--requests", type=int, default=48, help="requests per step per GPU")
    p.add_argument("--rate", type=float, default=0.0, help="Poisson rate (req/s); 0 = saturation")
    p.add_argument("--n-hi", type=int, default=8192)
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--cpu-budget", type=float, default=15.0, help="seconds of CPU work")
    p.add_argument("--budget-gb", type=float, default=120.0)
    p.add_argument("--seed", type=int, default=4)
    p.add_argument("--splr-workers", type=int, default=SPLR_WORKERS)
    p.add_argument("--chunk", type=int, default=CHUNK, help="Sinkhorn ticks per graph launch")
    p.add_argument("--in-flight", type=int, default=IN_FLIGHT,
                   help="saturation: requests kept in flight by the closed-loop client")
    return p.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_setup(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _reduce_over_ranks(x, world, op_name):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    # NCCL reduces device tensors; gloo (the CPU test harness) host tensors
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(x, world):
    return _reduce_over_ranks(x, world, "MAX")


def sum_over_ranks(x, world):
    return _reduce_over_ranks(x, world, "SUM")


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def step_specs(args, step, rank, warm):
    from curegot_backward_b200.synthetic import stream_specs
    # warm-up steps draw from the same size distribution (other seeds), so
    # first-use costs of every size class stay out of the timed steps
    count = args.requests
    n_hi = args.n_hi
    seed = args.seed * 1000003 + (step + (1 << 16 if warm else 0)) * 131 + rank
    return stream_specs(count, seed=seed, rate=args.rate or None, n_hi=n_hi)


def make_step(specs, device):
    import torch
    from curegot_backward_b200.synthetic import stream_problem
    probs = []
    for s in specs:
        M, a, b = stream_problem(s, device=device)
        probs.append((s, M, a, b))
    torch.cuda.synchronize()
    return probs


def to_host_pinned(probs):
    out = []
    for s, M, a, b in probs:
        out.append((s, M.cpu().pin_memory(), a.cpu().pin_memory(), b.cpu().pin_memory()))
    return out


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"cg_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx.append(float(f[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        except OSError:
            return None
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# engine passes
# ---------------------------------------------------------------------------
def run_engine_step(eng, probs, host, rate, window=0):
    """Serve a list of requests and wait for all of them.

    rate > 0: Poisson arrivals (each request's offset is honoured).
    rate == 0 (saturation): a closed loop that keeps `window` requests in
    flight (all of them when window is 0), submitting the next request as
    each result comes back.  Latency runs from a request's submission (or
    arrival) to its result."""
    t0 = eng.clock()
    pending = {}
    k = 0
    results = []
    while k < len(probs) or pending:
        now = eng.clock() - t0
        while k < len(probs) and (probs[k][0].arrival <= now if rate else
                                  (not window or len(pending) < window)):
            s, M, a, b = probs[k]
            t_sub = eng.clock()
            rid = eng.submit(M, a, b, eta=s.eta, algo=s.algo, tol=TOL, tag=k)
            pending[rid] = (s, t0 + s.arrival if rate else t_sub)
            k += 1
        wait = 1 if (k < len(probs) and rate) else 50
        for r in eng.poll(wait_ms=wait):
            s, arr = pending.pop(r["id"])
            r["latency"] = r["t_done"] - arr
            r["spec"] = s
            results.append(r)
    return results


def stream_of(steps, rate):
    """Concatenate the steps' requests into one stream; with Poisson arrivals,
    each step's offsets continue from the previous step's last arrival."""
    import dataclasses
    out, base = [], 0.0
    for probs in steps:
        last = 0.0
        for s, M, a, b in probs:
            s2 = dataclasses.replace(s, arrival=base + s.arrival) if rate else s
            out.append((s2, M, a, b))
            last = max(last, s.arrival)
        base += last
    return out


def timed_engine_pass(eng, steps, host, rate, world, window):
    """One timed region over all steps: the requests of the K steps form one
    stream (closed loop of `window` in flight, or Poisson arrivals), bracketed
    by a barrier and a device synchronize on both sides."""
    import torch
    probs = stream_of(steps, rate)
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    res = run_engine_step(eng, probs, host, rate, window)
    e1.record()
    torch.cuda.synchronize()
    barrier(world)
    total = max_over_ranks(e0.elapsed_time(e1), world)
    # map stream positions back to (step, index in step) and the step's spec
    where = [(i, k, p[0]) for i, probs_ in enumerate(steps) for k, p in enumerate(probs_)]
    for r in res:
        r["step"], r["tag"], r["spec"] = where[r["tag"]]
    return total, res


def plain_fp64_pass(steps, world):
    """The plain FP64 path, one request at a time, inputs resident in HBM.
    Returns the per-step times and each request's duals (keyed by the spec's
    id), which the accuracy report uses as the FP64 reference solution."""
    import torch
    from curegot_backward_b200 import _solvers
    step_ms = []
    duals = {}
    for probs in steps:
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for s, M64, a, b in probs:
            if s.algo == "bcd":
                _, _, dual = _solvers._bcd_device(M64, a, b, s.eta, TOL, 100000, None, "fp64",
                                                  want_plan=False)
            else:
                dmax = min(10.0 / min(s.n, s.m), 1.0)
                dual = _solvers._splr_device(M64, a, b, s.eta, TOL, 1000, 0, None, "fp64", dmax,
                                             1e-3, 30, 3, want_plan=False)["dual"]
            duals[id(s)] = dual
        e1.record()
        torch.cuda.synchronize()
        barrier(world)
        step_ms.append(max_over_ranks(e0.elapsed_time(e1), world))
    return step_ms, duals


def _dual_objective(M64, al, be, a, b, eta):
    """f(alpha, beta) = eta * sum(T) - <alpha, a> - <beta, b>, the dual objective
    the SPLR solver minimises, with T = exp((alpha + beta - M) / eta), in FP64."""
    import torch
    T = torch.exp((al[:, None] + be[None, :] - M64) / eta)
    return float(eta * T.sum() - (al * a).sum() - (be * b).sum()), T


def accuracy_report(probs, results, plain_duals):
    """FP64-checked errors of the engine's results, on the FP32-valued M upcast
    exactly to FP64: the row and column marginal errors ||T1 - a||_2,
    ||T^T 1 - b||_2, and the relative dual-objective error against the plain
    FP64 path's solution of the same request (None without the plain pass)."""
    import torch
    out = []
    by_tag = {r["tag"]: r for r in results}
    for k, (s, M, a, b) in enumerate(probs):
        r = by_tag[k]
        M64 = M.double()
        dual = r["dual"].to(M.device)
        f, P = _dual_objective(M64, dual[: s.n], dual[s.n:], a, b, s.eta)
        e_r = float(torch.linalg.norm(P.sum(1) - a))
        e_c = float(torch.linalg.norm(P.sum(0) - b))
        del P
        e_f = None
        ref = plain_duals.get((id(s))) if plain_duals is not None else None
        if ref is not None:
            ref = ref.to(M.device)
            f64, P = _dual_objective(M64, ref[: s.n], ref[s.n:], a, b, s.eta)
            del P
            e_f = abs(f - f64) / max(abs(f64), 1e-300)
        out.append({"algo": s.algo, "row": e_r, "col": e_c, "obj": e_f, "niter": r["niter"]})
        del M64
    return out


def summarize_accuracy(errs, ok):
    acc = {"all_status_ok": ok}
    for algo in ("bcd", "splr"):
        sub = [e for e in errs if e["algo"] == algo]
        if not sub:
            continue
        acc[f"max_row_marginal_err_{algo}"] = max(e["row"] for e in sub)
        acc[f"max_col_marginal_err_{algo}"] = max(e["col"] for e in sub)
        objs = [e["obj"] for e in sub if e["obj"] is not None]
        acc[f"max_rel_objective_err_{algo}"] = max(objs) if objs else None
    acc["frac_rows_and_cols_le_1e-8"] = float(np.mean([e["row"] <= TOL and e["col"] <= TOL
                                                         for e in errs]))
    acc["objective_reference"] = "plain FP64 path's solution of the same request, FP64-evaluated"
    return acc


# ---------------------------------------------------------------------------
# CPU restatement (reference algorithm on the host cores)
# ---------------------------------------------------------------------------
def _predicted_cpu_cost(spec):
    """Relative CPU cost of one request (only steers the sampling probabilities;
    the estimate stays unbiased whatever it predicts): BCD ~ n m iterations,
    SPLR ~ its passes over M plus the dense Cholesky of min(n, m - 1)."""
    nm = float(spec.n) * spec.m
    iters = 0.5 / spec.eta * 20.0
    if spec.algo == "bcd":
        return nm * iters
    k = float(min(spec.n, spec.m - 1))
    return 40.0 * (6.0 * nm + k ** 3 / 30.0)


def cpu_sample(specs, get_problem, budget_s, seed=0):
    """CPU solves/s of the oracle on a request set, estimated from a sample.

    Every request i is solved with probability p_i = min(1, lam / c_i), where
    c_i is its predicted cost and lam is set so that the expected CPU time
    (sum of min(c_i, lam), calibrated on the cheapest request, which is always
    solved) fits the budget.  The CPU time of the whole set is estimated by
    the Horvitz-Thompson sum of t_i / p_i over the solved requests, which is
    unbiased for any prediction; solves/s = requests / estimated time.
    get_problem(i) returns (M, a, b) as host tensors.  Returns (solves/s,
    threads, description)."""
    import oracle
    cores = oracle.num_threads()
    N = len(specs)
    cost = np.array([_predicted_cpu_cost(s) for s in specs])
    rng = np.random.default_rng(seed)
    u = rng.uniform(size=N)

    def solve(i):
        s = specs[i]
        M, a, b = get_problem(i)
        Mn, an, bn = M.double().numpy(), a.double().numpy(), b.double().numpy()
        t = time.perf_counter()
        if s.algo == "bcd":
            oracle.bcd(Mn, an, bn, s.eta, tol=TOL, max_iter=100000, want_plan=False)
        else:
            oracle.splr(Mn, an, bn, s.eta, tol=TOL, max_iter=1000, want_plan=False)
        return time.perf_counter() - t

    first = int(np.argmin(cost))
    solve(first)  # untimed: thread-pool start-up and first touches stay out of the calibration
    t_first = solve(first)
    sec_per_cost = t_first / max(cost[first], 1.0)
    # water-filling: sum_i min(c_i, lam) * sec_per_cost = remaining budget
    remaining = max(budget_s - t_first, 0.0) / max(sec_per_cost, 1e-30)
    others = np.delete(np.arange(N), first)
    cs = np.sort(cost[others])
    lam, acc = cs[-1] if len(cs) else 0.0, 0.0
    for k, c in enumerate(cs):
        rest = len(cs) - k
        if acc + c * rest >= remaining:
            lam = (remaining - acc) / rest
            break
        acc += c
    p = np.minimum(1.0, lam / np.maximum(cost, 1e-30))
    p[first] = 1.0
    est = t_first
    solved, cpu_s = 1, t_first
    for i in others:
        if u[i] < p[i]:
            t = solve(int(i))
            est += t / p[i]
            cpu_s += t
            solved += 1
    sps = N / max(est, 1e-12)
    desc = (f"{solved} of {N} requests solved by the CPU restatement ({cpu_s:.1f} s on {cores} "
            f"threads), each with probability min(1, lam/predicted cost); whole-set CPU time "
            f"estimated as the Horvitz-Thompson sum of t_i/p_i ({est:.1f} s)")
    return sps, cores, desc


def reference_arm(args, world, rank):
    """--impl reference: the reference algorithm on the host cores, on the
    requests the timed steps of the repo arm serve (same specs and seeds)."""
    if rank != 0:
        return
    import oracle
    from curegot_backward_b200.synthetic import stream_problem
    oracle.set_num_threads(os.cpu_count() or 1)
    specs = [s for st in range(args.steps) for s in step_specs(args, st, 0, False)]

    def get_problem(i):
        M, a, b = stream_problem(specs[i], device="cpu")
        return M, a, b

    budget = min(max(args.cpu_budget, 3.0 * args.steps), 90.0)
    value, cores, desc = cpu_sample(specs, get_problem, budget)
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * args.requests / value if value else None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "requests_per_step": args.requests,
                       "requests": len(specs)},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores,
                             "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def per_step_rates(results, per_step):
    """Solves/s of consecutive groups of `per_step` completions (in completion
    order): a throughput drop along the stream shows up here."""
    done = sorted(r["t_done"] for r in results)
    first = min(r["t_submit"] for r in results)
    out, prev = [], first
    for k in range(per_step - 1, len(done), per_step):
        out.append(per_step / max(done[k] - prev, 1e-9))
        prev = done[k]
    return out


def main():
    args = parse()
    import torch
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        reference_arm(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    from curegot_backward_b200 import _native
    from curegot_backward_b200.serving import OTEngine
    dev = torch.device("cuda", local if world > 1 else 0)
    _native.lib().cg_launch_count_reset()
    eng = OTEngine(budget_bytes=args.budget_gb * 1e9, max_batch=64, splr_workers=args.splr_workers,
                   chunk=args.chunk)

    # warm-up steps (untimed): device inputs, and host inputs for the e2e pass
    for st in range(args.warmup):
        probs = make_step(step_specs(args, st, rank, True), dev)
        run_engine_step(eng, probs, False, 0.0)
        if not args.no_e2e and st < 2:
            run_engine_step(eng, to_host_pinned(probs), True, 0.0)
    # timed steps: data generated up front (each step streams far more than L2)
    steps = [make_step(step_specs(args, st, rank, False), dev) for st in range(args.steps)]
    n_req = sum(len(p) for p in steps)
    sampler = ClockSampler(torch.cuda.current_device())
    s0 = eng.stats()
    l0 = _native.lib().cg_launch_count()
    sampler.start()
    total_ms, results = timed_engine_pass(eng, steps, False, args.rate, world, args.in_flight)
    clocks = sampler.stop()
    launches = _native.lib().cg_launch_count() - l0
    s1 = eng.stats()
    total_req = sum_over_ranks(n_req, world)
    value = total_req / (total_ms / 1000.0)
    lat = np.array([r["latency"] for r in results]) * 1000.0
    ok = all(r["status"] == 0 for r in results)
    step_rates = per_step_rates(results, args.requests)

    # roofline of the dominant kernels (the batched Sinkhorn row/column passes):
    # algorithmic bytes (2 n m sizeof(M) per tick of each running problem)
    # over the device time of the chunks that ran them, from CUDA events on
    # the batch streams.  DRAM traffic of these launches comes from an ncu
    # capture, not from this run, so it is not reported here.
    bytes_ = s1["bcd_bytes"] - s0["bcd_bytes"]
    gms = s1["bcd_gpu_ms"] - s0["bcd_gpu_ms"]
    peak, peak_kind = measured_hbm_peak()
    achieved = bytes_ / (gms / 1000.0) / 1e9 if gms > 0 else 0.0
    launches_per_chunk = 2 * args.chunk
    n_chunks = s1["chunks"] - s0["chunks"]

    # e2e: host inputs, copies inside the timed region
    e2e = None
    if not args.no_e2e:
        hsteps = [to_host_pinned(p) for p in steps]
        h2d = sum(p[1].numel() * 4 + (p[0].n + p[0].m) * 8 for st in hsteps for p in st)
        d2h = sum((p[0].n + p[0].m) * 8 for st in hsteps for p in st)
        e_ms, e_res = timed_engine_pass(eng, hsteps, True, args.rate, world, args.in_flight)
        e_lat = np.array([r["latency"] for r in e_res]) * 1000.0
        e2e = {"value": total_req / (e_ms / 1000.0), "unit": "solves/s",
               "h2d_bytes_per_step": int(h2d / max(args.steps, 1)),
               "d2h_bytes_per_step": int(d2h / max(args.steps, 1)),
               "latency_ms": {"p50": float(np.percentile(e_lat, 50)),
                              "p99": float(np.percentile(e_lat, 99))},
               "all_status_ok": all(r["status"] == 0 for r in e_res),
               "solves_per_s_by_step": per_step_rates(e_res, args.requests)}
        del hsteps

    # plain FP64 path on the same requests (also the FP64 reference solutions)
    plain, plain_duals = None, None
    if not args.no_plain:
        p64 = [[(s, M.double(), a, b) for (s, M, a, b) in probs] for probs in steps]
        p_ms, plain_duals = plain_fp64_pass(p64, world)
        pv = total_req / (sum(p_ms) / 1000.0)
        plain = {"value": pv, "unit": "solves/s", "ms_per_step": float(np.mean(p_ms)),
                 "engine_over_plain": value / pv}
        del p64

    # accuracy (FP64-checked, untimed)
    errs = []
    for k, probs in enumerate(steps):
        sub = [r for r in results if any(r["spec"] is p[0] for p in probs)]
        errs.extend(accuracy_report(probs, sub, plain_duals))
    accuracy = summarize_accuracy(errs, ok)
    plain_duals = None

    cpu = None
    if rank == 0:
        import oracle
        oracle.set_num_threads(os.cpu_count() or 1)
        specs0 = [p[0] for p in steps[0]]

        def get0(i):
            _, M, a, b = steps[0][i]
            return M.cpu(), a.cpu(), b.cpu()

        sps, cores, desc = cpu_sample(specs0, get0, args.cpu_budget)
        cpu = {"value": sps, "unit": "solves/s", "cores": cores, "kind": "port",
               "sample": desc + " (requests of the first timed step)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / max(args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32-M/f64", "data": "synthetic",
            "config": {"workload": WORKLOAD,
                       "requests_per_step": args.requests,
                       "arrivals": (f"poisson {args.rate}/s, one stream over the timed steps" if args.rate else
                                    f"saturation: closed loop over the timed steps' {n_req} requests, "
                                    f"{args.in_flight} in flight"),
                       "l2": "inputs larger than L2 (each step streams > 126 MB of M)",
                       "engine": f"max_batch 64, up to {args.splr_workers} SPLR solves in flight on "
                                 f"{(args.splr_workers + 7) // 8} scheduler threads, {args.chunk} ticks per graph launch",
                       "parallelism": f"replicas x{world}"},
            "latency_ms": {"p50": float(np.percentile(lat, 50)),
                           "p99": float(np.percentile(lat, 99)), "max": float(lat.max())},
            "solves_per_s_by_step": step_rates,
            "accuracy": accuracy,
            "plain_fp64": plain,
            "e2e": e2e,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if peak else None, "traffic": None,
                         "peak_kind": peak_kind,
                         "kernel": "bcd_row_kernel<float> + bcd_col_kernel<float> (batched)",
                         "note": f"{bytes_/1e9:.2f} GB algorithmic over {n_chunks} chunks of "
                                 f"{launches_per_chunk} launches ({gms:.1f} ms device time); "
                                 f"DRAM traffic of these kernels is in the committed ncu summaries"},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": int(launches),
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
