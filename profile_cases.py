"""Fixed single-GPU cases of the hot kernels, for timing and for profilers.

    python profile_cases.py bcd --n 8192 --m 8192 --precision mixed
    python profile_cases.py splr --n 4096 --m 4096 --density 0.1
    python profile_cases.py backward --n 2048 --m 2560
    python profile_cases.py precision --n 16384 --algo splr
    python profile_cases.py points --n 16384 --m 16384 --d 32 --iters 20
    python profile_cases.py batch --n 512 --m 640 --batch 16

Each case builds a seeded synthetic problem on cuda:0, runs it once to warm
up, then times `--reps` runs with CUDA events on the launching stream and
prints one JSON line.  Achieved bandwidth uses algorithmic bytes:
  bcd       2 * n * m * sizeof(M) per iteration (one row pass + one column
            pass, each reading M once), iterations fixed by --iters (tol 0);
  backward  n * m * 8 per PCG iteration (one fused pass over T), plus the
            right-hand-side and gradient-assembly passes (2 * n * m * 8 reads
            of T and G, n * m * 8 written).
The SPLR case reports wall time, iterations and the direction-solve path.
The points case times Sinkhorn iterations on a cost recomputed from BF16
point clouds on the tensor cores (never stored) for a fixed iteration
count, and, with --compare, the stored-cost passes on the same cost;
throughput is reported as cost elements per second (one exponential
each) against the nominal SFU rate of 148 SMs x 16 ex2/clk x 1.965 GHz.
The batch case times splr_ot_batch (forward and backward of a weighted sum
of the plans) against one splr_ot call per problem in a loop.
The precision case solves the precision-form problem (X, Y ~ N(0, I_32),
M = |x - y|^2 / median stored in FP32, Dirichlet(1) marginals floored at
1e-7, eta = 1e-3) in mixed precision once and reports its time, iterations
and the marginal errors of the returned duals evaluated in FP64 (torch, on
the FP32-valued M upcast exactly).
"""

from __future__ import annotations

import argparse
import json
import os

import sys

import torch

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from curegot_backward_b200 import _solvers, synthetic  # noqa: E402
from curegot_backward_b200.backward import solve_backward  # noqa: E402


def _peak():
    p = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _gauss(n, m, d, seed, dev, dtype):
    spec = synthetic.StreamSpec(0, n, m, d, 0.0, "bcd", seed, 0.0)
    return synthetic.stream_problem(spec, dev, dtype)


def _time(fn, reps):
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = None
    for _ in range(reps):
        out = fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps, out


def case_bcd(a):
    import curegot_backward_b200 as cg
    cg.set_bcd_cluster_path(a.path != "multi")
    cg.set_bcd_staging(a.staging == "on")
    dev = torch.device("cuda", 0)
    dtype = torch.float32 if a.precision == "mixed" else torch.float64
    M, am, bm = _gauss(a.n, a.m, a.d, a.seed, dev, dtype)
    run = lambda: _solvers._bcd_device(M, am, bm, a.eta, 0.0, a.iters, None, a.precision,
                                       want_plan=False)
    ms, out = _time(run, a.reps)
    niter = out[0]
    bytes_ = 2.0 * a.n * a.m * M.element_size() * niter
    gbs = bytes_ / (ms / 1e3) / 1e9
    peak, kind = _peak()
    return {"case": "bcd", "path": a.path, "staging": a.staging, "l2pf": a.l2pf, "lse": a.lse, "n": a.n, "m": a.m,
            "precision": a.precision, "eta": a.eta,
            "iterations": niter, "ms_per_solve": ms, "us_per_iteration": 1e3 * ms / niter,
            "algorithmic_GBps": gbs, "peak_GBps": peak, "peak_kind": kind, "frac": gbs / peak}


def case_c0(a):
    """Sinkhorn at the C0 configuration (n = 512, m = 640, X, Y ~ U[0,1]^8,
    M = mean squared difference, uniform marginals, eta = 0.05, tol = 1e-8):
    the reference's own GPU solver (cuda_sinkhorn_bcd built from its sources
    into oracle/_ref, device-resident inputs and outputs) beside this
    library's FP64 solver (cluster path and multi-CTA passes) and mixed
    solver, each timed with CUDA events over --reps solves, plan included."""
    import ctypes

    import numpy as np

    import curegot_backward_b200 as cg
    import oracle
    dev = torch.device("cuda", 0)
    M, an, bn, eta = synthetic.config0()
    Md = torch.tensor(M, device=dev)
    ad, bd = torch.tensor(an, device=dev), torch.tensor(bn, device=dev)
    n, m = M.shape
    P = torch.empty((n, m), dtype=torch.float64, device=dev)
    dual = torch.empty(n + m, dtype=torch.float64, device=dev)
    out = {"case": "c0", "n": n, "m": m, "eta": eta, "tol": 1e-8, "reps": a.reps}
    if oracle.ref_bcd_available():
        ms, it = _time(lambda: oracle.ref_bcd_device(Md.data_ptr(), ad.data_ptr(), bd.data_ptr(),
                                                     P.data_ptr(), eta, 1e-8, 100000, n, m,
                                                     dual.data_ptr()), a.reps)
        ref_dual = dual.clone()
        out["reference_gpu"] = {"ms_per_solve": ms, "niter": it}
    else:
        ref_dual = None
        out["reference_gpu"] = None
    for name, cluster, prec in (("ours_fp64_cluster", True, "fp64"),
                                ("ours_fp64_passes", False, "fp64"),
                                ("ours_mixed_cluster", True, "mixed")):
        cg.set_bcd_cluster_path(cluster)
        Mx = Md if prec == "fp64" else Md.float()
        ms, res = _time(lambda: _solvers._bcd_device(Mx, ad, bd, eta, 1e-8, 100000, None, prec),
                        a.reps)
        entry = {"ms_per_solve": ms, "niter": res[0]}
        if ref_dual is not None and prec == "fp64":
            d = (res[2] - ref_dual).abs().max().item()
            entry["max_dual_diff_vs_reference"] = d
        out[name] = entry
    cg.set_bcd_cluster_path(True)
    if out["reference_gpu"]:
        out["speedup_fp64_cluster"] = out["reference_gpu"]["ms_per_solve"] / \
            out["ours_fp64_cluster"]["ms_per_solve"]
    return out


def case_splr(a):
    import curegot_backward_b200 as cg
    dev = torch.device("cuda", 0)
    dtype = torch.float32 if a.precision == "mixed" else torch.float64
    M, am, bm = _gauss(a.n, a.m, a.d, a.seed, dev, dtype)
    if a.solver:
        cg.set_direction_solver(a.solver)
    kw = {} if a.density is None else {"density": a.density}
    run = lambda: cg.torch.sinkhorn_splr(M, am, bm, a.eta, tol=a.tol, max_iter=1000,
                                         precision=a.precision, **kw)
    ms, out = _time(run, a.reps)
    return {"case": "splr", "l2pf": a.l2pf, "n": a.n, "m": a.m, "precision": a.precision, "eta": a.eta,
            "density": a.density, "iterations": out["niter"], "ms_per_solve": ms,
            "direction_solver": cg.last_direction_solver()}


def case_backward(a):
    import curegot_backward_b200 as cg
    dev = torch.device("cuda", 0)
    M, am, bm = _gauss(a.n, a.m, a.d, a.seed, dev, torch.float64)
    out = cg.torch.sinkhorn_splr_bwd(M, am, bm, a.eta, 1e-8, 1000, 0)
    dual, ctx = out["dual"], out["context"]
    T = torch.exp((dual[: a.n, None] + dual[None, a.n:] - M) / a.eta)
    G = 2.0 * T
    run = lambda: solve_backward(T, G, ctx, a.eta, preconditioner=a.precond, tol=1e-12)
    ms, res = _time(run, a.reps)
    it = res["iterations"]
    bytes_ = a.n * a.m * 8.0 * (it + 3)
    gbs = bytes_ / (ms / 1e3) / 1e9
    peak, kind = _peak()
    return {"case": "backward", "n": a.n, "m": a.m, "eta": a.eta, "preconditioner": a.precond,
            "pcg_iterations": it, "ms_per_solve": ms, "algorithmic_GBps": gbs,
            "peak_GBps": peak, "peak_kind": kind, "frac": gbs / peak}


def dual_objective(M64, a, b, dual, eta, rows_per_chunk=1024):
    """f = eta * sum(T) - <alpha, a> - <beta, b> in FP64 (row chunks), the
    dual objective the SPLR solver minimises."""
    n, m = M64.shape
    al, be = dual[:n].double(), dual[n:].double()
    tot = 0.0
    for i0 in range(0, n, rows_per_chunk):
        i1 = min(n, i0 + rows_per_chunk)
        tot += float(torch.exp((al[i0:i1, None] + be[None, :] - M64[i0:i1]) / eta).sum())
    return eta * tot - float((al * a).sum()) - float((be * b).sum())


def fp64_marginal_errors(M, a, b, dual, eta, rows_per_chunk=1024):
    """||T 1 - a||_2 and ||T^T 1 - b||_2 of T = exp((alpha_i + beta_j - M_ij) / eta),
    evaluated in FP64 in row chunks."""
    n, m = M.shape
    al, be = dual[:n].double(), dual[n:].double()
    rows = torch.empty(n, dtype=torch.float64, device=M.device)
    cols = torch.zeros(m, dtype=torch.float64, device=M.device)
    for i0 in range(0, n, rows_per_chunk):
        i1 = min(n, i0 + rows_per_chunk)
        T = torch.exp((al[i0:i1, None] + be[None, :] - M[i0:i1].double()) / eta)
        rows[i0:i1] = T.sum(1)
        cols += T.sum(0)
    return float(torch.linalg.norm(rows - a)), float(torch.linalg.norm(cols - b))


def case_precision(a):
    dev = torch.device("cuda", 0)
    M, am, bm, eta = synthetic.config2(device=dev, n=a.n, m=a.n)
    if a.algo == "bcd":
        run = lambda: _solvers._bcd_device(M, am, bm, eta, a.tol, a.max_iter, None, "mixed",
                                           want_plan=False)
    else:
        run = lambda: _solvers._splr_device(M, am, bm, eta, a.tol, a.max_iter, 0, None, "mixed",
                                            0.01, 1e-3, 30, 3, want_plan=False)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = run()
    e1.record()
    torch.cuda.synchronize()
    niter, dual = (out[0], out[2]) if a.algo == "bcd" else (out["niter"], out["dual"])
    seconds = e0.elapsed_time(e1) / 1e3
    row_err, col_err = fp64_marginal_errors(M, am, bm, dual, eta)
    res = {"case": "precision", "algo": a.algo, "n": a.n, "m": a.n, "eta": eta,
           "M_dtype": "float32", "iterations": int(niter), "max_iter": a.max_iter,
           "seconds": seconds, "fp64_row_err": row_err, "fp64_col_err": col_err, "tol": a.tol}
    if a.fp64_reference:
        # objective error against the plain FP64 solve of the same FP32-valued
        # M (upcast exactly): the FP64 path is the one held to the oracle
        M64 = M.double()
        if a.algo == "bcd":
            _, _, ref = _solvers._bcd_device(M64, am, bm, eta, a.tol, a.max_iter, None, "fp64",
                                             want_plan=False)
        else:
            ref = _solvers._splr_device(M64, am, bm, eta, a.tol, a.max_iter, 0, None, "fp64",
                                        0.01, 1e-3, 30, 3, want_plan=False)["dual"]
        f_mixed = dual_objective(M64, am, bm, dual, eta)
        f_ref = dual_objective(M64, am, bm, ref, eta)
        del M64
        res["objective_fp64_ref"] = f_ref
        res["rel_objective_err"] = abs(f_mixed - f_ref) / abs(f_ref)
    return res


def case_points(a):
    from curegot_backward_b200.points import cost_from_points, sinkhorn_bcd_points
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(a.seed)
    X = torch.rand(a.n, a.d, generator=g, device=dev).bfloat16()
    Y = torch.rand(a.m, a.d, generator=g, device=dev).bfloat16()
    am = torch.full((a.n,), 1.0 / a.n, dtype=torch.float64, device=dev)
    bm = torch.full((a.m,), 1.0 / a.m, dtype=torch.float64, device=dev)
    run = lambda: sinkhorn_bcd_points(X, Y, am, bm, a.eta, tol=0.0, max_iter=a.iters,
                                      precision=a.precision)
    ms, out = _time(run, a.reps)
    it = out["niter"]
    elems = 2.0 * a.n * a.m * it
    sfu_peak = 148 * 16 * 1.965e9
    res = {"case": "points", "n": a.n, "m": a.m, "d": a.d, "eta": a.eta,
           "precision": a.precision, "iterations": it, "ms_per_iteration": ms / it,
           "elements_per_s": elems / (ms / 1e3), "sfu_nominal_per_s": sfu_peak,
           "frac_sfu_nominal": elems / (ms / 1e3) / sfu_peak,
           "point_bytes_per_pass": (a.n + a.m) * a.d * 2}
    if a.compare:
        M = cost_from_points(X, Y)
        if a.precision == "fp64":
            M = M.double()
        run2 = lambda: _solvers._bcd_device(M, am, bm, a.eta, 0.0, a.iters, None, a.precision,
                                            want_plan=False)
        ms2, _ = _time(run2, a.reps)
        res["stored_cost_ms_per_iteration"] = ms2 / a.iters
        del M
    return res


def case_batch(a):
    import curegot_backward_b200 as cg
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(a.seed)
    B, n, m = a.batch, a.n, a.m
    X = torch.rand(B, n, a.d, generator=g, device=dev, dtype=torch.float64)
    Y = torch.rand(B, m, a.d, generator=g, device=dev, dtype=torch.float64)
    M = ((X[:, :, None, :] - Y[:, None, :, :]) ** 2).mean(-1)
    am = torch.full((B, n), 1.0 / n, dtype=torch.float64, device=dev)
    bm = torch.full((B, m), 1.0 / m, dtype=torch.float64, device=dev)
    W = torch.rand(B, n, m, generator=g, device=dev, dtype=torch.float64)

    def batched():
        Mr = M.clone().requires_grad_(True)
        (cg.torch.splr_ot_batch(Mr, am, bm, eta=a.eta, tol=a.tol) * W).sum().backward()
        return Mr.grad

    def loop():
        Mr = M.clone().requires_grad_(True)
        T = torch.stack([cg.torch.splr_ot(Mr[i], am[i], bm[i], eta=a.eta, tol=a.tol)
                         for i in range(B)])
        (T * W).sum().backward()
        return Mr.grad

    ms_b, gb = _time(batched, a.reps)
    ms_l, gl = _time(loop, a.reps)
    return {"case": "batch", "batch": B, "n": n, "m": m, "eta": a.eta, "tol": a.tol,
            "ms_batch": ms_b, "ms_loop": ms_l, "speedup": ms_l / ms_b,
            "grads_bitwise_equal": bool(torch.equal(gb, gl))}


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    p.add_argument("case", choices=["bcd", "splr", "backward", "precision", "points", "batch",
                                    "c0"])
    p.add_argument("--n", type=int, default=8192)
    p.add_argument("--m", type=int, default=8192)
    p.add_argument("--d", type=int, default=16)
    p.add_argument("--eta", type=float, default=0.01)
    p.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    p.add_argument("--iters", type=int, default=100, help="bcd: fixed iteration count")
    p.add_argument("--path", default="auto", choices=["auto", "multi"],
                   help="bcd: auto = cluster-resident solver when the problem fits")
    p.add_argument("--density", type=float, default=None, help="splr: density_max kwarg")
    p.add_argument("--l2pf", type=int, default=None, help="L2 prefetch distance of the Sinkhorn and plan passes")
    p.add_argument("--lse", default="shifted", choices=["shifted", "online"],
                   help="Sinkhorn passes: shifted sums or running maximum in every pass")
    p.add_argument("--staging", default="off", choices=["on", "off"],
                   help="bcd: shared-memory staging of the passes")
    p.add_argument("--solver", default=None, choices=[None, "auto", "dense", "peel", "sparse"])
    p.add_argument("--tol", type=float, default=1e-8)
    p.add_argument("--precond", default="diag", choices=["none", "diag", "splr"])
    p.add_argument("--reps", type=int, default=3)
    p.add_argument("--seed", type=int, default=7)
    p.add_argument("--algo", default="splr", choices=["bcd", "splr"], help="precision case")
    p.add_argument("--max-iter", type=int, default=100000, help="precision case")
    p.add_argument("--fp64-reference", action="store_true",
                   help="precision case: also solve in plain FP64 and report the relative "
                        "objective error of the mixed solution")
    p.add_argument("--compare", action="store_true", help="points: also time the stored cost")
    p.add_argument("--batch", type=int, default=16, help="batch case: problems per batch")
    a = p.parse_args(argv)
    import curegot_backward_b200 as cg
    if a.l2pf is not None:
        cg.set_bcd_l2_prefetch(a.l2pf)
    cg.set_bcd_shifted_lse(a.lse == "shifted")
    res = {"bcd": case_bcd, "splr": case_splr, "backward": case_backward,
           "precision": case_precision, "points": case_points, "batch": case_batch,
           "c0": case_c0}[a.case](a)
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
