"""GPU parity of the Sinkhorn BCD path against the CPU oracle and against the
reference's own GPU BCD solver (oracle/_ref, built from the reference sources).

Bar (FP64 plain path): identical niter, duals within 1e-10 relative (to the
largest dual magnitude), plan within 1e-12 absolute.
"""
import numpy as np
import pytest
import torch

import curegot_backward_b200 as cg
import oracle

pytestmark = pytest.mark.gpu

DUAL_RTOL = 1e-10
PLAN_ATOL = 1e-12


def config0(seed=0):
    rng = np.random.default_rng(seed)
    n, m = 512, 640
    X = rng.uniform(size=(n, 8)); Y = rng.uniform(size=(m, 8))
    M = ((X[:, None, :] - Y[None, :, :]) ** 2).mean(-1)
    return M, np.full(n, 1.0 / n), np.full(m, 1.0 / m)


def rand_problem(n, m, seed):
    rng = np.random.default_rng(seed)
    M = rng.uniform(size=(n, m))
    a = rng.uniform(0.5, 1.5, size=n); a /= a.sum()
    b = rng.uniform(0.5, 1.5, size=m); b /= b.sum()
    return M, a, b


def assert_close(got, ref):
    assert got["niter"] == ref["niter"], (got["niter"], ref["niter"])
    scale = max(np.abs(ref["dual"]).max(), 1e-300)
    assert np.abs(got["dual"] - ref["dual"]).max() <= DUAL_RTOL * scale
    assert np.abs(got["plan"] - ref["plan"]).max() <= PLAN_ATOL


def test_config0_matches_oracle(cuda_dev):
    M, a, b = config0()
    got = cg.numpy.sinkhorn_bcd(M, a, b, 0.05, tol=1e-8, max_iter=1000)
    ref = oracle.bcd(M, a, b, 0.05, tol=1e-8, max_iter=1000)
    assert_close(got, ref)
    assert np.linalg.norm(got["plan"].sum(1) - a) < 1e-8


@pytest.mark.parametrize("n,m,reg,tol", [
    (80, 60, 0.01, 1e-6), (60, 80, 0.01, 1e-8), (50, 40, 0.05, 1e-8), (1, 1, 0.1, 1e-8),
    (1, 7, 0.1, 1e-8), (7, 1, 0.1, 1e-8), (33, 31, 0.02, 1e-8), (3, 1000, 0.05, 1e-8),
    (1000, 3, 0.05, 1e-8), (257, 129, 0.03, 1e-9), (2048, 96, 0.05, 1e-8),
    (96, 4099, 0.05, 1e-8),
])
def test_shapes_match_oracle(cuda_dev, n, m, reg, tol):
    M, a, b = rand_problem(n, m, n * 1000 + m)
    got = cg.numpy.sinkhorn_bcd(M, a, b, reg, tol=tol, max_iter=3000)
    ref = oracle.bcd(M, a, b, reg, tol=tol, max_iter=3000)
    assert_close(got, ref)


def test_truncation_and_zero_iterations(cuda_dev):
    M, a, b = rand_problem(50, 40, 456)
    got = cg.numpy.sinkhorn_bcd(M, a, b, 0.01, tol=1e-12, max_iter=10)
    assert got["niter"] == 10
    assert_close(got, oracle.bcd(M, a, b, 0.01, tol=1e-12, max_iter=10))
    z = cg.numpy.sinkhorn_bcd(M, a, b, 0.01, tol=1e-8, max_iter=0)
    assert z["niter"] == 0
    assert_close(z, oracle.bcd(M, a, b, 0.01, tol=1e-8, max_iter=0))


def test_warm_start(cuda_dev):
    M, a, b = rand_problem(50, 40, 789)
    r = cg.numpy.sinkhorn_bcd(M, a, b, 0.01, tol=1e-8, max_iter=5000)
    r2 = cg.numpy.sinkhorn_bcd(M, a, b, 0.01, tol=1e-8, max_iter=5000, x0=r["dual"])
    assert r2["niter"] <= r["niter"]
    assert np.abs(r2["plan"] - r["plan"]).max() <= 1e-8
    assert_close(r2, oracle.bcd(M, a, b, 0.01, tol=1e-8, max_iter=5000, x0=r["dual"]))


def test_torch_api_dtype_device_roundtrip(cuda_dev):
    M, a, b = rand_problem(64, 48, 3)
    Mt = torch.tensor(M, dtype=torch.float32)  # CPU float32 in -> CPU float32 out
    out = cg.torch.sinkhorn_bcd(Mt, torch.tensor(a), torch.tensor(b), 0.05, tol=1e-8)
    assert out["plan"].dtype == torch.float32 and out["plan"].device.type == "cpu"
    Mc = torch.tensor(M, device=cuda_dev)
    out = cg.torch.sinkhorn_bcd(Mc, torch.tensor(a, device=cuda_dev),
                                torch.tensor(b, device=cuda_dev), 0.05, tol=1e-8)
    assert out["plan"].is_cuda and out["plan"].dtype == torch.float64
    ref = oracle.bcd(Mt.double().numpy(), a, b, 0.05, tol=1e-8)
    assert out["niter"] == ref["niter"]


def test_deterministic(cuda_dev):
    M, a, b = rand_problem(300, 500, 11)
    r1 = cg.numpy.sinkhorn_bcd(M, a, b, 0.02, tol=1e-9, max_iter=2000)
    r2 = cg.numpy.sinkhorn_bcd(M, a, b, 0.02, tol=1e-9, max_iter=2000)
    assert np.array_equal(r1["dual"], r2["dual"])


def test_mixed_precision_fp64_checked(cuda_dev):
    M, a, b = rand_problem(700, 900, 5)
    M32 = M.astype(np.float32)
    got = cg.numpy.sinkhorn_bcd(M32, a, b, 0.05, tol=1e-8, max_iter=3000, precision="mixed")
    ref = oracle.bcd(M32.astype(np.float64), a, b, 0.05, tol=1e-8, max_iter=3000)
    # FP64-checked marginal error of the returned duals on the FP32-valued M
    al, be = got["dual"][:700], got["dual"][700:]
    P = np.exp((al[:, None] + be[None, :] - M32.astype(np.float64)) / 0.05)
    assert np.linalg.norm(P.sum(1) - a) < 1e-8
    assert np.linalg.norm(P.sum(0) - b) < 1e-8
    assert got["niter"] < 3000
    # duals agree with the FP64 oracle's to the accuracy a 1e-8 marginal allows
    g = got["dual"] - ref["dual"]
    g -= g.mean()  # gauge
    assert np.abs(g).max() < 1e-6


def test_exp2_implementations_vs_cuda(cuda_dev):
    from curegot_backward_b200 import _native
    x = torch.linspace(-1019.0, 1023.0, 2_000_003, dtype=torch.float64, device=cuda_dev)
    y = torch.empty_like(x)
    _native.call("cg_diag_exp2", x.data_ptr(), y.data_ptr(), x.numel(), 0,
                 torch.cuda.current_stream().cuda_stream)
    ref = torch.exp2(x)
    rel = ((y - ref).abs() / ref).max().item()
    assert rel < 2e-15, rel
    xn = torch.linspace(-120.0, 0.0, 1_000_003, dtype=torch.float64, device=cuda_dev)
    yn = torch.empty_like(xn)
    _native.call("cg_diag_exp2", xn.data_ptr(), yn.data_ptr(), xn.numel(), 1,
                 torch.cuda.current_stream().cuda_stream)
    refn = torch.exp2(xn)
    # one FP32 rounding of x (relative |x| 2^-24 ln2) plus the SFU's ~2^-22
    bound = 2.5e-7 + xn.abs() * 4.2e-8
    assert bool(((yn - refn).abs() / refn <= bound).all())


@pytest.mark.skipif(not oracle.ref_bcd_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("which", ["config0", "rand"])
def test_matches_reference_gpu_solver(cuda_dev, which):
    if which == "config0":
        M, a, b = config0()
        reg = 0.05
    else:
        M, a, b = rand_problem(120, 90, 7)
        reg = 0.02
    ref = oracle.ref_bcd(M, a, b, reg, tol=1e-8, max_iter=2000)
    got = cg.numpy.sinkhorn_bcd(M, a, b, reg, tol=1e-8, max_iter=2000)
    assert_close(got, ref)
    # and the oracle agrees with the reference's own solver
    assert_close(oracle.bcd(M, a, b, reg, tol=1e-8, max_iter=2000), ref)


@pytest.fixture
def bcd_path():
    """Selects the Sinkhorn path for one test; restores the default afterwards."""
    yield cg.set_bcd_cluster_path
    cg.set_bcd_cluster_path(True)


@pytest.mark.parametrize("path", ["cluster", "multi"])
@pytest.mark.parametrize("n,m,reg,tol", [
    (256, 320, 0.05, 1e-8), (17, 1000, 0.05, 1e-8), (1000, 3, 0.05, 1e-8), (3, 5, 0.1, 1e-8),
    (1, 1, 0.1, 1e-8), (600, 1200, 0.01, 1e-8), (100, 100, 0.01, 1e-10), (33, 31, 0.02, 1e-8),
])
def test_paths_match_oracle(cuda_dev, bcd_path, path, n, m, reg, tol):
    # the cluster-resident solver and the multi-CTA passes meet the same bar
    bcd_path(path == "cluster")
    M, a, b = rand_problem(n, m, 7 * n + m)
    got = cg.numpy.sinkhorn_bcd(M, a, b, reg, tol=tol, max_iter=5000)
    ref = oracle.bcd(M, a, b, reg, tol=tol, max_iter=5000)
    assert_close(got, ref)


def test_cluster_path_is_one_launch(cuda_dev, bcd_path):
    # problems of up to 768 KB of M take the cluster-resident path
    from curegot_backward_b200 import _native
    bcd_path(True)
    M, a, b = rand_problem(240, 360, 4)
    L = _native.lib()
    l0 = L.cg_launch_count()
    got = cg.numpy.sinkhorn_bcd(M, a, b, 0.05, tol=1e-8, max_iter=1000)
    # one cluster launch for the whole solve + the plan kernel
    assert L.cg_launch_count() - l0 <= 2
    ref = oracle.bcd(M, a, b, 0.05, tol=1e-8, max_iter=1000)
    assert_close(got, ref)


def test_cluster_path_warm_start_and_truncation(cuda_dev, bcd_path):
    bcd_path(True)
    M, a, b = rand_problem(300, 200, 3)
    r = cg.numpy.sinkhorn_bcd(M, a, b, 0.02, tol=1e-9, max_iter=7)
    o = oracle.bcd(M, a, b, 0.02, tol=1e-9, max_iter=7)
    assert r["niter"] == 7 == o["niter"]
    assert_close(r, o)
    full = cg.numpy.sinkhorn_bcd(M, a, b, 0.02, tol=1e-9, max_iter=5000)
    warm = cg.numpy.sinkhorn_bcd(M, a, b, 0.02, tol=1e-9, max_iter=5000, x0=full["dual"])
    ow = oracle.bcd(M, a, b, 0.02, tol=1e-9, max_iter=5000, x0=full["dual"])
    assert warm["niter"] == ow["niter"]
    assert np.abs(warm["plan"] - ow["plan"]).max() <= 1e-12


@pytest.mark.parametrize("precision,n,m", [("fp64", 1500, 4096), ("mixed", 2300, 8192),
                                           ("mixed", 3000, 2052), ("fp64", 700, 5003)])
def test_staged_passes_are_bitwise_the_unstaged_ones(cuda_dev, precision, n, m):
    """The shared-memory staging of the passes changes the memory pipeline
    only: duals and iteration counts are bitwise those of the register
    path (m = 5003 is not a multiple of the vector width: both take the
    scalar path)."""
    import torch
    from curegot_backward_b200 import _solvers
    g = torch.Generator(device=cuda_dev).manual_seed(n + m)
    X = torch.randn(n, 8, generator=g, device=cuda_dev, dtype=torch.float64)
    Y = torch.randn(m, 8, generator=g, device=cuda_dev, dtype=torch.float64)
    M = torch.cdist(X, Y) ** 2
    M = M / M.max()
    if precision == "mixed":
        M = M.float()
    a = torch.full((n,), 1.0 / n, dtype=torch.float64, device=cuda_dev)
    b = torch.full((m,), 1.0 / m, dtype=torch.float64, device=cuda_dev)
    out = {}
    try:
        for on in (True, False):
            cg.set_bcd_staging(on)
            out[on] = _solvers._bcd_device(M, a, b, 0.02, 1e-8, 3000, None, precision,
                                           want_plan=False)
    finally:
        cg.set_bcd_staging(False)  # the library default
    assert out[True][0] == out[False][0]
    assert torch.equal(out[True][2], out[False][2])


@pytest.mark.parametrize("precision,n,m,eta", [("fp64", 1500, 4096, 0.02), ("fp64", 700, 5003, 0.01),
                                               ("mixed", 2300, 8192, 0.02), ("fp64", 4000, 300, 0.01)])
def test_shifted_lse_agrees_with_running_maximum(cuda_dev, precision, n, m, eta):
    """Passes that sum relative to the previous LSE (no running maximum)
    against passes that keep the running maximum in every pass: same
    iteration count, duals within rounding, and both against the oracle's
    marginal bar.  At these eta the first iterations move the duals by more
    than the drift bound (|d beta| log2(e) / eta > 40), so both modes occur
    within one solve."""
    import torch
    from curegot_backward_b200 import _solvers
    g = torch.Generator(device=cuda_dev).manual_seed(3 * n + m)
    X = torch.randn(n, 8, generator=g, device=cuda_dev, dtype=torch.float64)
    Y = torch.randn(m, 8, generator=g, device=cuda_dev, dtype=torch.float64)
    M = torch.cdist(X, Y) ** 2
    M = M / M.max()
    if precision == "mixed":
        M = M.float()
    a = torch.rand(n, generator=g, device=cuda_dev, dtype=torch.float64) + 0.5
    b = torch.rand(m, generator=g, device=cuda_dev, dtype=torch.float64) + 0.5
    a, b = a / a.sum(), b / b.sum()
    out = {}
    try:
        for on in (True, False):
            cg.set_bcd_shifted_lse(on)
            out[on] = _solvers._bcd_device(M, a, b, eta, 1e-8, 5000, None, precision,
                                           want_plan=False)
    finally:
        cg.set_bcd_shifted_lse(True)  # the library default
    assert out[True][0] < 5000
    d1, d0 = out[True][2], out[False][2]
    if precision == "fp64":
        assert out[True][0] == out[False][0]
        assert (d1 - d0).abs().max().item() <= 1e-9 * d0.abs().max().item()
    else:
        # the SFU passes only decide when FP64 passes take over, so the two
        # solves may stop at neighbouring iterates, both within tol
        assert abs(out[True][0] - out[False][0]) <= 2
        assert (d1 - d0).abs().max().item() <= 1e-6 * d0.abs().max().item()
    # the marginal error of the shifted result, in FP64
    Md = M.double()
    P = torch.exp((d1[:n, None] + d1[None, n:] - Md) / eta)
    err = torch.sqrt(((P.sum(1) - a) ** 2).sum()).item()
    assert err < 1e-8
