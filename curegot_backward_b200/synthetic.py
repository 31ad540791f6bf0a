"""Seeded synthetic OT problems with the shapes and value distributions of the
benchmark configurations (no external datasets are used).

    config0()        Sinkhorn FP64, n=512, m=640: X~U[0,1]^{512x8}, Y~U[0,1]^{640x8},
                     M_ij = mean_d (x_i - y_j)^2, uniform marginals, eta 0.05
    config1()        SPLR FP64, n=m=4096: X,Y~N(0,I_16), M = |x-y|^2 / max,
                     marginals U[0.5,1.5] normalised, eta 0.01
    config2()        precision form, n=m=16384: X,Y~N(0,I_32), M = |x-y|^2 / median
                     stored FP32, Dirichlet(1) marginals floored at 1e-7, eta 1e-3
    config3()        differentiation, n=2048, m=2560: config-0 costs with d=32, eta 0.05
    stream_specs()   serving stream: n, m log-uniform in [64, 8192], d in {8, 32},
                     Gaussian clouds / max, eta in {0.1, 0.05, 0.01}, 70% Sinkhorn /
                     30% SPLR, tol 1e-8, Poisson arrivals
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch


def _sqdist(X, Y):
    """Squared Euclidean distances (FP64 accumulation), clamped at 0."""
    X = X.double()
    Y = Y.double()
    D = (X * X).sum(1)[:, None] + (Y * Y).sum(1)[None, :] - 2.0 * (X @ Y.T)
    return D.clamp_min_(0.0)


def config0(seed=0):
    rng = np.random.default_rng(seed)
    n, m = 512, 640
    X, Y = rng.uniform(size=(n, 8)), rng.uniform(size=(m, 8))
    M = ((X[:, None, :] - Y[None, :, :]) ** 2).mean(-1)
    return M, np.full(n, 1.0 / n), np.full(m, 1.0 / m), 0.05


def config1(seed=1, device="cuda"):
    g = torch.Generator(device=device).manual_seed(seed)
    n = m = 4096
    X = torch.randn(n, 16, generator=g, device=device)
    Y = torch.randn(m, 16, generator=g, device=device)
    M = _sqdist(X, Y)
    M /= M.max()
    a = torch.rand(n, generator=g, device=device, dtype=torch.float64) + 0.5
    b = torch.rand(m, generator=g, device=device, dtype=torch.float64) + 0.5
    return M, a / a.sum(), b / b.sum(), 0.01


def _dirichlet1(k, g, device):
    e = -torch.log(torch.rand(k, generator=g, device=device, dtype=torch.float64))
    w = e / e.sum()
    w = w.clamp_min(1e-7)
    return w / w.sum()


def config2(seed=2, device="cuda", n=16384, m=16384):
    g = torch.Generator(device=device).manual_seed(seed)
    X = torch.randn(n, 32, generator=g, device=device)
    Y = torch.randn(m, 32, generator=g, device=device)
    M = _sqdist(X, Y)
    med = torch.quantile(M.flatten()[:: max(1, M.numel() // (1 << 24))].float(), 0.5).double()
    M = (M / med).float()
    return M, _dirichlet1(n, g, device), _dirichlet1(m, g, device), 1e-3


def config3(seed=3, n=2048, m=2560):
    rng = np.random.default_rng(seed)
    X, Y = rng.uniform(size=(n, 32)), rng.uniform(size=(m, 32))
    M = (_sqdist(torch.from_numpy(X), torch.from_numpy(Y)) / 32.0).numpy()
    return M, np.full(n, 1.0 / n), np.full(m, 1.0 / m), 0.05


@dataclass
class StreamSpec:
    idx: int
    n: int
    m: int
    d: int
    eta: float
    algo: str
    seed: int
    arrival: float  # seconds after the stream start


def stream_specs(count=4096, seed=4, rate=None, n_lo=64, n_hi=8192):
    """Request specs of the serving stream.  rate=None: all arrive at t=0
    (saturation); else Poisson arrivals with that mean rate (requests/s)."""
    rng = np.random.default_rng(seed)
    lo, hi = math.log(n_lo), math.log(n_hi)
    t = 0.0
    specs = []
    for k in range(count):
        n = int(round(math.exp(rng.uniform(lo, hi))))
        m = int(round(math.exp(rng.uniform(lo, hi))))
        d = int(rng.choice([8, 32]))
        eta = float(rng.choice([0.1, 0.05, 0.01]))
        algo = "bcd" if rng.uniform() < 0.7 else "splr"
        if rate:
            t += float(rng.exponential(1.0 / rate))
        specs.append(StreamSpec(k, n, m, d, eta, algo, int(rng.integers(1 << 31)), t))
    return specs


def stream_problem(spec: StreamSpec, device="cuda", dtype=torch.float32):
    """Cost matrix (Gaussian clouds / max) and uniform marginals of one request."""
    g = torch.Generator(device=device).manual_seed(spec.seed)
    X = torch.randn(spec.n, spec.d, generator=g, device=device)
    Y = torch.randn(spec.m, spec.d, generator=g, device=device)
    M = _sqdist(X, Y)
    M /= M.max()
    a = torch.full((spec.n,), 1.0 / spec.n, dtype=torch.float64, device=device)
    b = torch.full((spec.m,), 1.0 / spec.m, dtype=torch.float64, device=device)
    return M.to(dtype), a, b
