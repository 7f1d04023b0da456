"""LSQR least squares for the host-side bulk solve.

The reference calls ``IterativeSolvers.lsqr!(x, A, b)`` from
`src/NonlinearSolvers/residual/AndersonResidual.jl:123` (and from
`fixed_point/AndersonMixing.jl:142` on the inhomogeneous path).  IterativeSolvers.jl
is an unpinned, un-vendored dependency; this is the published Paige-Saunders
algorithm (ACM TOMS 8(1):43-71, 1982) with that package's defaults:
``atol = btol = sqrt(eps)``, ``conlim = 1/sqrt(eps)``, ``maxiter = max(m, n)``,
no damping, and ``x`` used as the warm start (the bidiagonalisation starts from
``b - A x``).  The device solve and the CPU oracle implement the same recurrences.
"""
from __future__ import annotations

import math

import numpy as np

_EPS = float(np.finfo(np.float64).eps)


def lsqr_inplace(x: np.ndarray, A: np.ndarray, b: np.ndarray,
                 atol: float = math.sqrt(_EPS), btol: float = math.sqrt(_EPS),
                 conlim: float = 1.0 / math.sqrt(_EPS), maxiter: int | None = None) -> int:
    """Overwrites ``x`` with the LSQR solution of min ||A x - b||; returns istop."""
    m, n = A.shape
    if maxiter is None:
        maxiter = max(m, n)
    ctol = 1.0 / conlim if conlim > 0 else 0.0
    u = b - A @ x
    v = np.zeros(n)
    alpha = 0.0
    beta = float(np.linalg.norm(u))
    if beta > 0:
        u = u / beta
        v = A.T @ u
        alpha = float(np.linalg.norm(v))
    if alpha > 0:
        v = v / alpha
    w = v.copy()
    arnorm = alpha * beta
    if arnorm == 0:
        return 0
    anorm = acond = ddnorm = res2 = xxnorm = z = sn2 = 0.0
    cs2 = -1.0
    rhobar = alpha
    phibar = bnorm = beta
    itn = 0
    istop = 0
    while itn < maxiter and istop == 0:
        itn += 1
        u = A @ v - alpha * u
        beta = float(np.linalg.norm(u))
        if beta > 0:
            u = u / beta
            anorm = math.sqrt(anorm * anorm + alpha * alpha + beta * beta)
            v = A.T @ u - beta * v
            alpha = float(np.linalg.norm(v))
            if alpha > 0:
                v = v / alpha
        rhobar1 = rhobar  # no damping
        psi = 0.0
        rho = math.sqrt(rhobar1 * rhobar1 + beta * beta)
        cs = rhobar1 / rho
        sn = beta / rho
        theta = sn * alpha
        rhobar = -cs * alpha
        phi = cs * phibar
        phibar = sn * phibar
        tau = sn * phi
        t1 = phi / rho
        t2 = -theta / rho
        dk = w / rho
        x += t1 * w
        w = v + t2 * w
        ddnorm += float(dk @ dk)
        delta = sn2 * rho
        gambar = -cs2 * rho
        rhs = phi - delta * z
        zbar = rhs / gambar
        xnorm = math.sqrt(xxnorm + zbar * zbar)
        gamma = math.sqrt(gambar * gambar + theta * theta)
        cs2 = gambar / gamma
        sn2 = theta / gamma
        z = rhs / gamma
        xxnorm += z * z
        acond = anorm * math.sqrt(ddnorm)
        res1 = phibar * phibar
        res2 += psi * psi
        rnorm = math.sqrt(res1 + res2)
        arnorm = alpha * abs(tau)
        test1 = rnorm / bnorm
        test2 = arnorm / (anorm * rnorm) if anorm * rnorm != 0 else math.inf
        test3 = 1.0 / acond if acond != 0 else math.inf
        t1b = test1 / (1.0 + anorm * xnorm / bnorm)
        rtol = btol + atol * anorm * xnorm / bnorm
        if itn >= maxiter:
            istop = 7
        if 1.0 + test3 <= 1.0:
            istop = 6
        if 1.0 + test2 <= 1.0:
            istop = 5
        if 1.0 + t1b <= 1.0:
            istop = 4
        if test3 <= ctol:
            istop = 3
        if test2 <= atol:
            istop = 2
        if test1 <= rtol:
            istop = 1
    return istop
