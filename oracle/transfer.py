"""CPU oracle of the exact Stokes step (test infrastructure only).

polarized_transfer.stokes_step_exact (python/blackhole_sim/
polarized_transfer.py:51-70) forms exp(A ds) of the 5x5 augmented matrix
A = [[-K, j], [0, 0]] with scipy.linalg.expm (scipy 1.18 in the reference's
environment: Pade approximation with scaling and squaring) and applies it to
[S; 1].  Restated here with the Taylor series and scaling and squaring
(Moler & Van Loan 2003, method 3) in float64; only tests import this module.
"""

from __future__ import annotations

import math

import numpy as np


def propagation_matrix(c) -> np.ndarray:
    """synchrotron.py:82-94 for COEFF_NAMES-ordered coefficients."""
    ai, aq, au, av, rv, rq, ru = (float(x) for x in c[4:11])
    return np.array([[ai, aq, au, av], [aq, ai, rv, -ru], [au, -rv, ai, rq], [av, ru, -rq, ai]])


def expm(A: np.ndarray) -> np.ndarray:
    """exp(A) by scaling (||A/2^s||_1 <= 1/4) and an order-18 Taylor series."""
    norm = float(np.max(np.abs(A).sum(axis=0)))
    s = max(0, math.ceil(math.log2(norm / 0.25))) if norm > 0.25 else 0
    X = A / 2.0 ** s
    E = np.eye(A.shape[0])
    term = np.eye(A.shape[0])
    for m in range(1, 19):
        term = term @ X / m
        E = E + term
    for _ in range(s):
        E = E @ E
    return E


def stokes_step_exact(stokes, c, ds: float) -> np.ndarray:
    """polarized_transfer.py:51-70."""
    if ds <= 0.0:
        return np.asarray(stokes, dtype=float)
    A = np.zeros((5, 5))
    A[:4, :4] = -propagation_matrix(c)
    A[:4, 4] = np.asarray(c[:4], dtype=float)
    y = np.ones(5)
    y[:4] = np.asarray(stokes, dtype=float)
    return (expm(A * ds) @ y)[:4]
