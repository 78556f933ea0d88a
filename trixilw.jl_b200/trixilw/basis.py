"""Gauss-Lobatto-Legendre nodes and weights on the host (Trixi LobattoLegendreBasis nodes/weights),
used for node coordinates, quadrature in error norms and boundary time levels. The device library
builds its own copy of the basis (derivative matrices) in C++."""
from __future__ import annotations

import functools

import numpy as np


def _q_and_l(N: int, x: float):
    # Kopriva, "Implementing Spectral Methods for PDEs", Alg. 24
    a, b, da, db = 1.0, x, 0.0, 1.0
    for k in range(2, N + 1):
        c = ((2 * k - 1) * x * b - (k - 1) * a) / k
        dc = da + (2 * k - 1) * b
        a, b, da, db = b, c, db, dc
    k = N + 1
    c = ((2 * k - 1) * x * b - (k - 1) * a) / k
    dc = da + (2 * k - 1) * b
    return c - a, dc - da, b


@functools.lru_cache(maxsize=None)
def _gll(N: int):
    # Kopriva Alg. 25
    if N == 1:
        return np.array([-1.0, 1.0]), np.array([1.0, 1.0])
    x = np.zeros(N + 1)
    w = np.zeros(N + 1)
    x[0], x[N] = -1.0, 1.0
    w[0] = w[N] = 2.0 / (N * (N + 1))
    for j in range(1, (N + 1) // 2):
        xj = -np.cos((j + 0.25) * np.pi / N - 3.0 / (8.0 * N * np.pi * (j + 0.25)))
        for _ in range(100):
            q, dq, _ = _q_and_l(N, xj)
            d = -q / dq
            xj += d
            if abs(d) <= 4 * np.finfo(float).eps * abs(xj):
                break
        _, _, LN = _q_and_l(N, xj)
        x[j], x[N - j] = xj, -xj
        w[j] = w[N - j] = 2.0 / (N * (N + 1) * LN * LN)
    if N % 2 == 0:
        _, _, LN = _q_and_l(N, 0.0)
        x[N // 2] = 0.0
        w[N // 2] = 2.0 / (N * (N + 1) * LN * LN)
    return x, w


def gauss_lobatto(N: int):
    """(nodes, weights) of the N+1 point Gauss-Lobatto-Legendre rule on [-1, 1]."""
    x, w = _gll(int(N))
    return x.copy(), w.copy()


@functools.lru_cache(maxsize=None)
def _dmat(N: int):
    # Kopriva Algs. 30 and 37: barycentric weights, then the polynomial derivative matrix
    x, _ = _gll(N)
    n = N + 1
    wb = np.array([1.0 / np.prod([x[c] - x[k] for k in range(n) if k != c]) for c in range(n)])
    D = np.zeros((n, n))
    for r in range(n):
        for c in range(n):
            if c != r:
                D[r, c] = wb[c] / wb[r] / (x[r] - x[c])
                D[r, r] -= D[r, c]
    return D


def derivative_matrix(N: int) -> np.ndarray:
    """D[r, c] = l_c'(x_r) on the N+1 GLL nodes (Trixi derivative_matrix)."""
    return _dmat(int(N)).copy()
