"""Seeded synthetic matrices of the shapes the benchmarks use (no datasets
are downloaded; the reference's tests read SuiteSparse matrices, which are
not available offline).

All generators return a symmetric scipy CSC matrix (both triangles).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def _weights(rng, m, lo, hi, dist):
    if dist == "loguniform":
        return np.exp(rng.uniform(np.log(lo), np.log(hi), size=m))
    if dist == "uniform":
        return rng.uniform(lo, hi, size=m)
    if dist == "unit":
        return np.ones(m)
    raise ValueError(dist)


def _laplacian(n, i, j, w, shift):
    """Weighted graph Laplacian with diagonal = row sum of weights + shift."""
    rows = np.concatenate([i, j])
    cols = np.concatenate([j, i])
    vals = np.concatenate([-w, -w])
    deg = np.zeros(n)
    np.add.at(deg, i, w)
    np.add.at(deg, j, w)
    A = sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsc()
    A = A + sp.diags(deg + shift, format="csc")
    A = sp.csc_matrix(A)
    A.sum_duplicates()
    A.sort_indices()
    return A


def grid_edges(nx, ny, nz=1, stencil=5):
    """Edges (i < j) of a 2D 5-point, 2D 9-point or 3D 7-point stencil;
    vertex id x + nx*(y + ny*z)."""
    idx = np.arange(nx * ny * nz).reshape(nz, ny, nx)
    e = []
    e.append((idx[:, :, :-1].ravel(), idx[:, :, 1:].ravel()))
    e.append((idx[:, :-1, :].ravel(), idx[:, 1:, :].ravel()))
    if nz > 1:
        e.append((idx[:-1, :, :].ravel(), idx[1:, :, :].ravel()))
    if stencil == 9:
        e.append((idx[:, :-1, :-1].ravel(), idx[:, 1:, 1:].ravel()))
        e.append((idx[:, :-1, 1:].ravel(), idx[:, 1:, :-1].ravel()))
    i = np.concatenate([a for a, _ in e]).astype(np.int64)
    j = np.concatenate([b for _, b in e]).astype(np.int64)
    lo = np.minimum(i, j)
    hi = np.maximum(i, j)
    return lo, hi


def grid_laplacian(nx, ny, nz=1, *, stencil=None, seed=0, lo=0.1, hi=10.0, dist="loguniform", shift=1e-2):
    """SPD stencil matrix: off-diagonals -w (w seeded), diagonal = row sum + shift."""
    if stencil is None:
        stencil = 7 if nz > 1 else 5
    i, j = grid_edges(nx, ny, nz, 9 if stencil == 9 else 5)
    rng = np.random.default_rng(seed)
    w = _weights(rng, i.size, lo, hi, dist)
    return _laplacian(nx * ny * nz, i, j, w, shift)


def config1(seed=1):
    """2D 5-point 100x100, log-uniform [0.1, 10] weights, diagonal + 1e-2."""
    return grid_laplacian(100, 100, seed=seed, lo=0.1, hi=10.0, shift=1e-2)


def config2(side=80, seed=2):
    """3D 7-point side^3, log-uniform [1e-3, 1e3] coefficients, diagonal + 1e-6."""
    return grid_laplacian(side, side, side, seed=seed, lo=1e-3, hi=1e3, shift=1e-6)


def config3_matrix(side, seed):
    """2D 9-point side x side, uniform [0.5, 2] weights, diagonal + 1e-3."""
    return grid_laplacian(side, side, stencil=9, seed=seed, lo=0.5, hi=2.0, dist="uniform", shift=1e-3)


def config4(side=40, m=16000, per_row=6, delta=1e-6, seed=4):
    """K = [H A^T; A -delta I]: H = 3D 7-point side^3 Laplacian (unit weights)
    + 1e-4 I, A is m x side^3 with `per_row` N(0,1) entries per row at
    uniform random columns."""
    nh = side ** 3
    i, j = grid_edges(side, side, side)
    H = _laplacian(nh, i, j, np.ones(i.size), 0.0) + 1e-4 * sp.eye(nh, format="csc")
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(m), per_row)
    cols = np.empty(m * per_row, np.int64)
    for r in range(m):
        cols[r * per_row:(r + 1) * per_row] = rng.choice(nh, size=per_row, replace=False)
    vals = rng.standard_normal(m * per_row)
    A = sp.csc_matrix((vals, (rows, cols)), shape=(m, nh))
    K = sp.bmat([[H, A.T], [A, -delta * sp.eye(m)]], format="csc")
    K.sum_duplicates()
    K.sort_indices()
    return K


def rhs(n, k=1, seed=0):
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((n, k))
    return np.asfortranarray(B)


def backward_error(A, X, B):
    """Normwise backward error per column: ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf)."""
    X = np.asarray(X).reshape(A.shape[0], -1)
    B = np.asarray(B).reshape(A.shape[0], -1)
    R = B - A @ X
    anorm = abs(A).sum(axis=1).max()
    return np.abs(R).max(axis=0) / (anorm * np.abs(X).max(axis=0) + np.abs(B).max(axis=0))
