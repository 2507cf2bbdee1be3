"""Host-only checks of the device execution plan (mf_plan_info: no CUDA call)."""
import numpy as np
import pytest

import multifrontal as mf
from multifrontal import _native, testmatrices as tm
from multifrontal._native import ptr64


def plan(S, monkeypatch, amalg):
    monkeypatch.setenv("MF_AMALGAMATE", amalg)
    lib = _native.gpulib()
    out = np.zeros(8, np.int64)
    rc = lib.mf_plan_info(S.n, S.nfr, ptr64(S.resptr), ptr64(S.sepptr), ptr64(S.septgt), ptr64(S.reltgt),
                          ptr64(S.chdptr), ptr64(S.chdtgt), ptr64(S.Dptr), ptr64(S.Lptr), 16, ptr64(out))
    assert rc == 0, lib.mf_last_error()
    return out


def test_amalgamation_merges_chains(monkeypatch):
    A = tm.grid_laplacian(24, 24, 24, lo=1e-3, hi=1e3, shift=1e-6)
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(24, 24, 24))
    exact = plan(S, monkeypatch, "0")
    merged = plan(S, monkeypatch, "1")
    assert exact[0] == S.nfr
    assert merged[0] < S.nfr // 4          # far fewer execution fronts
    assert merged[1] < exact[1] // 4       # far fewer levels
    # panel storage grows only by the explicit zeros of the merged chains
    nn, nj = S.nn(), S.nn() + S.na()
    assert exact[2] == int(np.sum(((nj + 3) // 4 * 4) * nn))   # panels nj x nn, ld padded to 4
    assert merged[2] < 1.3 * exact[2]


def test_plan_rejects_corrupted_symbolic(monkeypatch):
    A = tm.grid_laplacian(8, 8)
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(8, 8, 1))
    bad = S.reltgt.copy()
    j = int(np.nonzero(S.na() > 1)[0][0])
    bad[S.sepptr[j]] += 1
    lib = _native.gpulib()
    out = np.zeros(8, np.int64)
    rc = lib.mf_plan_info(S.n, S.nfr, ptr64(S.resptr), ptr64(S.sepptr), ptr64(S.septgt), ptr64(bad),
                          ptr64(S.chdptr), ptr64(S.chdtgt), ptr64(S.Dptr), ptr64(S.Lptr), 16, ptr64(out))
    assert rc == -2
    assert b"rel" in lib.mf_last_error()
