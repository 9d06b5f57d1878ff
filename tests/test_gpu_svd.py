"""The device SVD (bm::svd3, the step kernels' SVD::compute) against the
reference's own outputs (GPU).

tests/golden/svd_cases.npz holds 512 matrices with the U, S, V that the
reference's SVD::compute (include/basements/core/math/svd.h:18-108) returns
for them. The device code follows the same cyclic Jacobi (skip below 1e-6,
stop below 1e-5, at most 5 sweeps, singular values unsorted, no sign fix,
U = F V / S) but contracts multiply-adds, so it may round differently. The
checks: S to 2e-6 of the largest singular value and in the reference's
order (unsorted), V to 1e-4, U diag(S) = F V (the columns of U scaled by
their singular values, which does not amplify rounding the way U = F V / S
does for the fixture's small singular values, down to 0) to 1e-4 of |F|, and
F = U S V^T as closely as the reference's own factors give it back. A sort, a
determinant or sign fix, or a changed threshold moves S, V or U S by O(1) on
the fixture's unsorted, near-identity and degenerate matrices.
"""
import os

import numpy as np
import pytest

import basements_b200 as bm

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("fast_math", [False, True], ids=["ieee", "fast"])
def test_device_svd_matches_reference_outputs(fast_math):
    d = np.load(os.path.join(GOLD, "svd_cases.npz"))
    F, U0, S0, V0 = (d[k].astype(np.float64) for k in ("F", "U", "S", "V"))
    U, S, V = (a.astype(np.float64) for a in bm.device_svd3(d["F"], fast_math=fast_math))
    scale = np.maximum(1.0, np.abs(S0).max(axis=1))
    nF = np.maximum(1.0, np.abs(F).reshape(-1, 9).max(axis=1))
    eS = np.abs(S - S0).max(axis=1) / scale
    eV = np.abs(V - V0).reshape(-1, 9).max(axis=1)
    eUS = np.abs(U * S[:, None, :] - U0 * S0[:, None, :]).reshape(-1, 9).max(axis=1) / nF
    eU = np.abs(U - U0).reshape(-1, 9).max(axis=1)
    rec = np.einsum("nij,nj,nkj->nik", U, S, V)
    eR = np.abs(rec - F).reshape(-1, 9).max(axis=1) / nF
    exact = np.mean((U == U0).all(axis=(1, 2)) & (S == S0).all(axis=1) & (V == V0).all(axis=(1, 2)))
    print(f"{'fast' if fast_math else 'ieee'}: bit-equal {exact:.3f}, max |S - S_ref| {eS.max():.2e}, "
          f"|V - V_ref| {eV.max():.2e}, |U S - (U S)_ref| {eUS.max():.2e}, |U - U_ref| {eU.max():.2e} "
          f"(smallest singular value there {S0[np.argmax(eU)].min():.2e}), reconstruction {eR.max():.2e}")
    assert eS.max() < 2e-6
    assert eV.max() < 1e-4
    assert eUS.max() < 1e-4
    # V orthonormal, as the reference's rotations keep it
    VtV = np.einsum("nji,njk->nik", V, V)
    assert np.abs(VtV - np.eye(3)).max() < 2e-5
    # F = U S V^T as well as the reference's own factors give it back
    rec0 = np.einsum("nij,nj,nkj->nik", U0, S0, V0)
    eR0 = np.abs(rec0 - F).reshape(-1, 9).max(axis=1) / nF
    assert (eR <= eR0 + 2e-5).all()
