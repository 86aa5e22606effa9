"""CPU checks of the learned-SPAI oracle (oracle/spai_ref.py) before it is
used to check the GPU kernels: its parameter gradient equals central finite
differences of its loss, the untrained network is Jacobi, and the scaled
preconditioner Mh is symmetric positive definite for arbitrary weights."""
import numpy as np
import pytest

from high_precision_blas1_b200 import problems, spai
from oracle import spai_ref as R


@pytest.fixture
def system():
    A = problems.diffusion3d_lognormal(4, seed=3, sigma=1.5, corr=2.0)
    offs, dslot = spai.stencil7(4)
    return A, offs, dslot


def test_gradient_matches_finite_differences(system, monkeypatch):
    A, offs, dslot = system
    monkeypatch.setattr(R, "bf16", lambda x: np.asarray(x, dtype=np.float64))  # smooth in w for the differences
    rng = np.random.default_rng(0)
    w = rng.standard_normal(R.NP) * 0.3
    res = [rng.standard_normal(A.n) for _ in range(2)]
    _, _, _, g = R.loss_and_grad(A, offs, dslot, w, res, 1.0, 0.7)
    for idx in (R.W1 + 7, R.B1 + 3, R.W2 + 100, R.B2 + 9, R.W3 + 5, R.B3 + 1, R.B3 + dslot):
        e = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[idx] += e
        wm[idx] -= e
        fd = (R.loss_and_grad(A, offs, dslot, wp, res, 1.0, 0.7)[0] -
              R.loss_and_grad(A, offs, dslot, wm, res, 1.0, 0.7)[0]) / (2 * e)
        assert g[idx] == pytest.approx(fd, rel=1e-5, abs=1e-9), idx


def test_zero_output_layer_is_jacobi(system):
    A, offs, dslot = system
    w = np.zeros(R.NP)
    w[R.W1:R.B1] = 0.3
    X, diag = R.features(A, offs, dslot)
    _, _, out = R.forward(w, X)
    m = R.assemble(A, offs, dslot, out, diag)
    rows = np.repeat(np.arange(A.n), np.diff(A.row_ptr))
    want = np.where(rows == A.col_ind, 1.0 / A.val.astype(np.float32).astype(np.float64), 0.0)
    assert np.allclose(m, want, rtol=1e-12, atol=0)


def test_scaled_preconditioner_is_spd_for_any_weights(system):
    A, offs, dslot = system
    rng = np.random.default_rng(4)
    for _ in range(3):
        w = rng.standard_normal(R.NP) * 2.0
        X, _ = R.features(A, offs, dslot)
        _, _, out = R.forward(w, X)
        mh = R.assemble_scaled(A, offs, out, dslot)
        M = np.zeros((A.n, A.n))
        M[np.repeat(np.arange(A.n), np.diff(A.row_ptr)), A.col_ind] = mh
        assert np.allclose(M, M.T)
        assert np.linalg.eigvalsh(M).min() > 0
