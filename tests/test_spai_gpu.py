"""Learned sparse approximate inverse: the GPU forward/backward kernels
against the float64 CPU oracle (oracle/spai_ref.py), the untrained network
being exactly Jacobi, and a short training run on the GPU that must beat
Jacobi on held-out systems of the family.

Tolerances (binary32 features, MLP and loss kernels on the GPU, binary64 in
the oracle, same bf16 weights): assembled M within 1e-4 relative to its
largest entry, losses within 1e-4 relative, gradient
||g_gpu - g_ref|| <= 2e-3 ||g_ref||."""
import ctypes as C

import numpy as np
import pytest

from gpu_utils import dev, host
from high_precision_blas1_b200 import _lib, problems, spai

pytestmark = pytest.mark.gpu


def test_gradient_matches_cpu_oracle(gpu):
    from oracle import spai_ref
    ctx, torch = gpu
    N = 6
    A = problems.diffusion3d_lognormal(N, seed=3, sigma=1.5, corr=2.0)
    offs, dslot = spai.stencil7(N)
    net = spai.SpaiNet(offs, dslot, seed=1)
    rng = np.random.default_rng(0)
    w = (rng.standard_normal(spai.NUM_PARAMS) * 0.2).astype(np.float32)
    net.set_weights(w)
    D = spai.DeviceCSR(torch, A)
    res = rng.standard_normal((2, A.n)).astype(np.float32)
    D.res = torch.from_numpy(res).cuda()
    D.nres = 2
    m_gpu = host(net.assemble(torch, D)).astype(np.float64)
    X, diag = spai_ref.features(A, offs, dslot)
    _, _, out = spai_ref.forward(w, X)
    m_ref = spai_ref.assemble(A, offs, dslot, out, diag)
    assert np.max(np.abs(m_gpu - m_ref)) <= 1e-4 * np.max(np.abs(m_ref))
    # the assembled preconditioner is symmetric
    Ms = problems.CSR(A.n, A.row_ptr, A.col_ind, m_gpu)
    v = np.random.default_rng(1).standard_normal(A.n)
    u = np.random.default_rng(2).standard_normal(A.n)
    assert abs(u @ Ms.matvec(v) - v @ Ms.matvec(u)) <= 1e-5 * np.linalg.norm(u) * np.linalg.norm(Ms.matvec(v))
    for wf, wr in ((1.0, 0.0), (0.0, 1.0), (1.0, 0.5)):
        loss, g = net.loss_grad(D, wf, wr, want_grad=True)
        tot, lf, lr, gref = spai_ref.loss_and_grad(A, offs, dslot, w, [r for r in res], wf, wr)
        assert loss[1] == pytest.approx(lf, rel=1e-4) and loss[2] == pytest.approx(lr, rel=1e-4)
        err = np.linalg.norm(g.astype(np.float64) - gref) / np.linalg.norm(gref)
        assert err <= 2e-3, (wf, wr, err)
    net.adam(0.0, 1.0)  # clears the accumulated gradient
    net.close()


@pytest.mark.parametrize("rows", [1, 127, 128, 129, 4999, 70001])
def test_tcgen05_forward_matches_warp_kernel_and_oracle(gpu, rows):
    """The tensor-memory MLP forward (128-row tiles, ragged last tile) against
    the warp-level mma.sync kernel (the same bf16 hi/lo products in another
    summation order: 2e-5 of the largest output) and the binary64 oracle
    forward with the same bf16 weights (1e-4)."""
    from oracle import spai_ref
    ctx, torch = gpu
    offs, dslot = spai.stencil7(8)
    net = spai.SpaiNet(offs, dslot, seed=3)
    rng = np.random.default_rng(rows)
    w = (rng.standard_normal(spai.NUM_PARAMS) * 0.3).astype(np.float32)
    net.set_weights(w)
    X = rng.standard_normal((rows, 16)).astype(np.float32)
    dX = dev(torch, X)
    out_tc = host(net.forward(torch, dX, path=1)).astype(np.float64)
    out_ws = host(net.forward(torch, dX, path=0)).astype(np.float64)
    _, _, ref = spai_ref.forward(w, X.astype(np.float64))
    scale = np.abs(ref).max()
    assert np.abs(out_tc - ref).max() <= 1e-4 * scale
    assert np.abs(out_tc - out_ws).max() <= 2e-5 * scale
    # repeatable
    assert np.array_equal(host(net.forward(torch, dX, path=1)).astype(np.float64), out_tc)
    net.close()


def test_untrained_network_is_jacobi(gpu):
    ctx, torch = gpu
    N = 8
    A = problems.diffusion3d_lognormal(N, seed=5)
    offs, dslot = spai.stencil7(N)
    net = spai.SpaiNet(offs, dslot, seed=2)
    D = spai.DeviceCSR(torch, A)
    m = host(net.assemble(torch, D))
    rows = np.repeat(np.arange(A.n), np.diff(A.row_ptr))
    diag = A.val[rows == A.col_ind].astype(np.float32)
    want = np.where(rows == A.col_ind, 1.0 / A.val.astype(np.float32), 0.0)
    assert np.allclose(m, want, rtol=1e-6)
    assert diag.size == A.n
    net.close()


def ir_iters(torch, A, b, precond, M=None, basis=30):
    d = [dev(torch, a) for a in (A.row_ptr, A.col_ind, A.val, b, np.zeros(A.n))]
    p = _lib.ir_params("gmres", basis=basis, inner_rel_tol=1e-5, precond=precond, rel_tol=1e-10)
    rep = _lib.hpb_ir_report()
    mp = [None, None, None, 0] if M is None else [d[0].data_ptr(), d[1].data_ptr(), M.data_ptr(), A.nnz]
    st = _lib.lib.hpb_ir_solve_f64(C.byref(p), A.n, A.nnz, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), None,
                                   mp[0], mp[1], mp[2], mp[3], d[3].data_ptr(), d[4].data_ptr(), C.byref(rep), None, 0)
    torch.cuda.synchronize()
    x = host(d[4])
    return st, rep, np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b)


def test_trained_network_beats_jacobi_on_held_out_systems(gpu):
    ctx, torch = gpu
    N = 12
    w, hist = spai.train(torch, n_systems=48, N=N, epochs=4, batch=4, lr=3e-3, seed=5000, log=lambda *a: None)
    assert hist[-1] < hist[0]  # the loss goes down
    offs, dslot = spai.stencil7(16)
    net = spai.SpaiNet(offs, dslot)
    net.set_weights(w)
    gains = []
    for seed in (91, 92):  # held-out seeds, larger grid than training
        A = spai.family(16, seed)
        b = problems.rhs_uniform(A.n, seed)
        M = net.assemble(torch, spai.DeviceCSR(torch, A))
        st_j, rep_j, rel_j = ir_iters(torch, A, b, "jacobi")
        st_m, rep_m, rel_m = ir_iters(torch, A, b, "matrix", M=M)
        assert st_j == 0 and st_m == 0 and rel_j <= 1.05e-10 and rel_m <= 1.05e-10
        gains.append(rep_j.inner_iters / rep_m.inner_iters)
    net.close()
    assert min(gains) > 1.0, gains
