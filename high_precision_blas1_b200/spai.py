"""Training and use of the learned sparse approximate inverse (per-row MLP,
see include/hpblas1.h, hpb_spai_*).

Everything that computes runs in libhpblas1.so: features, the MLP forward
and backward kernels, the loss gradients, Adam, the SpMVs and vector updates
that produce the residual histories.  torch only holds device memory.

    python -m high_precision_blas1_b200.spai train --systems 2000 --grid 24 --out weights.npy
"""
from __future__ import annotations

import argparse
import ctypes as C
import time
from pathlib import Path

import numpy as np

from . import _lib, problems

L = _lib.lib
P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64


hpb_spai_system = _lib.hpb_spai_system

NUM_PARAMS = L.hpb_spai_num_params()
# weights trained on the GPU by `python -m high_precision_blas1_b200.spai train --systems 2000 --grid 24`
WEIGHTS_FILE = Path(__file__).resolve().parent / "data" / "spai_lognormal3d_w64.npy"


def stencil7(N: int):
    return [-N * N, -N, -1, 0, 1, N, N * N], 3


def stencil5(N: int):
    return [-N, -1, 0, 1, N], 2


def check(st, what):
    if st != 0:
        raise _lib.HpbError(st, what)


class DeviceCSR:
    """A binary32 CSR copy of a problems.CSR on the device (torch tensors)."""

    def __init__(self, torch, A: problems.CSR):
        self.n, self.nnz = A.n, A.nnz
        self.rp = torch.from_numpy(A.row_ptr).cuda()
        self.ci = torch.from_numpy(A.col_ind).cuda()
        self.val = torch.from_numpy(A.val.astype(np.float32)).cuda()
        self.res = None
        self.nres = 0

    def system(self):
        return hpb_spai_system(self.n, self.nnz, self.rp.data_ptr(), self.ci.data_ptr(), self.val.data_ptr(),
                               self.nres, self.res.data_ptr() if self.res is not None else None)


def jacobi_residuals(torch, ctx, D: DeviceCSR, seed: int, snapshots=(2, 8, 32)):
    """Residual vectors of the damped Jacobi iteration on A x = b from x = 0,
    b uniform in [-1, 1]: r_{k+1} = r_k - (2/3) A D^{-1} r_k (the residual
    history of the plain stationary solver), normalised, at `snapshots`."""
    n = D.n
    d = torch.empty(n, dtype=torch.float32, device="cuda")
    check(L.hpb_csr_diag_f32(ctx.h, n, D.rp.data_ptr(), D.ci.data_ptr(), D.val.data_ptr(), d.data_ptr()), "diag")
    r = torch.empty(n, dtype=torch.float32, device="cuda")
    check(L.hpb_random_f32(ctx.h, n, seed, -1.0, 1.0, r.data_ptr()), "random")
    t = torch.empty_like(r)
    u = torch.empty_like(r)
    out = torch.empty((len(snapshots), n), dtype=torch.float32, device="cuda")
    k = 0
    for it in range(max(snapshots) + 1):
        if it in snapshots:
            nrm = np.zeros(4)
            check(L.hpb_nrm2_f32_host(ctx.h, n, r.data_ptr(), nrm.ctypes.data), "nrm2")
            check(L.hpb_scal_f32(ctx.h, n, 1.0 / nrm[0], r.data_ptr(), out[k].data_ptr()), "scal")
            k += 1
        # t = r ./ d ; u = A t ; r = r - (2/3) u
        check(L.hpb_div_pointwise_f32(ctx.h, n, 1.0, r.data_ptr(), 1.0, d.data_ptr(), t.data_ptr()), "div")
        check(L.hpb_csr_spmv_f32(ctx.h, n, n, D.nnz, D.rp.data_ptr(), D.ci.data_ptr(), D.val.data_ptr(), 1.0,
                                 t.data_ptr(), 0.0, u.data_ptr()), "spmv")
        check(L.hpb_axpy_f32(ctx.h, n, -2.0 / 3.0, u.data_ptr(), r.data_ptr()), "axpy")
    D.res = out
    D.nres = len(snapshots)


class SpaiNet:
    def __init__(self, offsets, dslot, seed=0):
        self.h = P()
        arr = (C.c_int * len(offsets))(*offsets)
        check(L.hpb_spai_create(C.byref(self.h), len(offsets), dslot, arr, seed), "hpb_spai_create")

    def close(self):
        if self.h:
            L.hpb_spai_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def weights(self) -> np.ndarray:
        w = np.zeros(NUM_PARAMS, dtype=np.float32)
        check(L.hpb_spai_get_weights(self.h, w.ctypes.data), "get_weights")
        return w

    def set_weights(self, w: np.ndarray):
        w = np.ascontiguousarray(w, dtype=np.float32)
        check(L.hpb_spai_set_weights(self.h, w.ctypes.data), "set_weights")

    def loss_grad(self, D: DeviceCSR, w_frob=1.0, w_resid=1.0, want_grad=False):
        loss = np.zeros(3)
        g = np.zeros(NUM_PARAMS, dtype=np.float32) if want_grad else None
        sysd = D.system()
        check(L.hpb_spai_loss_grad(self.h, C.byref(sysd), w_frob, w_resid, loss.ctypes.data,
                                   g.ctypes.data if want_grad else None), "loss_grad")
        return loss, g

    def loss(self, D: DeviceCSR, w_frob=1.0, w_resid=1.0):
        out = np.zeros(3)
        sysd = D.system()
        check(L.hpb_spai_loss(self.h, C.byref(sysd), w_frob, w_resid, out.ctypes.data), "loss")
        return out

    def adam(self, lr, scale=1.0):
        check(L.hpb_spai_adam(self.h, lr, scale), "adam")

    def assemble(self, torch, D: DeviceCSR):
        m = torch.empty(D.nnz, dtype=torch.float32, device="cuda")
        sysd = D.system()
        check(L.hpb_spai_assemble(self.h, C.byref(sysd), m.data_ptr()), "assemble")
        return m

    def forward(self, torch, feat, path=1):
        """The MLP alone on a (rows, 16) binary32 device tensor: (rows, 8)
        outputs; path 1 the tcgen05 kernel, path 0 the warp-level mma.sync one."""
        feat = feat.contiguous()
        out = torch.empty((feat.shape[0], 8), dtype=torch.float32, device=feat.device)
        check(L.hpb_spai_forward(self.h, feat.shape[0], feat.data_ptr(), out.data_ptr(), path), "forward")
        return out


def family(N: int, seed: int) -> problems.CSR:
    """The config-5 family: 3-D 7-point -div(kappa grad u), lognormal kappa,
    log-std 2.3, correlation length 8 cells."""
    return problems.diffusion3d_lognormal(N, seed=seed, sigma=2.3, corr=8.0)


def train(torch, n_systems=2000, N=24, epochs=3, batch=8, lr=3e-3, w_frob=1.0, w_resid=1.0, seed=1000, n_val=32,
          log=print):
    """Train on n_systems seeded systems of the family (seeds seed..seed+n-1);
    n_val further seeds are held out and the weights of the epoch with the
    lowest held-out loss are returned.  Returns (weights, history), history
    = mean training loss per epoch."""
    from . import Context
    offs, dslot = stencil7(N)
    net = SpaiNet(offs, dslot, seed=7)
    hist = []
    with Context(0, torch.cuda.current_stream().cuda_stream) as ctx:
        t0 = time.time()
        data, val = [], []
        for s in range(n_systems + n_val):
            D = DeviceCSR(torch, family(N, seed + s))
            jacobi_residuals(torch, ctx, D, seed=seed + s)
            (data if s < n_systems else val).append(D)
        log(f"generated {n_systems} + {n_val} systems of {N}^3 in {time.time() - t0:.1f}s")

        def val_loss():
            return float(np.mean([net.loss(D, w_frob, w_resid)[0] for D in val])) if val else 0.0

        best, best_w = val_loss(), net.weights()
        log(f"untrained (Jacobi): held-out loss {best:.5f}")
        rng = np.random.default_rng(seed)
        for ep in range(epochs):
            te = time.time()
            order = rng.permutation(n_systems)
            tot = 0.0
            for b0 in range(0, n_systems, batch):
                idx = order[b0:b0 + batch]
                for i in idx:
                    loss, _ = net.loss_grad(data[i], w_frob, w_resid)
                    tot += loss[0]
                net.adam(lr, 1.0 / len(idx))
            hist.append(tot / n_systems)
            vl = val_loss()
            if vl < best or not val:
                best, best_w = vl, net.weights()
            log(f"epoch {ep}: mean training loss {tot / n_systems:.5f}, held-out {vl:.5f}, "
                f"epoch {time.time() - te:.1f}s ({time.time() - t0:.1f}s total)")
    net.close()
    return best_w, hist


def main(argv=None):
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--systems", type=int, default=2000)
    t.add_argument("--grid", type=int, default=24)
    t.add_argument("--epochs", type=int, default=3)
    t.add_argument("--lr", type=float, default=3e-3)
    t.add_argument("--out", type=str, required=True)
    a = ap.parse_args(argv)
    import torch
    w, hist = train(torch, n_systems=a.systems, N=a.grid, epochs=a.epochs, lr=a.lr)
    np.save(Path(a.out), w)
    print("saved", a.out, "loss history", hist)


if __name__ == "__main__":
    main()
