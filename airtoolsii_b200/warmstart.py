"""Learned warm start for SIRT (no counterpart in the reference; it reaches
the solvers only through their x0 argument, sirt/sirt.m:5).

For one fixed paralleltomo geometry a U-Net maps the normalised
back-projection of the data, u = D.*A'(M.*b) with the SART weights (one SART
step from zero with relaxpar 1), to a starting point x0; cimmino then runs
from x0 to the discrepancy-principle stop.  Training pairs come from
seeded random-ellipse phantoms: the input u of the noisy sinogram and, as
target, the DP-stopped cimmino solution that the GPU SIRT computes for it.
Plain SIRT from zero stays the fallback, and the DP residual of SIRT judges
every warm-started answer.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import _lib
from ._lib import check, dptr, lib
from .batch import ParallelBatch
from .solvers import cimmino, sart
from .testprobs import parallel_operator, parallel_tables
from .unet import UNet


def ellipse_params(N_seeds, count=10):
    """Per seed `count` ellipses (amp, a, b, x0, y0, cos phi, sin phi):
    centres U[-0.6,0.6]^2, semi-axes U[0.05,0.4], rotation U[0,pi),
    intensity U[0.1,1]."""
    out = np.zeros((len(N_seeds), count, 7))
    for k, s in enumerate(N_seeds):
        rng = np.random.default_rng(int(s))
        for e in range(count):
            cx, cy = rng.uniform(-0.6, 0.6, 2)
            a, b = rng.uniform(0.05, 0.4, 2)
            phi = rng.uniform(0.0, math.pi)
            amp = rng.uniform(0.1, 1.0)
            out[k, e] = (amp, a, b, cx, cy, math.cos(phi), math.sin(phi))
    return out


class WarmStart:
    """Warm-start pipeline for one paralleltomo geometry (N, theta, p).

    Every stage runs on the GPU with device-resident data: phantoms
    (airt_phantom_ellipses), sinograms (airt_apply_device plus seeded
    Gaussian noise scaled to eta*||b||), the network input (one batched SART
    step), the training targets (batched cimmino to the per-instance DP
    stop), training (airt_unet_train_step) and inference
    (airt_unet_forward_f64).  Batches of `chunk` instances share one
    block-diagonal system."""

    def __init__(self, N=256, theta=None, p=None, base=32, levels=4, method="cimmino",
                 tau=1.02, max_batch=16, seed=0, chunk=64):
        import torch
        self.torch = torch
        theta = np.arange(0.0, 180.0, 3.0) if theta is None else np.asarray(theta, float)
        th, p, d, ct, st, off = parallel_tables(N, theta, p)
        self.N, self.theta, self.p = N, th, p
        self.n, self.m = N * N, p * len(th)
        self.A = parallel_operator(N, ct, st, off)
        self.method, self.tau, self.chunk = method, tau, chunk
        r = C.c_double()
        check(lib().airt_rho(self.A.handle, _lib.METHODS[method], None, None, 1e-7, 200, C.byref(r)))
        self.rho = float(r.value)
        self.net = UNet(N, N, base, levels, max_batch, seed)
        self.max_batch = max_batch
        self._batches = {}

    def batch(self, K) -> ParallelBatch:
        if K not in self._batches:
            self._batches[K] = ParallelBatch([self.N] * K, [self.theta] * K, [self.p] * K)
        return self._batches[K]

    # ------------------------------------------------------------ data
    def phantoms(self, seeds, count=10):
        """Device FP64 tensor (len(seeds), n) of random-ellipse phantoms."""
        torch = self.torch
        prm = np.ascontiguousarray(ellipse_params(seeds, count).reshape(-1))
        out = torch.empty((len(seeds), self.n), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        check(lib().airt_phantom_ellipses(self.N, len(seeds), count, dptr(prm), 0.0, 1.0,
                                          C.c_void_p(out.data_ptr()), None))
        return out

    def sinograms(self, X, eta, seed):
        """b = A x + e with ||e|| = eta ||A x|| per row of X (device); returns
        (device b, host delta = ||e||)."""
        torch = self.torch
        K = X.shape[0]
        B0 = torch.empty((K, self.m), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        for k in range(K):
            check(lib().airt_apply_device(self.A.handle, C.c_void_p(X[k].data_ptr()),
                                          C.c_void_p(B0[k].data_ptr()), 0))
        g = torch.Generator(device="cuda")
        g.manual_seed(10_000_019 + int(seed))
        E = torch.randn((K, self.m), generator=g, dtype=torch.float64, device="cuda")
        scale = eta * torch.linalg.norm(B0, dim=1) / torch.linalg.norm(E, dim=1)
        E *= scale[:, None]
        return B0 + E, torch.linalg.norm(E, dim=1).cpu().numpy()

    def net_input(self, d_b, d_u, K):
        """u = D.*A'(M.*b), one SART step from zero with relaxpar 1 (device);
        returns the device time in ms."""
        return self.batch(K).backproject_device("sart", d_b, d_u)

    def dp_solve(self, d_b, d_x, K, taudelta, d_x0=None, kmax=2000):
        return self.batch(K).sirt_device(self.method, d_b, d_x, kmax, taudelta=taudelta,
                                         rho=np.full(K, self.rho), d_x0=d_x0)

    def prepare(self, seeds, eta=0.02):
        """Device tensors u (network input), target (DP-stopped cimmino
        solution), x (phantom) as FP32 (K, n); b (FP64 (K, m)); host
        taudelta and DP iteration counts."""
        torch = self.torch
        K = len(seeds)
        U = torch.empty((K, self.n), dtype=torch.float32, device="cuda")
        T = torch.empty_like(U)
        Xs = torch.empty_like(U)
        Bs = torch.empty((K, self.m), dtype=torch.float64, device="cuda")
        td = np.zeros(K)
        its = np.zeros(K, np.int64)
        for c0 in range(0, K, self.chunk):
            sl = list(seeds[c0:c0 + self.chunk])
            k = len(sl)
            X = self.phantoms(sl)
            b, delta = self.sinograms(X, eta, sl[0])
            td[c0:c0 + k] = self.tau * delta
            u = torch.empty((k, self.n), dtype=torch.float64, device="cuda")
            x = torch.empty_like(u)
            self.net_input(b.data_ptr(), u.data_ptr(), k)
            info = self.dp_solve(b.data_ptr(), x.data_ptr(), k, td[c0:c0 + k])
            U[c0:c0 + k] = u
            T[c0:c0 + k] = x
            Xs[c0:c0 + k] = X
            Bs[c0:c0 + k] = b
            its[c0:c0 + k] = info["finaliter"]
        torch.cuda.synchronize()
        return dict(u=U, target=T, x=Xs, b=Bs, taudelta=td, iters=its)

    # ------------------------------------------------------------ training
    def train(self, U, T, epochs=4, batch=16, lr=1e-3, decay_every=1, log=None):
        """Adam on (U, T) (device FP32 (K, n)); the learning rate halves every
        `decay_every` epochs."""
        torch = self.torch
        K = U.shape[0]
        rng = np.random.default_rng(0)
        steps = max(1, K // batch)
        hist = []
        for ep in range(epochs):
            perm = torch.from_numpy(rng.permutation(K)).cuda()
            lr_e = lr * (0.5 ** (ep // decay_every))
            tot = 0.0
            for s in range(steps):
                idx = perm[s * batch:(s + 1) * batch]
                bu = U.index_select(0, idx).contiguous()
                bt = T.index_select(0, idx).contiguous()
                torch.cuda.current_stream().synchronize()
                tot += self.net.train_step(bu.data_ptr(), bt.data_ptr(), idx.numel(), lr_e)
            hist.append(tot / steps)
            if log:
                log(f"epoch {ep}: mse {hist[-1]:.3e}")
        return hist

    def predict(self, d_u, d_x0, K, stream=0):
        """x0 = net(u) for K FP64 device images."""
        self.net.forward_f64(d_u, d_x0, K, stream)

    # ------------------------------------------------------------ comparison
    def compare_batched(self, data, sel=None, kmax=2000):
        """Time to the DP stop for the instances `sel` of `data`, solved as one
        batch: plain cimmino from zero vs SART step + network + cimmino from
        x0.  Both pipelines run from device-resident sinograms to
        device-resident solutions; times are host wall times around each
        whole pipeline (synchronised), plus the solvers' device times."""
        torch = self.torch
        sel = np.arange(data["b"].shape[0]) if sel is None else np.asarray(sel)
        K = len(sel)
        isel = torch.from_numpy(sel).cuda()
        d_b = data["b"].index_select(0, isel).contiguous()
        td = data["taudelta"][sel]
        Bt = self.batch(K)
        xp = torch.empty((K, self.n), dtype=torch.float64, device="cuda")
        xw, u, x0 = torch.empty_like(xp), torch.empty_like(xp), torch.empty_like(xp)
        rho = np.full(K, self.rho)
        stream = Bt.stream_ptr()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ip = Bt.sirt_device(self.method, d_b.data_ptr(), xp.data_ptr(), kmax, taudelta=td,
                            rho=rho)
        torch.cuda.synchronize()
        wall_plain = time.perf_counter() - t0
        t0 = time.perf_counter()
        u_ms = self.net_input(d_b.data_ptr(), u.data_ptr(), K)
        self.predict(u.data_ptr(), x0.data_ptr(), K, stream)
        iw = Bt.sirt_device(self.method, d_b.data_ptr(), xw.data_ptr(), kmax, taudelta=td,
                            rho=rho, d_x0=x0.data_ptr())
        torch.cuda.synchronize()
        wall_warm = time.perf_counter() - t0
        # the network alone, for the breakdown
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        self.predict(u.data_ptr(), x0.data_ptr(), K, stream)
        torch.cuda.synchronize()
        t_net = time.perf_counter() - t1
        xt = data["x"].index_select(0, isel).double()
        err = lambda xs: (torch.linalg.norm(xs - xt, dim=1)  # noqa: E731
                          / torch.linalg.norm(xt, dim=1)).cpu().numpy()
        return dict(K=K, plain_iters=ip["finaliter"], warm_iters=iw["finaliter"],
                    plain_gpu_ms=ip["gpu_ms"], warm_gpu_ms=u_ms + iw["gpu_ms"],
                    net_wall_s=t_net, plain_wall_s=wall_plain, warm_wall_s=wall_warm,
                    plain_relerr=err(xp), warm_relerr=err(xw), x0_relerr=err(x0))

    def time_to_dp_shared(self, data, batch, kmax=2000):
        """time_to_dp with the same-geometry engine: every batch of `batch`
        sinograms is solved as K right-hand sides of the one stored matrix
        (airt_sirt_multi_device: the matrix is read once per iteration for
        the whole batch).  plain: cimmino from zero; warm: u = D.*A'(M.*b)
        (one SART step from zero, through the same engine), x0 = U-Net(u),
        cimmino from x0.  Same clocks and outputs as time_to_dp (no fbp arm).
        (Queueing every batch's network on its own stream, so that it runs
        beside the solves of earlier batches, was measured: no faster.)"""
        from .batch import sirt_multi_device
        torch = self.torch
        total = data["b"].shape[0]
        nb = total // batch
        if nb < 1:
            raise ValueError("need at least one full batch")
        sels = [np.arange(i * batch, (i + 1) * batch) for i in range(nb)]
        d_b = [data["b"].index_select(0, torch.from_numpy(sl).cuda()).contiguous() for sl in sels]
        xp = [torch.empty((batch, self.n), dtype=torch.float64, device="cuda") for _ in range(nb)]
        xw = [torch.empty_like(xp[0]) for _ in range(nb)]
        u = [torch.empty_like(xp[0]) for _ in range(nb)]
        x0 = [torch.empty_like(xp[0]) for _ in range(nb)]
        tds = [data["taudelta"][sl] for sl in sels]
        stream = self.A.stream_ptr()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ip = [sirt_multi_device(self.A, self.method, d_b[i].data_ptr(), xp[i].data_ptr(), batch,
                                kmax, taudelta=tds[i], rho=self.rho) for i in range(nb)]
        torch.cuda.synchronize()
        wall_plain = time.perf_counter() - t0
        t0 = time.perf_counter()
        iw = []
        for i in range(nb):
            sirt_multi_device(self.A, "sart", d_b[i].data_ptr(), u[i].data_ptr(), batch, 1,
                              relaxpar=1.0)
            self.predict(u[i].data_ptr(), x0[i].data_ptr(), batch, stream)
            iw.append(sirt_multi_device(self.A, self.method, d_b[i].data_ptr(), xw[i].data_ptr(),
                                        batch, kmax, taudelta=tds[i], rho=self.rho,
                                        d_X0=x0[i].data_ptr()))
        torch.cuda.synchronize()
        wall_warm = time.perf_counter() - t0
        xt = data["x"].double()

        def err(xs):
            out = []
            for i, sl in enumerate(sels):
                ref = xt.index_select(0, torch.from_numpy(sl).cuda())
                out.append((torch.linalg.norm(xs[i] - ref, dim=1) / torch.linalg.norm(ref, dim=1)).cpu().numpy())
            return np.concatenate(out)
        return dict(instances=nb * batch, batch=batch, plain_wall_s=wall_plain, warm_wall_s=wall_warm,
                    plain_iters=np.concatenate([r["finaliter"] for r in ip]),
                    warm_iters=np.concatenate([r["finaliter"] for r in iw]),
                    plain_relerr=err(xp), warm_relerr=err(xw), x0_relerr=err(x0),
                    plain_solver_gpu_ms=sum(r["gpu_ms"] for r in ip),
                    warm_solver_gpu_ms=sum(r["gpu_ms"] for r in iw))

    def time_to_dp(self, data, batch, kmax=2000, fbp_filter="hamming"):
        """Time to the DP stop for all instances of `data`, `batch` at a time
        (a multiple of batch instances): plain, fbp warm start and learned
        warm start.

        plain: batched cimmino from zero, batch after batch.
        fbp: per batch, the filtered back projection (auxil/fbp.m, filter
        `fbp_filter`) as x0, then batched cimmino from it.
        warm: per batch, the back-projection u, the network's x0 and batched
        cimmino from x0, in that order on the solver's stream.  (Running the
        next batch's network on its own stream during a solve was measured
        slower: the convolutions take bandwidth from the HBM-bound SpMVs.)

        Inputs (sinograms) are resident on the device before the clocks start
        and the solutions stay there; times are host wall clocks around each
        synchronised pipeline.  Returns per-instance iterations and relative
        errors and the two wall times."""
        torch = self.torch
        total = data["b"].shape[0]
        nb = total // batch
        if nb < 1:
            raise ValueError("need at least one full batch")
        Bt = self.batch(batch)
        sels = [np.arange(i * batch, (i + 1) * batch) for i in range(nb)]
        d_b = [data["b"].index_select(0, torch.from_numpy(sl).cuda()).contiguous() for sl in sels]
        xp = [torch.empty((batch, self.n), dtype=torch.float64, device="cuda") for _ in range(nb)]
        xw = [torch.empty_like(xp[0]) for _ in range(nb)]
        u = [torch.empty_like(xp[0]) for _ in range(nb)]
        x0 = [torch.empty_like(xp[0]) for _ in range(nb)]
        xf = [torch.empty_like(xp[0]) for _ in range(nb)]
        xf0 = [torch.empty_like(xp[0]) for _ in range(nb)]
        rho = np.full(batch, self.rho)
        tds = [data["taudelta"][sl] for sl in sels]
        stream = Bt.stream_ptr()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ip = [Bt.sirt_device(self.method, d_b[i].data_ptr(), xp[i].data_ptr(), kmax, taudelta=tds[i],
                             rho=rho) for i in range(nb)]
        torch.cuda.synchronize()
        wall_plain = time.perf_counter() - t0
        t0 = time.perf_counter()
        iF = []
        wall_filter = 0.0
        for i in range(nb):
            t1 = time.perf_counter()
            Bt.fbp_device(d_b[i].data_ptr(), xf0[i].data_ptr(), fbp_filter)  # returns synchronised
            wall_filter += time.perf_counter() - t1
            iF.append(Bt.sirt_device(self.method, d_b[i].data_ptr(), xf[i].data_ptr(), kmax,
                                     taudelta=tds[i], rho=rho, d_x0=xf0[i].data_ptr()))
        torch.cuda.synchronize()
        wall_fbp = time.perf_counter() - t0
        t0 = time.perf_counter()
        iw = []
        for i in range(nb):
            self.net_input(d_b[i].data_ptr(), u[i].data_ptr(), batch)
            self.predict(u[i].data_ptr(), x0[i].data_ptr(), batch, stream)
            iw.append(Bt.sirt_device(self.method, d_b[i].data_ptr(), xw[i].data_ptr(), kmax,
                                     taudelta=tds[i], rho=rho, d_x0=x0[i].data_ptr()))
        torch.cuda.synchronize()
        wall_warm = time.perf_counter() - t0
        xt = data["x"].double()
        def err(xs):  # noqa: E306
            out = []
            for i, sl in enumerate(sels):
                ref = xt.index_select(0, torch.from_numpy(sl).cuda())
                out.append((torch.linalg.norm(xs[i] - ref, dim=1) / torch.linalg.norm(ref, dim=1)).cpu().numpy())
            return np.concatenate(out)
        return dict(instances=nb * batch, batch=batch, plain_wall_s=wall_plain, warm_wall_s=wall_warm,
                    fbp_wall_s=wall_fbp, fbp_filter_wall_s=wall_filter, fbp_filter=fbp_filter,
                    plain_iters=np.concatenate([r["finaliter"] for r in ip]),
                    warm_iters=np.concatenate([r["finaliter"] for r in iw]),
                    fbp_iters=np.concatenate([r["finaliter"] for r in iF]),
                    plain_relerr=err(xp), warm_relerr=err(xw), x0_relerr=err(x0),
                    fbp_relerr=err(xf), fbp_x0_relerr=err(xf0),
                    plain_solver_gpu_ms=sum(r["gpu_ms"] for r in ip),
                    warm_solver_gpu_ms=sum(r["gpu_ms"] for r in iw),
                    fbp_solver_gpu_ms=sum(r["gpu_ms"] for r in iF))


# ---------------------------------------------------------------- training CLI
# The configuration the checkpoint in airtoolsii_b200/weights was trained
# with: N=256, 60 angles (0:3:177 degrees), 2% noise, 20000 phantoms (seeds
# 1000..20999), 8 epochs of Adam, batch 16, learning rate 1e-3 halved every
# 2 epochs.  Training runs on the GPU only (the network's gradients use
# atomics, so runs agree statistically, not bit for bit).
C5 = dict(N=256, theta_step=3.0, angles=60, eta=0.02, base=32, levels=4, train_seeds=(1000, 21000),
          epochs=8, batch=16, lr=1e-3, decay_every=2, net_seed=0)
CHECKPOINT = "weights/unet_paralleltomo_n256_a60.npz"


def checkpoint_path() -> str:
    import os
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), CHECKPOINT)


def c5_warmstart(max_batch=32, chunk=128) -> WarmStart:
    c = C5
    return WarmStart(N=c["N"], theta=np.arange(c["angles"]) * c["theta_step"], base=c["base"],
                     levels=c["levels"], max_batch=max_batch, seed=c["net_seed"], chunk=chunk)


def train_c5(out=None, log=print) -> dict:
    """Generate the training pairs on the GPU, train, and write the checkpoint."""
    c = C5
    ws = c5_warmstart()
    t0 = time.perf_counter()
    tr = ws.prepare(list(range(*c["train_seeds"])), eta=c["eta"])
    t1 = time.perf_counter()
    hist = ws.train(tr["u"], tr["target"], epochs=c["epochs"], batch=c["batch"], lr=c["lr"],
                    decay_every=c["decay_every"], log=log)
    ws.torch.cuda.synchronize()
    t2 = time.perf_counter()
    meta = dict(c, prepare_s=round(t1 - t0, 2), train_s=round(t2 - t1, 2), final_mse=hist[-1],
                mean_dp_iters=float(tr["iters"].mean()))
    ws.net.save(out or checkpoint_path(), **meta)
    return meta


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description="train the N=256 / 60-angle warm-start U-Net")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    print(train_c5(a.out))
