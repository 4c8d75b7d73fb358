"""Learned subgrid closure for coarse 2D runs: training data from filtered DNS, training on the
GPU with the library's own CNN kernels, and a-posteriori evaluation against filtered DNS.

Filtering is a sharp spectral cutoff: the coarse field keeps |kx| < Nc/2 and -Nc/2 < kz < Nc/2
of the fine field.  With FN the solver's nonlinear term (d omega/dt = FN + viscous), the
filtered DNS obeys d w_bar/dt = FN_c(w_bar) + F + viscous with the subgrid forcing
    F = trunc(FN_f(w)) - FN_c(w_bar)   (= -(filtered(u.grad w) - u_bar.grad w_bar)).
The CNN maps (w_bar, u_bar, v_bar) on the coarse 3/2 grid to F on the same grid.
"""
from __future__ import annotations

import time

import numpy as np

from . import CNN, Solver


def truncate(om_f: np.ndarray, Nc: int) -> np.ndarray:
    """Sharp spectral cutoff of a compact [iz][ix] spectrum to Nc (the kz = -Nc/2 row is 0)."""
    Nf = om_f.shape[0]
    Hc = Nc // 2
    out = np.zeros((Nc, Hc), dtype=om_f.dtype)
    out[:Hc, :] = om_f[:Hc, :Hc]
    out[Hc + 1:, :] = om_f[Nf - Hc + 1:, :Hc]
    return out


class _Coarse:
    """Coarse-grid helper state: nonlinear term and physical fields of a given spectrum."""

    def __init__(self, Nc, Re, K0, cfl):
        self.s = Solver(Nc, Re, K0, cfl)

    def fields(self, om_c):
        s = self.s
        s.init_vorticity(om_c)
        s.velocity_phys()
        s.om2phys()
        return np.stack([s.phys(2), s.phys(0), s.phys(1)])  # (omega, u, w)

    def nonlinear(self, om_c):
        s = self.s
        s.init_vorticity(om_c)
        s.next_dt()
        s.step(1)
        return s.fnm1()

    def physical(self, spec):
        s = self.s
        s.init_vorticity(spec)
        s.om2phys()
        return s.phys(2)


def generate(Nf=512, Nc=64, Re=1e4, K0=4.0, cfl=0.1, seeds=range(8), steps=4000, every=50, warm=200):
    """Training pairs (inputs [n][3][Lc][Lc], targets [n][1][Lc][Lc]) from filtered DNS."""
    X, T = [], []
    co = _Coarse(Nc, Re, K0, cfl)
    for sd in seeds:
        f = Solver(Nf, Re, K0, cfl)
        f.init_k4(int(sd))
        f.next_dt()
        f.step(1)
        f.next_dt()
        it = 1
        while it < steps:
            n = min(every, steps - it)
            f.step(n)
            it += n
            if it % 100 == 0:
                f.next_dt()
            if it < warm:
                continue
            om_f = f.om2()
            f.step(1)  # fnm1 <- FN(om_f)
            it += 1
            fn_f = f.fnm1()
            om_c = truncate(om_f, Nc)
            F_hat = truncate(fn_f, Nc) - co.nonlinear(om_c)
            X.append(co.fields(om_c))
            T.append(co.physical(F_hat)[None])
        f.close()
    return np.asarray(X, dtype=np.float32), np.asarray(T, dtype=np.float32)


def train(X, T, layers=6, channels=32, iters=2000, batch=32, lr=1e-3, seed=0, tensor_cores=False):
    """Normalise, train on the GPU (convolutions as tcgen05 GEMMs with tensor_cores); returns
    (network, scales, losses)."""
    s_om = float(X[:, 0].std())
    s_u = float(np.sqrt(0.5 * (X[:, 1].var() + X[:, 2].var())))
    s_out = float(T.std())
    scales = np.array([s_om, s_u, s_u, s_out], dtype=np.float32)
    Xn = X / scales[None, :3, None, None]
    Tn = T / s_out
    net = CNN(layers, channels, seed=seed)
    net.set_train_tc(tensor_cores)
    net.set_dataset(Xn, Tn)
    losses = net.train(iters, batch, lr, seed=seed + 1)
    return net, scales, losses


def shells(om: np.ndarray) -> np.ndarray:
    """E(k) = 1/2 sum_{round|k| = k} w |om|^2 / K^2 of a compact spectrum (w = 1 on kx = 0)."""
    N, H = om.shape
    kz = np.where(np.arange(N) < H, np.arange(N), np.arange(N) - N)[:, None]
    kx = np.arange(H)[None, :]
    k2 = (kx * kx + kz * kz).astype(np.float64)
    w = np.where(kx == 0, 1.0, 2.0)
    p = np.abs(om.astype(np.complex128)) ** 2
    e = np.where(k2 > 0, 0.5 * w * p / np.maximum(k2, 1), 0.0)
    sh = np.rint(np.sqrt(k2)).astype(int)
    return np.bincount(sh.ravel(), weights=e.ravel(), minlength=N)


def evaluate(net, scales, Nf=512, Nc=64, Re=1e4, K0=4.0, cfl=0.1, seed=100, fine_steps=2000, update=100, check=1,
             clamp=0.0):
    """Filtered DNS vs coarse runs with and without the closure over the same physical time."""
    f = Solver(Nf, Re, K0, cfl)
    f.init_k4(seed)
    om0 = truncate(f.om2(), Nc)
    f.next_dt()
    t0 = time.perf_counter()
    it = 0
    while it < fine_steps:
        n = 1 if it == 0 else min(update - it % update, fine_steps - it)
        f.step(n)
        it += n
        if it == 1 or it % update == 0:
            f.next_dt()
    f.sync()
    wall_f = time.perf_counter() - t0
    t_end = f.scalars()["t"]
    ref = truncate(f.om2(), Nc)
    f.close()

    def coarse(with_closure):
        c = Solver(Nc, Re, K0, cfl)
        c.init_vorticity(om0)
        c.next_dt()
        if with_closure:
            c.attach_closure(net, scales, energy_check=check)
            if clamp > 0.0:
                c.closure_clamp(clamp)
        # same diagnostic cadence as the DNS; stop at the step closest to the DNS end time
        t0 = time.perf_counter()
        n = 0
        while True:
            sc = c.scalars()
            left = int(round((t_end - sc["t"]) / sc["dt"])) if sc["dt"] > 0 else 0
            if left <= 0:
                break
            k = 1 if n == 0 else min(left, update - n % update)
            c.step(k)
            n += k
            if n == 1 or n % update == 0:
                c.next_dt()
        c.sync()
        wall = time.perf_counter() - t0
        stats = c.closure_stats() if with_closure else (0, 0)
        om = c.om2()
        tc = c.scalars()["t"]
        c.close()
        return om, wall, n, tc, stats

    out = {"t_end": t_end, "wall_dns": wall_f, "fine_steps": fine_steps, "clamp": clamp}
    E_ref = shells(ref)
    Z_ref = float(np.sum(np.abs(ref.astype(np.complex128)) ** 2 * np.where(np.arange(Nc // 2) == 0, 0.5, 1.0)))
    kmax = Nc // 2 - 1
    for name, flag in (("plain", False), ("closure", True)):
        om, wall, n, tc, stats = coarse(flag)
        E = shells(om)
        rel = np.abs(E[1:kmax + 1] / E_ref[1:kmax + 1] - 1.0)
        Z = float(np.sum(np.abs(om.astype(np.complex128)) ** 2 * np.where(np.arange(Nc // 2) == 0, 0.5, 1.0)))
        out[name] = {"wall": wall, "steps": n, "t": tc, "shell_err_max": float(rel.max()),
                     "shell_err_mean": float(rel.mean()), "enstrophy_err": abs(Z / Z_ref - 1.0),
                     "closure_steps": stats[0], "fallbacks": stats[1]}
    return out


def main(argv=None):
    """The closure experiment at a given scale: filtered-DNS data, GPU training for a time
    budget, a-posteriori evaluation on a held-out seed (energy gate with and without the forcing
    limiter, and ungated) at 1/4 and all of the run.  Prints one JSON line per evaluation.

        python -m optimizec_b200.closure --nf 2048 --nc 256 --re 1e5 --seeds 8 --steps 67000 \\
            --every 1000 --train-seconds 420 --batch 4
    """
    import argparse
    import json

    ap = argparse.ArgumentParser()
    ap.add_argument("--nf", type=int, default=2048)
    ap.add_argument("--nc", type=int, default=256)
    ap.add_argument("--re", type=float, default=1e5)
    ap.add_argument("--seeds", type=int, default=8)
    ap.add_argument("--steps", type=int, default=67000)
    ap.add_argument("--every", type=int, default=1000)
    ap.add_argument("--train-seconds", type=float, default=420.0)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--clamp", type=float, default=1.0, help="forcing limiter alpha (0: off)")
    ap.add_argument("--checks", default=None,
                    help="evaluations as energy_check:alpha pairs, e.g. 1:1,3:1 (default: 1:clamp,1:0,0:0)")
    ap.add_argument("--fp32-training", action="store_true",
                    help="train with the FP32 SIMT convolutions instead of the tensor-core GEMMs")
    ap.add_argument("--timing-only", action="store_true",
                    help="no data or training: time the DNS, plain and closed runs (energy_check 1, the "
                         "limiter at --clamp) with an untrained 6 x 32 network; the wall-time ratio does "
                         "not depend on the weights")
    a = ap.parse_args(argv)
    if a.timing_only:
        from . import CNN
        net = CNN(6, 32, seed=1)
        r = evaluate(net, np.array([5.0, 1.0, 1.0, 0.01], np.float32), Nf=a.nf, Nc=a.nc, Re=a.re, K0=4.0,
                     seed=100, fine_steps=a.steps, update=1000, check=1, clamp=a.clamp)
        print(json.dumps({"wall_dns": r["wall_dns"], "closure_wall": r["closure"]["wall"],
                          "closure_steps": r["closure"]["steps"], "plain_wall": r["plain"]["wall"],
                          "speedup_closure_vs_dns": r["wall_dns"] / r["closure"]["wall"]}), flush=True)
        net.close()
        return
    runs = ([(int(c), float(al)) for c, al in (x.split(":") for x in a.checks.split(","))] if a.checks
            else [(1, a.clamp), (1, 0.0), (0, 0.0)])
    cfg = dict(Nf=a.nf, Nc=a.nc, Re=a.re, K0=4.0, cfl=0.1)
    t = time.time()
    X, T = generate(seeds=range(a.seeds), steps=a.steps, every=a.every, warm=a.every, **cfg)
    print(json.dumps({"data": list(X.shape), "generate_s": round(time.time() - t, 1)}), flush=True)
    net, sc, _ = train(X, T, iters=20, batch=a.batch, lr=1e-3, tensor_cores=not a.fp32_training)
    t = time.time()  # the rate of an iteration, without the network's creation and the dataset upload
    net.train(20, a.batch, 1e-3, seed=3)
    per = (time.time() - t) / 20
    iters = max(100, int(a.train_seconds / per))
    t = time.time()
    losses = net.train(iters, a.batch, 1e-3, seed=7)
    print(json.dumps({"train_iters": iters, "train_s": round(time.time() - t, 1),
                      "loss_first": float(np.mean(losses[:20])), "loss_last": float(np.mean(losses[-50:]))}),
          flush=True)
    for chk, clamp in runs:
        for fs in (a.steps // 4, a.steps):
            r = evaluate(net, sc, seed=100, fine_steps=fs, update=100, check=chk, clamp=clamp, **cfg)
            r["energy_check"] = chk
            r["clamp"] = clamp
            r["speedup_closure_vs_dns"] = r["wall_dns"] / r["closure"]["wall"]
            print(json.dumps(r), flush=True)
    net.close()


if __name__ == "__main__":
    main()
