"""Learned closure coupled to the solver: the forcing spectrum against the FP64 oracle (CNN
forward + 2D transform), one closed step against the plain step plus the forcing term of the
CN/AB2 update, the energy gate (device gate and host rollback), and the a-posteriori gain of a
trained closure over the plain coarse run measured against filtered DNS."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 32
RE = 2000.0


@pytest.fixture(scope="module")
def pkg():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import optimizec_b200 as pk

    pk.lib()
    return pk


def _state(pk, seed=3):
    s = pk.Solver(N, RE, 4.0, 0.1)
    s.init_k4(seed)
    s.next_dt()
    return s


def _retained(spec_full, N):
    """Compact [iz][kx] retained modes of a [kz mod L][kx] spectrum (the kz = -N/2 row zero)."""
    H = N // 2
    L = spec_full.shape[0]
    out = np.zeros((N, H), dtype=np.complex128)
    for iz in range(N):
        kz = iz if iz < H else iz - N
        if kz == -H:
            continue
        out[iz] = spec_full[kz % L, :H]
    return out


def _identity_net(pk, s_om):
    """2-layer network whose output is omega / s_om (GELU run where it is the identity to 1e-20)."""
    from oracle import cnn_oracle as co

    net = pk.CNN(2, 4, seed=0)
    p = np.zeros(net.num_params(), dtype=np.float32)
    (ci0, co0), (ci1, co1) = co.layer_shapes(2, 4)
    w0 = np.zeros((co0, ci0, 3, 3), np.float32)
    b0 = np.zeros(co0, np.float32)
    w0[0, 0, 1, 1] = 1.0
    b0[0] = 10.0
    w1 = np.zeros((co1, ci1, 3, 3), np.float32)
    w1[0, 0, 1, 1] = 1.0
    b1 = np.array([-10.0], np.float32)
    p[:] = np.concatenate([w0.ravel(), b0, w1.ravel(), b1])
    net.set_params(p)
    return net


def test_forcing_spectrum_matches_oracle(pkg):
    from oracle import cnn_oracle as co
    from oracle import oracle as orc

    s = _state(pkg)
    net = pkg.CNN(3, 8, seed=7)
    s.velocity_phys()
    s.om2phys()
    u, w, om = s.phys(0), s.phys(1), s.phys(2)
    scales = np.array([om.std(), u.std(), w.std(), 0.37], dtype=np.float32)
    s.attach_closure(net, scales, energy_check=0)
    F = s.closure_forcing().astype(np.complex128)

    x = np.stack([om / scales[0], u / scales[1], w / scales[2]])[None].astype(np.float64)
    y, _ = co.forward(net.params(), 3, 8, x)
    L = s.L
    ref = _retained(orc.fwd2d(y[0, 0] * float(scales[3])) / (L * L), N)
    err = np.abs(F - ref).max()
    assert err <= 2e-5 * np.abs(ref).max(), (err, np.abs(ref).max())
    s.close()
    net.close()


def test_closed_step_adds_forcing_term(pkg):
    s_p = _state(pkg)
    s_c = _state(pkg)
    net = pkg.CNN(3, 8, seed=11)
    s_c.velocity_phys()
    s_c.om2phys()
    sc = np.array([s_c.phys(2).std(), s_c.phys(0).std(), s_c.phys(1).std(), 5.0], dtype=np.float32)
    s_c.attach_closure(net, sc, energy_check=0)
    F = s_c.closure_forcing().astype(np.complex128)
    d = s_c.scalars()
    s_p.step(1)
    s_c.step(1)
    assert s_c.closure_stats() == (1, 0)

    fn_p, fn_c = s_p.fnm1().astype(np.complex128), s_c.fnm1().astype(np.complex128)
    scale_fn = np.abs(fn_p).max() + np.abs(F).max()
    assert np.abs(fn_c - (fn_p + F)).max() <= 1e-6 * scale_fn

    H = N // 2
    kz = np.where(np.arange(N) < H, np.arange(N), np.arange(N) - N)[:, None]
    kx = np.arange(H)[None, :]
    K2 = (kx * kx + kz * kz).astype(np.float64)
    visc = 1.0 / RE
    coef = 0.5 * d["dt"] * (2.0 + d["cnm1"]) / (1.0 + 0.5 * visc * d["dt"] * K2)
    om_p, om_c = s_p.om2().astype(np.complex128), s_c.om2().astype(np.complex128)
    want = om_p + coef * F
    # the forcing term is resolved well above float rounding of the update
    assert np.abs(om_c - want).max() <= 2e-6 * np.abs(om_p).max()
    assert np.abs(om_c - want).max() <= 0.01 * np.abs(om_c - om_p).max()
    for x in (s_p, s_c, net):
        x.close()


@pytest.mark.parametrize("check", [1, 2])
def test_energy_gate_drops_anti_dissipative_forcing(pkg, check):
    """F = omega (energy input 2E per unit time, far above 2 nu Z): every step falls back and the
    run is bit-identical to the plain run; without the gate the energy grows."""
    steps = 40
    s_p = _state(pkg)
    s_p.velocity_phys()
    s_p.om2phys()
    s_om = float(np.abs(s_p.phys(2)).max()) * 2.0
    net = _identity_net(pkg, s_om)
    sc = np.array([s_om, 1.0, 1.0, s_om], dtype=np.float32)

    s_g = _state(pkg)
    s_g.attach_closure(net, sc, energy_check=check)
    E_p, _ = s_p.step(steps, history=True)
    E_g, _ = s_g.step(steps, history=True)
    st = s_g.closure_stats()
    assert st[1] == steps, st
    np.testing.assert_array_equal(s_g.om2(), s_p.om2())
    np.testing.assert_array_equal(E_g, E_p)

    s_n = _state(pkg)
    s_n.attach_closure(net, sc, energy_check=0)
    E_n, _ = s_n.step(steps, history=True)
    assert s_n.closure_stats() == (steps, 0)
    assert E_n[-1] > E_p[-1] * 1.001
    for x in (s_p, s_g, s_n, net):
        x.close()


def test_energy_scaling_caps_the_forcing_input(pkg):
    """energy_check 3 with the anti-dissipative F = omega: every step is limited (scaled, not
    dropped), so the run differs from the plain one, and the forcing's input only replaces the
    viscous loss: the energy drifts by less than 5 % of the plain run's viscous decay (the time
    stepping's own O(dt^2) error), where an unlimited F = omega makes it grow."""
    steps = 40
    s_p = _state(pkg)
    s_p.velocity_phys()
    s_p.om2phys()
    s_om = float(np.abs(s_p.phys(2)).max()) * 2.0
    net = _identity_net(pkg, s_om)
    sc = np.array([s_om, 1.0, 1.0, s_om], dtype=np.float32)
    E0, _ = s_p.energy_enstrophy()
    s_s = _state(pkg)
    s_s.attach_closure(net, sc, energy_check=3)
    E_p, _ = s_p.step(steps, history=True)
    E_s, _ = s_s.step(steps, history=True)
    assert s_s.closure_stats() == (steps, steps)
    decay = E0 - E_p[-1]
    assert decay > 0
    assert np.max(np.abs(E_s - E0)) < 0.05 * decay
    assert not np.array_equal(s_s.om2(), s_p.om2())
    for x in (s_p, s_s, net):
        x.close()


def test_trained_closure_improves_coarse_run(pkg):
    """Train on filtered N=256 DNS, run N=32 with and without the closure to the DNS end time."""
    from optimizec_b200 import closure as CL

    cfg = dict(Nf=256, Nc=32, Re=RE, K0=4.0, cfl=0.1)
    X, T = CL.generate(seeds=range(4), steps=3000, every=40, warm=200, **cfg)
    assert X.shape == (280, 3, 48, 48) and T.shape == (280, 1, 48, 48)
    net, scales, losses = CL.train(X, T, iters=600, batch=32, lr=1e-3)
    assert np.mean(losses[-50:]) < 0.25 * np.mean(losses[:10])
    r = CL.evaluate(net, scales, seed=100, fine_steps=4000, check=1, **cfg)
    p, c = r["plain"], r["closure"]
    assert abs(c["t"] - r["t_end"]) < 0.01 * r["t_end"]
    assert c["closure_steps"] == c["steps"]
    assert c["shell_err_mean"] < 0.5 * p["shell_err_mean"], r
    assert c["shell_err_max"] < 0.5 * p["shell_err_max"], r
    assert c["enstrophy_err"] < p["enstrophy_err"], r
    net.close()


def test_tensor_core_forcing_matches_fp32_forcing(pkg):
    """N = 256 (L = 384): the closure runs its hidden layers on the BF16 tensor-core path by
    default; its forcing spectrum agrees with the FP32 network's within bf16 rounding."""
    s = pkg.Solver(256, 1e5, 4.0, 0.1)
    s.init_k4(2)
    s.next_dt()
    net = pkg.CNN(6, 32, seed=4)
    s.velocity_phys()
    s.om2phys()
    sc = np.array([s.phys(2).std(), s.phys(0).std(), s.phys(1).std(), 0.3], dtype=np.float32)
    s.attach_closure(net, sc, energy_check=1)
    F_tc = s.closure_forcing().astype(np.complex128)
    s.closure_tensor_cores(False)
    F_32 = s.closure_forcing().astype(np.complex128)
    s.closure_tensor_cores(True)
    assert np.linalg.norm(F_tc - F_32) <= 3e-2 * np.linalg.norm(F_32)
    assert np.linalg.norm(F_tc - F_32) > 0.0  # the two paths differ (bf16), so both ran
    s.step(10)
    assert s.closure_stats()[0] == 10
    s.close()
    net.close()


def test_forcing_limiter_bounds_each_mode(pkg):
    """With closure_clamp(alpha), the forcing a closed step adds to FN (closed FNM1 minus the plain
    step's FNM1 from the same state) is at most alpha |FN| on every mode, and binds on some."""
    alpha = 0.5
    s_p = _state(pkg)
    s_c = _state(pkg)
    net = pkg.CNN(3, 8, seed=11)
    s_c.velocity_phys()
    s_c.om2phys()
    sc = np.array([s_c.phys(2).std(), s_c.phys(0).std(), s_c.phys(1).std(), 5.0], dtype=np.float32)
    s_c.attach_closure(net, sc, energy_check=0)
    F = s_c.closure_forcing().astype(np.complex128)
    s_c.closure_clamp(alpha)
    s_p.step(1)
    s_c.step(1)
    fn = s_p.fnm1().astype(np.complex128)
    applied = s_c.fnm1().astype(np.complex128) - fn
    tol = 1e-6 * (np.abs(fn).max() + np.abs(F).max())
    assert np.all(np.abs(applied) <= alpha * np.abs(fn) * (1 + 1e-5) + tol)
    limited = np.abs(F) > alpha * np.abs(fn) * 1.01 + tol
    assert limited.any()
    # where it does not bind, the forcing is applied unchanged
    free = np.abs(F) < alpha * np.abs(fn) * 0.99
    assert np.abs(applied[free] - F[free]).max() <= tol
    for x in (s_p, s_c, net):
        x.close()
