"""GPU tests of the batched ensemble (dns2d_batch_*): every member must follow exactly the run
that a single-state solver with the same N, Re, K0, CFL and seed produces (same kernels, same
float scalar bookkeeping), and the ensemble configuration itself must be well formed."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_batch_members_equal_single_runs():
    import optimizec_b200 as P
    members = [(64, 2.0e3, 3.0, 0.1, 0), (128, 5.0e4, 4.0, 0.1, 1), (64, 1.0e4, 6.0, 0.2, 2),
               (128, 1.5e3, 2.0, 0.1, 3), (256, 1.0e5, 8.0, 0.1, 4)]
    b = P.Batch(members)
    b.init_k4()
    b.next_dt()
    E1, Z1 = b.step(1, history=True)
    b.next_dt()
    E2, Z2 = b.step(30, history=True)
    b.next_dt()
    for m, (N, Re, K0, cfl, seed) in enumerate(members):
        s = P.Solver(N, Re, K0, cfl)
        s.init_k4(seed)
        s.next_dt()
        e1, z1 = s.step(1, history=True)
        s.next_dt()
        e2, z2 = s.step(30, history=True)
        s.next_dt()
        np.testing.assert_array_equal(b.om2(m), s.om2())
        np.testing.assert_allclose(np.concatenate([E1[m], E2[m]]), np.concatenate([e1, e2]), rtol=1e-12)
        sb, ss = b.scalars(m), s.scalars()
        for k in ("it", "t", "dt", "cn", "cnm1", "cflm", "visc"):
            assert sb[k] == ss[k], (m, k)
        s.close()
    b.close()


def test_ensemble_configuration():
    import optimizec_b200 as P
    ms = P.ensemble_members()
    assert len(ms) == 64
    assert [m[0] for m in ms].count(128) == 32 and [m[0] for m in ms].count(256) == 24
    assert all(1e3 <= m[1] <= 1e5 and 2 <= m[2] <= 8 for m in ms)
    assert [m[4] for m in ms] == list(range(64))
    b = P.Batch(ms)
    b.init_k4()
    b.next_dt()
    E, Z = b.step(20, history=True)
    assert np.all(np.isfinite(E)) and np.all(np.abs(E - 0.5) < 1e-3)
    # decaying turbulence: over 20 steps the energy of every member decreases; per step the
    # viscous decay of the high-Re members (~1e-8) is below FP32 rounding of the nonlinear term
    assert np.all(E[:, -1] < E[:, 0])
    b.close()


def test_batch_autotune_keeps_results():
    """dns2d_batch_autotune (before init) picks kernel variants per size group: the tuned batch
    reproduces the untuned one bit for bit where the group keeps its default radix plans, and to
    FP32 rounding (relative L2 <= 1e-6 after 10 steps) where the tuner picked another plan."""
    import optimizec_b200 as P
    ms = [(128, 3e3, 3.0, 0.1, 1), (256, 1e4, 4.0, 0.1, 2), (128, 1e4, 5.0, 0.1, 3), (1024, 1e4, 4.0, 0.1, 4)]
    out = []
    for tune in (False, True):
        b = P.Batch(ms)
        if tune:
            b.autotune()
        b.init_k4()
        b.next_dt()
        b.step(1)
        b.next_dt()
        b.step(9)
        out.append([b.om2(m) for m in range(len(ms))])
        b.close()
    for a, c in zip(out[0], out[1]):
        a, c = a.astype(np.complex128), c.astype(np.complex128)
        assert np.linalg.norm(a - c) / np.linalg.norm(a) <= 1e-6


def test_batch_prepare_builds_graphs_without_stepping():
    """dns2d_batch_prepare captures the chunk graphs of a later dns2d_batch_step without running
    them: the members do not move, and the prepared batch steps like an unprepared one."""
    import optimizec_b200 as P
    ms = [(128, 3e3, 3.0, 0.1, 1), (256, 1e4, 4.0, 0.1, 2)]
    out = []
    for prep in (False, True):
        b = P.Batch(ms)
        b.init_k4()
        b.next_dt()
        before = [b.om2(m) for m in range(len(ms))]
        if prep:
            b.prepare(150)
            b.sync()
            for m in range(len(ms)):
                np.testing.assert_array_equal(b.om2(m), before[m])
                assert b.scalars(m)["it"] == 0
        b.step(150)
        out.append([b.om2(m) for m in range(len(ms))])
        b.close()
    for a, c in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, c)
