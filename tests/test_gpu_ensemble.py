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


PERSISTENT_MEMBERS = [(64, 2.0e3, 3.0, 0.1, 0), (128, 5.0e4, 4.0, 0.1, 1), (512, 1.0e4, 6.0, 0.2, 2),
                      (256, 1.5e3, 2.0, 0.1, 3), (128, 1.0e5, 8.0, 0.1, 4), (256, 3.0e4, 5.0, 0.1, 5)]


def _run(mode, members, steps=(1, 150)):
    import optimizec_b200 as P
    b = P.Batch(members)
    b.set_mode(mode)
    b.init_k4()
    b.next_dt()
    E1, Z1 = b.step(steps[0], history=True)
    b.next_dt()
    E2, Z2 = b.step(steps[1], history=True)
    b.next_dt()
    out = ([b.om2(m) for m in range(len(members))], np.concatenate([E1, E2], axis=1),
           np.concatenate([Z1, Z2], axis=1), [b.scalars(m) for m in range(len(members))])
    b.close()
    return out


def test_persistent_launch_equals_graph_mode():
    """Mode 1 (every member of sizes 64 ... 512 advanced inside one persistent launch per chunk of
    up to 128 steps, work items in dependency order) against mode 0 (one graph per chunk, a
    branch per size group): 151 steps, across a chunk boundary -- the same fields bit for bit, the
    energy / enstrophy histories to 1e-12 (their FP64 partials are summed per item instead of per
    column), the same scalars."""
    g = _run(0, PERSISTENT_MEMBERS)
    p = _run(1, PERSISTENT_MEMBERS)
    for m in range(len(PERSISTENT_MEMBERS)):
        np.testing.assert_array_equal(p[0][m], g[0][m])
        for k in ("it", "t", "dt", "cn", "cnm1", "cflm", "visc"):
            assert p[3][m][k] == g[3][m][k], (m, k)
    np.testing.assert_allclose(p[1], g[1], rtol=1e-12)
    np.testing.assert_allclose(p[2], g[2], rtol=1e-12)


def test_persistent_launch_wait_times_out():
    """A dependency wait of the persistent launch that nothing satisfies (member 1's column items
    wait for a row count that is never reached) gives up after its poll limit: dns2d_batch_step
    returns DNS2D_ERR_TIMEOUT, every CTA stops, and the context stays usable (the batch steps again
    from a fresh field, and a new solver runs)."""
    import optimizec_b200 as P
    members = [(128, 1e4, 4.0, 0.1, 0), (256, 1e4, 4.0, 0.1, 1)]
    b = P.Batch(members)
    b.set_mode(1)
    b.init_k4()
    b.next_dt()
    b.set_waits(20000, 1)
    with pytest.raises(P.Dns2dError, match="wait ran out"):
        b.step(3)
    b.set_waits(1 << 22, -1)
    b.init_k4()
    b.next_dt()
    E, _ = b.step(3, history=True)
    assert np.all(np.isfinite(E)) and np.all(np.abs(E - 0.5) < 1e-3)
    b.close()
    s = P.Solver(64, 1e4, 4.0, 0.1)
    s.init_k4(0)
    s.next_dt()
    s.step(2)
    s.sync()
    s.close()


def test_persistent_mode_sizes():
    """The persistent launch serves the sizes 64, 128, 256 and 512; a batch with another size keeps
    the graph mode (DNS2D_ERR_SIZE)."""
    import optimizec_b200 as P
    b = P.Batch([(128, 1e4, 4.0, 0.1, 0), (1024, 1e4, 4.0, 0.1, 1)])
    with pytest.raises(P.Dns2dError):
        b.set_mode(1)
    b.close()
