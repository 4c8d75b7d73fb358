"""Autotuner: rows per CTA, thread groups per column CTA and L2 prefetch distances give
bit-identical fields (they do not change the arithmetic); the radix plans of the small-grid passes
change the FP32 rounding, and every plan meets the FP64 oracle tolerances of the parity tests."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def P():
    import optimizec_b200 as mod

    return mod


def _run(N, steps=12):
    s = P().Solver(N, 1e4, 4.0, 0.1)
    s.init_k4(9)
    s.next_dt()
    s.step(1)
    s.next_dt()
    E, _ = s.step(steps - 1, history=True)
    om = s.om2()
    s.close()
    return om, E


@pytest.mark.parametrize("N", [128, 512, 2048])
def test_autotuned_variants_give_identical_fields(N):
    """Bit-identical when the tuner keeps the default radix plans, within FP32 rounding when it
    picks another plan."""
    om0, _ = _run(N)
    cfg = P().autotune(N)
    if N >= 1024:
        assert cfg["cols_groups"] in (1, 2) and cfg["pf_rows"] in (0, 148, 296, 444, 592)
        assert cfg["pf_cols"] in (0, 37, 74, 148)
        assert cfg["plan_rows"] == cfg["plan_cols"] == 0
    else:
        assert cfg["rows_tile"] in (2, 4, 8)
        assert cfg["plan_rows"] in (0, 1, 2) and cfg["plan_cols"] in (0, 1, 2)
    om1, _ = _run(N)
    P().set_tuning(N)
    if cfg["plan_rows"] == cfg["plan_cols"] == 0:
        np.testing.assert_array_equal(om1, om0)
    else:
        a, b = om1.astype(np.complex128), om0.astype(np.complex128)
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-6


@pytest.mark.parametrize("N", [64, 128, 256, 512])
@pytest.mark.parametrize("plan_rows,plan_cols", [(0, 0), (1, 1), (2, 2), (1, 2)])
def test_every_radix_plan_matches_oracle(N, plan_rows, plan_cols):
    """Each radix plan the tuner can choose: 20 steps from the seeded k^4 field against the FP64
    oracle, vorticity relative L2 <= 1e-5 and energy history <= 1e-6 relative."""
    from oracle import oracle as O
    om0 = O.k4_spectrum(N, 4.0, 5)
    o = O.Oracle(N, 1e4, 4.0, 0.1)
    o.init_om2(om0)
    P().set_tuning(N, plan_rows=plan_rows, plan_cols=plan_cols)
    try:
        s = P().Solver(N, 1e4, 4.0, 0.1)
    finally:
        P().set_tuning(N)
    s.init_vorticity(om0)
    s.next_dt()
    E, _ = s.step(1, history=True)
    s.next_dt()
    E2, _ = s.step(19, history=True)
    Er, _, _ = o.run(20, 1000, 20, want_diag=False)  # NEXTDT at init, it = 1 and it = 20
    a, b = s.om2().astype(np.complex128), o.om2()
    s.close()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-5
    E = np.concatenate([E, E2])
    assert np.max(np.abs(E / Er - 1)) <= 1e-6


@pytest.mark.parametrize("N,configs", [
    (256, [(2, 0, 296, 74), (4, 0, 296, 74), (8, 0, 296, 74), (2, 0, 296, 74, 1, 2), (8, 0, 296, 74, 1, 2)]),
    (2048, [(0, 1, 0, 0), (0, 2, 296, 74), (0, 1, 592, 148), (0, 2, 148, 37)]),
])
def test_every_variant_gives_identical_fields(N, configs):
    """Each configuration the autotuner can choose, pinned in turn: with the same radix plans,
    bit-identical fields and the FP64 energy history to rounding (the column kernels' per-thread
    partial sums differ in order)."""
    ref = {}
    for cfg in configs:
        P().set_tuning(N, *cfg)
        om, E = _run(N)
        plans = tuple(cfg[4:]) or (0, 0)
        if plans not in ref:
            ref[plans] = (om, E)
            continue
        np.testing.assert_array_equal(om, ref[plans][0])
        np.testing.assert_allclose(E, ref[plans][1], rtol=1e-14, atol=0)
    P().set_tuning(N)
    assert len(ref) == (2 if N == 256 else 1)
