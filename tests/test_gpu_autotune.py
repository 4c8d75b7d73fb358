"""Autotuner: the chosen kernel variants give bit-identical fields (the variants differ in rows
per CTA, thread groups per column CTA and L2 prefetch distances, not in arithmetic)."""
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
    om0, _ = _run(N)
    cfg = P().autotune(N)
    if N >= 1024:
        assert cfg["cols_groups"] in (1, 2) and cfg["pf_rows"] in (0, 148, 296, 592)
        assert cfg["pf_cols"] in (0, 37, 74, 148)
    else:
        assert cfg["rows_tile"] in (2, 4, 8)
    om1, _ = _run(N)
    np.testing.assert_array_equal(om1, om0)


@pytest.mark.parametrize("N,configs", [
    (256, [(2, 0, 296, 74), (4, 0, 296, 74), (8, 0, 296, 74)]),
    (2048, [(0, 1, 0, 0), (0, 2, 296, 74), (0, 1, 592, 148), (0, 2, 148, 37)]),
])
def test_every_variant_gives_identical_fields(N, configs):
    """Each configuration the autotuner can choose, pinned in turn: bit-identical fields; the FP64
    energy history to rounding (the column kernels' per-thread partial sums differ in order)."""
    P().set_tuning(N, *configs[0])
    om_ref, E_ref = _run(N)
    for cfg in configs[1:]:
        P().set_tuning(N, *cfg)
        om, E = _run(N)
        np.testing.assert_array_equal(om, om_ref)
        np.testing.assert_allclose(E, E_ref, rtol=1e-14, atol=0)
    P().set_tuning(N)
