"""CPU tests of the FP64 oracle: its FFT against numpy.fft, its PAO-k^-3 port and its full step
against the reference's recorded stdout (tests/golden/reference_stdout.json)."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("L", [6, 12, 24, 48, 72, 96, 192, 384, 768, 1536, 6144, 44100, 210, 35, 2 * 3 * 5 * 7 * 4])
def test_fft_c2c_matches_numpy(L):
    rng = np.random.default_rng(L)
    x = rng.standard_normal(L) + 1j * rng.standard_normal(L)
    ref = np.fft.fft(x)
    got = O.fft_c2c(x)
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    inv = O.fft_c2c(x, inverse=True)
    assert np.abs(inv - np.fft.ifft(x) * L).max() <= 1e-13 * np.abs(inv).max()


@pytest.mark.parametrize("L", [24, 48, 96, 192])
def test_2d_transforms_match_numpy(L):
    rng = np.random.default_rng(L)
    a = rng.standard_normal((L, L))
    s = O.fwd2d(a)
    assert np.abs(s - np.fft.rfft2(a)).max() <= 1e-12 * np.abs(s).max()
    b = O.inv2d(s)
    assert np.abs(b - a * L * L).max() <= 1e-11 * np.abs(b).max()


def _golden_run(golden, n):
    for r in golden["runs"]:
        if r["file"].startswith(f"sim_output_{n}"):
            return r
    raise KeyError(n)


@pytest.mark.parametrize("name", ["512", "4096"])
def test_pao_stats_match_reference_stdout(golden, name):
    run = _golden_run(golden, name)
    _, stats, seed = O.pao_spectrum(run["N"], run["K0"], run["Re"])
    assert seed == run["pao_seed"]
    for key, txt in run["pao"].items():
        # printed with %12.7f / %12.5f / %12.4f / %12.1f: compare at the printed precision
        decimals = len(txt.split(".")[1]) if "." in txt else 0
        assert round(stats[key], decimals) == pytest.approx(float(txt), abs=1.5 * 10 ** -decimals), key


def test_pao_stats_n16384(golden):
    # the two N=16384 runs share the PAO seed; their K0/Re differ
    for name in ["16384_21", "16384_101"]:
        run = _golden_run(golden, name)
        _, stats, seed = O.pao_spectrum(run["N"], run["K0"], run["Re"])
        assert seed == run["pao_seed"]
        for key in ["Energy", "WiWi", "Epsilon", "a11", "e11"]:
            txt = run["pao"][key]
            decimals = len(txt.split(".")[1])
            assert stats[key] == pytest.approx(float(txt), abs=1.5 * 10 ** -decimals), key


def test_step_matches_reference_trajectory_n512(golden):
    """Init CFLM and the it=1 / it=100 lines of the reference's N=512 run (CFL 0.25, K0 10)."""
    run = _golden_run(golden, "512")
    o = O.Oracle(run["N"], run["Re"], run["K0"], run["CFL"])
    o.init_pao()
    sc = o.scalars()
    assert sc["cflm"] == pytest.approx(run["nextdt_init"]["CFLM"], rel=2e-7)
    assert sc["dt"] == pytest.approx(run["nextdt_init"]["DT"], abs=1e-7)
    its = {r["it"]: r for r in run["iterations"]}
    _, _, d = o.run(1, run["UPDATE"], run["STEPS"])
    g = its[1]
    assert d[1] == pytest.approx(g["T"], abs=2e-10)
    assert d[3] == pytest.approx(g["CN"], abs=2e-8)
    assert d[4] == pytest.approx(g["CFLM"], rel=3e-7)
    assert int(d[5]) == g["SIG"]
    _, _, d = o.run(99, run["UPDATE"], run["STEPS"])
    g = its[100]
    assert d[1] == pytest.approx(g["T"], abs=2e-10)
    assert d[2] == pytest.approx(g["DT"], abs=1e-8)
    assert d[3] == pytest.approx(g["CN"], abs=2e-8)
    assert d[4] == pytest.approx(g["CFLM"], rel=3e-7)
    assert int(d[5]) == g["SIG"]


@pytest.mark.parametrize("N,K0,seed", [(64, 4.0, 0), (512, 4.0, 7), (128, 8.0, 63)])
def test_k4_spectrum_properties(N, K0, seed):
    om = O.k4_spectrum(N, K0, seed)
    H = N // 2
    E, Z = O.energy_enstrophy(om.astype(np.complex128))
    assert E == pytest.approx(0.5, rel=1e-6)
    assert om[0, 0] == 0
    assert np.all(om[H, :] == 0)  # kz = -N/2 row
    # Hermitian kx = 0 column
    for iz in range(1, H):
        assert om[N - iz, 0] == np.conj(om[iz, 0])
    # shell spectrum peaks near K0 with the k^4 exp(-2 (k/K0)^2) shape
    Ek = O.shell_spectrum(om.astype(np.complex128))
    assert abs(int(np.argmax(Ek)) - K0) <= 2


def test_k4_product_generator_matches_oracle():
    """The library's host IC generator and the oracle's produce identical bytes."""
    import optimizec_b200 as P
    for N, K0, seed in [(64, 4.0, 0), (256, 4.0, 5), (512, 3.0, 11)]:
        a = O.k4_spectrum(N, K0, seed)
        b = P.k4_spectrum(N, K0, seed)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_oracle_energy_history_is_monotone_decay():
    o = O.Oracle(64, 1e3, 4.0, 0.1)
    o.init_om2(O.k4_spectrum(64, 4.0, 1))
    E, Z, _ = o.run(20, 100, 20)
    assert np.all(np.diff(E) < 0)  # 2D decaying turbulence: energy decays monotonically
    assert np.all(Z > 0)


def test_movie_restatement_rules():
    """Colour table stops, the reference's per-size downsampling factors, constant planes."""
    lut = O.inferno_lut()
    assert lut[0].tolist() == [0, 0, 4] and lut[255].tolist() == [252, 255, 164]
    assert [O.movie_scale(n) for n in (256, 2560, 4096, 9216, 16384, 29400)] == [1, 1, 2, 8, 12, 14]
    rgb, sigma = O.render_frame(np.full((12, 12), 3.0, np.float32), 5)
    assert rgb.shape == (3, 3, 3) and sigma == 0.0 and np.all(rgb == lut[128])


def test_restart_v2_writer_layout(tmp_path):
    """The oracle's restart.bin v2 writer (how the seeded field reaches the reference's own
    loader): 144-byte header with the dims and scalars of the state, UR planes u, w of the
    oracle's recovered velocity, OM2 equal to the seeded field, FNM1 zero."""
    import struct
    N, Re, K0, cfl = 16, 1e4, 4.0, 0.1
    o = O.Oracle(N, Re, K0, cfl)
    om = O.k4_spectrum(N, K0, 3)
    o.init_om2(om)
    path = tmp_path / "restart.bin"
    n = O.write_restart_v2(str(path), o, Re, K0, cfl)
    b = path.read_bytes()
    L, H = 3 * N // 2, N // 2
    assert len(b) == n == 144 + 3 * L * L * 4 + 2 * N * H * 8
    h = struct.unpack("<16s4I10i9f4x4Q", b[:144])
    assert h[0].rstrip(b"\0") == b"CTRB_RESTART" and h[1:5] == (2, 144, 4, 8)
    assert h[5:15] == (N, N, N, N, 3 * N // 4 + 1, L, L, 3 * N // 4 + 1, 0, 1)
    sc = o.scalars()
    Re_, K0_, visc, t, dt, cn, cnm1, cflnum, cflm = h[15:24]
    assert (t, cn, cnm1) == (0.0, 1.0, 0.0) and dt == np.float32(sc["dt"]) and dt > 0
    assert cflm == np.float32(sc["cflm"]) and cflnum == np.float32(cfl) and Re_ == np.float32(Re)
    assert h[24:] == (0, N * H, N * H, 3 * L * L)
    ur = np.frombuffer(b, dtype=np.float32, count=3 * L * L, offset=144).reshape(3, L, L)
    assert np.array_equal(ur[0], o.ur(0).astype(np.float32)) and not ur[2].any()
    om2 = np.frombuffer(b, dtype=np.complex64, count=N * H, offset=144 + 12 * L * L).reshape(N, H)
    assert np.array_equal(om2, om)
    assert not np.frombuffer(b, dtype=np.complex64, offset=144 + 12 * L * L + 8 * N * H).any()
    o.close()
