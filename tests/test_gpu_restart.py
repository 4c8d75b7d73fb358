"""restart.bin through the pinned staging pipeline: file bytes against the state's own arrays at
sizes where the file spans one to many staging chunks (chunk boundaries fall inside the header,
the UR planes and OM2/FNM1), v1 and v2 files with and without a UC payload, short files."""
import struct
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HDR = "<16s4I10i9f4x4Q"   # v2 header, 144 bytes (cuda/mem_cuda.cu:1019-1054)
HDR1 = "<16s4I10i9f4x3Q"  # v1 header, 136 bytes


def P():
    import optimizec_b200
    return optimizec_b200


def _state(N, seed=5, steps=6):
    s = P().Solver(N, 1e4, 4.0, 0.1)
    s.init_k4(seed)
    s.next_dt()
    s.step(steps)
    return s


def _header(N, version=2, uc=False, it=17, t=0.25):
    L, H = 3 * N // 2, N // 2
    nk = L // 2 + 1
    ucn = nk * L * 3 if (version == 1 or uc) else 0
    counts = (ucn, N * H, N * H) + ((3 * L * L,) if version == 2 else ())
    fmt = HDR if version == 2 else HDR1
    return struct.pack(fmt, b"CTRB_RESTART", version, struct.calcsize(fmt), 4, 8,
                       N, N, N, N, nk, L, L, nk, it, 1,
                       1e4, 4.0, 1e-4, t, 1e-3, 0.5, 0.25, 0.1, 0.09, *counts), ucn


@pytest.mark.parametrize("N", [128, 512, 2048])
def test_saved_bytes_are_the_state(N, tmp_path):
    s = _state(N)
    path = tmp_path / "r.bin"
    s.save_restart(str(path))
    L, H = 3 * N // 2, N // 2
    data = path.read_bytes()
    assert len(data) == 144 + 3 * L * L * 4 + 2 * N * H * 8
    h = struct.unpack(HDR, data[:144])
    sc = s.scalars()
    assert h[0].rstrip(b"\0") == b"CTRB_RESTART" and h[1:5] == (2, 144, 4, 8)
    assert h[5:15] == (N, N, N, N, L // 2 + 1, L, L, L // 2 + 1, sc["it"], 1)
    assert h[24:] == (0, N * H, N * H, 3 * L * L)
    ur = np.frombuffer(data, np.float32, 3 * L * L, 144).reshape(3, L, L)
    for c in range(3):
        np.testing.assert_array_equal(ur[c], s.phys(c))   # the save computed the velocity planes
    off = 144 + 3 * L * L * 4
    om = np.frombuffer(data, np.complex64, N * H, off).reshape(N, H)
    fn = np.frombuffer(data, np.complex64, N * H, off + N * H * 8).reshape(N, H)
    np.testing.assert_array_equal(om, s.om2())
    np.testing.assert_array_equal(fn, s.fnm1())


@pytest.mark.parametrize("N,version,uc", [(256, 2, False), (256, 2, True), (256, 1, True), (1024, 2, False)])
def test_load_places_every_byte(N, version, uc, tmp_path):
    L, H = 3 * N // 2, N // 2
    rng = np.random.default_rng(N + version)
    head, ucn = _header(N, version, uc)
    om = ((rng.standard_normal((N, H)) + 1j * rng.standard_normal((N, H))) * 1e-3).astype(np.complex64)
    fn = ((rng.standard_normal((N, H)) + 1j * rng.standard_normal((N, H))) * 1e-3).astype(np.complex64)
    parts = [head, rng.standard_normal(2 * ucn).astype(np.float32).tobytes()]
    if version == 2:
        parts.append(rng.standard_normal(3 * L * L).astype(np.float32).tobytes())
    parts += [om.tobytes(), fn.tobytes()]
    path = tmp_path / "in.bin"
    path.write_bytes(b"".join(parts))
    s = P().Solver(N, 1e4, 4.0, 0.1)
    s.load_restart(str(path))
    np.testing.assert_array_equal(s.om2(), om)
    np.testing.assert_array_equal(s.fnm1(), fn)
    sc = s.scalars()
    assert sc["it"] == 17 and sc["t"] == 0.25 and sc["cn"] == 0.5 and sc["cnm1"] == 0.25
    # a short file is refused before the state is touched
    path.write_bytes(b"".join(parts)[:-8])
    s2 = P().Solver(N, 1e4, 4.0, 0.1)
    with pytest.raises(P().Dns2dError, match="short payload"):
        s2.load_restart(str(path))


def test_staged_roundtrip_continues_exactly(tmp_path):
    """N=4096 (a 520 MB file, nine staging chunks): save, load into a fresh state: the same OM2,
    FNM1 and scalars, and the two states step on together (the loaded velocity is the forward
    transform of the saved physical planes, equal to FP32 rounding); save/load throughput printed
    for the record."""
    N = 4096
    s = _state(N, seed=2, steps=3)
    path = str(tmp_path / "big.bin")
    s.save_restart(path)   # the first call allocates the staging buffers
    t0 = time.perf_counter()
    s.save_restart(path)
    t_save = time.perf_counter() - t0
    s2 = P().Solver(N, 1e4, 4.0, 0.1)
    s2.load_restart(path)
    t0 = time.perf_counter()
    s2.load_restart(path)
    t_load = time.perf_counter() - t0
    size = 144 + 27 * N * N + 8 * N * (N // 2)
    print(f"restart N={N}: {size / 1e6:.0f} MB, save {size / t_save / 1e9:.2f} GB/s, load {size / t_load / 1e9:.2f} GB/s")
    assert s2.scalars() == s.scalars()
    np.testing.assert_array_equal(s2.om2(), s.om2())
    np.testing.assert_array_equal(s2.fnm1(), s.fnm1())
    s.step(4)
    s2.step(4)
    a, b = s2.om2().astype(np.complex128), s.om2().astype(np.complex128)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5   # 1.7e-6 measured at N=4096


def test_library_reads_oracle_written_restart(tmp_path):
    """The restart.bin v2 file that the bench writes (from the FP64 oracle) for the reference's
    loader is also read by this library: same field, same scalars, and the run continues along the
    same trajectory as a run started from the field itself."""
    from oracle import oracle as O
    N, Re, K0, cfl = 256, 1e4, 4.0, 0.1
    om = O.k4_spectrum(N, K0, 9)
    o = O.Oracle(N, Re, K0, cfl)
    o.init_om2(om)
    path = str(tmp_path / "restart.bin")
    O.write_restart_v2(path, o, Re, K0, cfl)
    a = P().Solver(N, Re, K0, cfl)
    a.load_restart(path)
    assert np.array_equal(a.om2(), om)
    sa = a.scalars()
    assert sa["it"] == 0 and sa["dt"] == np.float32(o.scalars()["dt"])
    b = P().Solver(N, Re, K0, cfl)
    b.init_vorticity(om)
    b.next_dt()
    assert sa["dt"] == pytest.approx(b.scalars()["dt"], rel=2e-6)
    b.set_scalars(dt=sa["dt"], visc=sa["visc"])
    for s in (a, b):
        s.step(1)
        s.next_dt()
        s.step(9)
    x, y = a.om2().astype(np.complex128), b.om2().astype(np.complex128)
    assert np.linalg.norm(x - y) / np.linalg.norm(y) <= 1e-6
    o.close()
