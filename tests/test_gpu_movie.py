"""Movie frames: the library's inferno rendering against the oracle's restatement (bit-exact),
and the CLI's PNG frames (folder naming, frame numbering across runs, decodable PNG) against the
reference's own mem_cuda MOV frames when that binary is present."""
import os
import struct
import subprocess
import zlib

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(REPO, "optimizec_b200", "mem_cuda")
REF = os.path.join(REPO, "oracle", "_ref", "mem_cuda")


def read_png(path):
    """Decode an 8-bit RGB, non-interlaced PNG with filter-0 rows; checks every chunk CRC and the
    zlib Adler-32 (zlib.decompress does)."""
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat = 8, b""
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        typ = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        crc, = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert zlib.crc32(typ + body) & 0xFFFFFFFF == crc
        if typ == b"IHDR":
            w, h, depth, ctype, comp, filt, inter = struct.unpack(">IIBBBBB", body)
            assert (depth, ctype, comp, filt, inter) == (8, 2, 0, 0, 0)
        elif typ == b"IDAT":
            idat += body
        elif typ == b"IEND":
            break
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), dtype=np.uint8).reshape(h, 3 * w + 1)
    assert np.all(raw[:, 0] == 0)
    return raw[:, 1:].reshape(h, w, 3).copy()


@pytest.mark.parametrize("N,F", [(128, 0), (256, 1), (256, 3), (1024, 0), (2048, 0)])
def test_frame_matches_oracle(N, F):
    """Bit-exact against the restatement, including F = 1 frames larger than one scratch band."""
    import optimizec_b200 as P
    s = P.Solver(N, 1e4, 4.0, 0.1)
    s.init_k4(3)
    s.next_dt()
    s.step(20)
    s.om2phys()
    rgb, sigma = s.movie_frame(2, F)
    ref, ref_sigma = O.render_frame(s.phys(2), F or O.movie_scale(N))
    assert rgb.shape == ref.shape
    assert sigma == ref_sigma
    assert np.array_equal(rgb, ref)


def test_frame_constant_and_nonfinite():
    """A constant plane renders pixel 128 everywhere; non-finite points are pixel 128 and do not
    enter the min/max."""
    import optimizec_b200 as P
    s = P.Solver(128, 1e4, 4.0, 0.1)
    L = s.L
    zero = np.zeros((L, L), np.float32)
    s.set_velocity_phys(zero, zero)   # planes 0 and 1
    rgb, sigma = s.movie_frame(0, 1)
    assert sigma == 0.0
    assert np.all(rgb == O.inferno_lut()[128])
    f = np.random.default_rng(5).standard_normal((L, L)).astype(np.float32)
    f[3, 7] = np.inf
    f[10, 0] = np.nan
    s.set_velocity_phys(f, zero)
    rgb, sigma = s.movie_frame(0, 1)
    ref, ref_sigma = O.render_frame(f, 1)
    assert sigma == ref_sigma
    assert np.array_equal(rgb, ref)


def _run(exe, args, cwd, movdir, mov=None):
    env = dict(os.environ, MOV_DIR=str(movdir))
    env.pop("MOV", None)
    if mov is not None:
        env["MOV"] = mov
    return subprocess.run([exe, *map(str, args)], cwd=cwd, env=env, capture_output=True, text=True, timeout=300)


def test_cli_frames_and_numbering(tmp_path):
    N, update = 256, 25
    args = [N, 10000, 4, 50, 0.1, update, 0, "MOV"]
    r = _run(CLI, args, tmp_path, tmp_path / "mov")
    assert r.returncode == 0, r.stderr
    folder = tmp_path / "mov" / "cuda_256_4_1E04_0.100_U25"
    assert f"[MOV] Saving omega_inferno_%05d.png every {update} steps to {folder} (F=1, next=00001)" in r.stdout
    assert sorted(os.listdir(folder)) == ["omega_inferno_00001.png", "omega_inferno_00002.png"]
    assert f"[MOV] Wrote {folder / 'omega_inferno_00002.png'} (Inferno PNG, 384x384, F=1, comp=2, sigma=" in r.stdout
    img = read_png(folder / "omega_inferno_00002.png")
    assert img.shape == (384, 384, 3)
    # a second run appends after the frames already in the folder
    r2 = _run(CLI, args, tmp_path, tmp_path / "mov")
    assert r2.returncode == 0, r2.stderr
    assert "(F=1, next=00003)" in r2.stdout
    assert sorted(os.listdir(folder))[-1] == "omega_inferno_00004.png"
    # same trajectory both times (PAO initial condition), so the same picture
    assert np.array_equal(read_png(folder / "omega_inferno_00004.png"), img)
    # MOV=0 in the environment overrides the argument
    r3 = _run(CLI, args, tmp_path, tmp_path / "off", mov="0")
    assert r3.returncode == 0 and "[MOV]" not in r3.stdout and not (tmp_path / "off").exists()


@pytest.mark.skipif(not os.path.exists(REF), reason="reference binary not built")
def test_cli_frames_match_reference(tmp_path):
    """Same run, same frames as the reference's mem_cuda: the fields differ by FP32 transform noise,
    so a pixel's colour index may move by one step at a boundary."""
    N, update = 512, 50
    args = [N, 10000, 4, 100, 0.1, update, 0, "MOV"]
    (tmp_path / "r").mkdir()
    r = _run(REF, args, tmp_path / "r", tmp_path / "rm")
    o = _run(CLI, args, tmp_path, tmp_path / "om")
    assert r.returncode == 0, r.stderr
    assert o.returncode == 0, o.stderr
    sub = "cuda_512_4_1E04_0.100_U50"
    for k in (1, 2):
        name = f"omega_inferno_{k:05d}.png"
        a = read_png(tmp_path / "rm" / sub / name).astype(int)
        b = read_png(tmp_path / "om" / sub / name).astype(int)
        assert a.shape == b.shape
        same = np.all(a == b, axis=2).mean()
        assert same >= 0.99, same
        assert np.abs(a - b).max() <= 8
        # same PNG layout (stored deflate of the same size)
        assert os.path.getsize(tmp_path / "rm" / sub / name) == os.path.getsize(tmp_path / "om" / sub / name)
