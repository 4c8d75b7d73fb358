"""ctypes front end of the FP64 oracle (test infrastructure only).

Loaded by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` as the
checker of the CUDA path; the product never imports this module.  The C source is
``oracle/dns2d_oracle.c``; ``make -C oracle`` (or ``__graft_entry__.build()``) builds it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

PAO_STAT_NAMES = [
    "Reynolds n.", "Energy", "WiWi", "Epsilon", "a11", "e11", "Time scale", "Kolmogorov",
    "Viscosity", "dx/Kol.", "2Pi/Nlamda", "2Pi/Lux", "2Pi/Luz", "2Pi/Lwx", "2Pi/Lwz",
    "Deps.", "Ceps2", "E1", "E3",
]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.check_call(["make", "-s", "-C", _HERE, "oracle"])
        L = C.CDLL(path)
        dp = C.POINTER(C.c_double)
        fp = C.POINTER(C.c_float)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_fft_c2c.argtypes = [C.c_int, dp, dp, C.c_int]
        L.orc_pao_spectrum.argtypes = [C.c_int, C.c_float, C.c_float, fp, dp, C.POINTER(C.c_int)]
        L.orc_k4_spectrum.argtypes = [C.c_int, C.c_double, C.c_uint64, fp]
        L.orc_init_pao.restype = C.c_int
        L.orc_init_pao.argtypes = [C.c_void_p, dp]
        L.orc_init_om2.argtypes = [C.c_void_p, fp]
        L.orc_run.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, dp, dp, dp]
        L.orc_run_fixed.argtypes = [C.c_void_p, C.c_int, fp, fp, dp, dp]
        L.orc_get_scalars.argtypes = [C.c_void_p, dp]
        L.orc_set_f32_cn.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_scalars.argtypes = [C.c_void_p, dp]
        L.orc_get_om2.argtypes = [C.c_void_p, dp]
        L.orc_get_fnm1.argtypes = [C.c_void_p, dp]
        L.orc_get_ur.argtypes = [C.c_void_p, C.c_int, dp]
        L.orc_om2phys.argtypes = [C.c_void_p, dp]
        L.orc_display_sigma.restype = C.c_double
        L.orc_display_sigma.argtypes = [dp, C.c_size_t]
        L.orc_energy_enstrophy.argtypes = [C.c_int, dp, dp, dp]
        L.orc_shell_spectrum.argtypes = [C.c_int, dp, dp, C.c_int]
        L.orc_fwd2d.argtypes = [C.c_int, dp, dp]
        L.orc_inv2d.argtypes = [C.c_int, dp, dp]
        L.orc_threads.restype = C.c_int
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def fft_c2c(x: np.ndarray, inverse: bool = False) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    lib().orc_fft_c2c(x.size, _dp(x.view(np.float64)), _dp(out.view(np.float64)), int(inverse))
    return out


def fwd2d(plane: np.ndarray) -> np.ndarray:
    plane = np.ascontiguousarray(plane, dtype=np.float64)
    L = plane.shape[0]
    out = np.empty((L, L // 2 + 1), dtype=np.complex128)
    lib().orc_fwd2d(L, _dp(plane), _dp(out.view(np.float64)))
    return out


def inv2d(spec: np.ndarray) -> np.ndarray:
    spec = np.ascontiguousarray(spec, dtype=np.complex128)
    L = spec.shape[0]
    out = np.empty((L, L), dtype=np.float64)
    lib().orc_inv2d(L, _dp(spec.view(np.float64)), _dp(out))
    return out


def pao_spectrum(N: int, K0: float, Re: float):
    """PAO-k^-3 initial velocity spectrum: (uw [N][N/2][2] complex64, stats dict, seed)."""
    uw = np.zeros((N, N // 2, 2), dtype=np.complex64)
    stats = np.zeros(19, dtype=np.float64)
    seed = C.c_int(0)
    lib().orc_pao_spectrum(N, K0, Re, _fp(uw.view(np.float32)), _dp(stats), C.byref(seed))
    return uw, dict(zip(PAO_STAT_NAMES, stats.tolist())), seed.value


def k4_spectrum(N: int, K0: float, seed: int) -> np.ndarray:
    """Seeded k^4 exp(-2(k/K0)^2) vorticity field, [N][N/2] complex64 (compact order)."""
    om = np.zeros((N, N // 2), dtype=np.complex64)
    lib().orc_k4_spectrum(N, float(K0), C.c_uint64(seed), _fp(om.view(np.float32)))
    return om


def energy_enstrophy(om2: np.ndarray):
    om2 = np.ascontiguousarray(om2, dtype=np.complex128)
    E, Z = C.c_double(), C.c_double()
    lib().orc_energy_enstrophy(om2.shape[0], _dp(om2.view(np.float64)), C.byref(E), C.byref(Z))
    return E.value, Z.value


def shell_spectrum(om2: np.ndarray, nb: int | None = None) -> np.ndarray:
    om2 = np.ascontiguousarray(om2, dtype=np.complex128)
    N = om2.shape[0]
    nb = nb or (N // 2 + N // 4 + 2)
    Ek = np.zeros(nb, dtype=np.float64)
    lib().orc_shell_spectrum(N, _dp(om2.view(np.float64)), _dp(Ek), nb)
    return Ek


def display_sigma(field: np.ndarray) -> float:
    f = np.ascontiguousarray(field, dtype=np.float64)
    return lib().orc_display_sigma(_dp(f), f.size)


def movie_scale(N: int) -> int:
    """Frame downsampling factor for size N (cuda/color_cuda.cu:491-498)."""
    return {9216: 8, 16384: 12, 29400: 14}.get(N, max(1, (3 * N // 2 + 3839) // 3840))


def inferno_lut() -> np.ndarray:
    """256x3 colour table: five stops, linear in between, float32 arithmetic truncated to bytes
    (cuda/color_cuda.cu:37-70)."""
    pos = np.array([0.0, 0.25, 0.5, 0.75, 1.0], dtype=np.float32)
    col = np.array([[0, 0, 4], [87, 15, 109], [187, 55, 84], [249, 142, 8], [252, 255, 164]], dtype=np.float32)
    lut = np.zeros((256, 3), dtype=np.uint8)
    for i in range(256):
        x = np.float32(i) / np.float32(255)
        k = 0
        while k + 1 < 5 and x > pos[k + 1]:
            k += 1
        k1 = min(k + 1, 4)
        span = max(np.float32(1e-12), pos[k1] - pos[k])
        t = np.float32(min(np.float32(1), max(np.float32(0), (x - pos[k]) / span)))
        for c in range(3):
            v = (np.float32(1) - t) * col[k, c] + t * col[k1, c]
            lut[i, c] = int(np.float32(v))
    return lut


def frame_pixels(field: np.ndarray) -> np.ndarray:
    """Pixel values 1..255 of a float32 plane (cuda/color_cuda.cu:95-185, :518-540): min/max over
    the finite values, pix = trunc(clamp(1 + 254 norm)) with 1 + 254 norm one fused multiply-add as
    the device computes it, 128 for non-finite values and for a constant plane."""
    f = np.ascontiguousarray(field, dtype=np.float32)
    fin = np.isfinite(f)
    if not fin.any():
        return np.full(f.shape, 128, dtype=np.int64)
    minv, maxv = np.float32(f[fin].min()), np.float32(f[fin].max())
    rng = np.float32(maxv - minv)
    if not rng > np.float32(1e-12):
        return np.full(f.shape, 128, dtype=np.int64)
    inv = np.float32(np.float32(1) / rng)
    with np.errstate(invalid="ignore", over="ignore"):
        norm = (f - minv).astype(np.float32) * inv                      # two float32 roundings
        pf = (norm.astype(np.float64) * 254.0 + 1.0).astype(np.float32)  # one rounding: fma(norm, 254, 1)
        pf = np.clip(pf, np.float32(1), np.float32(255))
        return np.where(fin, np.trunc(np.nan_to_num(pf)), 128).astype(np.int64)


def render_frame(field: np.ndarray, F: int):
    """Inferno RGB frame (uint8 [h][w][3]) of a float32 plane sampled every F points, and the
    plane's pixel sigma (cuda/color_cuda.cu:186-232, :500-597): colour index = pix, or
    round((pix - lo) * 255 / (hi - lo)) clamped to [0, 255] with lo/hi = mean -/+ 2.5 sigma of all
    pixels when sigma >= 1."""
    pix = frame_pixels(field)
    n = pix.size
    mean = float(pix.sum()) / n
    sigma = float(np.sqrt(max(0.0, float((pix * pix).sum()) / n - mean * mean)))
    nz, nx = pix.shape
    oh, ow = (nz + F - 1) // F, (nx + F - 1) // F
    ys = np.minimum(np.arange(oh) * F, nz - 1)
    xs = np.minimum(np.arange(ow) * F, nx - 1)
    p = pix[np.ix_(ys, xs)]
    ci = p.copy()
    lo, hi = mean - 2.5 * sigma, mean + 2.5 * sigma
    if sigma >= 1.0 and hi > lo:
        ci = np.clip(np.floor((p.astype(np.float64) - lo) * 255.0 / (hi - lo) + 0.5), 0, 255).astype(np.int64)
    return inferno_lut()[ci], sigma


def threads() -> int:
    return lib().orc_threads()


def write_restart_v2(path: str, o: "Oracle", Re: float, K0: float, cflnum: float) -> int:
    """Write the oracle's current state as a restart.bin v2 file that the reference's own
    mem_cuda loads unchanged (header: cuda/mem_cuda.cu:1019-1054; payload order UR_full f32
    [3][L][L], OM2 c64 [N][N/2], FNM1 c64 [N][N/2]: cuda/mem_cuda.cu:1236-1285).  This is how one
    seeded field reaches the reference without a change to its source.  UR plane 2 is written as
    zeros: the reference's next step overwrites it with the uw product before reading it.
    Returns the number of bytes written."""
    import struct
    N, L = o.N, o.L
    sc = o.scalars()
    Nk = 3 * N // 4 + 1
    hdr = struct.pack("<16s4I10i9f4x4Q", b"CTRB_RESTART", 2, 144, 4, 8,
                      N, N, N, N, Nk, L, L, Nk, int(sc["it"]), 1,
                      Re, K0, sc["visc"], sc["t"], sc["dt"], sc["cn"], sc["cnm1"], cflnum, sc["cflm"],
                      0, N * (N // 2), N * (N // 2), 3 * L * L)
    assert len(hdr) == 144
    with open(path, "wb") as f:
        f.write(hdr)
        for c in (0, 1):
            f.write(o.ur(c).astype(np.float32).tobytes())
        f.write(np.zeros((L, L), dtype=np.float32).tobytes())
        f.write(o.om2().astype(np.complex64).tobytes())
        f.write(o.fnm1().astype(np.complex64).tobytes())
    return 144 + 3 * L * L * 4 + 2 * N * (N // 2) * 8


class Oracle:
    """FP64 solver state mirroring the reference's DnsDeviceState + mem_cuda loop."""

    def __init__(self, N: int, Re: float, K0: float, cfl: float):
        self.N = N
        self.H = N // 2
        self.L = 3 * N // 2
        self._s = lib().orc_create(N, Re, K0, cfl)
        if not self._s:
            raise ValueError(f"oracle: unsupported N={N}")

    def close(self):
        if self._s:
            lib().orc_destroy(self._s)
            self._s = None

    def __del__(self):
        self.close()

    def init_pao(self):
        stats = np.zeros(19, dtype=np.float64)
        seed = lib().orc_init_pao(self._s, _dp(stats))
        return dict(zip(PAO_STAT_NAMES, stats.tolist())), seed

    def init_om2(self, om2: np.ndarray):
        om2 = np.ascontiguousarray(om2, dtype=np.complex64)
        lib().orc_init_om2(self._s, _fp(om2.view(np.float32)))

    def run(self, nsteps: int, update: int, steps_total: int, want_diag: bool = True):
        E = np.zeros(nsteps)
        Z = np.zeros(nsteps)
        diag = np.zeros(6)
        lib().orc_run(self._s, nsteps, update, steps_total, _dp(E), _dp(Z),
                      _dp(diag) if want_diag else None)
        return E, Z, diag

    def run_fixed(self, dts, cns):
        dts = np.ascontiguousarray(dts, dtype=np.float32)
        cns = np.ascontiguousarray(cns, dtype=np.float32)
        n = dts.size
        E = np.zeros(n)
        Z = np.zeros(n)
        lib().orc_run_fixed(self._s, n, _fp(dts), _fp(cns), _dp(E), _dp(Z))
        return E, Z

    def f32_cn(self, on: bool = True):
        """Form the Crank-Nicolson factors in float, rounded in the reference's operation order
        (cuda/step3_cuda.cu:82-91), instead of FP64: the variant that isolates how far the
        reference's own FP32 factors move it from the FP64 scheme."""
        lib().orc_set_f32_cn(self._s, int(on))

    def scalars(self) -> dict:
        v = np.zeros(8)
        lib().orc_get_scalars(self._s, _dp(v))
        keys = ["it", "t", "dt", "cn", "cnm1", "cflm", "visc", "cflnum"]
        return dict(zip(keys, v.tolist()))

    def set_scalars(self, d: dict):
        keys = ["it", "t", "dt", "cn", "cnm1", "cflm", "visc", "cflnum"]
        cur = self.scalars()
        cur.update(d)
        v = np.array([cur[k] for k in keys], dtype=np.float64)
        lib().orc_set_scalars(self._s, _dp(v))

    def om2(self) -> np.ndarray:
        out = np.zeros((self.N, self.H), dtype=np.complex128)
        lib().orc_get_om2(self._s, _dp(out.view(np.float64)))
        return out

    def fnm1(self) -> np.ndarray:
        out = np.zeros((self.N, self.H), dtype=np.complex128)
        lib().orc_get_fnm1(self._s, _dp(out.view(np.float64)))
        return out

    def ur(self, c: int) -> np.ndarray:
        out = np.zeros((self.L, self.L), dtype=np.float64)
        lib().orc_get_ur(self._s, c, _dp(out))
        return out

    def omega_phys(self) -> np.ndarray:
        out = np.zeros((self.L, self.L), dtype=np.float64)
        lib().orc_om2phys(self._s, _dp(out))
        return out
