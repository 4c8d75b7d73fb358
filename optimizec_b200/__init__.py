"""optimizec_b200 — B200 (sm_100a) replacement for cudaturbo's 2D pseudo-spectral vorticity step.

The product is the C ABI library ``libdns2d.so`` (declared in ``include/dns2d.h``) and the
drop-in ``mem_cuda`` CLI.  This module is a thin ctypes front end over that library, with one
method per entry point of the reference's in-process solver API (cuda/cuda_dns.h:108-202):

    reference (cuda_dns.h)            here
    dnsCudaCreate / dnsCudaDestroy    Solver(N, Re, K0, cfl) / Solver.close()
    dnsCudaInit (PAO + CALCOM)        Solver.init_pao()
    dnsCudaStep2B/Step3/Step2A        Solver.step(n)
    next_dt_gpu                       Solver.next_dt()
    dnsCudaOm2Phys                    Solver.om2phys()
    dnsCudaStreamFunc / Kinetic       Solver.stream_func() / Solver.kinetic()

Errors raise ``Dns2dError`` with the library's message; there is no CPU fallback: if the
shared library or a CUDA device is missing the constructor raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdns2d.so")
REPO = os.path.dirname(_HERE)

SYMBOLS = [
    "dns2d_create", "dns2d_destroy", "dns2d_strerror", "dns2d_last_error", "dns2d_supported",
    "dns2d_device_bytes", "dns2d_init_pao", "dns2d_init_vorticity", "dns2d_init_k4",
    "dns2d_k4_spectrum", "dns2d_step", "dns2d_next_dt", "dns2d_stream", "dns2d_sync", "dns2d_om2phys",
    "dns2d_stream_func", "dns2d_velocity_phys", "dns2d_kinetic", "dns2d_display_sigma",
    "dns2d_energy_enstrophy", "dns2d_shell_spectrum", "dns2d_palin",
    "dns2d_velocity_spectrum_bins", "dns2d_get_scalars", "dns2d_set_scalars", "dns2d_get_om2",
    "dns2d_get_fnm1", "dns2d_get_phys", "dns2d_set_velocity_phys", "dns2d_save_restart",
    "dns2d_load_restart", "dns2d_phase_timing", "dns2d_phase_report", "dns2d_step_noalloc",
    "dns2d_batch_create", "dns2d_batch_destroy", "dns2d_batch_last_error", "dns2d_batch_stream",
    "dns2d_batch_init_k4", "dns2d_batch_next_dt", "dns2d_batch_step", "dns2d_batch_sync",
    "dns2d_batch_get_om2", "dns2d_batch_get_scalars",
    "dns2d_cnn_create", "dns2d_cnn_destroy", "dns2d_cnn_last_error", "dns2d_cnn_num_params",
    "dns2d_cnn_get_params", "dns2d_cnn_set_params", "dns2d_cnn_forward", "dns2d_cnn_loss_grad",
    "dns2d_cnn_set_dataset", "dns2d_cnn_train", "dns2d_closure_attach", "dns2d_closure_forcing", "dns2d_closure_stats",
    "dns2d_cnn_forward_tc", "dns2d_closure_tensor_cores", "dns2d_autotune", "dns2d_set_tuning", "dns2d_batch_autotune", "dns2d_closure_clamp",
    "dns2d_movie_scale", "dns2d_movie_frame", "dns2d_prepare", "dns2d_batch_prepare", "dns2d_batch_set_mode",
    "dns2d_batch_set_waits", "dns2d_batch_set_items", "dns2d_cnn_set_tc_mode", "dns2d_cnn_tc_info",
    "dns2d_cnn_set_trace", "dns2d_cnn_read_trace", "dns2d_cnn_set_train_tc",
]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
# translation units of libdns2d.so: the C ABI and one unit per group of compiled grid sizes
SOURCES = ["dns2d_api.cu", "ensemble.cu", "cnn_net.cu", "cnn_gemm.cu", "sets_small.cu", "sets_256.cu", "sets_mid.cu", "sets_4096.cu", "sets_cluster.cu", "sets_16384.cu",
           "sets_29400.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr"]


class Dns2dError(RuntimeError):
    pass


class Scalars(C.Structure):
    _fields_ = [("N", C.c_int32), ("NX_full", C.c_int32), ("NK_full", C.c_int32),
                ("it", C.c_int32), ("ifn", C.c_int32), ("Re", C.c_float), ("K0", C.c_float),
                ("visc", C.c_float), ("t", C.c_float), ("dt", C.c_float), ("cn", C.c_float),
                ("cnm1", C.c_float), ("cflnum", C.c_float), ("cflm", C.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Member(C.Structure):
    _fields_ = [("N", C.c_int32), ("Re", C.c_float), ("K0", C.c_float), ("cflnum", C.c_float),
                ("seed", C.c_uint64)]


def build(verbose: bool = False) -> str:
    """Compile libdns2d.so (sm_100a) and the mem_cuda CLI in-tree."""
    import tempfile
    with tempfile.TemporaryDirectory(prefix="dns2d_build_") as tmp:
        objs, procs = [], []
        for src in SOURCES:  # one nvcc per translation unit, in parallel
            obj = os.path.join(tmp, src.replace(".cu", ".o"))
            cmd = [NVCC, *ARCH, *CUFLAGS, "-Xcompiler", "-fPIC", "-c", "-o", obj, os.path.join(_HERE, "csrc", src)]
            if verbose:
                print(" ".join(cmd))
            objs.append(obj)
            procs.append((cmd, subprocess.Popen(cmd)))
        failed = [cmd for cmd, pr in procs if pr.wait() != 0]
        if failed:
            raise subprocess.CalledProcessError(1, failed[0])
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB_PATH, *objs]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    cli_src = os.path.join(_HERE, "cli", "mem_cuda.cpp")
    if os.path.exists(cli_src):
        cli = os.path.join(_HERE, "mem_cuda")
        cmd = [NVCC, *ARCH, "-O2", "-std=c++17", "-o", cli, cli_src, "-L" + _HERE, "-ldns2d",
               "-Xlinker", "-rpath,$ORIGIN", "-I" + os.path.join(REPO, "include")]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB_PATH


_LIB = None


def lib():
    """Load libdns2d.so (building it first when absent)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        build()
    L = C.CDLL(LIB_PATH)
    vp, fp, dp, ip = C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int)
    sig = {
        "dns2d_create": (C.c_int, [C.POINTER(vp), C.c_int, C.c_float, C.c_float, C.c_float, C.c_int]),
        "dns2d_destroy": (None, [vp]),
        "dns2d_strerror": (C.c_char_p, [C.c_int]),
        "dns2d_last_error": (C.c_char_p, [vp]),
        "dns2d_supported": (C.c_int, [C.c_int]),
        "dns2d_device_bytes": (C.c_size_t, [C.c_int]),
        "dns2d_init_pao": (C.c_int, [vp, dp, ip]),
        "dns2d_init_vorticity": (C.c_int, [vp, fp, fp]),
        "dns2d_init_k4": (C.c_int, [vp, C.c_uint64]),
        "dns2d_k4_spectrum": (C.c_int, [C.c_int, C.c_float, C.c_uint64, fp]),
        "dns2d_step": (C.c_int, [vp, C.c_int, dp, dp]),
        "dns2d_next_dt": (C.c_int, [vp, fp]),
        "dns2d_stream": (vp, [vp]),
        "dns2d_sync": (C.c_int, [vp, C.c_int]),
        "dns2d_om2phys": (C.c_int, [vp]),
        "dns2d_stream_func": (C.c_int, [vp]),
        "dns2d_velocity_phys": (C.c_int, [vp]),
        "dns2d_kinetic": (C.c_int, [vp]),
        "dns2d_display_sigma": (C.c_int, [vp, C.c_int, dp]),
        "dns2d_energy_enstrophy": (C.c_int, [vp, dp, dp]),
        "dns2d_shell_spectrum": (C.c_int, [vp, dp, C.c_int]),
        "dns2d_palin": (C.c_int, [vp, dp]),
        "dns2d_velocity_spectrum_bins": (C.c_int, [vp, dp, ip, C.c_int]),
        "dns2d_get_scalars": (C.c_int, [vp, C.POINTER(Scalars)]),
        "dns2d_set_scalars": (C.c_int, [vp, C.POINTER(Scalars)]),
        "dns2d_get_om2": (C.c_int, [vp, fp]),
        "dns2d_get_fnm1": (C.c_int, [vp, fp]),
        "dns2d_get_phys": (C.c_int, [vp, C.c_int, fp]),
        "dns2d_set_velocity_phys": (C.c_int, [vp, fp, fp]),
        "dns2d_save_restart": (C.c_int, [vp, C.c_char_p]),
        "dns2d_load_restart": (C.c_int, [vp, C.c_char_p]),
        "dns2d_phase_timing": (C.c_int, [vp, C.c_int]),
        "dns2d_phase_report": (C.c_int, [vp, dp, C.POINTER(C.c_longlong)]),
        "dns2d_step_noalloc": (C.c_int, [C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int,
                                         vp, vp, vp]),
        "dns2d_batch_create": (C.c_int, [C.POINTER(vp), C.POINTER(Member), C.c_int, C.c_int]),
        "dns2d_batch_destroy": (None, [vp]),
        "dns2d_batch_last_error": (C.c_char_p, [vp]),
        "dns2d_batch_stream": (vp, [vp]),
        "dns2d_batch_init_k4": (C.c_int, [vp]),
        "dns2d_batch_next_dt": (C.c_int, [vp, fp]),
        "dns2d_batch_step": (C.c_int, [vp, C.c_int, dp, dp]),
        "dns2d_batch_sync": (C.c_int, [vp]),
        "dns2d_batch_get_om2": (C.c_int, [vp, C.c_int, fp]),
        "dns2d_batch_get_scalars": (C.c_int, [vp, C.c_int, C.POINTER(Scalars)]),
        "dns2d_cnn_create": (C.c_int, [C.POINTER(vp), C.c_int, C.c_int, C.c_uint64, C.c_int]),
        "dns2d_cnn_destroy": (None, [vp]),
        "dns2d_cnn_last_error": (C.c_char_p, [vp]),
        "dns2d_cnn_num_params": (C.c_int, [vp]),
        "dns2d_cnn_get_params": (C.c_int, [vp, fp]),
        "dns2d_cnn_set_params": (C.c_int, [vp, fp]),
        "dns2d_cnn_forward": (C.c_int, [vp, fp, C.c_int, C.c_int, C.c_int, fp]),
        "dns2d_cnn_loss_grad": (C.c_int, [vp, fp, fp, C.c_int, C.c_int, C.c_int, dp, fp]),
        "dns2d_cnn_set_dataset": (C.c_int, [vp, fp, fp, C.c_int, C.c_int, C.c_int]),
        "dns2d_cnn_train": (C.c_int, [vp, C.c_int, C.c_int, C.c_float, C.c_uint64, dp]),
        "dns2d_closure_attach": (C.c_int, [vp, vp, fp, C.c_int]),
        "dns2d_closure_forcing": (C.c_int, [vp, fp]),
        "dns2d_cnn_forward_tc": (C.c_int, [vp, fp, C.c_int, C.c_int, C.c_int, fp]),
        "dns2d_cnn_set_tc_mode": (C.c_int, [vp, C.c_int]),
        "dns2d_cnn_tc_info": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "dns2d_cnn_set_trace": (C.c_int, [vp, C.c_int]),
        "dns2d_cnn_set_train_tc": (C.c_int, [vp, C.c_int]),
        "dns2d_cnn_read_trace": (C.c_int, [vp, C.POINTER(C.c_uint64), C.c_int, C.POINTER(C.c_int)]),
        "dns2d_closure_tensor_cores": (C.c_int, [vp, C.c_int]),
        "dns2d_autotune": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int)]),
        "dns2d_set_tuning": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int)]),
        "dns2d_batch_autotune": (C.c_int, [vp]),
        "dns2d_closure_clamp": (C.c_int, [vp, C.c_float]),
        "dns2d_closure_stats": (C.c_int, [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
        "dns2d_movie_scale": (C.c_int, [C.c_int]),
        "dns2d_prepare": (C.c_int, [vp, C.c_int]),
        "dns2d_batch_prepare": (C.c_int, [vp, C.c_int]),
        "dns2d_batch_set_mode": (C.c_int, [vp, C.c_int]),
        "dns2d_batch_set_waits": (C.c_int, [vp, C.c_longlong, C.c_int]),
        "dns2d_batch_set_items": (C.c_int, [vp, C.c_int, C.c_int]),
        "dns2d_movie_frame": (C.c_int, [vp, C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                        C.POINTER(C.c_double)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _LIB = L
    return L


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def supported(N: int) -> bool:
    return bool(lib().dns2d_supported(N))


def autotune(N: int, device: int = 0) -> dict:
    """Time the kernel variants of size N and keep the fastest (dns2d_autotune)."""
    cfg = (C.c_int * 6)()
    rc = lib().dns2d_autotune(N, device, cfg)
    if rc:
        raise Dns2dError(f"dns2d_autotune: {lib().dns2d_strerror(rc).decode()}")
    return dict(zip(("rows_tile", "cols_groups", "pf_rows", "pf_cols", "plan_rows", "plan_cols"), list(cfg)))


def set_tuning(N: int, rows_tile=0, cols_groups=0, pf_rows=296, pf_cols=74, plan_rows=0, plan_cols=0,
               device: int = 0):
    """Pin the kernel configuration of size N (dns2d_set_tuning)."""
    cfg = (C.c_int * 6)(rows_tile, cols_groups, pf_rows, pf_cols, plan_rows, plan_cols)
    rc = lib().dns2d_set_tuning(N, device, cfg)
    if rc:
        raise Dns2dError(f"dns2d_set_tuning: {lib().dns2d_strerror(rc).decode()}")


def k4_spectrum(N: int, K0: float, seed: int) -> np.ndarray:
    out = np.zeros((N, N // 2), dtype=np.complex64)
    rc = lib().dns2d_k4_spectrum(N, K0, seed, _fp(out.view(np.float32)))
    if rc:
        raise Dns2dError(lib().dns2d_strerror(rc).decode())
    return out


class Solver:
    """One simulation on one GPU (owns a dns2d_state)."""

    def __init__(self, N: int, Re: float, K0: float, cfl: float, device: int = 0):
        self.N, self.H, self.L = N, N // 2, 3 * N // 2
        self._L = lib()
        self._s = C.c_void_p()
        rc = self._L.dns2d_create(C.byref(self._s), N, Re, K0, cfl, device)
        if rc:
            raise Dns2dError(f"dns2d_create(N={N}): {self._L.dns2d_strerror(rc).decode()}")

    def _chk(self, rc):
        if rc:
            msg = self._L.dns2d_last_error(self._s).decode() if self._s else ""
            raise Dns2dError(f"{self._L.dns2d_strerror(rc).decode()}: {msg}")

    def close(self):
        if self._s:
            self._L.dns2d_destroy(self._s)
            self._s = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- initial conditions ----
    def init_pao(self):
        stats = np.zeros(19)
        seed = C.c_int(0)
        self._chk(self._L.dns2d_init_pao(self._s, _dp(stats), C.byref(seed)))
        return stats, seed.value

    def init_vorticity(self, om2: np.ndarray, fnm1: np.ndarray | None = None):
        om2 = np.ascontiguousarray(om2, dtype=np.complex64)
        f = None if fnm1 is None else np.ascontiguousarray(fnm1, dtype=np.complex64)
        self._chk(self._L.dns2d_init_vorticity(self._s, _fp(om2.view(np.float32)),
                                               None if f is None else _fp(f.view(np.float32))))

    def init_k4(self, seed: int):
        self._chk(self._L.dns2d_init_k4(self._s, seed))

    # ---- stepping ----
    def step(self, n: int, history: bool = False):
        if history:
            E = np.zeros(n)
            Z = np.zeros(n)
            self._chk(self._L.dns2d_step(self._s, n, _dp(E), _dp(Z)))
            return E, Z
        self._chk(self._L.dns2d_step(self._s, n, None, None))
        return None

    def prepare(self, n: int):
        """Build the CUDA graphs step(n) will launch, without running them (dns2d_prepare)."""
        self._chk(self._L.dns2d_prepare(self._s, int(n)))

    def next_dt(self) -> float:
        c = C.c_float(0)
        self._chk(self._L.dns2d_next_dt(self._s, C.byref(c)))
        return c.value

    def stream(self) -> int:
        """the state's cudaStream_t as an integer handle"""
        return self._L.dns2d_stream(self._s) or 0

    def sync(self, timeout_ms: int = 0):
        self._chk(self._L.dns2d_sync(self._s, timeout_ms))

    # ---- diagnostics ----
    def om2phys(self):
        self._chk(self._L.dns2d_om2phys(self._s))

    def stream_func(self):
        self._chk(self._L.dns2d_stream_func(self._s))

    def velocity_phys(self):
        self._chk(self._L.dns2d_velocity_phys(self._s))

    def kinetic(self):
        self._chk(self._L.dns2d_kinetic(self._s))

    def display_sigma(self, comp: int = 2) -> float:
        v = C.c_double(0)
        self._chk(self._L.dns2d_display_sigma(self._s, comp, C.byref(v)))
        return v.value

    def energy_enstrophy(self):
        E, Z = C.c_double(0), C.c_double(0)
        self._chk(self._L.dns2d_energy_enstrophy(self._s, C.byref(E), C.byref(Z)))
        return E.value, Z.value

    def shell_spectrum(self, nb: int | None = None) -> np.ndarray:
        nb = nb or (self.N // 2 + self.N // 4 + 2)
        out = np.zeros(nb)
        self._chk(self._L.dns2d_shell_spectrum(self._s, _dp(out), nb))
        return out

    def palin(self) -> float:
        v = C.c_double(0)
        self._chk(self._L.dns2d_palin(self._s, C.byref(v)))
        return v.value

    def velocity_spectrum_bins(self, nbins: int | None = None):
        nbins = nbins or max(32, 2 * self.L)
        e = np.zeros(nbins)
        c = np.zeros(nbins, dtype=np.int32)
        self._chk(self._L.dns2d_velocity_spectrum_bins(self._s, _dp(e), c.ctypes.data_as(C.POINTER(C.c_int)), nbins))
        return e, c

    # ---- state ----
    def scalars(self) -> dict:
        s = Scalars()
        self._chk(self._L.dns2d_get_scalars(self._s, C.byref(s)))
        return s.as_dict()

    def set_scalars(self, **kw):
        s = Scalars()
        self._chk(self._L.dns2d_get_scalars(self._s, C.byref(s)))
        for k, v in kw.items():
            setattr(s, k, v)
        self._chk(self._L.dns2d_set_scalars(self._s, C.byref(s)))

    def _spectrum_out(self, out):
        if out is None:
            return np.zeros((self.N, self.H), dtype=np.complex64)
        if out.dtype != np.complex64 or out.shape != (self.N, self.H) or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous complex64 array of shape ({self.N}, {self.H})")
        return out

    def om2(self, out: np.ndarray | None = None) -> np.ndarray:
        """Vorticity [iz][ix] (N x N/2 complex64); `out` (e.g. a view of pinned memory) is filled
        in place when given."""
        out = self._spectrum_out(out)
        self._chk(self._L.dns2d_get_om2(self._s, _fp(out.view(np.float32))))
        return out

    def fnm1(self, out: np.ndarray | None = None) -> np.ndarray:
        out = self._spectrum_out(out)
        self._chk(self._L.dns2d_get_fnm1(self._s, _fp(out.view(np.float32))))
        return out

    def phys(self, comp: int) -> np.ndarray:
        out = np.zeros((self.L, self.L), dtype=np.float32)
        self._chk(self._L.dns2d_get_phys(self._s, comp, _fp(out)))
        return out

    def set_velocity_phys(self, u: np.ndarray, w: np.ndarray):
        u = np.ascontiguousarray(u, dtype=np.float32)
        w = np.ascontiguousarray(w, dtype=np.float32)
        self._chk(self._L.dns2d_set_velocity_phys(self._s, _fp(u), _fp(w)))

    def save_restart(self, path: str):
        self._chk(self._L.dns2d_save_restart(self._s, path.encode()))

    def load_restart(self, path: str):
        self._chk(self._L.dns2d_load_restart(self._s, path.encode()))

    def attach_closure(self, net, scales, energy_check: int = 1):
        """Couple a trained CNN (or None to detach); scales = (s_omega, s_u, s_w, s_out);
        energy_check 0 off, 1 device-side gate (graph-captured), 2 host rollback, 3 device-side
        scaling of an energy-raising forcing to the viscous loss."""
        sc = np.ascontiguousarray(scales, dtype=np.float32)
        self._closure_net = net  # keep the network alive while attached
        self._chk(self._L.dns2d_closure_attach(self._s, net.handle if net is not None else None, _fp(sc),
                                               int(energy_check)))

    def closure_forcing(self) -> np.ndarray:
        out = np.zeros((self.N, self.H), dtype=np.complex64)
        self._chk(self._L.dns2d_closure_forcing(self._s, _fp(out.view(np.float32))))
        return out

    def movie_frame(self, comp: int = 2, scale_f: int = 0):
        """Inferno RGB frame of physical plane comp (uint8 [h][w][3]) and the plane's pixel sigma;
        scale_f 0 = the reference's factor for this N."""
        F = scale_f or self._L.dns2d_movie_scale(self.N)
        w, h = C.c_int(0), C.c_int(0)
        self._chk(self._L.dns2d_movie_frame(self._s, comp, F, None, C.byref(w), C.byref(h), None))
        out = np.zeros((h.value, w.value, 3), dtype=np.uint8)
        sig = C.c_double(0)
        self._chk(self._L.dns2d_movie_frame(self._s, comp, F, out.ctypes.data_as(C.c_void_p), C.byref(w),
                                            C.byref(h), C.byref(sig)))
        return out, sig.value

    def closure_clamp(self, alpha: float):
        """Limit each mode's closure forcing to alpha |FN| (0: off)."""
        self._chk(self._L.dns2d_closure_clamp(self._s, float(alpha)))

    def closure_tensor_cores(self, enable: bool):
        self._chk(self._L.dns2d_closure_tensor_cores(self._s, int(enable)))

    def closure_stats(self):
        a, b = C.c_longlong(0), C.c_longlong(0)
        self._chk(self._L.dns2d_closure_stats(self._s, C.byref(a), C.byref(b)))
        return a.value, b.value

    def phase_timing(self, on: bool):
        self._chk(self._L.dns2d_phase_timing(self._s, int(on)))

    def phase_report(self):
        ms = np.zeros(4)
        n = np.zeros(4, dtype=np.int64)
        self._chk(self._L.dns2d_phase_report(self._s, _dp(ms), n.ctypes.data_as(C.POINTER(C.c_longlong))))
        return ms, n


class Batch:
    """An ensemble of independent runs advanced together (dns2d_batch_*)."""

    def __init__(self, members, device: int = 0):
        """members: sequence of (N, Re, K0, cfl, seed)"""
        self._L = lib()
        self.members = [tuple(m) for m in members]
        arr = (Member * len(self.members))(*[Member(int(N), Re, K0, c, int(sd)) for N, Re, K0, c, sd in self.members])
        self._b = C.c_void_p()
        rc = self._L.dns2d_batch_create(C.byref(self._b), arr, len(self.members), device)
        if rc:
            raise Dns2dError(f"dns2d_batch_create: {self._L.dns2d_strerror(rc).decode()}")

    def _chk(self, rc):
        if rc:
            raise Dns2dError(f"{self._L.dns2d_strerror(rc).decode()}: {self._L.dns2d_batch_last_error(self._b).decode()}")

    def close(self):
        if self._b:
            self._L.dns2d_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def autotune(self):
        """Time each size group's kernel variants at its member count (before init_k4)."""
        self._chk(self._L.dns2d_batch_autotune(self._b))

    def set_mode(self, mode: int):
        """0: one CUDA graph per chunk, a branch per size group; 1: one persistent launch per
        chunk (dns2d_batch_set_mode)."""
        self._chk(self._L.dns2d_batch_set_mode(self._b, int(mode)))

    def set_items(self, tiles_per_item: int, groups_per_item: int):
        """Work-item size of the persistent launch (dns2d_batch_set_items)."""
        self._chk(self._L.dns2d_batch_set_items(self._b, int(tiles_per_item), int(groups_per_item)))

    def set_waits(self, spin_limit: int, stall_member: int = -1):
        """Dependency waits of the persistent launch (dns2d_batch_set_waits)."""
        self._chk(self._L.dns2d_batch_set_waits(self._b, int(spin_limit), int(stall_member)))

    def prepare(self, n: int):
        """Build the graphs step(n) will launch, without running them (dns2d_batch_prepare)."""
        self._chk(self._L.dns2d_batch_prepare(self._b, int(n)))

    def init_k4(self):
        self._chk(self._L.dns2d_batch_init_k4(self._b))

    def next_dt(self) -> np.ndarray:
        out = np.zeros(len(self.members), dtype=np.float32)
        self._chk(self._L.dns2d_batch_next_dt(self._b, _fp(out)))
        return out

    def step(self, n: int, history: bool = False):
        if history:
            E = np.zeros((len(self.members), n))
            Z = np.zeros((len(self.members), n))
            self._chk(self._L.dns2d_batch_step(self._b, n, _dp(E), _dp(Z)))
            return E, Z
        self._chk(self._L.dns2d_batch_step(self._b, n, None, None))
        return None

    def sync(self):
        self._chk(self._L.dns2d_batch_sync(self._b))

    def stream(self) -> int:
        return self._L.dns2d_batch_stream(self._b) or 0

    def om2(self, m: int) -> np.ndarray:
        N = self.members[m][0]
        out = np.zeros((N, N // 2), dtype=np.complex64)
        self._chk(self._L.dns2d_batch_get_om2(self._b, m, _fp(out.view(np.float32))))
        return out

    def scalars(self, m: int) -> dict:
        s = Scalars()
        self._chk(self._L.dns2d_batch_get_scalars(self._b, m, C.byref(s)))
        return s.as_dict()


def ensemble_members(counts=((128, 32), (256, 24), (512, 8)), cfl: float = 0.1):
    """The 64-member ensemble configuration: sizes by count, seeds 0..63, Re log-uniform in
    [1e3, 1e5] and K0 uniform-integer in [2, 8], both drawn from splitmix64(seed)."""
    def sm64(x):
        x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        return x ^ (x >> 31)
    out = []
    seed = 0
    for N, n in counts:
        for _ in range(n):
            r1 = sm64(seed)
            r2 = sm64(r1)
            u1 = (r1 >> 11) / float(1 << 53)
            u2 = (r2 >> 11) / float(1 << 53)
            Re = 10.0 ** (3.0 + 2.0 * u1)
            K0 = float(2 + min(6, int(7 * u2)))
            out.append((N, Re, K0, cfl, seed))
            seed += 1
    return out


class CNN:
    """The closure network (dns2d_cnn_*): periodic 3x3 CNN, 3 inputs -> 1 output."""

    def __init__(self, layers: int = 6, channels: int = 32, seed: int = 0, device: int = 0):
        self._L = lib()
        self.layers, self.channels = layers, channels
        self._n = C.c_void_p()
        rc = self._L.dns2d_cnn_create(C.byref(self._n), layers, channels, seed, device)
        if rc:
            raise Dns2dError(f"dns2d_cnn_create: {self._L.dns2d_strerror(rc).decode()}")

    def _chk(self, rc):
        if rc:
            raise Dns2dError(f"{self._L.dns2d_strerror(rc).decode()}: {self._L.dns2d_cnn_last_error(self._n).decode()}")

    def close(self):
        if self._n:
            self._L.dns2d_cnn_destroy(self._n)
            self._n = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._n

    def num_params(self) -> int:
        return self._L.dns2d_cnn_num_params(self._n)

    def params(self) -> np.ndarray:
        p = np.zeros(self.num_params(), dtype=np.float32)
        self._chk(self._L.dns2d_cnn_get_params(self._n, _fp(p)))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._chk(self._L.dns2d_cnn_set_params(self._n, _fp(p)))

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        B, _, H, W = x.shape
        y = np.zeros((B, 1, H, W), dtype=np.float32)
        self._chk(self._L.dns2d_cnn_forward(self._n, _fp(x), B, H, W, _fp(y)))
        return y

    def forward_tc(self, x: np.ndarray) -> np.ndarray:
        """Forward on the BF16 tensor-core path (hidden layers on tcgen05); W % 128 == 0."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        B, _, H, W = x.shape
        y = np.zeros((B, 1, H, W), dtype=np.float32)
        self._chk(self._L.dns2d_cnn_forward_tc(self._n, _fp(x), B, H, W, _fp(y)))
        return y

    def set_tc_mode(self, mode: int):
        """1 (default): layers 1 .. L-1 of the tensor-core path in one persistent launch where their
        weights fit in shared memory; 0: one launch per layer (same values bit for bit)."""
        self._chk(self._L.dns2d_cnn_set_tc_mode(self._n, int(mode)))

    def set_train_tc(self, on: bool):
        """Training convolutions (forward, data and weight gradients) as tcgen05 GEMMs over bf16
        operands with FP32 accumulation (off by default)."""
        self._chk(self._L.dns2d_cnn_set_train_tc(self._n, int(bool(on))))

    def set_trace(self, on: bool):
        """Record per-tile timestamps in each persistent launch (off by default)."""
        self._chk(self._L.dns2d_cnn_set_trace(self._n, int(bool(on))))

    def read_trace(self) -> np.ndarray:
        """[tiles, 10] uint64 ns of the last persistent launch (tiles in layer order, tile rows
        rotated by one per layer): taken, input rows complete, stage free, copy issued, copy
        landed, MMAs issued and committed, epilogue started, accumulator read, stores issued,
        released."""
        tiles = C.c_int(0)
        self._chk(self._L.dns2d_cnn_read_trace(self._n, (C.c_uint64 * 1)(), 0, C.byref(tiles)))
        out = np.zeros((tiles.value, 10), dtype=np.uint64)
        if tiles.value:
            self._chk(self._L.dns2d_cnn_read_trace(self._n, out.ctypes.data_as(C.POINTER(C.c_uint64)),
                                                   tiles.value, C.byref(tiles)))
        return out

    def tc_info(self):
        """(mode, grid of the last persistent launch; 0 before any)."""
        m, g = C.c_int(0), C.c_int(0)
        self._chk(self._L.dns2d_cnn_tc_info(self._n, C.byref(m), C.byref(g)))
        return m.value, g.value

    def loss_grad(self, x: np.ndarray, t: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        B, _, H, W = x.shape
        loss = C.c_double(0)
        g = np.zeros(self.num_params(), dtype=np.float32)
        self._chk(self._L.dns2d_cnn_loss_grad(self._n, _fp(x), _fp(t), B, H, W, C.byref(loss), _fp(g)))
        return loss.value, g

    def set_dataset(self, x: np.ndarray, t: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        n, _, H, W = x.shape
        self._chk(self._L.dns2d_cnn_set_dataset(self._n, _fp(x), _fp(t), n, H, W))

    def train(self, iters: int, batch: int, lr: float, seed: int = 0) -> np.ndarray:
        losses = np.zeros(iters)
        self._chk(self._L.dns2d_cnn_train(self._n, iters, batch, lr, seed, _dp(losses)))
        return losses
