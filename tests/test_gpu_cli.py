"""GPU tests of the drop-in mem_cuda CLI: stdout lines, signals, output files, restart.bin
round trips, and restart.bin interchange with the reference's own binary (oracle/_ref/mem_cuda,
built from the reference sources) when that binary is present."""
import os
import re
import signal
import subprocess
import time

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(REPO, "optimizec_b200", "mem_cuda")
REF = os.path.join(REPO, "oracle", "_ref", "mem_cuda")
ITER_RE = re.compile(r"ITERATION\s+(\d+) T=([-0-9.eE]+) DT=([-0-9.eE]+) CN=([-0-9.eE]+) CFLM=([-0-9.eE]+) "
                     r"Re=\s*([-0-9.eE+]+) VISC=\s*([-0-9.eE+]+) PALIN=(\d+) SIG=(\d+)")


def iterations(text):
    return {int(m[1]): dict(T=float(m[2]), DT=float(m[3]), CN=float(m[4]), CFLM=float(m[5]), Re=float(m[6]),
                            VISC=float(m[7]), PALIN=int(m[8]), SIG=int(m[9]))
            for m in ITER_RE.finditer(text)}


def run_cli(args, cwd, env=None, timeout=300, exe=CLI):
    e = dict(os.environ)
    if env:
        e.update(env)
    return subprocess.run([exe, *map(str, args)], cwd=cwd, env=e, capture_output=True, text=True, timeout=timeout)


def test_cli_trajectory_matches_oracle(tmp_path):
    """PAO start, N=128: every printed diagnostic line against the FP64 oracle."""
    N, Re, K0, steps, cfl, update = 128, 1e4, 10.0, 60, 0.25, 20
    p = run_cli([N, int(Re), int(K0), steps, cfl, update, 0], tmp_path)
    assert p.returncode == 0, p.stderr
    assert "PAO seed" in p.stdout and "[OUTPUT] Normal completion" in p.stdout
    got = iterations(p.stdout)
    assert sorted(got) == [1, 20, 40, 60]
    o = O.Oracle(N, Re, K0, cfl)
    o.init_pao()
    done = 0
    for it in sorted(got):
        _, _, d = o.run(it - done, update, steps)
        done = it
        g = got[it]
        assert g["T"] == pytest.approx(d[1], rel=1e-6)
        assert g["DT"] == pytest.approx(d[2], rel=1e-5, abs=2e-8)
        assert g["CN"] == pytest.approx(d[3], abs=2e-7)
        assert g["CFLM"] == pytest.approx(d[4], rel=1e-6)
        assert abs(g["SIG"] - int(d[5])) <= 1


def _start(args, cwd, env=None):
    e = dict(os.environ)
    if env:
        e.update(env)
    return subprocess.Popen([CLI, *map(str, args)], cwd=cwd, env=e, stdout=subprocess.PIPE,
                            stderr=subprocess.PIPE, text=True)


def _wait_for(proc, pattern, timeout=60):
    t0 = time.time()
    buf = ""
    while time.time() - t0 < timeout:
        line = proc.stdout.readline()
        if not line:
            break
        buf += line
        if re.search(pattern, buf):
            return buf
    raise AssertionError(f"pattern {pattern!r} not seen; got:\n{buf[-2000:]}")


def test_signals_save_restart_and_exit(tmp_path):
    N = 64
    proc = _start([N, 10000, 4, 1000000, 0.1, 10, 0], tmp_path)
    try:
        _wait_for(proc, r"ITERATION\s+20 ")
        proc.send_signal(signal.SIGUSR1)
        _wait_for(proc, r"Wrote .*meta\.csv")
        proc.send_signal(signal.SIGRTMIN)
        _wait_for(proc, r"_restart/meta\.csv")
        proc.send_signal(signal.SIGHUP)
        out, err = proc.communicate(timeout=60)
    finally:
        if proc.poll() is None:
            proc.kill()
    assert proc.returncode == 128 + signal.SIGHUP
    folders = sorted(d for d in os.listdir(tmp_path) if d.startswith("output_64_4_1E04_0.10_"))
    assert len(folders) >= 3, folders
    rfold = [d for d in folders if d.endswith("_restart")]
    assert len(rfold) == 1
    for d in folders:
        files = set(os.listdir(tmp_path / d))
        for f in ["u_velocity.pgm", "v_velocity.pgm", "kinetic.pgm", "omega.pgm", "stream.pgm",
                  "energy_spectrum.csv", "metrics.csv", "meta.csv"]:
            assert f in files, (d, f)
    L = 3 * N // 2
    rb = tmp_path / rfold[0] / "restart.bin"
    assert rb.stat().st_size == 144 + 3 * L * L * 4 + 2 * N * (N // 2) * 8
    pgm = (tmp_path / rfold[0] / "omega.pgm").read_bytes()
    assert pgm.startswith(f"P5\n{L} {L}\n255\n".encode())
    meta = (tmp_path / rfold[0] / "meta.csv").read_text().splitlines()
    assert meta[0].startswith("timestamp,N,K0,Re,CFL,visc,T,IT,Update")
    assert meta[1].endswith(",CUDA")
    # RESTART mode resumes from the folder at the saved iteration
    it0 = int(meta[1].split(",")[7])
    p = run_cli(["RESTART", str(tmp_path / rfold[0])], tmp_path, env={"RESTART_STEPS": str(it0 + 10)})
    assert p.returncode == 0, p.stderr + p.stdout
    assert f"at iteration {it0}" in p.stdout
    assert max(iterations(p.stdout)) == it0 + 10


def test_sigint_exits_without_files(tmp_path):
    proc = _start([64, 10000, 4, 1000000, 0.1, 10, 0], tmp_path)
    try:
        _wait_for(proc, r"ITERATION\s+10 ")
        proc.send_signal(signal.SIGINT)
        out, _ = proc.communicate(timeout=60)
    finally:
        if proc.poll() is None:
            proc.kill()
    assert proc.returncode == 128 + signal.SIGINT
    assert "exiting without saving" in out
    assert not [d for d in os.listdir(tmp_path) if d.startswith("output_")]


def test_restart_file_continues_exactly(tmp_path):
    """restart.bin written after k steps and reloaded gives the same continuation."""
    import optimizec_b200 as P
    N = 128
    s = P.Solver(N, 1e4, 4.0, 0.1)
    s.init_k4(3)
    s.next_dt()
    s.step(1)
    s.next_dt()
    s.step(9)
    path = str(tmp_path / "restart.bin")
    s.save_restart(path)
    a = run_cli([N, 10000, 4, 30, 0.1, 10, 0, path], tmp_path)
    assert a.returncode == 0, a.stderr
    s.step(10)
    s.next_dt()
    s.step(10)
    s.next_dt()
    got = iterations(a.stdout)
    sc = s.scalars()
    assert got[30]["T"] == pytest.approx(sc["t"], rel=1e-7)
    assert got[30]["CFLM"] == pytest.approx(sc["cflm"], rel=1e-6)


@pytest.mark.skipif(not os.path.exists(REF), reason="reference binary not built")
def test_restart_interchange_with_reference(tmp_path):
    """A restart.bin written by this library is read by the reference's own mem_cuda, and both
    continue along the same trajectory (printed T, DT, CN, CFLM, SIG)."""
    import optimizec_b200 as P
    N, Re, K0, cfl, update = 256, 1e4, 4.0, 0.1, 10
    s = P.Solver(N, Re, K0, cfl)
    s.init_k4(11)
    s.next_dt()
    path = str(tmp_path / "restart.bin")
    s.save_restart(path)
    args = [N, int(Re), int(K0), 40, cfl, update, 0, path]
    ref = run_cli(args, tmp_path, exe=REF)
    ours = run_cli(args, tmp_path)
    assert ref.returncode == 0, ref.stderr
    assert ours.returncode == 0, ours.stderr
    r, o = iterations(ref.stdout), iterations(ours.stdout)
    assert sorted(r) == sorted(o) == [1, 10, 20, 30, 40]
    for it in r:
        assert o[it]["T"] == pytest.approx(r[it]["T"], rel=1e-7)
        assert o[it]["DT"] == pytest.approx(r[it]["DT"], rel=2e-6, abs=2e-8)
        assert o[it]["CN"] == pytest.approx(r[it]["CN"], abs=2e-7)
        assert o[it]["CFLM"] == pytest.approx(r[it]["CFLM"], rel=2e-6)
        assert abs(o[it]["SIG"] - r[it]["SIG"]) <= 1


def _ref_harness(N, Re, K0, cfl, steps, update, om0, tmp_path):
    """The reference's cuFFT path (oracle/_ref/ref_harness) from om0: per-step E, Z, the DIAG lines
    {it: [t, dt, cn, cflm, sigma]} and the final vorticity."""
    f = tmp_path / "om2.bin"
    om0.tofile(f)
    h = subprocess.run([os.path.join(REPO, "oracle", "_ref", "ref_harness"), str(N), str(Re), str(K0), str(cfl),
                        str(steps), str(update), str(f), str(tmp_path / "ref")], capture_output=True, text=True,
                       timeout=900)
    assert h.returncode == 0, h.stderr
    lines = h.stdout.splitlines()
    E = np.array([float(l.split()[2]) for l in lines if l.startswith("STEP ")])
    Z = np.array([float(l.split()[3]) for l in lines if l.startswith("STEP ")])
    diag = {int(float(l.split()[1])): [float(x) for x in l.split()[2:]] for l in lines if l.startswith("DIAG ")}
    om = np.fromfile(tmp_path / "ref.om2", dtype=np.complex64).reshape(N, N // 2).astype(np.complex128)
    return E, Z, diag, om


def _ours(N, Re, K0, cfl, steps, update, om0):
    """This library with the reference's cadence (NEXTDT + OM2PHYS at it = 1, every UPDATE steps
    and the last step): per-step E, Z, {it: [t, dt, cn, cflm, sigma]}, final vorticity."""
    import optimizec_b200 as P
    s = P.Solver(N, Re, K0, cfl)
    s.init_vorticity(om0)
    s.next_dt()
    E, Z, diag = [], [], {}
    while s.scalars()["it"] < steps:
        it = s.scalars()["it"]
        nxt = 1 if it < 1 else min(steps, (it // update + 1) * update)
        e, z = s.step(nxt - it, history=True)
        E.append(e)
        Z.append(z)
        s.next_dt()
        s.om2phys()
        sc = s.scalars()
        diag[nxt] = [sc["t"], sc["dt"], sc["cn"], sc["cflm"], s.display_sigma(2)]
    om = s.om2().astype(np.complex128)
    s.close()
    return np.concatenate(E), np.concatenate(Z), diag, om


def _oracle(N, Re, K0, cfl, steps, update, om0, f32_cn=False):
    o = O.Oracle(N, Re, K0, cfl)
    o.f32_cn(f32_cn)
    o.init_om2(om0)
    E, Z, _ = o.run(steps, update, steps, want_diag=False)
    om = o.om2()
    o.close()
    return E, Z, om


def _rl2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.skipif(not os.path.exists(os.path.join(REPO, "oracle", "_ref", "ref_harness")),
                    reason="reference harness not built")
@pytest.mark.parametrize("N,Re", [(256, 1e4), (512, 1e4), (4096, 1e5)])
def test_twenty_steps_match_reference_cufft(N, Re, tmp_path):
    """20 steps from the same seeded field (K0 = 4, CFL = 0.1, dt fixed after step 1), this library
    against the reference's own cuFFT path and the FP64 oracle.  (4096, 1e5) is the headline
    configuration.  Required of this library: vorticity within 1e-5 (relative L2) of the FP64
    oracle, energy and enstrophy histories within 1e-6 of both the oracle and the reference, and
    energy spectra within 1e-5 per shell (plus a floor of 1e-10 of the total energy) of both.
    Against the reference's field: within 1e-5 where the reference itself is (N = 256, 512).  At the
    headline size the reference's own field is 1.35e-5 from the FP64 oracle (its FP32 transform
    rounding, amplified by K^2 in the nearly empty high-k modes; not its float Crank-Nicolson
    factors, which move it by 1e-7), so no implementation can be within 1e-5 of both: there the
    test requires this library to be at most 1e-5 from the oracle, and at most 1e-5 farther from
    the reference than the reference is from the oracle."""
    K0, cfl, steps = 4.0, 0.1, 20
    om0 = O.k4_spectrum(N, K0, 5 if N < 4096 else 0)
    E_ref, Z_ref, _, om_ref = _ref_harness(N, Re, K0, cfl, steps, 1000, om0, tmp_path)
    E, Z, _, om = _ours(N, Re, K0, cfl, steps, 1000, om0)
    E_o, Z_o, om_o = _oracle(N, Re, K0, cfl, steps, 1000, om0)
    ours_o, ref_o, ours_ref = _rl2(om, om_o), _rl2(om_ref, om_o), _rl2(om, om_ref)
    assert ours_o <= 1e-5, ours_o
    if ref_o <= 1e-5:
        assert ours_ref <= 1e-5, (ours_ref, ref_o)
    else:
        assert ours_ref <= ref_o + 1e-5, (ours_ref, ref_o)
    for a, b in ((E, E_ref), (Z, Z_ref), (E, E_o), (Z, Z_o)):
        assert np.max(np.abs(a / b - 1)) <= 1e-6
    Ek = O.shell_spectrum(om)
    for other in (om_ref, om_o):
        Ek_r = O.shell_spectrum(other)
        assert np.all(np.abs(Ek - Ek_r) <= 1e-5 * Ek_r + 1e-10 * Ek_r.sum())


@pytest.mark.skipif(not os.path.exists(os.path.join(REPO, "oracle", "_ref", "ref_harness")),
                    reason="reference harness not built")
def test_c1_thousand_steps_match_reference_cufft(tmp_path):
    """The N = 512 configuration (Re = 1e4, K0 = 4, CFL = 0.1, UPDATE = 100, 1000 steps) with the
    reference's diagnostic cadence, this library against the FP64 oracle and the reference's
    cuFFT path.
    - Against the FP64 oracle: energy and enstrophy histories within 1e-6 over all 1000 steps, and
      the vorticity within 1e-4 at step 1000 (FP32 rounding grows through the dynamics: 1e-5 is
      the 20-step bound).
    - The reference forms its Crank-Nicolson factors in float (cuda/step3_cuda.cu:82-91): at
      Re = 1e4 the viscous decrement of the energy-bearing modes (~1e-7 K^2 per step) is of the
      order of the float spacing below 1, which biases its energy decay (+6.8e-6 after 1000 steps
      against the FP64 scheme).  Its energy history is compared with the oracle run with the same
      float factors (within 2e-6), which isolates that bias; this library's history then lies
      within the FP64-to-float-factor gap plus 2e-6 of the reference's.
    - Every printed diagnostic: DT and CFLM within 3e-5 (each run's CFLM is the maximum over its
      own field, and the two fields are ~4e-5 apart by step 1000), CN within 2e-6, T within 2e-5
      (the float sum of the DT sequence), and SIG within one pixel level."""
    N, Re, K0, cfl, steps, update = 512, 1e4, 4.0, 0.1, 1000, 100
    om0 = O.k4_spectrum(N, K0, 0)
    E_ref, Z_ref, diag_ref, om_ref = _ref_harness(N, Re, K0, cfl, steps, update, om0, tmp_path)
    E, Z, diag, om = _ours(N, Re, K0, cfl, steps, update, om0)
    E_o, Z_o, om_o = _oracle(N, Re, K0, cfl, steps, update, om0)
    E_f, _, _ = _oracle(N, Re, K0, cfl, steps, update, om0, f32_cn=True)
    assert E.size == E_ref.size == E_o.size == steps
    assert np.max(np.abs(E / E_o - 1)) <= 1e-6
    assert np.max(np.abs(Z / Z_o - 1)) <= 1e-6
    assert _rl2(om, om_o) <= 1e-4
    assert np.max(np.abs(E_ref / E_f - 1)) <= 2e-6
    gap = np.max(np.abs(E_f / E_o - 1))
    assert np.max(np.abs(E / E_ref - 1)) <= gap + 2e-6
    assert sorted(diag) == sorted(diag_ref) == [1] + list(range(100, 1001, 100))
    for it, (t, dt, cn, cflm, sig) in diag_ref.items():
        g = diag[it]
        assert g[0] == pytest.approx(t, rel=2e-5)
        assert g[1] == pytest.approx(dt, rel=3e-5)
        assert g[2] == pytest.approx(cn, abs=2e-6)
        assert g[3] == pytest.approx(cflm, rel=3e-5)
        assert abs(g[4] - sig) <= 1.0


@pytest.mark.skipif(not os.path.exists(REF), reason="reference binary not built")
@pytest.mark.parametrize("args", [[16384, "1E6", 5, 21, 0.2, 10, 0], [2048, "1E5", 4, 200, 0.1, 50, 0]])
def test_cli_matches_reference_binary(args, tmp_path):
    """The reference's own command lines (its recorded N=16384 run on the cluster path, and an
    N=2048 run), both binaries from their PAO start on the same GPU: the PAO seed and every printed
    iteration line (T, DT, CN, CFLM, SIG) agree to FP32 transform rounding."""
    (tmp_path / "r").mkdir()
    (tmp_path / "o").mkdir()
    env = {"BENCH_WARMUP_STEPS": "0"}
    ref = run_cli(args, tmp_path / "r", env=env, exe=REF, timeout=900)
    ours = run_cli(args, tmp_path / "o", env=env, timeout=900)
    assert ref.returncode == 0, ref.stderr[-2000:]
    assert ours.returncode == 0, ours.stderr[-2000:]
    seed = re.compile(r"PAO seed\s*=\s*(\d+)")
    assert seed.search(ref.stdout)[1] == seed.search(ours.stdout)[1]
    r, o = iterations(ref.stdout), iterations(ours.stdout)
    assert sorted(r) == sorted(o) and len(r) >= 3
    for it in r:
        # T is printed with 10 decimals: one unit of the last digit is 1e-10
        assert o[it]["T"] == pytest.approx(r[it]["T"], rel=1e-6, abs=1.5e-10)
        assert o[it]["DT"] == pytest.approx(r[it]["DT"], rel=1e-5, abs=2e-8)
        assert o[it]["CN"] == pytest.approx(r[it]["CN"], abs=2e-6)
        assert o[it]["CFLM"] == pytest.approx(r[it]["CFLM"], rel=1e-5)
        assert abs(o[it]["SIG"] - r[it]["SIG"]) <= 1



def _spectrum_bins(u, w, nbins):
    """energy_spectrum.csv bins (cuda/mem_cuda.cu:599-626) of the physical planes u, w, in FP64:
    forward R2C of each, p = |U|^2 + |W|^2 doubled for 0 < kx < L/2, binned by |k| / (L/2) / sqrt 2."""
    L = u.shape[0]
    U, W = np.fft.rfft2(u), np.fft.rfft2(w)
    p = np.abs(U) ** 2 + np.abs(W) ** 2
    kx = np.arange(L // 2 + 1)[None, :]
    z = np.arange(L)[:, None]
    kz = np.where(z <= L // 2, z, z - L)
    r = np.sqrt((kx * kx + kz * kz).astype(np.float64)) / (0.5 * L)
    b = np.clip(np.floor(r / np.sqrt(2.0) * nbins).astype(np.int64), 0, nbins - 1)
    dbl = (kx > 0) & (kx < L // 2)
    keep = ~((kx == 0) & (kz == 0))
    e = np.bincount(b[keep], weights=np.where(dbl, 2 * p, p)[keep], minlength=nbins)
    c = np.bincount(b[keep], weights=np.broadcast_to(np.where(dbl, 2, 1), b.shape)[keep], minlength=nbins)
    return e, c.astype(np.int64)


def test_energy_spectrum_bins_match_oracle():
    """The energy_spectrum.csv bins of this library (the forward R2C of the physical velocity over
    every mode, binned like the reference) against the same binning of the FP64 oracle's velocity
    after 10 steps: equal counts in every bin; bins with energy above 1e-12 of the total within
    1e-5 relative (plus a floor of 1e-10 of the total); the bins beyond the retained radius hold
    only rounding noise, below 1e-9 of the total."""
    import optimizec_b200 as P
    N, Re, K0, cfl = 128, 1e4, 4.0, 0.1
    om0 = O.k4_spectrum(N, K0, 2)
    s = P.Solver(N, Re, K0, cfl)
    s.init_vorticity(om0)
    s.next_dt()
    s.step(10)
    o = O.Oracle(N, Re, K0, cfl)
    o.init_om2(om0)
    o.run_fixed([s.scalars()["dt"]] * 10, [1.0] * 10)
    nbins = 3 * N
    e, c = s.velocity_spectrum_bins(nbins)
    e_o, c_o = _spectrum_bins(o.ur(0), o.ur(1), nbins)
    o.close()
    assert np.array_equal(c, c_o)
    tot = e_o.sum()
    big = e_o > 1e-12 * tot
    assert big.sum() >= 20  # the k^4 field at K0 = 4 fills the low-k shells only
    assert np.all(np.abs(e[big] - e_o[big]) <= 1e-5 * e_o[big] + 1e-10 * tot)
    assert np.all(e[~big] <= 1e-9 * tot)


def _pgm(path):
    b = open(path, "rb").read()
    parts = b.split(b"\n", 3)
    w, h = map(int, parts[1].split())
    return np.frombuffer(parts[3], dtype=np.uint8).reshape(h, w)


def _csv_rows(path):
    lines = open(path).read().splitlines()
    return lines[0], [tuple(float(x) for x in l.split(",")) for l in lines[1:]]


@pytest.mark.skipif(not os.path.exists(REF), reason="reference binary not built")
def test_dump_files_match_reference_binary(tmp_path):
    """The files of a signal save, against the reference binary's own: the reference runs from a
    seeded restart.bin and is sent SIGRTMIN, which writes restart.bin and every dump file of the
    same state into its _restart folder; this CLI's DUMP mode renders that restart.bin.
    - u_velocity, v_velocity, kinetic, omega (0.1 % / 99.9 % percentile clip), stream PGMs:
      same header, at most one grey level apart, and at least 99.9 % of the pixels identical (the
      velocities are rebuilt from the file through this library's transforms, so values sitting on
      a grey-level boundary can round the other way).
    - energy_spectrum.csv: the same header and the same rows (bin radius and count), and every
      energy within 1e-5 relative plus an absolute floor of 1e-10 of the total (the two codes'
      FP32 transform rounding in the nearly empty high-k bins); the bins below that floor hold the
      transforms' rounding noise in both files and are compared only for being below 1e-9 of the
      total."""
    N, Re, K0, cfl = 256, 1e4, 4.0, 0.1
    o = O.Oracle(N, Re, K0, cfl)
    o.init_om2(O.k4_spectrum(N, K0, 4))
    rb = tmp_path / "start.bin"
    O.write_restart_v2(str(rb), o, Re, K0, cfl)
    o.close()
    run = tmp_path / "ref"
    run.mkdir()
    proc = subprocess.Popen([REF, str(N), "10000", "4", "1000000", "0.1", "50", "0", str(rb)], cwd=run,
                            stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
    try:
        _wait_for(proc, r"ITERATION\s+100 ", timeout=120)
        proc.send_signal(signal.SIGRTMIN)
        _wait_for(proc, r"_restart/meta\.csv", timeout=120)
        proc.send_signal(signal.SIGINT)
        proc.communicate(timeout=60)
    finally:
        if proc.poll() is None:
            proc.kill()
    folders = [d for d in os.listdir(run) if d.endswith("_restart")]
    assert len(folders) == 1, folders
    ref = run / folders[0]
    ours = tmp_path / "ours"
    p = subprocess.run([CLI, "DUMP", str(ref / "restart.bin"), str(ours), "50"], capture_output=True, text=True,
                       timeout=300)
    assert p.returncode == 0, p.stderr + p.stdout
    for f in ["u_velocity.pgm", "v_velocity.pgm", "kinetic.pgm", "omega.pgm", "stream.pgm"]:
        a, b = _pgm(ours / f), _pgm(ref / f)
        assert a.shape == b.shape == (3 * N // 2, 3 * N // 2), f
        d = np.abs(a.astype(np.int64) - b.astype(np.int64))
        assert d.max() <= 1 and (d == 0).mean() >= 0.999, (f, int(d.max()), float((d == 0).mean()))
    ha, ra = _csv_rows(ours / "energy_spectrum.csv")
    hb, rb_ = _csv_rows(ref / "energy_spectrum.csv")
    assert ha == hb == "normalized_radius,shell_sum_energy,count"
    assert [(r[0], r[2]) for r in ra] == [(r[0], r[2]) for r in rb_]
    ea, eb = np.array([r[1] for r in ra]), np.array([r[1] for r in rb_])
    tot = eb.sum()
    big = eb > 1e-10 * tot
    assert np.all(np.abs(ea[big] - eb[big]) <= 1e-5 * eb[big] + 1e-10 * tot), np.max(np.abs(ea[big] / eb[big] - 1))
    assert np.all(ea[~big] <= 1e-9 * tot)


def _palin_fp64(om2):
    """The reference's palinstrophy ratio (cuda/mem_cuda.cu:872-940) in FP64 on [iz][ix] om2:
    sum w k^2 |om|^2 / ((sum w |om|^2 - |om_00|^2) kmax^2), w = 1 on ix = 0 and ix = N/2 - 1, else 2."""
    N, H = om2.shape
    ax = np.arange(H, dtype=np.float64)[None, :]
    iz = np.arange(N)[:, None]
    gz = np.where(iz < N // 2, iz, iz - N).astype(np.float64)
    k2 = ax * ax + gz * gz
    w = np.where((np.arange(H) == 0) | (np.arange(H) == H - 1), 1.0, 2.0)[None, :]
    p = np.abs(om2.astype(np.complex128)) ** 2
    total = float((w * p).sum()) - float(p[0, 0])
    return float((w * k2 * p).sum()) / (total * float(k2.max()))


@pytest.mark.parametrize("N", [64, 512, 2048])
def test_palin_matches_fp64_formula(N):
    """dns2d_palin (FP64 reduction on the GPU) against the reference's formula evaluated in FP64 on
    the host from the same field, after 5 steps of a seeded run: 1e-12 relative."""
    import optimizec_b200 as P
    s = P.Solver(N, 1e4, 4.0, 0.1)
    s.init_vorticity(O.k4_spectrum(N, 4.0, 3))
    s.next_dt()
    s.step(5)
    got = s.palin()
    want = _palin_fp64(s.om2())
    s.close()
    assert got == pytest.approx(want, rel=1e-12)


@pytest.mark.skipif(not os.path.exists(REF), reason="reference binary not built")
def test_adaptive_viscosity_matches_reference_binary(tmp_path):
    """ADAPT_VISC=1: both binaries from the same seeded restart.bin (N = 256, 600 steps, UPDATE =
    20), the PD controller on the filtered palinstrophy ratio moving the viscosity at the diagnostic
    steps: every printed PALIN within one unit, VISC and Re within 1e-4 relative (printed to 6
    digits), DT within 1e-5, and the viscosity does change during the run."""
    N, Re, K0, cfl = 256, 1e4, 4.0, 0.1
    o = O.Oracle(N, Re, K0, cfl)
    o.init_om2(O.k4_spectrum(N, K0, 6))
    rb = tmp_path / "start.bin"
    O.write_restart_v2(str(rb), o, Re, K0, cfl)
    o.close()
    args = [N, 10000, 4, 600, 0.1, 20, 1, str(rb)]
    (tmp_path / "r").mkdir()
    (tmp_path / "o").mkdir()
    ref = run_cli(args, tmp_path / "r", exe=REF)
    ours = run_cli(args, tmp_path / "o")
    assert ref.returncode == 0, ref.stderr
    assert ours.returncode == 0, ours.stderr
    r, g = iterations(ref.stdout), iterations(ours.stdout)
    assert sorted(r) == sorted(g) and len(r) == 31
    for it in r:
        assert abs(g[it]["PALIN"] - r[it]["PALIN"]) <= 1, it
        assert g[it]["VISC"] == pytest.approx(r[it]["VISC"], rel=1e-4), it
        assert g[it]["Re"] == pytest.approx(r[it]["Re"], rel=1e-4), it
        assert g[it]["DT"] == pytest.approx(r[it]["DT"], rel=1e-5, abs=2e-8), it
    assert len({r[it]["VISC"] for it in r}) > 1  # the controller acted
