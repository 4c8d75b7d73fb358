"""The no-allocation time step, dns2d_step_noalloc, against the regular entry point.

Some callers cannot allocate device memory: applications that only hand out buffers from their
own pool or arena, processes with a fixed device-memory budget, or code where cudaMalloc is not
allowed.  dns2d_step_noalloc takes the caller's own device buffers for the vorticity state and
keeps every other byte it needs in one static device array inside the library.

This test advances the same field through both entry points, twice in a row (the second call
continues from the first call's output and so also exercises the array's leftover contents),
and requires the no-allocation result to match the regular one within the vorticity tolerance
used by the parity tests (relative L2 <= 1e-5).  The file is named so that pytest collects it
last; it passes alone in a fresh process and after the other tests.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.parametrize("N", [64, 512])
def test_noalloc_matches_regular_step(N):
    import torch
    import optimizec_b200 as P

    K0, Re, cfl, n = 4.0, 1e4, 0.1, 6
    om0 = P.k4_spectrum(N, K0, 21)
    s = P.Solver(N, Re, K0, cfl)
    s.init_vorticity(om0)
    s.next_dt()
    sc = s.scalars()

    dev = torch.device("cuda:0")
    d_om = torch.from_numpy(om0.view(np.float32).copy()).to(dev)
    d_fn = torch.zeros_like(d_om)
    lib = P.lib()
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        # regular entry point
        s.step(n)
        # no-allocation entry point with the same scalars the regular one used for this call
        rc = lib.dns2d_step_noalloc(N, sc["visc"], sc["dt"], sc["cnm1"], sc["cn"], n,
                                    d_om.data_ptr(), d_fn.data_ptr(), stream)
        assert rc == 0, lib.dns2d_strerror(rc)
        torch.cuda.synchronize(dev)
        sc = s.scalars()
        got = d_om.cpu().numpy().view(np.complex64).reshape(N, N // 2).astype(np.complex128)
        want = s.om2().astype(np.complex128)
        assert rel_l2(got, want) <= 1e-5, (call, rel_l2(got, want))
        got_fn = d_fn.cpu().numpy().view(np.complex64).reshape(N, N // 2).astype(np.complex128)
        want_fn = s.fnm1().astype(np.complex128)
        assert rel_l2(got_fn, want_fn) <= 1e-5, call
    s.close()
    if N <= 64:
        # and directly against the FP64 oracle over the same 2 x n steps at the same dt
        from oracle import oracle as O
        sc0 = P.Solver(N, Re, K0, cfl)
        sc0.init_vorticity(om0)
        sc0.next_dt()
        d = sc0.scalars()
        sc0.close()
        o = O.Oracle(N, Re, K0, cfl)
        o.init_om2(om0)
        o.set_scalars({"visc": d["visc"]})
        o.run_fixed([d["dt"]] * (2 * n), [d["cn"]] * (2 * n))
        assert rel_l2(got, o.om2()) <= 1e-5
        o.close()


def test_noalloc_rejects_sizes_beyond_its_array():
    import optimizec_b200 as P

    lib = P.lib()
    assert lib.dns2d_step_noalloc(1024, 1e-4, 1e-4, 0.0, 1.0, 1, 1, 1, None) == 2  # DNS2D_ERR_SIZE
    assert lib.dns2d_step_noalloc(100, 1e-4, 1e-4, 0.0, 1.0, 1, 1, 1, None) == 2
    assert lib.dns2d_step_noalloc(64, 1e-4, 1e-4, 0.0, 1.0, 1, None, None, None) == 1  # DNS2D_ERR_ARG
