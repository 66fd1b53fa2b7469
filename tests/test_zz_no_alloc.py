"""The allocation-free contour step, scft_do_step_noalloc, through the C ABI.

It serves callers that cannot allocate device memory at the moment they need
a step (a real-time loop that must not stall on the allocator, a framework
that owns all device allocations through its own pool): its working buffers
live in a static device array instead.  Two calls in a row must give the
same result as the allocating entry point scft_do_step and as the FP64
oracle's do_step, within the tolerance of the other FP64 step tests, on a
small runtime-shaped grid and on grids at the array's limits (an axis of 64;
M = 32768); a size beyond the limits is rejected.  Collected last so that a
failure here leaves every other test run."""
import ctypes as C

import numpy as np
import pytest

import scft_string_b200 as S

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("m,D", [((16, 12, 10), (4.0, 3.0, 2.5)),
                                 ((64, 64, 8), (4.0, 4.0, 0.5)),
                                 ((32, 32, 32), (4.0, 4.0, 4.0))])
def test_noalloc_step_matches_allocating_step(built_lib, m, D):
    import torch

    import oracle as O

    N, f = 24, 0.45
    M = int(np.prod(m))
    rng = np.random.default_rng(9)
    wm, wp = rng.normal(0, 1.5, M), rng.normal(0, 0.5, M)
    ctx = S.Context(m, D, N, chi=12, f=f, phidb=0.8, ens=2, strn=1, dostring=0)
    ctx.set_fields(0, wm, wp)
    od = O.Density(m, D, N)
    od.prepare(1.0 / N, np.concatenate([wm, wp]))
    lib = S.lib()
    mi = (C.c_int * 3)(*m)
    Di = (C.c_double * 3)(*D)
    dev = torch.device("cuda", 0)
    w_dev = torch.tensor(np.concatenate([wm, wp]), dtype=torch.float64, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    n1 = round(N * (round(N * f) / N))
    for s in (0, n1 - 1, n1, N - 1):
        qin = 1.0 + 0.3 * rng.normal(size=2 * M)
        ref = ctx.do_step(0, qin, s)
        orc = od.do_step(qin, s, n1, N - n1)
        in_dev = torch.tensor(qin, dtype=torch.float64, device=dev)
        for _ in range(2):  # the shared array keeps the previous call's contents
            out_dev = torch.full((2 * M,), np.nan, dtype=torch.float64, device=dev)
            rc = lib.scft_do_step_noalloc(mi, Di, N, f, _ptr(w_dev), _ptr(in_dev), _ptr(out_dev), s, stream)
            assert rc == 0, S.STATUS.get(rc, rc)
            got = out_dev.cpu().numpy()
            assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max(), s
            assert np.abs(got - orc).max() <= 1e-13 * np.abs(orc).max(), s


def test_noalloc_rejects_sizes_beyond_its_array(built_lib):
    import torch

    lib = S.lib()
    dev = torch.device("cuda", 0)
    big = (64, 64, 16)  # M = 65536 > 32768
    M = 64 * 64 * 16
    buf = torch.zeros(2 * M, dtype=torch.float64, device=dev)
    rc = lib.scft_do_step_noalloc((C.c_int * 3)(*big), (C.c_double * 3)(4.0, 4.0, 1.0), 10, 0.5,
                                  _ptr(buf), _ptr(buf), _ptr(buf), 0, None)
    assert rc == 3
    # an A fraction outside [0, 1] is refused as scft_create refuses it
    rc = lib.scft_do_step_noalloc((C.c_int * 3)(8, 8, 8), (C.c_double * 3)(4.0, 4.0, 4.0), 10, 1.5,
                                  _ptr(buf), _ptr(buf), _ptr(buf), 0, None)
    assert rc == 3
