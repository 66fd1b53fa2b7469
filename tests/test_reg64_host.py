"""The register-resident 64-point transforms and warp slab phases of the
64^3 FP32 step kernels (scft_string_b200/csrc/reg64.cuh), built for the host
and checked against numpy's FFT in float64: the 64-point FFT in both orders,
the forward slab (64 x 64 real -> 64 x 33 half spectrum, two-for-one z pass and
joined kz = 0/32 column) and the inverse slab (half-complex-to-real).  No GPU."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _cuda_include():
    home = os.environ.get("CUDA_HOME") or os.environ.get("CUDA_PATH")
    if not home:
        nvcc = shutil.which("nvcc")
        home = os.path.dirname(os.path.dirname(nvcc)) if nvcc else None
    inc = os.path.join(home, "include") if home else None
    return inc if inc and os.path.exists(os.path.join(inc, "cuda_runtime.h")) else None


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    inc = _cuda_include()
    if inc is None or shutil.which("g++") is None:
        pytest.skip("needs g++ and the CUDA headers")
    out = str(tmp_path_factory.mktemp("reg64") / "libreg64_host.so")
    subprocess.run(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-I" + inc, "-o", out,
                    os.path.join(HERE, "reg64_host.cpp")], check=True)
    L = C.CDLL(out)
    fp = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    L.h_fft64.argtypes = [C.c_int, C.c_int, fp]
    L.h_perm.restype = C.c_int
    L.h_slab_forward.argtypes = [fp, fp]
    L.h_slab_inverse.argtypes = [fp, fp]
    return L


def _c64(a):
    return np.ascontiguousarray(np.stack([a.real, a.imag], -1).astype(np.float32).reshape(-1))


def _cplx(f):
    f = f.reshape(-1, 2).astype(np.float64)
    return f[:, 0] + 1j * f[:, 1]


@pytest.mark.parametrize("sign", [-1, 1])
def test_fft64_both_orders(lib, sign):
    rng = np.random.default_rng(1)
    x = rng.normal(size=64) + 1j * rng.normal(size=64)
    ref = np.fft.fft(x) if sign < 0 else np.fft.ifft(x) * 64
    buf = _c64(x)
    lib.h_fft64(sign, 0, buf)
    got = _cplx(buf)
    perm = [lib.h_perm(k) for k in range(64)]
    assert sorted(perm) == list(range(64))
    np.testing.assert_allclose(got[perm], ref, atol=2e-5 * np.abs(ref).max())
    # permuted input, natural output
    xp = np.empty(64, complex)
    xp[perm] = x
    buf = _c64(xp)
    lib.h_fft64(sign, 1, buf)
    np.testing.assert_allclose(_cplx(buf), ref, atol=2e-5 * np.abs(ref).max())


def test_slab_forward_matches_rfft2(lib):
    rng = np.random.default_rng(2)
    real = np.exp(rng.normal(0, 0.5, (64, 64)))
    spec = np.zeros(64 * 33 * 2, np.float32)
    lib.h_slab_forward(np.ascontiguousarray(real, np.float32), spec)
    got = _cplx(spec).reshape(64, 33)
    ref = np.fft.rfft2(real.astype(np.float32).astype(np.float64))
    assert np.abs(got - ref).max() <= 2e-6 * np.abs(ref).max()


def test_slab_inverse_matches_irfft2(lib):
    rng = np.random.default_rng(3)
    real = np.exp(rng.normal(0, 0.5, (64, 64)))
    spec = np.fft.rfft2(real)
    out = np.zeros(64 * 64, np.float32)
    lib.h_slab_inverse(_c64(spec), out)
    ref = np.fft.irfft2(_cplx(_c64(spec)).reshape(64, 33), s=(64, 64)) * 4096
    assert np.abs(out.reshape(64, 64) - ref).max() <= 2e-6 * np.abs(ref).max()
    # round trip
    np.testing.assert_allclose(out.reshape(64, 64) / 4096, real, rtol=3e-6)
