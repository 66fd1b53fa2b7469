"""The octet (eight-lane) 64-point transforms of the shuffle x pass
(k_pencil_sh), restated lane by lane in numpy:

* the decomposition n = s + 8 n2, k = k1 + 8 k2 (8-point DFT, twiddle
  w64^(s k1), 8 x 8 transpose by three xor exchanges, 8-point DFT) gives the
  DFT, and forward, pointwise multiply, inverse gives back x'[s + 8 j] in the
  lane that loaded x[s + 8 j] (octet_fft64_fwd / octet_fft64_inv, fft.cuh);
* the shared-memory addresses of the 128-byte-swizzled pencil tiles
  (PencilSh::at, props_kernels.cu) spread every half-warp of 8-byte (FP32)
  and every octet of 16-byte (FP64) complex elements over distinct banks.
  This is a model: ncu still counts 18-22 % bank-conflict wavefronts for the
  FP32 kernel on a B200, so the hardware groups a warp's requests
  differently;
* every tile index stays inside its tile.
CPU only."""
import numpy as np
import pytest


def dft8(v, sign):
    k = np.arange(8)
    return np.exp(sign * 2j * np.pi * np.outer(k, k) / 8) @ v


def octet_transpose(a):
    """a[lane][slot] -> the exchanges of octet_transpose, mask 1, 2, 4."""
    a = [list(x) for x in a]
    for m in (1, 2, 4):
        new = [list(x) for x in a]
        for s in range(8):
            up = bool(s & m)
            p = s ^ m
            for j in range(8):
                if j & m:
                    continue
                recv = a[p][j] if (p & m) else a[p][j | m]   # what the partner sends
                if up:
                    new[s][j] = recv
                else:
                    new[s][j | m] = recv
        a = new
    return a


W64 = np.exp(-2j * np.pi * np.arange(64) / 64)


def octet_fwd(lanes):
    out = []
    for s in range(8):
        v = dft8(np.array(lanes[s]), -1)
        out.append(v * W64[s * np.arange(8)])
    return [dft8(np.array(r), -1) for r in octet_transpose(out)]


def octet_inv(lanes):
    out = []
    for s in range(8):
        v = dft8(np.array(lanes[s]), +1)
        out.append(v * np.conj(W64[s * np.arange(8)]))
    return [dft8(np.array(r), +1) for r in octet_transpose(out)]


def test_transpose_is_a_transpose():
    a = np.arange(64).reshape(8, 8)
    assert np.array_equal(np.array(octet_transpose(a.tolist())), a.T)


def test_forward_multiply_inverse():
    rng = np.random.default_rng(3)
    x = rng.normal(size=64) + 1j * rng.normal(size=64)
    K = rng.uniform(0.2, 1.0, 64)
    lanes = [x[s + 8 * np.arange(8)] for s in range(8)]
    X = octet_fwd(lanes)
    got = np.zeros(64, complex)
    for s in range(8):
        got[s + 8 * np.arange(8)] = X[s]
    np.testing.assert_allclose(got, np.fft.fft(x), atol=1e-12)
    Y = octet_inv([X[s] * K[s + 8 * np.arange(8)] for s in range(8)])
    back = np.zeros(64, complex)
    for s in range(8):
        back[s + 8 * np.arange(8)] = Y[s]
    np.testing.assert_allclose(back, np.fft.ifft(np.fft.fft(x) * K) * 64, atol=1e-11)


def pencil_at(x, c, m0, esize):
    """PencilSh<T>::at: complex index of element (x, c) of a swizzled tile."""
    cpb = 128 // (2 * esize)
    b, cc = divmod(c, cpb)
    chunk = cc >> 1 if esize == 4 else cc
    sw = chunk ^ (x & 7)
    return b * cpb * m0 + x * cpb + ((sw << 1) | (cc & 1) if esize == 4 else sw)


def groups(esize):
    """lanes served by one shared-memory wavefront: 16 lanes of 8-byte, 8 of 16-byte elements"""
    n = 16 if esize == 4 else 8
    return [range(g, g + n) for g in range(0, 32, n)]


def conflict_free(addr_of_lane, esize):
    """addresses (complex index) of the lanes of a warp: distinct addresses in
    a wavefront must fall in distinct 128-byte bank slots"""
    cb = 2 * esize  # bytes per complex
    for grp in groups(esize):
        seen = {}
        for lane in grp:
            a = addr_of_lane(lane)
            bank = (a * cb) % 128 // cb
            if bank in seen and seen[bank] != a:
                return False
            seen[bank] = a
    return True


@pytest.mark.parametrize("esize,tc", [(4, 32), (4, 64), (8, 16), (8, 32)])
def test_pencil_tile_is_conflict_free_and_in_bounds(esize, tc):
    m0 = 64
    idx = {pencil_at(x, c, m0, esize) for x in range(m0) for c in range(tc)}
    assert idx == set(range(tc * m0))   # a permutation of the tile
    for warp in range(8):
        for line0 in range(0, 2 * tc, 32):
            for j in range(8):
                def addr(lane):
                    s, oct_ = lane & 7, warp * 4 + (lane >> 3)
                    t = (line0 + oct_) % tc
                    return pencil_at(s + 8 * j, t, m0, esize)
                assert conflict_free(addr, esize)
