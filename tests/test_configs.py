"""CPU checks of the workload definitions and seeded field generators used by
the benchmark modes (no GPU, no library calls)."""
import numpy as np

from scft_string_b200.configs import (ADJOINT_96, MIXED_128, STRING_64, fields, gyroid_fields,
                                      hex_fields)


def test_workload_parameters():
    # canonical runs converge only with even n1, n2 and alpha N (scft.cu:1032-1040)
    c = ADJOINT_96
    assert c["ens"] == 1
    for v in (c["N"] * c["f"], c["N"] * (1 - c["f"]), c["alpha"] * c["N"]):
        assert abs(v - round(v)) < 1e-9 and round(v) % 2 == 0
    assert MIXED_128["m"] == (128, 128, 128) and MIXED_128["dostring"] == 0
    assert STRING_64["strn"] == 16 and STRING_64["ens"] == 2


def test_gyroid_fields_shape_seed_and_symmetry():
    c = dict(MIXED_128, m=(16, 16, 16), strn=3)
    wm, wp = gyroid_fields(c)
    assert wm.shape == (3, 16 ** 3) and wp.shape == wm.shape and not wp.any()
    wm2, _ = gyroid_fields(c)
    np.testing.assert_array_equal(wm, wm2)           # seeded
    assert not np.allclose(wm[0], wm[1])              # per-replica noise
    # the noiseless part is odd under r -> -r (each term is odd in one coordinate)
    base = wm.mean(axis=0).reshape(16, 16, 16)
    flipped = np.roll(base[::-1, ::-1, ::-1], 1, axis=(0, 1, 2))
    assert np.abs(base + flipped).max() < 6 * 0.03 * c["chi"] / np.sqrt(3) + 1e-12


def test_hex_fields_sixfold_pattern():
    c = dict(ADJOINT_96, m=(24, 24, 8), seed=11)
    wm, wp = hex_fields(c)
    assert wm.shape == (1, 24 * 24 * 8) and not wp.any()
    w = wm[0].reshape(24, 24, 8)
    # constant along z up to the noise; mean close to zero
    assert np.abs(w - w.mean(axis=2, keepdims=True)).max() < 10 * 0.02 * c["chi"]
    assert abs(w.mean()) < 0.1 * c["chi"]
    # the maximum of sum_j cos(G_j.r) is 3 at the origin
    assert abs(w[0, 0].mean() - 1.5 * c["chi"]) < 0.1 * c["chi"]


def test_string_fields_reproducible():
    c = dict(STRING_64, m=(8, 8, 8), strn=4)
    a = fields(c)
    b = fields(c)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    assert a[0].shape == (4, 512)


def test_lamellar_fields_vary_along_z_only():
    from scft_string_b200.configs import lamellar_fields
    c = dict(ADJOINT_96, m=(8, 8, 24), seed=2)
    wm, wp = lamellar_fields(c)
    w = wm[0].reshape(8, 8, 24)
    assert not wp.any()
    assert np.abs(w - w.mean(axis=(0, 1), keepdims=True)).max() < 10 * 0.02 * c["chi"]
    assert abs(w[:, :, 0].mean() - 0.4 * c["chi"]) < 0.05 * c["chi"]
