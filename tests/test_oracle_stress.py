"""The oracle's box-stress adjoint (oc_stress: dS/dL applied in real space)
against fourth-order central differences of the oracle's own lnQ in the box
lengths (h = 1e-3, truncation error about 1e-12 here), at fixed fields, in
both ensembles."""
import numpy as np
import pytest

import oracle as O


def _fields(m, D, seed):
    rng = np.random.default_rng(seed)
    x = [np.arange(m[i]) * D[i] / m[i] for i in range(3)]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    wm = 3.0 * (np.cos(2 * np.pi * X / D[0]) + 0.5 * np.sin(2 * np.pi * Y / D[1]) * np.cos(2 * np.pi * Z / D[2]))
    wm += 0.2 * rng.normal(size=m)
    wp = 0.3 * rng.normal(size=m)
    return np.concatenate([wm.ravel(), wp.ravel()])


def _lnq(m, D, N, W, f, ens):
    d = O.Density(m, D, N)
    w = np.zeros(3 * W.size)
    w[:W.size] = W
    return d.props(w, N, 0.1, 0.8, f, ens)[0]


@pytest.mark.parametrize("m,D,N,ens", [((8, 12, 10), (2.0, 3.0, 2.5), 20, 1),
                                        ((12, 8, 16), (3.1, 2.2, 4.0), 24, 2)])
def test_oracle_stress_matches_finite_differences(m, D, N, ens):
    D = np.array(D)
    W = _fields(m, D, 1)
    f = round(N * 0.45) / N
    dl = O.Density(m, D, N).stress(W, N, 0.1, 0.8, f, ens)
    h = 1e-3
    for i in range(3):
        e = np.eye(3)[i]
        L = [_lnq(m, D + k * h * e, N, W, f, ens) for k in (-2, -1, 1, 2)]
        fd = (L[0] - 8 * L[1] + 8 * L[2] - L[3]) / (12 * h)
        assert abs(dl[i] - fd) <= 1e-10 * max(1.0, abs(fd)), (i, dl[i], fd)
