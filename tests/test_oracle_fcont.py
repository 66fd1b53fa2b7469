"""The oracle's continuous-f restatement (oc_props_fcont; no reference
counterpart): theta = 0 is the reference discretisation bit for bit; lnQ is
continuous where N f crosses an integer (the junction step turns from pure A
into pure B smoothly) and smooth inside a step.  The oracle's derivatives of
the variant (oc_dlnq_df, oc_stress_fcont) against central finite differences
of its lnQ at fixed fields."""
import numpy as np
import pytest

import oracle as O

M3, D3, N = (8, 12, 10), (2.0, 3.0, 2.5), 20


def _w(seed=0):
    M = int(np.prod(M3))
    rng = np.random.default_rng(seed)
    w = np.zeros(6 * M)
    w[:M] = rng.normal(0, 1.5, M)
    w[M:2 * M] = rng.normal(0, 0.5, M)
    return w


def _fd4(fn, x, h):
    """(-F(x+2h) + 8F(x+h) - 8F(x-h) + F(x-2h)) / 12h: error O(h^4)."""
    return (-fn(x + 2 * h) + 8 * fn(x + h) - 8 * fn(x - h) + fn(x - 2 * h)) / (12 * h)


def _lnq(f, ens, cont=True, seed=0):
    d = O.Density(M3, D3, N)
    w = _w(seed)
    q, phis = (d.props_fcont if cont else d.props)(w, N, 0.1, 0.8, f, ens)
    return q, phis, w[2 * w.size // 6:]


def test_theta_zero_is_the_reference_discretisation():
    for ens in (1, 2):
        q0, p0, c0 = _lnq(0.45, ens, cont=False)   # N f = 9 exactly
        q1, p1, c1 = _lnq(0.45, ens, cont=True)
        assert q0 == q1
        np.testing.assert_array_equal(p0, p1)
        np.testing.assert_array_equal(c0, c1)


def test_lnq_continuous_across_a_step_boundary():
    for ens in (1, 2):
        below, _, _ = _lnq(0.5 - 1e-9, ens)   # n1 = 9, theta -> 1: the junction step is pure A
        at, _, _ = _lnq(0.5, ens)             # n1 = 10, theta = 0
        assert abs(below - at) <= 1e-6 * max(1.0, abs(at)), (below, at)


def test_lnq_smooth_inside_a_step():
    f0 = 0.47   # N f = 9.4
    for ens in (1, 2):
        d1 = (_lnq(f0 + 1e-3, ens)[0] - _lnq(f0 - 1e-3, ens)[0]) / 2e-3
        d2 = (_lnq(f0 + 5e-4, ens)[0] - _lnq(f0 - 5e-4, ens)[0]) / 1e-3
        assert abs(d1 - d2) <= 1e-5 * max(1.0, abs(d2)), (d1, d2)
        assert abs(d2) > 1e-6   # f does move lnQ


@pytest.mark.parametrize("ens,f", [(1, 0.47), (2, 0.47), (1, 0.43), (2, 0.512)])
def test_dlnq_df_matches_finite_differences(ens, f):
    """d lnQ/df by dS/dtheta of the junction step against the fourth-order
    central difference of lnQ, h = 1e-3, with N f away from an integer (the
    stencil stays inside one contour step).  Its truncation error is about
    3e-13 here, so the adjoint is exact, not an approximation."""
    w = _w(3)
    W = w[:2 * w.size // 6].copy()
    dl = O.Density(M3, D3, N).dlnq_df(W, N, 0.1, 0.8, f, ens)
    fd = _fd4(lambda x: _lnq(x, ens, seed=3)[0], f, 1e-3)
    print("ens", ens, "f", f, "adjoint", dl, "fd", fd)
    assert abs(dl - fd) <= 1e-10 * max(1.0, abs(fd)), (dl, fd)


def test_dlnq_df_refuses_what_props_refuses():
    w = _w(3)
    W = w[:2 * w.size // 6].copy()
    with pytest.raises(ValueError):
        O.Density(M3, D3, N).dlnq_df(W, N, 0.1, 0.8, 0.47, 3)


@pytest.mark.parametrize("ens", [1, 2])
def test_stress_with_the_junction_step_matches_finite_differences(ens):
    """oc_stress_fcont against fourth-order differences of props_fcont's lnQ
    in the box lengths (h = 1e-3); at theta = 0 it equals oc_stress bit for
    bit."""
    D = np.array(D3)
    w = _w(4)
    W = w[:2 * w.size // 6].copy()
    f, h = 0.47, 1e-3
    dl = O.Density(M3, D, N).stress(W, N, 0.1, 0.8, f, ens, fcont=True)

    def lnq(Dx):
        ww = np.zeros_like(w)
        ww[:W.size] = W
        return O.Density(M3, Dx, N).props_fcont(ww, N, 0.1, 0.8, f, ens)[0]

    for i in range(3):
        e = np.eye(3)[i]
        fd = _fd4(lambda x: lnq(D + x * e), 0.0, h)
        assert abs(dl[i] - fd) <= 1e-10 * max(1.0, abs(fd)), (i, dl[i], fd)
    s0 = O.Density(M3, D, N).stress(W, N, 0.1, 0.8, 0.45, ens)
    s1 = O.Density(M3, D, N).stress(W, N, 0.1, 0.8, 0.45, ens, fcont=True)
    np.testing.assert_array_equal(s0, s1)
