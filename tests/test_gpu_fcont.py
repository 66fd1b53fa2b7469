"""Continuous A fraction (scft_problem.fcont, no reference counterpart): the
junction step's field theta wA + (1 - theta) wB makes lnQ and F smooth in f.
Checked here: theta = 0 reproduces the reference discretisation bit for bit;
the adjoint d lnQ/df and the box stress against central finite differences at
fixed fields; dF/df at a converged saddle point against differences of
re-converged free energies."""
import numpy as np
import pytest

import scft_string_b200 as S

pytestmark = pytest.mark.gpu


def _fields(m, D, seed):
    rng = np.random.default_rng(seed)
    x = [np.arange(m[i]) * D[i] / m[i] for i in range(3)]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    wm = 3.0 * (np.cos(2 * np.pi * X / D[0]) + 0.5 * np.sin(2 * np.pi * Y / D[1]) * np.cos(2 * np.pi * Z / D[2]))
    wm += 0.2 * rng.normal(size=m)
    wp = 0.3 * rng.normal(size=m)
    return wm.ravel(), wp.ravel()


def _ctx(m, D, N, f, ens, fcont=1, precision="fp64"):
    return S.Context(m, D, N, chi=12, f=f, phidb=0.8, ens=ens, alpha=0.1, strn=1, dostring=0,
                     precision=precision, fcont=fcont)


def _lnq(ctx, wm, wp):
    ctx.set_fields(0, wm, wp)
    ctx.props(0)
    return ctx.get_conc(0)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_theta_zero_is_the_reference_discretisation(built_lib, precision):
    m, D, N = (8, 12, 10), (2.0, 3.0, 2.5), 20
    wm, wp = _fields(m, D, 4)
    c0, q0, p0 = _lnq(_ctx(m, D, N, 0.45, 1, fcont=0, precision=precision), wm, wp)
    c1, q1, p1 = _lnq(_ctx(m, D, N, 0.45, 1, fcont=1, precision=precision), wm, wp)
    assert q0 == q1
    np.testing.assert_array_equal(c0, c1)
    np.testing.assert_array_equal(p0, p1)


@pytest.mark.parametrize("ens", [1, 2])
def test_dlnq_df_matches_finite_differences(built_lib, ens):
    m, D, N, f = (8, 12, 10), (2.0, 3.0, 2.5), 20, 0.47   # N f = 9.4: theta = 0.4
    wm, wp = _fields(m, D, 5)
    ctx = _ctx(m, D, N, f, ens)
    ctx.set_fields(0, wm, wp)
    dlnq, dF = ctx.dF_df(0)
    assert dF == -dlnq
    h = 1e-4
    qp = _lnq(_ctx(m, D, N, f + h, ens), wm, wp)[1]
    qm = _lnq(_ctx(m, D, N, f - h, ens), wm, wp)[1]
    fd = (qp - qm) / (2 * h)
    print("ens", ens, "d lnQ/df adjoint", dlnq, "fd", fd)
    assert abs(dlnq - fd) <= 1e-6 * max(1.0, abs(fd))
    c32 = _ctx(m, D, N, f, ens, precision="fp32")
    c32.set_fields(0, wm, wp)
    d32, _ = c32.dF_df(0)
    assert abs(d32 - dlnq) <= 1e-3 * max(1.0, abs(dlnq))


def test_box_stress_with_junction_step(built_lib):
    """The box stress adjoint (full store and checkpointed) with the junction
    step inside the chain."""
    m, D, N, f = (12, 8, 16), np.array([3.1, 2.2, 4.0]), 24, 0.43   # theta = 0.32
    wm, wp = _fields(m, D, 6)
    ctx = _ctx(m, D, N, f, 1)
    ctx.set_fields(0, wm, wp)
    dlnq, _ = ctx.stress(0)
    ck, _, _ = ctx.stress_ckpt(0, 5)
    assert np.abs(ck - dlnq).max() <= 1e-11 * np.abs(dlnq).max()
    h = 1e-4
    for i in range(3):
        Dp, Dm = D.copy(), D.copy()
        Dp[i] += h
        Dm[i] -= h
        ctx.set_box(Dp)
        ctx.props(0)
        qp = ctx.get_conc(0)[1]
        ctx.set_box(Dm)
        ctx.props(0)
        qm = ctx.get_conc(0)[1]
        fd = (qp - qm) / (2 * h)
        assert abs(dlnq[i] - fd) <= 1e-6 * max(1.0, abs(fd)), (i, dlnq[i], fd)


def _saddle(f, chi=14.0, m=(8, 8, 24), N=20, D=(2.0, 2.0, 4.6)):
    ctx = S.Context(m, D, N, chi=chi, f=f, phidb=0.8, ens=1, alpha=0.1, strn=1, dostring=0, fcont=1)
    z = np.arange(m[2]) * D[2] / m[2]
    wm = np.broadcast_to(0.4 * chi * np.cos(2 * np.pi * z / D[2]), m).ravel()
    ctx.set_fields(0, wm, np.zeros_like(wm))
    n, err = ctx.anderson_solve(0, maxIter=3000, tol=1e-10, nhist=12, lam=0.1)
    M = ctx.M
    ctx.props(0)
    conc, lnQ, _ = ctx.get_conc(0)
    W = ctx.get_fields(0)
    pA, pB = conc[:M], conc[M:2 * M]
    wa, wb = W[:M] + W[M:], W[M:] - W[:M]
    F = -lnQ + np.mean(chi * pA * pB - wa * pA - wb * pB)
    return ctx, F, err


def test_saddle_point_dF_df(built_lib):
    """dF/df = -d lnQ/df at the saddle point against central differences of
    re-converged free energies, f inside one contour step: N f = 10.2, so the
    A and B Simpson blocks (10 and 10 steps) and Nh = 2 are even, as a
    canonical saddle point needs (odd blocks bias the weights and leave
    <phiA + phiB> != 1)."""
    f, h = 0.51, 1e-4
    ctx, F0, err = _saddle(f)
    assert err <= 1e-10
    _, dF = ctx.dF_df(0)
    _, Fp, ep = _saddle(f + h)
    _, Fm, em = _saddle(f - h)
    assert max(ep, em) <= 1e-10
    fd = (Fp - Fm) / (2 * h)
    print("dF/df adjoint", dF, "fd", fd, "rel", abs(dF - fd) / abs(fd))
    assert abs(dF - fd) <= 2e-3 * max(1.0, abs(fd))


def test_gradients_entry_point(built_lib):
    """scft_gradients returns what the individual derivative calls return."""
    m, D, N = (8, 12, 10), np.array([2.0, 3.0, 2.5]), 20
    wm, wp = _fields(m, D, 7)
    for fcont in (0, 1):
        ctx = _ctx(m, D, N, 0.47, 1, fcont=fcont)
        ctx.set_fields(0, wm, wp)
        dL, dchi, df = ctx.gradients(0)
        np.testing.assert_array_equal(dL, ctx.stress(0)[1])
        assert dchi == ctx.dF_dchi(0)
        if fcont:
            assert df == ctx.dF_df(0)[1]
        else:
            assert np.isnan(df)


@pytest.mark.parametrize("m,D,N,f,ens,prec,tol", [
    ((8, 12, 10), (2.0, 3.0, 2.5), 20, 0.47, 1, "fp64", 1e-11),
    ((8, 12, 10), (2.0, 3.0, 2.5), 20, 0.47, 2, "fp64", 1e-11),
    ((32, 32, 32), (4.0, 4.0, 4.0), 24, 0.43, 1, "fp64", 1e-11),
    ((32, 32, 32), (4.0, 4.0, 4.0), 24, 0.43, 1, "fp32", 5e-5),
])
def test_fcont_props_match_the_oracle(built_lib, m, D, N, f, ens, prec, tol):
    """The CUDA continuous-f props against the oracle's FP64 restatement of the
    same variant (oc_props_fcont): lnQ and the four density fields."""
    import oracle as O
    wm, wp = _fields(m, D, 8)
    M = int(np.prod(m))
    ctx = _ctx(m, D, N, f, ens, fcont=1, precision=prec)
    conc, lnq, phis = _lnq(ctx, wm, wp)
    od = O.Density(m, D, N)
    w = np.zeros(6 * M)
    w[:M], w[M:2 * M] = wm, wp
    lnq0, phis0 = od.props_fcont(w, N, 0.1, 0.8, f, ens)
    assert abs(lnq - lnq0) <= tol * max(1.0, abs(lnq0)), (lnq, lnq0)
    assert np.abs(conc - w[2 * M:]).max() <= tol, np.abs(conc - w[2 * M:]).max()
    np.testing.assert_allclose(phis, phis0, rtol=0, atol=tol)


@pytest.mark.parametrize("m,D,N,f,ens", [
    ((8, 12, 10), (2.0, 3.0, 2.5), 20, 0.47, 1),
    ((8, 12, 10), (2.0, 3.0, 2.5), 20, 0.47, 2),
    ((8, 12, 10), (2.0, 3.0, 2.5), 20, 0.512, 2),
    ((32, 32, 32), (4.0, 4.0, 4.0), 24, 0.43, 1),
])
def test_fcont_derivatives_match_the_oracle(built_lib, m, D, N, f, ens):
    """The CUDA d lnQ/df (junction adjoint, Parseval form) and box stress
    with the junction step against the oracle's FP64 restatements
    (oc_dlnq_df, oc_stress_fcont: dS/dtheta and dS/dL applied in real space),
    at the same fields, FP64."""
    import oracle as O
    wm, wp = _fields(m, D, 9)
    ctx = _ctx(m, D, N, f, ens)
    ctx.set_fields(0, wm, wp)
    dlnq, _ = ctx.dF_df(0)
    dl, _ = ctx.stress(0)
    od = O.Density(m, D, N)
    W = np.concatenate([wm, wp])
    dlnq0 = od.dlnq_df(W, N, 0.1, 0.8, f, ens)
    dl0 = od.stress(W, N, 0.1, 0.8, f, ens, fcont=True)
    print("d lnQ/df", dlnq, dlnq0, "stress", dl, dl0)
    assert abs(dlnq - dlnq0) <= 1e-9 * max(1.0, abs(dlnq0)), (dlnq, dlnq0)
    np.testing.assert_allclose(dl, dl0, rtol=1e-9, atol=1e-12)
