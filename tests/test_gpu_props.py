"""CUDA propagator, density and spline kernels against the FP64 oracle through
the C ABI (density::props, step::do_step, the spline services)."""
import numpy as np
import pytest

import oracle as O
import scft_string_b200 as S

pytestmark = pytest.mark.gpu

GRIDS = [
    ((8, 8, 8), (4.0, 4.0, 4.0), 20, 0.5, 1),
    ((12, 10, 6), (3.0, 2.5, 2.0), 21, 0.45, 2),
    ((6, 5, 9), (2.0, 2.0, 3.0), 17, 0.3, 1),
    ((16, 12, 20), (4.0, 3.0, 5.0), 24, 0.4, 2),
    ((14, 7, 10), (3.5, 1.75, 2.5), 12, 0.5, 2),
]


def fields(m, seed, amp=1.0):
    rng = np.random.default_rng(seed)
    return rng.normal(0, amp, m).ravel(), rng.normal(0, 0.5 * amp, m).ravel()


@pytest.mark.parametrize("m,D,Ns,f,ens", GRIDS)
def test_do_step_fp64(built_lib, m, D, Ns, f, ens):
    M = int(np.prod(m))
    wm, wp = fields(m, 1)
    ctx = S.Context(m, D, Ns, chi=10, f=f, phidb=0.8, ens=ens, strn=1, dostring=0)
    ctx.set_fields(0, wm, wp)
    od = O.Density(m, D, Ns)
    od.prepare(1.0 / Ns, np.concatenate([wm, wp]))
    rng = np.random.default_rng(2)
    qin = 1.0 + 0.3 * rng.normal(size=2 * M)
    n1 = int(round(Ns * (round(Ns * f) / Ns)))
    for s in [0, n1 - 1, n1, Ns - 1]:
        ref = od.do_step(qin, s, n1, Ns - n1)
        got = ctx.do_step(0, qin, s)
        assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max(), s


@pytest.mark.parametrize("m,D,Ns,f,ens", GRIDS)
def test_props_fp64(built_lib, m, D, Ns, f, ens):
    M = int(np.prod(m))
    wm, wp = fields(m, 3, 2.0)
    alpha, phic = 0.2, 0.8
    od = O.Density(m, D, Ns)
    w0 = np.zeros(6 * M)
    w0[:M], w0[M:2 * M] = wm, wp
    lnQ0, phis0 = od.props(w0, Ns, alpha, phic, f, ens)
    dens = S.Density(m, D, Ns, ens, alpha, phic, f)
    w1 = np.zeros(6 * M)
    w1[:M], w1[M:2 * M] = wm, wp
    lnQ1, phis1 = dens.props(w1, Ns, alpha, phic, f)
    assert abs(lnQ1 - lnQ0) <= 1e-12 * max(1.0, abs(lnQ0))
    assert np.allclose(phis1, phis0, rtol=1e-12, atol=1e-14)
    assert np.abs(w1[2 * M:] - w0[2 * M:]).max() <= 1e-12 * np.abs(w0[2 * M:]).max()
    # propagators
    ctx = dens.ctx
    n1 = int(round(Ns * (round(Ns * f) / Ns)))
    for which, s in [(0, Ns), (1, Ns), (0, n1), (1, 3)]:
        got = ctx.propagator(ctx.strn, which, s)
        ref = od.q(which, s)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("m,D,Ns,f,ens", GRIDS[:3])
def test_props_fp32_close_to_fp64(built_lib, m, D, Ns, f, ens):
    M = int(np.prod(m))
    wm, wp = fields(m, 5, 1.0)
    alpha, phic = 0.2, 0.8
    od = O.Density(m, D, Ns)
    w0 = np.zeros(6 * M)
    w0[:M], w0[M:2 * M] = wm, wp
    lnQ0, phis0 = od.props(w0, Ns, alpha, phic, f, ens)
    dens = S.Density(m, D, Ns, ens, alpha, phic, f, precision="fp32")
    w1 = np.zeros(6 * M)
    w1[:M], w1[M:2 * M] = wm, wp
    lnQ1, phis1 = dens.props(w1, Ns, alpha, phic, f)
    assert abs(lnQ1 - lnQ0) <= 2e-6 * max(1.0, abs(lnQ0))
    assert np.abs(w1[2 * M:3 * M] - w0[2 * M:3 * M]).max() <= 1e-5


def test_spline_services_fp64(built_lib):
    rng = np.random.default_rng(7)
    strn, m = 6, (4, 4, 4)
    M = 64
    ctx = S.Context(m, (2, 2, 2), 10, chi=10, f=0.5, phidb=0.8, ens=2, strn=strn)
    x = np.array([0.0, 0.15, 0.3, 0.52, 0.8, 1.0])
    xref = np.linspace(0, 1, strn)
    Wm = rng.normal(size=(strn, M))
    doiis = np.array([0, 1, 1, 1, 1, 0], np.int32)
    ref = O.spline_derivs(x, Wm, doiis)
    got = ctx.spline_derivs(x, Wm, doiis)
    assert np.allclose(got[doiis == 1], ref[doiis == 1], rtol=1e-13, atol=1e-13)
    ref = O.spline_redist(x, xref, Wm, doiis, 0.37)
    got = ctx.spline_redist(x, xref, Wm, doiis, 0.37)
    assert np.allclose(got, ref, rtol=1e-13, atol=1e-13)


def test_bad_inputs_return_status(built_lib):
    with pytest.raises(S.ScftError) as e:
        S.Context((11, 8, 8), (2, 2, 2), 10, chi=10, f=0.5, phidb=0.8)
    assert e.value.status == 3
    ctx = S.Context((8, 8, 8), (2, 2, 2), 10, chi=10, f=0.5, phidb=0.8)
    with pytest.raises(S.ScftError) as e:
        ctx.props(5)
    assert e.value.status == 3


# grids with compile-time kernel instantiations
FIXED = [(32, 32, 32), (48, 48, 48), (64, 64, 64), (96, 96, 96), (128, 128, 128), (64, 64, 96)]


@pytest.mark.parametrize("m", FIXED)
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
def test_do_step_fixed_shapes(built_lib, m, prec, tol):
    M = int(np.prod(m))
    D = tuple(v / 16 for v in m)
    Ns, f = 16, 0.5
    wm, wp = fields(m, 11, 1.0)
    ctx = S.Context(m, D, Ns, chi=10, f=f, phidb=0.8, ens=2, strn=1, dostring=0, precision=prec)
    ctx.set_fields(0, wm, wp)
    od = O.Density(m, D, Ns)
    od.prepare(1.0 / Ns, np.concatenate([wm, wp]))
    rng = np.random.default_rng(4)
    qin = 1.0 + 0.3 * rng.normal(size=2 * M)
    for s in [0, Ns - 1]:
        ref = od.do_step(qin, s, 8, 8)
        got = ctx.do_step(0, qin, s)
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max(), (m, s)


@pytest.mark.parametrize("persist", ["0", "1"])
def test_register_kernels_64cubed_fp32(built_lib, monkeypatch, persist):
    """The register-resident 64^3 FP32 step kernels (SCFT_REG64=1), with four
    launches per contour step or one persistent launch: one step against the
    FP64 oracle at the FP32 step tolerance, and a props of the same fields
    against the oracle's lnQ and densities."""
    monkeypatch.setenv("SCFT_REG64", "1")
    monkeypatch.setenv("SCFT_NO_PERSIST", "0" if persist == "1" else "1")
    m = (64, 64, 64)
    M = int(np.prod(m))
    D = (4.0, 4.0, 4.0)
    Ns, f = 16, 0.5
    wm, wp = fields(m, 11, 1.0)
    ctx = S.Context(m, D, Ns, chi=10, f=f, phidb=0.8, ens=2, strn=1, dostring=0, precision="fp32")
    ctx.set_fields(0, wm, wp)
    od = O.Density(m, D, Ns)
    od.prepare(1.0 / Ns, np.concatenate([wm, wp]))
    qin = 1.0 + 0.3 * np.random.default_rng(4).normal(size=2 * M)
    for s in [0, 7, 8, Ns - 1]:
        ref = od.do_step(qin, s, 8, 8)
        got = ctx.do_step(0, qin, s)
        assert np.abs(got - ref).max() <= 2e-6 * np.abs(ref).max(), s
    ctx.props(0)
    conc, lnQ, phis = ctx.get_conc(0)
    w0 = np.zeros(6 * M)
    w0[:M], w0[M:2 * M] = wm, wp
    lnQ0, phis0 = O.Density(m, D, Ns).props(w0, Ns, 0.1, 0.8, f, 2)
    assert abs(lnQ - lnQ0) <= 1e-5 * abs(lnQ0)
    assert np.abs(conc - w0[2 * M:]).max() <= 1e-5


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("wide", ["0", "1"])
def test_shuffle_pencil_m0_64(built_lib, monkeypatch, prec, wide):
    """The x pass as octet register transforms with warp-shuffle transposes
    (SCFT_PENCIL_SHUFFLE=1, grids with m0 = 64), at both tile widths: steps
    against the FP64 oracle at the step tolerance of the precision, and a
    props round with one persistent launch per contour step equal bit for bit
    to one with four launches, both against the oracle's lnQ."""
    monkeypatch.setenv("SCFT_PENCIL_SHUFFLE", "1")
    monkeypatch.setenv("SCFT_PENCIL_TILE_WIDE", wide)
    tol = 1e-13 if prec == "fp64" else 2e-6
    Ns, f = 16, 0.5
    for m, D in [((64, 64, 64), (4.0, 4.0, 4.0)), ((64, 64, 96), (4.0, 4.0, 6.0))]:
        M = int(np.prod(m))
        wm, wp = fields(m, 11, 1.0)
        od = O.Density(m, D, Ns)
        od.prepare(1.0 / Ns, np.concatenate([wm, wp]))
        qin = 1.0 + 0.3 * np.random.default_rng(4).normal(size=2 * M)
        res = []
        for persist in ("0", "1"):
            monkeypatch.setenv("SCFT_PERSIST", persist)
            ctx = S.Context(m, D, Ns, chi=10, f=f, phidb=0.8, ens=2, strn=1, dostring=0, precision=prec)
            ctx.set_fields(0, wm, wp)
            if persist == "0":
                for s in [0, 7, 8, Ns - 1]:
                    ref = od.do_step(qin, s, 8, 8)
                    got = ctx.do_step(0, qin, s)
                    assert np.abs(got - ref).max() <= tol * np.abs(ref).max(), (m, s)
            ctx.props(0)
            res.append(ctx.get_conc(0))
        assert np.array_equal(res[0][0], res[1][0]) and res[0][1] == res[1][1], m
        w0 = np.zeros(6 * M)
        w0[:M], w0[M:2 * M] = wm, wp
        lnQ0, _ = O.Density(m, D, Ns).props(w0, Ns, 0.1, 0.8, f, 2)
        assert abs(res[0][1] - lnQ0) <= (1e-12 if prec == "fp64" else 1e-5) * abs(lnQ0), m
