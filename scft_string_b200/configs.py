"""Seeded synthetic inputs for the benchmark workloads and the parity cases.

Every workload is a reference ``input.dat`` (scft.cu:80-251 keys) plus one
``win<ii>`` file per replica holding W- and W+ in grid order
r = z + m2*(y + m1*x) (scft.cu:462-464, 1057-1064).  Fields:

* single replica: W- = amp*chiN*cos(2*pi*c/D) along ``axis`` plus Gaussian
  noise sigma*chiN drawn with ``numpy.random.default_rng(seed)``;
* string: replica 0 is the noiseless cosine, the last replica is Gaussian
  noise sigma*chiN (``default_rng(seed)``) and replica ii in between is the
  linear interpolation plus noise 0.5*sigma*chiN (``default_rng(seed+ii)``);
* W+ = 0.
"""
from __future__ import annotations

import numpy as np

# The string workload the headline metric is quoted on: 16 replicas, 64^3,
# N=128, chiN=14, f=0.45, phidb=0.85, D=5, fixed ends.  `ens` is not given for
# it, so the reference default ens=2 (scft.cu:37) applies.
STRING_64 = dict(name="string16_64cubed_N128", chi=14.0, f=0.45, ens=2, phidb=0.85, N=128,
                 alpha=0.1, m=(64, 64, 64), D=(5.0, 5.0, 5.0), fix=(1, 1), dostring=1, strn=16,
                 amp=0.6, sigma=0.02, axis=2, seed=1)

# Plain single-replica canonical blend: 32^3, N=100, chiN=15, f=0.5, phidb=0.8.
PLAIN_32 = dict(name="plain_32cubed_N100", chi=15.0, f=0.5, ens=1, phidb=0.8, N=100, alpha=0.1,
                m=(32, 32, 32), D=(4.0, 4.0, 4.0), fix=(0, 0), dostring=0, strn=1, amp=0.5,
                sigma=0.05, axis=0, seed=0)


def input_dat(c: dict) -> str:
    """The reference parameter file for workload ``c``."""
    return (
        f"chi = {c['chi']!r}\t# xN\n"
        f"f = {c['f']!r}\n"
        f"ens = {c['ens']}\n"
        f"phidb = {c['phidb']!r}\n"
        f"alpha = {c.get('alpha', 0.1)!r}\n"
        f"N = {c['N']}\n"
        f"m = {c['m'][0]} {c['m'][1]} {c['m'][2]}\n"
        f"D = {c['D'][0]!r} {c['D'][1]!r} {c['D'][2]!r}\n"
        f"fix = {c['fix'][0]} {c['fix'][1]}\n"
        f"readwin = 1\n"
        f"justFE = {c.get('justFE', 0)}\n"
        f"dostring = {c['dostring']}\n"
    )


def fields(c: dict):
    """(W-, W+) for every replica, each of shape (strn, M), float64."""
    m = tuple(c["m"])
    M = int(np.prod(m))
    strn = int(c["strn"])
    ax = int(c["axis"])
    chi = float(c["chi"])
    coord = np.arange(m[ax]) * c["D"][ax] / m[ax]
    shape = [1, 1, 1]
    shape[ax] = m[ax]
    lam = c["amp"] * chi * np.cos(2 * np.pi * coord / c["D"][ax]).reshape(shape)
    lam = np.broadcast_to(lam, m).reshape(-1)
    wm = np.zeros((strn, M))
    if strn == 1:
        wm[0] = lam + np.random.default_rng(c["seed"]).normal(0.0, c["sigma"] * chi, M)
    else:
        end1 = np.random.default_rng(c["seed"]).normal(0.0, c["sigma"] * chi, M)
        for ii in range(strn):
            t = ii / (strn - 1)
            wm[ii] = (1 - t) * lam + t * end1
            if 0 < ii < strn - 1:
                wm[ii] += np.random.default_rng(c["seed"] + ii).normal(0.0, 0.5 * c["sigma"] * chi, M)
    return wm, np.zeros((strn, M))


def win_text(wm_row, wp_row) -> str:
    """A ``win`` file with full double precision (read back exactly by
    ``fscanf("%lf %lf")`` in the reference, scft.cu:1062)."""
    return "".join(f"{a:.17g} {b:.17g}\n" for a, b in zip(wm_row, wp_row))


def uneven_batch(seed: int = 5):
    """The 24 independent solves of the uneven-batch workload: 8 at 48^3, 10
    at 64^3 and 6 at 96^3 (D = m/16), with N drawn from {64, 96, 128, 192,
    256}, chiN from U[12, 25], f from U[0.3, 0.5] and phidb from U[0.6, 1.0]
    by default_rng(seed) in that order per solve, and W- = Gaussian noise
    0.1*chiN from default_rng([seed, j]).  ens = 2 (the reference default):
    in the canonical ensemble alpha*N = 6.4 ... 25.6 is never an integer and
    the W+ relaxation cannot converge (see the notes on Nh)."""
    rng = np.random.default_rng(seed)
    grids = [48] * 8 + [64] * 10 + [96] * 6
    out = []
    for j, mm in enumerate(grids):
        N = int(rng.choice([64, 96, 128, 192, 256]))
        chi = float(rng.uniform(12, 25))
        f = float(rng.uniform(0.3, 0.5))
        phidb = float(rng.uniform(0.6, 1.0))
        out.append(dict(name=f"solve{j}_{mm}cubed_N{N}", chi=chi, f=f, ens=2, phidb=phidb, N=N, alpha=0.1,
                        m=(mm, mm, mm), D=(mm / 16.0,) * 3, fix=(0, 0), dostring=0, strn=1,
                        noise_seed=[seed, j]))
    return out


def noise_fields(c: dict):
    """W- = N(0, 0.1*chiN) from default_rng(c['noise_seed']), W+ = 0."""
    M = int(np.prod(c["m"]))
    wm = np.random.default_rng(c["noise_seed"]).normal(0.0, 0.1 * c["chi"], M)
    return wm, np.zeros(M)


# Mixed-precision scaling: 128^3, N=200, 8 independent replicas, grand canonical
# with fugacity 1.0, gyroid start with per-replica noise (seed 3 + ii).
MIXED_128 = dict(name="mixed8_128cubed_N200", chi=20.0, f=0.35, ens=2, phidb=1.0, N=200, alpha=0.1,
                 m=(128, 128, 128), D=(6.4, 6.4, 6.4), fix=(0, 0), dostring=0, strn=8, seed=3)

# Adjoint check: 64x64x96, Lx = Ly = 4.2, Lz = 6.3, N=160, canonical (alpha N = 16,
# n1 = 64, n2 = 96 all even), hexagonal start with noise (seed 4).
ADJOINT_96 = dict(name="adjoint_64x64x96_N160", chi=16.0, f=0.4, ens=1, phidb=0.9, N=160, alpha=0.1,
                  m=(64, 64, 96), D=(4.2, 4.2, 6.3), fix=(0, 0), dostring=0, strn=1, seed=4)


def gyroid_fields(c: dict):
    """W- = 0.4 chiN (sin X cos Y + sin Y cos Z + sin Z cos X) with X = 2 pi x / D,
    plus noise 0.03 chiN from default_rng(seed + ii) per replica; W+ = 0."""
    m, D = c["m"], c["D"]
    ax = [2 * np.pi * np.arange(m[i]) * (D[i] / m[i]) / D[i] for i in range(3)]
    X, Y, Z = np.meshgrid(*ax, indexing="ij")
    base = (0.4 * c["chi"] * (np.sin(X) * np.cos(Y) + np.sin(Y) * np.cos(Z) + np.sin(Z) * np.cos(X))).ravel()
    M = base.size
    wm = np.stack([base + np.random.default_rng(c["seed"] + ii).normal(0, 0.03 * c["chi"], M)
                   for ii in range(c["strn"])])
    return wm, np.zeros_like(wm)


def hex_fields(c: dict):
    """W- = 0.5 chiN sum_j cos(G_j . r), three in-plane wave vectors at 120 degrees
    with |G| = 2 pi / Lx, evaluated on the (square) grid, plus noise 0.02 chiN
    (default_rng(seed)); W+ = 0."""
    m, D = c["m"], c["D"]
    x = [np.arange(m[i]) * D[i] / m[i] for i in range(3)]
    X, Y, _ = np.meshgrid(*x, indexing="ij")
    g = 2 * np.pi / D[0]
    w = np.zeros(m)
    for j in range(3):
        a = 2 * np.pi * j / 3
        w += np.cos(g * (np.cos(a) * X + np.sin(a) * Y))
    wm = 0.5 * c["chi"] * w.ravel() + np.random.default_rng(c["seed"]).normal(0, 0.02 * c["chi"], w.size)
    return wm[None, :], np.zeros((1, w.size))


def lamellar_fields(c: dict):
    """W- = 0.4 chiN cos(2 pi z / Lz) (one period along axis 2) plus noise
    0.02 chiN (default_rng(seed)); W+ = 0."""
    m, D = c["m"], c["D"]
    z = np.arange(m[2]) * D[2] / m[2]
    w = np.broadcast_to(0.4 * c["chi"] * np.cos(2 * np.pi * z / D[2]), tuple(m)).ravel()
    wm = w + np.random.default_rng(c["seed"]).normal(0, 0.02 * c["chi"], w.size)
    return wm[None, :], np.zeros((1, w.size))
