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
