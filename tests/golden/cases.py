"""Small seeded problems for the golden fixtures and the parity tests.

Each case is a reference ``input.dat`` plus seeded ``win<ii>`` files built by
``scft_string_b200.configs.fields``; all are small enough for the FP64 oracle
to replay in seconds.  Canonical (ens=1) cases keep n1, n2 and Nh = alpha*N
even: the reference's Simpson weights (density.h:404-422) are biased for odd
counts, and the canonical W+ relaxation only converges when they are not.
"""
from __future__ import annotations

from scft_string_b200.configs import fields, input_dat, win_text  # noqa: F401

CASES = {
    # single replica, canonical blend, plain SCFT (dostring=0)
    "plain_c": dict(chi=15.0, f=0.5, ens=1, phidb=0.8, alpha=0.1, N=20, m=(12, 12, 12),
                    D=(4.0, 4.0, 4.0), fix=(0, 0), dostring=0, strn=1, nsterp=30, amp=0.25,
                    sigma=0.05, axis=0, seed=0),
    # canonical string (n1, n2, Nh even)
    "string_c": dict(chi=14.0, f=0.45, ens=1, phidb=0.85, alpha=0.1, N=40, m=(8, 8, 16),
                     D=(2.5, 2.5, 5.0), fix=(0, 0), dostring=1, strn=3, nsterp=8, amp=0.3,
                     sigma=0.02, axis=2, seed=3),
    # grand canonical string on a mixed-radix grid with odd n1
    "string_mixed": dict(chi=14.0, f=0.45, ens=2, phidb=0.85, alpha=0.1, N=21, m=(12, 10, 8),
                         D=(3.5, 3.0, 2.5), fix=(0, 0), dostring=1, strn=4, nsterp=55, amp=0.3,
                         sigma=0.03, axis=2, seed=1),
    # grand canonical, fixed ends, one missing win file (spring steps, scft.cu:1065-1078)
    "string_gc_fix": dict(chi=12.0, f=0.4, ens=2, phidb=1.0, alpha=0.1, N=20, m=(8, 8, 12),
                          D=(3.0, 3.0, 4.5), fix=(1, 1), dostring=1, strn=5, nsterp=12,
                          amp=0.3, sigma=0.02, axis=2, seed=2, missing=(2,)),
}
