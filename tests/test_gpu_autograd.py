"""torch.autograd wrappers of the adjoint: torch.autograd.gradcheck compares
their backward (the adjoint, full store and checkpointed) with central finite
differences of the forward (FP64)."""
import numpy as np
import pytest
import torch

import scft_string_b200 as S
from scft_string_b200.autograd import LnQOfBox, SaddleFreeEnergy

pytestmark = pytest.mark.gpu


def _fields(m, D, seed):
    rng = np.random.default_rng(seed)
    x = [np.arange(m[i]) * D[i] / m[i] for i in range(3)]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    wm = 3.0 * (np.cos(2 * np.pi * X / D[0]) + 0.5 * np.sin(2 * np.pi * Y / D[1]) * np.cos(2 * np.pi * Z / D[2]))
    wm += 0.2 * rng.normal(size=m)
    wp = 0.3 * rng.normal(size=m)
    return wm.ravel(), wp.ravel()


@pytest.mark.parametrize("K", [0, 3])
def test_lnq_of_box_gradcheck(built_lib, K):
    m, D, N = (8, 12, 10), (2.0, 3.0, 2.5), 20
    ctx = S.Context(m, D, N, chi=12, f=0.45, phidb=0.8, ens=1, alpha=0.1, strn=1, dostring=0)
    wm, wp = _fields(m, D, 3)
    ctx.set_fields(0, wm, wp)
    L = torch.tensor(D, dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(lambda x: LnQOfBox.apply(x, ctx, 0, K), (L,), eps=1e-4, atol=1e-6,
                                    rtol=1e-5)


def test_saddle_free_energy_gradcheck(built_lib):
    """dF/dL_z and dF/dchiN at a lamellar saddle point (re-converged to RMS
    1e-10 at every finite-difference point)."""
    m, N = (8, 8, 24), 20
    D0, chi0 = np.array([2.0, 2.0, 4.6]), 14.0
    z = np.arange(m[2]) * D0[2] / m[2]
    wm = np.broadcast_to(0.4 * chi0 * np.cos(2 * np.pi * z / D0[2]), m).ravel()
    w0 = np.concatenate([wm, np.zeros_like(wm)])

    def make(D, chi):
        return S.Context(m, D, N, chi=chi, f=0.5, phidb=0.8, ens=1, alpha=0.1, strn=1, dostring=0)

    p = torch.tensor([*D0, chi0], dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(lambda x: SaddleFreeEnergy.apply(x, make, w0), (p,), eps=1e-3,
                                    atol=2e-6, rtol=1e-5)
