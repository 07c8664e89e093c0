"""The reference-shaped API called in a loop: operators built from the same
device arrays are reused, in-place torch updates of those arrays are seen,
and a wrong mask is still refused."""
import numpy as np
import pytest
import torch

from oracle import dda_oracle as O

pytestmark = pytest.mark.gpu


def _problem(n=8, m=1.5 + 0.05j, seed=4):
    rng = np.random.default_rng(seed)
    k = 2 * np.pi / 0.5
    d = 0.5 / (abs(m) * k)
    occ = O.sphere_lattice(n, n / 2.0)
    alpha = np.where(occ, O.calculate_alpha(m, d, k, method="RR"), 0)
    x = rng.standard_normal((n, n, n, 3)) + 1j * rng.standard_normal((n, n, n, 3))
    return k, d, alpha, x


def test_interaction_mult_reuses_operator_and_sees_in_place_updates():
    import precondda_b200 as P
    from precondda_b200 import reference_api as R
    n = 8
    k, d, alpha, x = _problem(n)
    R.clear_operator_cache()
    inv_alpha, mask, G, _ = P.prepare_interaction_matrices((n, n, n), k, 1, 0, 0, 0, alpha, d)
    xt = torch.as_tensor(x, device="cuda").to(torch.complex64)
    y1 = P.interaction_mult(xt, None, G, inv_alpha, mask, None, n, n, n)
    op1 = R._op_from_reference(G, inv_alpha, n, n, n, torch.complex64, mask)
    y2 = P.interaction_mult(xt, None, G, inv_alpha, mask, None, n, n, n)
    assert R._op_from_reference(G, inv_alpha, n, n, n, torch.complex64, mask) is op1
    assert len(R._OP_CACHE) == 1
    assert torch.equal(y1, y2)
    ia_o, mask_o, G_o, _ = O.prepare_interaction_matrices(alpha, k, d)
    ref = O.interaction_mult(x, G_o, ia_o, mask_o).reshape(-1)
    assert np.abs(y1.cpu().numpy() - ref).max() / np.abs(ref).max() < 2e-5
    # an in-place update of the octant (torch bumps its version): new operator
    G.mul_(2.0)
    y3 = P.interaction_mult(xt, None, G, inv_alpha, mask, None, n, n, n)
    assert R._op_from_reference(G, inv_alpha, n, n, n, torch.complex64, mask) is not op1
    conv = (inv_alpha.reshape(n, n, n, 1) * xt - y1.reshape(n, n, n, 3))     # mask * conv(x)
    assert torch.allclose(y3.reshape(n, n, n, 3), inv_alpha.reshape(n, n, n, 1) * xt - 2 * conv,
                          rtol=0, atol=1e-4 * float(y1.abs().max()))
    with pytest.raises(ValueError):
        P.interaction_mult(xt, None, G, inv_alpha, ~mask, None, n, n, n)
    R.clear_operator_cache()
