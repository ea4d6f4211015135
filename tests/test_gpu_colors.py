"""GPU colour statistics (bd_color_statistics, colors.cu) against the
oracle's restatement, which is itself pinned to the reference's own
calculate_color on the CPU."""
import numpy as np
import pytest

from bd_aging_b200 import configs as CF
from bd_aging_b200 import lib as B
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SB, SS = float(CF.SIGMA_BIG), float(CF.SIGMA_SML)


@pytest.mark.parametrize("nb,ns,phi,jit", [(800, 800, 0.55, 0.15), (500, 1500, 0.5, 0.25), (60, 30, 0.3, 0.3)])
def test_colors_match_oracle(nb, ns, phi, jit):
    import torch
    side = float(np.float32(CF.side_from_phi(nb, ns, phi)))
    pos = CF.lattice_config(nb, ns, side, 5, jitter=jit)
    pars = B.setup_params(side, nb, ns, SB, SS)
    rb = torch.tensor(pos[:nb], device="cuda")
    rs = torch.tensor(pos[nb:], device="cuda")
    ids = torch.zeros(nb, dtype=torch.int32, device="cuda")
    counts = B.color_statistics(rb, rs, pars, ids)
    ids_o, counts_o = O.colors(pos[:nb], pos[nb:], side, SB, SS)
    np.testing.assert_array_equal(ids.cpu().numpy(), ids_o)
    np.testing.assert_array_equal(counts, counts_o)
    assert counts.sum() == nb
