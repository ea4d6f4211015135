"""Colour statistics of the snapshot writer: the oracle's restatement of
colors.cu against the reference's own calculate_color (oracle/_ref), and the
.pov text format."""
import numpy as np
import pytest

from bd_aging_b200 import configs as CF
from bd_aging_b200 import snapshots as SN
from oracle import oracle as O

SB, SS = float(CF.SIGMA_BIG), float(CF.SIGMA_SML)


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("nb,ns,phi,jit", [(300, 300, 0.5, 0.1), (200, 500, 0.58, 0.2), (120, 60, 0.3, 0.3)])
def test_colors_oracle_matches_reference(nb, ns, phi, jit):
    side = float(np.float32(CF.side_from_phi(nb, ns, phi)))
    pos = CF.lattice_config(nb, ns, side, 11, jitter=jit)
    ids, c = O.colors(pos[:nb], pos[nb:], side, SB, SS)
    ids_r, c_r = O.ref_colors(pos[:nb], pos[nb:], O.setup_params(side, nb, ns, SB, SS))
    np.testing.assert_array_equal(ids, ids_r)
    np.testing.assert_array_equal(c, c_r)


def test_pov_text(tmp_path):
    rb = np.array([[1.0, 2.0, 2.0], [3.0, 4.0, 5.0]], np.float32)
    rs = np.array([[1.5, 1.5, 2.0]], np.float32)
    p = tmp_path / "snapshot_1.pov"
    SN.write_pov(str(p), rb, rs, SB, SS, np.array([2, 0]))
    txt = p.read_text()
    assert txt.startswith('#include "colors.inc"\nglobal_settings {')
    assert "sphere{ <   1.000,   2.000,   2.000>,    0.786 pigment {Red} finish { specular 0.5 }}" in txt
    assert "5.000" not in txt  # outside the slab
    assert "sphere{ <   1.500   1.500   2.000>,    0.561 pigment {Yellow}" in txt
    assert SN.color_statistics_line(0.5, [3, 2, 1]) == "0.500000  1  2  3\n"
