"""CSF input (csf / csfmap sections of a .det file) expanded to the
determinant coefficients of every state as read_csfmap_file does; a
determinant shared by two CSFs accumulates both contributions."""
import numpy as np
import pytest

from champ_b200 import champ_io

DET = """determinants 4 1
 1.0 0.0 0.0 0.0
 1 2 1 2
 1 3 1 2
 1 2 1 3
 1 3 1 3
end
csf 3 2
 0.9 0.3 -0.2
 0.1 -0.7 0.5
end
csfmap 3 4 5
1
 1 1.0
2
 2 0.70710678118654752
 3 -0.70710678118654752
2
 4 1.0
 3 0.5
end
"""


def test_expand_csf(tmp_path):
    p = tmp_path / "x.det"
    p.write_text(DET)
    cst, iworbd = champ_io.read_det_states(str(p), 4)
    assert iworbd.shape == (4, 4)
    r = 0.70710678118654752
    want = np.array([[0.9, 0.3 * r, -0.3 * r + -0.2 * 0.5, -0.2],
                     [0.1, -0.7 * r, 0.7 * r + 0.5 * 0.5, 0.5]])
    assert np.allclose(cst, want, rtol=0, atol=1e-15)


def test_no_csf_section_is_one_state(tmp_path):
    p = tmp_path / "y.det"
    p.write_text(DET.split("csf")[0])
    cst, _ = champ_io.read_det_states(str(p), 4)
    assert cst.shape == (1, 4) and cst[0, 0] == 1.0


def test_bad_map(tmp_path):
    with pytest.raises(ValueError):
        champ_io.expand_csf([[1.0, 2.0]], [[(1, 1.0)], [(5, 1.0)]], 4)
