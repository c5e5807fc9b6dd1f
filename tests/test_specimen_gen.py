"""Host specimen generator (msf_amorphous_positions): count, box, periodic
minimum separation, determinism per seed."""
import numpy as np
import pytest
from scipy.spatial import cKDTree

import msf


@pytest.mark.parametrize("n,box", [(780, (25.0, 25.0, 25.0)), (5000, (50.0, 50.0, 40.0)),
                                   (40, (30.0, 30.0, 4.0))])
def test_positions_respect_box_and_separation(n, box):
    q = msf.amorphous_positions(n, box, 2.2, seed=3)
    assert q.shape == (n, 3)
    assert (q >= 0).all() and (q < np.array(box)).all()
    d, _ = cKDTree(q, boxsize=box).query(q, k=2)
    assert d[:, 1].min() >= 2.2


def test_seeded():
    a = msf.amorphous_positions(500, (25.0, 25.0, 25.0), 2.2, seed=9)
    b = msf.amorphous_positions(500, (25.0, 25.0, 25.0), 2.2, seed=9)
    c = msf.amorphous_positions(500, (25.0, 25.0, 25.0), 2.2, seed=10)
    assert np.array_equal(a, b) and not np.array_equal(a, c)


def test_overfull_box_fails():
    with pytest.raises(msf.MsfError):
        msf.amorphous_positions(2000, (10.0, 10.0, 10.0), 2.2, seed=1, max_proposals=100000)
