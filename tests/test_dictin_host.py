"""Host copies of small dictIn fields (no device access: mode 'gpu_transfer')."""
import numpy as np
import torch

from adaptivegriddiscretizations_b200.Eikonal import dictIn


def test_small_fields_answer_from_host_copy():
    d = dictIn({"mode": "gpu_transfer", "model": "Riemann2", "seeds": [[0.5, 0.25]]})
    d.SetRect([[0, 1], [0, 2]], dimx=10)
    assert d.shape == (10, 20)
    assert np.allclose(d.gridScales, [0.1, 0.1])
    assert np.allclose(d.host("seeds"), [[0.5, 0.25]])
    bottom, top = d.corners
    assert np.allclose(bottom, [0, 0]) and np.allclose(top, [1, 2])


def test_host_copy_follows_reassignment_and_deletion():
    d = dictIn({"mode": "gpu_transfer", "dims": [4, 5]})
    assert d.shape == (4, 5)
    d["dims"] = np.array([6, 7])
    assert d.shape == (6, 7)
    d["seed"] = [0.5, 0.5]
    assert d.host("seeds").shape == (1, 2)
    del d["seed"]
    assert "seeds" not in d and "seeds" not in d._shadow
    e = d.copy()
    assert e.shape == (6, 7)


def test_large_fields_keep_no_host_copy():
    d = dictIn({"mode": "gpu_transfer", "cost": np.ones((100, 100), np.float32)})
    assert "cost" not in d._shadow
    assert d.host("cost").shape == (100, 100)
    t = torch.zeros(3)
    d["origin"] = t
    assert np.allclose(d.host("origin"), 0)
