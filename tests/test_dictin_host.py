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


def test_uniform_batch_option_comparison():
    """SubmitBatch's check that dictIn differ only in their data compares the
    scalar and short-list options directly; it must agree with the comparison
    of their host forms (_option) wherever it answers."""
    from adaptivegriddiscretizations_b200.Eikonal.HFM_CUDA import _option, _same_option

    class Store:
        def __init__(self, v):
            self.v = v

        def raw(self, k):
            return self.v

        def host(self, k):
            return np.asarray(self.v)

    vals = [1, 1.0, 0.5, True, False, None, "Riemann2", "gpu", [512, 512], [512.0, 512.0], (0.0, 0.0), [0.0, 0.0],
            [np.float32(1), 2], [1, 2, 3], [float("nan")], float("nan"), -0.0, 0.0, [-0.0, 0.0], {"a": 1},
            np.array([1.0, 2.0]), np.array([1.0, 2.0], np.float32), np.array([512, 512]), np.array([-0.0, 0.0]),
            np.array([0.0, 0.0]), np.array([[1.0, 2.0]])]
    answered = 0
    for a in vals:
        for b in vals:
            r = _same_option(a, b)
            if r is None:
                continue
            answered += 1
            assert r == (_option(Store(a), "k") == _option(Store(b), "k")), (a, b)
    assert answered > 200
    assert _same_option([0.0, 1.0], [0.0, 1.0]) and not _same_option([0.0, 1.0], [0.0, 2.0])
    assert _same_option(np.zeros(65), np.zeros(65)) is None  # larger arrays: compared by _option
    assert _same_option(torch.zeros(2), torch.zeros(2)) is None
