"""Batched solves: several dictIn of mixed models in one persistent launch
(RunBatch), and batches submitted on two CUDA streams (SubmitBatch) so that one
batch is prepared while the other solves.  Each instance must give the values
of the reference's own kernels for that instance (1e-5 relative)."""
import numpy as np
import pytest
import torch

from conftest import load_case

pytestmark = pytest.mark.gpu
REL = 1e-5


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    fin = np.isfinite(b)
    assert np.array_equal(fin, np.isfinite(a)), "finite masks differ"
    return (np.abs(a[fin] - b[fin]) / np.maximum(np.abs(b[fin]), 1e-30)).max()


def _dictin(case, pinned=False):
    """dictIn of a golden case; with pinned, its arrays are page-locked host tensors."""
    from adaptivegriddiscretizations_b200 import Eikonal
    d = {"mode": "gpu", "verbosity": 0, "exportValues": True}
    for k, v in case.items():
        if pinned and isinstance(v, np.ndarray) and v.dtype == np.float32:
            v = torch.from_numpy(v).pin_memory()
        d[k] = v
    return Eikonal.dictIn(d)


def _inputs(names):
    cases, refs = [], []
    for name in names:
        case, ref = load_case(name)
        cases.append({k: v for k, v in case.items() if k not in ("tips", "sensitivity")})
        refs.append(ref["values"])
    return cases, refs


@pytest.mark.parametrize("names", [["iso2", "riem2", "riem2_aniso", "riem2_mp", "riem2"], ["iso3", "riem3", "iso3"]],
                         ids=["2d_mixed", "3d_mixed"])
def test_run_batch_mixed_models(names):
    from adaptivegriddiscretizations_b200 import Eikonal
    cases, refs = _inputs(names)
    outs = Eikonal.RunBatch([_dictin(c) for c in cases])
    assert len(outs) == len(cases)
    for out, ref in zip(outs, refs):
        assert _rel(out["values"].cpu().numpy(), ref) < REL
        assert out["stats"]["eikonal"]["niter_o"] > 0


def test_submit_batch_two_streams():
    from adaptivegriddiscretizations_b200 import Eikonal
    names_a, names_b = ["riem2", "iso2", "riem2_aniso"], ["riem2_aniso", "riem2"]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    jobs, refs = [], []
    for names, stream in zip((names_a, names_b, names_a), (streams[0], streams[1], streams[0])):
        cases, ref = _inputs(names)
        with torch.cuda.stream(stream):
            # host inputs in page-locked memory, uploaded without blocking the host
            jobs.append(Eikonal.SubmitBatch([_dictin(c, pinned=True) for c in cases]))
        refs.append(ref)
    for job, ref in zip(reversed(jobs), reversed(refs)):  # collect out of submission order
        outs = job.result()
        assert job.done()
        with torch.cuda.stream(job.stream):
            vals = [o["values"].cpu().numpy() for o in outs]
        for v, r in zip(vals, ref):
            assert _rel(v, r) < REL
        assert job.result() is outs


def _riemann2_cases(n, count, seed):
    import bench
    metrics, seeds = bench.make_fields(n, count, seed, sigma=4.0)
    return [dict(model="Riemann2", dims=np.array([n, n], np.float32), gridScales=np.full(2, 1.0 / n, np.float32),
                 origin=np.zeros(2, np.float32), metric=m, seeds=s) for m, s in zip(metrics, seeds)]


@pytest.mark.parametrize("pinned", [False, True])
def test_submit_batch_uniform_path(pinned):
    """dictIn that differ only in their data go through the batched preparation
    (one agd_prep_batch launch): values, iteration counts and the key
    bookkeeping per instance are those of RunGPU on each dictIn."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from adaptivegriddiscretizations_b200 import Eikonal
    from adaptivegriddiscretizations_b200.Eikonal.HFM_CUDA import UniformBatchJob
    from parity import assert_near_discrete
    cases = _riemann2_cases(96, 6, 17)
    for rep in range(2):  # the second batch reuses the cached solver
        job = Eikonal.SubmitBatch([_dictin(c, pinned=pinned) for c in cases])
        assert isinstance(job, UniformBatchJob)
        outs = job.result()
        for c, o in zip(cases, outs):
            ref = _dictin(c).Run()
            v = o["values"].cpu().numpy()
            assert_near_discrete(v, c)
            assert _rel(v, ref["values"].cpu().numpy()) < 1e-4
            assert o["stats"]["eikonal"]["niter_o"] > 0
            for k in ("used", "default", "help"):
                assert list(o["keys"][k]) == list(ref["keys"][k]), k
    # a batch whose options differ goes instance by instance
    mixed = [_dictin(c) for c in cases[:2]]
    mixed[1]["nitermax_o"] = 500
    assert not isinstance(Eikonal.SubmitBatch(mixed), UniformBatchJob)


def test_traits_auto(tmp_path, monkeypatch):
    """traits='auto': the autotuner's trial solves pick a tile shape and local
    iteration count (cached for the next call); the values meet the parity
    criteria like those of any traits."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from parity import assert_near_discrete
    monkeypatch.setenv("AGD_AUTOTUNE_CACHE", str(tmp_path / "autotune.json"))
    case = _riemann2_cases(128, 1, 23)[0]
    h = _dictin(dict(case, traits="auto"))
    out = h.Run()
    at = out["stats"]["autotune"]
    assert not at["cached"] and tuple(at["traits"]["shape_i"]) in {(8, 8), (16, 16)}
    assert_near_discrete(out["values"].cpu().numpy(), case)
    out2 = _dictin(dict(case, traits="auto")).Run()
    assert out2["stats"]["autotune"]["cached"] and out2["stats"]["autotune"]["traits"] == at["traits"]
