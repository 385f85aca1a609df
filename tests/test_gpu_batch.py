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
