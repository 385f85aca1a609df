"""The device watchdog: every wait of the persistent solver is bounded by
agd_launch.timeout_ns, after which the launch gives up with
AGD_STATUS_WATCHDOG in the statistics (the reference reports a solve that
does not finish as non-convergence, _solvers.py:53-57, _Kernel.py:363-366).

The test makes the limit run out on purpose: a Riemann2 512^2 solve whose
workers may wait 1 microsecond for the next queue entry, far less than an
epoch lasts.  The waits end with the error status, the kernel exits, the
stream stays usable, and the next solve with the default limit on the same
stream and workspace converges to the same values as a fresh one.
"""
import numpy as np
import pytest
import torch

from conftest import make_dictin

pytestmark = pytest.mark.gpu


def _interfaces(n=512, count=2):
    import bench
    from adaptivegriddiscretizations_b200.Eikonal.HFM_CUDA import Interface
    metrics, seeds = bench.make_fields(n, count, 77)
    itfs = []
    for m, s in zip(metrics, seeds):
        case = dict(model="Riemann2", dims=np.array([n, n], np.float32), gridScales=np.full(2, 1.0 / n, np.float32),
                    origin=np.zeros(2, np.float32), metric=m, seeds=s)
        it = Interface(make_dictin(case, extra={"exportValues": True}))
        it.SetKernelTraits()
        it.SetGeometry()
        it.SetArgs()
        itfs.append(it)
    return itfs


def test_watchdog_short_limit_returns_status():
    from adaptivegriddiscretizations_b200 import _lib
    from adaptivegriddiscretizations_b200.Eikonal.HFM_CUDA import BatchPlan
    itfs = _interfaces()
    short = BatchPlan(itfs, launch=_lib.AgdLaunch(ctas=0, warps_per_cta=4, timeout_ns=1000))
    short.run()
    torch.cuda.synchronize()  # the kernel exits: every wait gave up
    niter, status, visits = short.read_stats()
    assert (status & _lib.AGD_STATUS_WATCHDOG).all(), status
    with pytest.raises(_lib.AgdError):
        short.finish()
    # the same stream and workspace, default limit: the solve converges
    inf = float("inf")
    for it in itfs:
        it.values_t.fill_(inf)
    short.launch = None
    short.run()
    torch.cuda.synchronize()
    niter, status, visits = short.read_stats()
    assert not status.any() and (niter > 10).all()
    again = [it.squeeze(it.values_t).cpu().numpy() for it in itfs]
    for it in itfs:
        it.values_t.fill_(inf)
    fresh = BatchPlan(itfs)
    fresh.run()
    torch.cuda.synchronize()
    assert not fresh.read_stats()[1].any()
    for a, it in zip(again, itfs):
        b = it.squeeze(it.values_t).cpu().numpy()
        fin = np.isfinite(b)
        assert np.array_equal(fin, np.isfinite(a))
        assert (np.abs(a[fin] - b[fin]) / np.abs(b[fin]).clip(1e-30)).max() < 1e-4
