"""Parity criteria for solved values.

The scheme's discrete solution is the fixed point of its update; the float64
oracle run with tolerances of 1e-14 gives it.  A float32 solve stops when no
visit changes a value by more than atol + rtol*|u| (the reference's stopping
test), so where it stops depends on the visiting order: the reference's own
float32 run of a seeded 192^2 or 512^2 Riemann2 case sits up to 1.3e-5
relative from the discrete solution.  Hence:

  * with tight tolerances (atol = rtol = 1e-8) a solve must reach the discrete
    solution to float32 rounding: 2e-6 relative everywhere;
  * at the default tolerances, every point within 4 stopping tolerances
    (4 * (atol + rtol * |u|)) of the discrete solution, and 99.9 % of the points
    within 1e-5 relative;
  * against the golden fixtures made by the reference's own kernels on small
    cases, 1e-5 relative everywhere (tests compare with `rel_err`).
"""
import numpy as np

from oracle import oracle as O

REL = 1e-5
TIGHT = {"atol": 1e-8, "rtol": 1e-8}
TIGHT_REL = 2e-6


def rel_err(a, b):
    """Max relative error of a against b; the finite masks must agree."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    fin = np.isfinite(b)
    assert np.array_equal(fin, np.isfinite(a)), "finite masks differ"
    return (np.abs(a[fin] - b[fin]) / np.maximum(np.abs(b[fin]), 1e-30)).max()


def discrete_solution(case, nthreads=8):
    """The scheme's discrete solution: float64 oracle run to 1e-14."""
    return O.run(dict(case, atol=1e-14, rtol=1e-14), np.float64, nthreads=nthreads)["values"]


def default_tolerances(case):
    pr = O.prepare(case)
    return pr.atol, pr.rtol


def assert_near_discrete(v, case, exact=None, ntol=4.0, rel=REL):
    """Values of a solve at the case's stopping tolerances against the discrete
    solution: within ntol stopping tolerances everywhere, 99.9 % of the points
    within rel relative."""
    exact = discrete_solution(case) if exact is None else exact
    v, exact = np.asarray(v, np.float64), np.asarray(exact, np.float64)
    fin = np.isfinite(exact)
    assert np.array_equal(fin, np.isfinite(v)), "finite masks differ"
    atol, rtol = default_tolerances(case)
    err = np.abs(v[fin] - exact[fin])
    bound = ntol * (atol + rtol * np.abs(exact[fin]))
    worst = np.argmax(err / bound)
    assert (err <= bound).all(), f"{err[worst]:.3g} > {bound[worst]:.3g} at u = {exact[fin][worst]:.4g}"
    q = np.quantile(err / np.maximum(np.abs(exact[fin]), 1e-30), 0.999)
    assert q <= rel, f"99.9% quantile of the relative error {q:.3g}"
