"""The oracle's LSMR restatement (ext/KrylovExt.jl:97-132 with Fong & Saunders' recurrences), pinned on CPU: against
numpy's lstsq of the same damped problem on badly scaled block-structured matrices (the reference's LP1 test,
test/dampedlinearsolve_qrelimination.jl:235-247, at rtol 1e-6), a consistent system stopping on test 1, and the
reference's NotPositiveDefinite cases (rank deficient undamped, a block of D not positive definite, a non-finite r~)
and an itmax stop."""
import numpy as np
import pytest

import oracle as orc


def problem(seed, m=60, r_dims=(6, 6, 3, 6)):
    rng = np.random.default_rng(seed)
    nr = sum(r_dims)
    J = rng.standard_normal((m, nr)) * 10.0 ** rng.uniform(-3, 3, nr)
    return J, rng.standard_normal(m), np.array(r_dims), 0.5 + rng.random(nr)


def direct(J, r, lam, s_r):
    nr = J.shape[1]
    d = np.sqrt(lam * (np.ones(nr) if s_r is None else s_r))
    return np.linalg.lstsq(np.vstack([J, np.diag(d)]), np.concatenate([r, np.zeros(nr)]), rcond=None)[0]


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("lam,scaled", [(0.0, False), (1e-8, False), (1e-4, False), (1e-8, True), (1e-4, True)])
def test_equals_the_direct_solution(seed, lam, scaled):
    J, r, rd, s_r = problem(seed)
    s = s_r if scaled else None
    x, status, it, istop = orc.lsmr_reduced(J, r, rd, lam, s, atol=1e-12, btol=1e-12, conlim=1e14)
    ref = direct(J, r, lam, s)
    assert status == "ok" and istop in (1, 2, 4, 5) and 0 < it <= J.shape[0] + J.shape[1]
    assert np.linalg.norm(x - ref) <= 1e-6 * np.linalg.norm(ref)


def test_consistent_system_stops_on_the_residual():
    J, _, rd, _ = problem(4)
    xt = np.random.default_rng(5).standard_normal(J.shape[1])
    x, status, it, istop = orc.lsmr_reduced(J, J @ xt, rd, 0.0, atol=1e-10, btol=1e-10, conlim=1e14)
    assert status == "ok" and istop == 1
    assert np.linalg.norm(x - xt) <= 1e-6 * np.linalg.norm(xt)


def test_not_positive_definite_and_itmax():
    J, r, rd, _ = problem(6)
    assert orc.lsmr_reduced(J[:10], r[:10], rd, 0.0)[1] == "not_pd"            # fewer rows than columns, undamped
    Jz = J.copy()
    Jz[:, :6] = 0.0
    assert orc.lsmr_reduced(Jz, r, rd, 0.0)[1] == "not_pd"                     # a zero block of D
    assert orc.lsmr_reduced(Jz, r, rd, 1e-4, atol=1e-12, btol=1e-12, conlim=1e14)[1] == "ok"
    rn = r.copy()
    rn[3] = np.nan
    assert orc.lsmr_reduced(J, rn, rd, 1e-4)[1] == "not_pd"
    x, status, it, istop = orc.lsmr_reduced(J, r, rd, 1e-4, atol=0.0, btol=0.0, conlim=0.0, itmax=2)
    assert status == "itmax" and istop == 7 and it == 2
    x, status, it, istop = orc.lsmr_reduced(J, r, rd, 1e-4, itmax=0)
    assert status == "itmax" and istop == 7 and it == 0 and not x.any()
