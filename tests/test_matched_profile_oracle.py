"""The matched tight-tolerance profile on the oracle alone (CPU).

The 1e-6 parity tests at the configurations' sizes rest on one premise: under the matched profile
(Newton accepted at CNV 1e-8 / MB 1e-10, every CPR-FGMRES solve refined to a relative residual of
1e-10; tests/_matched.py) the Newton path does not depend on rounding.  Here the oracle is run with
the reference's left-to-right dot products and with two interleaved summation orders: every report
step must take the same Newton iterations, substeps and retries, and the fields must agree far
below the 1e-6 bar.
"""
from _matched import oracle_runs_parallel
from _parity import rel_err


def test_matched_profile_newton_path_is_rounding_independent():
    spec, dt, steps = ("variant", 142), 10.0, 2  # 30 x 22 x 5, 3,300 cells
    runs = oracle_runs_parallel([(spec, dt, steps, True, m) for m in (0, 2, 61)])
    base = runs[0][0]
    for (out, _), order in zip(runs[1:], (2, 61)):
        for s, (st, bhp, newton, sub, rc, ret) in enumerate(out):
            b = base[s]
            assert rc == 0 and b[4] == 0
            assert (newton, sub, ret) == (b[2], b[3], b[5]), (order, s)
            for k in ("pressure", "sat_water"):
                assert rel_err(st[k], b[0][k]) < 1e-10, (order, s, k)
            assert rel_err(bhp, b[1]) < 1e-10
