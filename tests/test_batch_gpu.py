"""Batched S2CN2 on the GPU: instances of uneven grid and velocity-set sizes advanced together.

Each instance of a batch must follow exactly the single-instance S2CN2 step: the same kernels on the
same data, so the comparison is bitwise.  One instance on a generated 24^2 table is also checked
against the oracle (1e-11).
"""
import numpy as np
import pytest

from ugks2d_high_order_b200.case import CouetteCase, batched_cases, velocity_table

HO_TOL = 1e-11


def _mixed(n=6):
    """n cases of the batched distribution at small grids, cycling the three velocity sets."""
    out = []
    for k, (c, _) in enumerate(batched_cases(n)):
        ny = (32, 32, 64)[k % 3]
        nva = (24, 32, 48)[k % 3]
        out.append((c.with_(ny=ny, dy=1.0 / ny), nva))
    return out


@pytest.mark.gpu
def test_batch_matches_single_instances_bitwise():
    from ugks2d_high_order_b200.batch import Batch
    from ugks2d_high_order_b200.solver import Solver
    cases = _mixed(6)
    tables = {n: velocity_table(n) for n in (24, 32, 48)}
    b = Batch([(c, tables[n]) for c, n in cases], max_streams=4)
    singles = [Solver(c, *tables[n]) for c, n in cases]
    try:
        b.init_freestream()
        for s in singles:
            s.init_freestream()
        for n in (4, 3):          # two graph pairs, then a pair and an odd tail
            done, st = b.run(n)
            assert list(done) == [n] * len(cases) and not st.any()
            for i, s in enumerate(singles):
                d, rep = s.step_s2cn2(n)
                assert d == n
                for x, y in zip(b.download(i), s.download()):
                    assert np.array_equal(x, y), (i, n)
                assert np.array_equal(b.report(i), rep)
                assert np.array_equal(b.wall_aero(i), s.wall_aero())
        k, ms = b.tune(steps=2)   # advances the batch; then both sides restart from the cold start
        assert 1 <= k <= 4 and ms > 0
        b.init_freestream()
        for s in singles:
            s.init_freestream()
        b.run(2)
        for i, s in enumerate(singles):
            s.step_s2cn2(2)
            for x, y in zip(b.download(i), s.download()):
                assert np.array_equal(x, y), ("after tune", i)
    finally:
        b.close()
        for s in singles:
            s.close()


@pytest.mark.gpu
def test_generated_table_instance_matches_oracle():
    from oracle.oracle import Oracle, set_threads
    from ugks2d_high_order_b200.batch import Batch
    set_threads(None)
    case, _ = _mixed(1)[0]
    table = velocity_table(24)
    b = Batch([(case, table)], max_streams=1)
    o = Oracle(case, *table)
    try:
        b.init_freestream()
        o.init_freestream()
        hg, bg, Wg = b.download(0)
        ho, bo, Wo = o.get_state()
        assert np.abs(hg - ho).max() <= 1e-12 * np.abs(ho).max()
        b.run(3)
        for _ in range(3):
            out = o.s2cn2_step()
        hg, bg, Wg = b.download(0)
        ho, bo, Wo = o.get_state()
        for x, y in ((hg, ho), (bg, bo), (Wg, Wo)):
            assert np.abs(x - y).max() <= HO_TOL * np.abs(y).max()
        rep = b.report(0)
        assert rep[1] <= 2e-12 and rep[2] <= 2e-12 and rep[9] <= 2e-12
        assert abs(rep[0] - out[0]) <= 1e-15 * out[0]
    finally:
        b.close()
