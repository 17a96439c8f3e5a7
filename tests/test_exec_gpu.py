"""The plan executor on the GPU: the benchmark plans written as JSON give exactly the
results of the same plans written against the C ABI (and the oracle's), variables are freed
after their last use, a budget too small fails cleanly, and inputs load from packed
relation files."""
import numpy as np
import pytest

from redfox_b200 import executor as X
from redfox_b200 import plans as PL

from helpers import join_aggregate_oracle, join_aggregate_oracle_data, to_np

pytestmark = pytest.mark.gpu


def _run_join_aggregate(r, s, budget=0):
    ex = X.Executor(X.join_aggregate_plan(), budget)
    ex.bind("R", r.clone())
    ex.bind("S", s.clone())
    ex.run()
    out = [ex.output(n) for n in ("keys", "sums", "counts")]
    st = ex.stats()
    ex.close()
    return out, st


@pytest.mark.parametrize("nr,ns,dom", [(1000, 4000, 256), (50000, 200000, 12500)])
def test_join_aggregate_plan_matches(cuda, nr, ns, dom):
    r, s = PL.gen_join_aggregate(nr, ns, key_domain=dom)
    (k, sm, c), st = _run_join_aggregate(r, s)
    ek, esum, ecnt, _ = join_aggregate_oracle(*join_aggregate_oracle_data(nr, ns, dom))
    assert np.array_equal(to_np(k).view(np.uint32).ravel(), ek)
    assert np.array_equal(to_np(sm).view(np.int64).ravel(), esum)
    assert np.array_equal(to_np(c).view(np.uint32).ravel(), ecnt)
    assert st["ops"] == 4


def test_liveness_and_budget(cuda):
    r, s = PL.gen_join_aggregate(50000, 200000, key_domain=12500)
    _, st = _run_join_aggregate(r, s)
    # J (the join output, 16 B x ~1M rows) and the workspaces are freed after their last
    # use; the outputs and the bound inputs stay
    assert st["in_use"] < st["peak"]
    with pytest.raises(X.PlanError, match="budget"):
        _run_join_aggregate(r, s, budget=1 << 20)


def test_three_relation_plan_matches(cuda):
    n1, n2, n3, l5, l2 = (PL.C2_D1_ROWS // 100, PL.C2_D2_ROWS // 100, PL.C2_F_ROWS // 100, PL.C2_L5 // 100,
                          PL.C2_L2 // 100)
    d1, d2, f, li, lo = PL.gen_three_relation(n1, n2, n3, l5, l2)
    ek, es, ec = PL.three_relation(d1, d2, f, li, lo)
    ex = X.Executor(X.three_relation_plan(PL.C2_SEGMENT, PL.C2_DATE_LO, PL.C2_DATE_HI))
    for name, t in (("D1", d1), ("D2", d2), ("F", f.clone()), ("Lin", li), ("Lout", lo)):
        ex.bind(name, t)
    ex.run()
    k, sm, c = (ex.output(n) for n in ("keys", "sums", "counts"))
    assert np.array_equal(to_np(k).view(np.uint32).ravel(), to_np(ek).view(np.uint32))
    assert np.array_equal(to_np(sm).view(np.int64).ravel(), to_np(es))
    assert np.array_equal(to_np(c).view(np.uint32).ravel(), to_np(ec).view(np.uint32))
    ex.close()


def test_inputs_from_packed_files(cuda, tmp_path):
    r, s = PL.gen_join_aggregate(3000, 12000, key_domain=700)
    (pr, ps) = (tmp_path / "R.bin", tmp_path / "S.bin")
    to_np(r).tofile(pr)
    to_np(s).tofile(ps)
    ex = X.Executor(X.join_aggregate_plan())
    ex.load("R", pr)
    ex.load("S", ps)
    ex.run()
    got = [to_np(ex.output(n)) for n in ("keys", "sums", "counts")]
    ex.close()
    (k, sm, c), _ = _run_join_aggregate(r, s)
    for a, b in zip(got, (k, sm, c)):
        assert np.array_equal(a, to_np(b))
    # a file whose size is not a whole number of rows is refused
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"123")
    ex = X.Executor(X.join_aggregate_plan())
    with pytest.raises(X.PlanError):
        ex.load("R", bad)
    ex.close()


def test_captured_plan_replays_the_eager_result(cuda):
    """Both benchmark plans captured as CUDA graphs: every replay gives the eager run's
    outputs, and the whole plan is one graph launch per replay."""
    import torch
    stream = torch.cuda.Stream()
    r, s = PL.gen_join_aggregate(50000, 200000, key_domain=12500)
    (ek, es, ec), _ = _run_join_aggregate(r, s)
    ex = X.Executor(X.join_aggregate_plan())
    ex.bind("R", r.clone())
    ex.bind("S", s.clone())
    ex.capture(stream)
    for _ in range(3):
        ex.replay(stream)
        k, sm, c = (ex.output(n) for n in ("keys", "sums", "counts"))
        assert torch.equal(k, ek) and torch.equal(sm, es) and torch.equal(c, ec)
    ex.close()

    n1, n2, n3, l5, l2 = (PL.C2_D1_ROWS // 100, PL.C2_D2_ROWS // 100, PL.C2_F_ROWS // 100, PL.C2_L5 // 100,
                          PL.C2_L2 // 100)
    d1, d2, f, li, lo = PL.gen_three_relation(n1, n2, n3, l5, l2)
    gk, gs, gc = PL.three_relation(d1, d2, f, li, lo)
    ex = X.Executor(X.three_relation_plan(PL.C2_SEGMENT, PL.C2_DATE_LO, PL.C2_DATE_HI))
    for name, t in (("D1", d1), ("D2", d2), ("F", f.clone()), ("Lin", li), ("Lout", lo)):
        ex.bind(name, t)
    ex.capture(stream)
    for _ in range(2):
        ex.replay(stream)
        k, sm, c = (ex.output(n) for n in ("keys", "sums", "counts"))
        assert np.array_equal(to_np(k).view(np.uint32).ravel(), to_np(gk).view(np.uint32))
        assert np.array_equal(to_np(sm).view(np.int64).ravel(), to_np(gs))
        assert np.array_equal(to_np(c).view(np.uint32).ravel(), to_np(gc).view(np.uint32))
    ex.close()


def test_replay_detects_a_changed_plan_shape(cuda):
    """New input contents of the same size that change an intermediate size (a different
    key domain: another join size) make the replay report RFX_ERR_CAPACITY; an eager run
    then gives the right result."""
    import torch
    stream = torch.cuda.Stream()
    r, s = PL.gen_join_aggregate(20000, 80000, key_domain=5000)
    r2, s2 = PL.gen_join_aggregate(20000, 80000, key_domain=900)
    rb, sb = r.clone(), s.clone()
    ex = X.Executor(X.join_aggregate_plan())
    ex.bind("R", rb)
    ex.bind("S", sb)
    ex.capture(stream)
    ex.replay(stream)
    rb.copy_(r2)
    sb.copy_(s2)
    torch.cuda.synchronize()
    with pytest.raises(X.PlanError, match="replay"):
        ex.replay(stream)
    rb.copy_(r2)
    sb.copy_(s2)
    ex.run()
    (ek, es, ec), _ = _run_join_aggregate(r2, s2)
    k, sm, c = (ex.output(n) for n in ("keys", "sums", "counts"))
    assert torch.equal(k, ek) and torch.equal(sm, es) and torch.equal(c, ec)
    ex.close()
