"""The RA plan builder without a GPU: operators lower to the reference's kernel sequences
(sorts only where an input is not sorted on the fields an operator needs, fused select +
project, aggregation over leading fields without a projection, a COUNT sharing a TOTAL's
reduce), the plans it emits are the benchmark plans, and malformed RA is refused."""
import pytest

from redfox_b200 import executor as X
from redfox_b200 import plan_builder as PB
from redfox_b200 import rfx as R


def _ops(b):
    return b.plan()["ops"]


def _strip(op):
    return {k: v for k, v in op.items() if k not in ("keys", "sums", "counts")}


def test_join_aggregate_lowers_to_the_benchmark_plan():
    ops = _ops(PB.join_aggregate_ra())
    hand = X.join_aggregate_plan()["ops"]
    assert [_strip(o) for o in ops[:4]] == [_strip(o) for o in hand]
    assert ops[3]["sums"] and ops[3]["counts"]          # one reduce for SUM and COUNT
    assert [o["op"] for o in ops[4:]] == ["merge", "merge"]
    X.Executor(PB.join_aggregate_ra().json()).close()   # the executor accepts it


def test_three_relation_lowers_to_the_benchmark_plan():
    ops = _ops(PB.three_relation_ra(2, 500, 2000))
    hand = X.three_relation_plan(2, 500, 2000)["ops"]
    assert [_strip(o) for o in ops[:len(hand)] if o["op"] != "sort" or o["rel"] != "K"] == \
        [_strip(o) for o in hand if o["op"] != "sort" or o["rel"] != "K"]
    kb = [o for o in ops if o["op"] == "sort" and o["rel"] == "K"]
    assert kb == [{"op": "sort", "rel": "K", "begin_bit": 0, "end_bit": 32}]
    X.Executor(PB.three_relation_ra(2, 500, 2000).json()).close()
    X.Executor(PB.three_relation_ra(1, 0, 100, with_lists=False).json()).close()


def test_sorted_inputs_are_not_sorted_again():
    b = PB.PlanBuilder().relation("R", [32, 32], sorted_fields=2).relation("S", [32, 64], sorted_fields=1)
    b.join("J", "R", "S", 1).agg("T", "J", [0], PB.AGG_TOTAL, 2).output("T")
    assert [o["op"] for o in _ops(b)] == ["join", "reduce", "merge"]
    assert b.schema("J") == ([32, 32, 64], 2)      # sorted as far as the left input is
    assert b.schema("T") == ([32, 64], 2)


def test_second_join_on_the_same_input_sorts_once():
    b = PB.PlanBuilder().relation("R", [32, 32]).relation("S", [32, 64]).relation("U", [32, 16])
    b.join("J1", "R", "S", 1).join("J2", "R", "U", 1).output("J1", "J2")
    assert [o["op"] for o in _ops(b)].count("sort") == 3   # R once, S, U


def test_aggregation_over_non_leading_fields_projects_and_sorts():
    b = PB.PlanBuilder().relation("A", [16, 16, 32], sorted_fields=3)
    b.agg("T", "A", [1], PB.AGG_TOTAL, 2).agg("C", "A", [1, 0], PB.AGG_COUNT).output("T", "C")
    ops = _ops(b)
    assert [o["op"] for o in ops] == ["project", "sort", "reduce", "merge", "project", "sort", "reduce", "merge"]
    assert ops[0]["map"] == [1, 2] and ops[4]["map"] == [1, 0]
    assert ops[2]["key_shift"] == 32 and ops[2]["value_bits"] == 32
    assert ops[6]["key_shift"] == 0
    assert b.schema("C") == ([16, 16, 32], 3)


def test_aggregation_sorts_its_input_in_place_when_needed():
    b = PB.PlanBuilder().relation("A", [32, 32])
    b.agg("T", "A", [0], PB.AGG_TOTAL, 1).agg("C", "A", [0], PB.AGG_COUNT).output("T", "C")
    assert [o["op"] for o in _ops(b)] == ["sort", "reduce", "merge", "merge"]


def test_set_operations_and_unique_sort_unsorted_inputs():
    b = PB.PlanBuilder().relation("A", [32]).relation("B", [32], sorted_fields=1)
    b.set_op("U", "A", "B", R.SET_UNION).unique("U").output("U")
    ops = _ops(b)
    assert [o["op"] for o in ops] == ["sort", "set", "unique"]
    assert ops[0] == {"op": "sort", "rel": "A", "begin_bit": 0, "end_bit": 32}


def test_fusion_waits_for_in_place_sorts():
    """A select is not moved past an in-place sort of its input."""
    b = PB.PlanBuilder().relation("A", [32, 32]).relation("B", [32, 32])
    b.select("As", "A", [(R.LT, (R.OPND_VAR, 1), (R.OPND_CONST, 5), R.I32)])
    b.join("J", "A", "B", 1)
    b.project("P", "As", [1, 0]).output("P", "J")
    kinds = [o["op"] for o in _ops(b)]
    assert "select_project" not in kinds and kinds.count("select") == 1


@pytest.mark.parametrize("build,msg", [
    (lambda b: b.join("J", "R", "Q", 1), "unknown relation"),
    (lambda b: b.join("R", "R", "S", 1), "in use"),
    (lambda b: b.join("J", "R", "S", 3), "key count"),
    (lambda b: b.join("J", "R", "W", 1), "widths differ"),
    (lambda b: b.join("J", "S", "S2", 1), "128-bit"),
    (lambda b: b.project("P", "R", [5]), "out of range"),
    (lambda b: b.agg("T", "R", [0], 7), "COUNT or TOTAL"),
    (lambda b: b.agg("T", "S2", [0, 1], PB.AGG_TOTAL, 1), "fit 128"),
    (lambda b: b.select("X", "R", [(R.EQ, (R.OPND_VAR, 9), (R.OPND_CONST, 1), R.I32)]), "out of range"),
    (lambda b: b.set_op("X", "R", "S", R.SET_UNION), "fields differ"),
])
def test_malformed_ra_is_refused(build, msg):
    b = PB.PlanBuilder().relation("R", [32, 32]).relation("S", [32, 64]).relation("W", [16, 8])
    b.relation("S2", [32, 64, 64])
    with pytest.raises(PB.PlanBuildError, match=msg):
        build(b)
