"""Plan executor front end without a GPU: plans are parsed and checked (unknown operators,
unknown variables, missing row widths, malformed JSON) before anything runs."""
import pytest

from redfox_b200 import executor as X


def test_benchmark_plans_parse():
    X.Executor(X.join_aggregate_plan()).close()
    X.Executor(X.three_relation_plan(2, 500, 2000)).close()
    X.Executor(X.three_relation_plan(1, 0, 100, with_lists=False)).close()


@pytest.mark.parametrize("plan,msg", [
    ('{"variables": {"R": {"row_bytes": 8}}, "ops": [{"op": "frobnicate", "rel": "R"}]}', "unknown kind"),
    ('{"variables": {"R": {"row_bytes": 8}}, "ops": [{"op": "sort", "rel": "Q"}]}', "unknown variable"),
    ('{"variables": {"R": {}}, "ops": []}', "row_bytes"),
    ('{"variables": {"R": {"row_bytes": 8}}, "ops": [}', "plan:"),
    ('[1, 2]', "plan:"),
    ('{"variables": {"R": {"row_bytes": 8}}, "ops": [], "outputs": ["Z"]}', "outputs"),
])
def test_bad_plans_are_rejected(plan, msg):
    with pytest.raises(X.PlanError, match=msg):
        X.Executor(plan)
