"""The block lists under oracle/plans/ (what the timed CPU baseline walks)
equal the planner's output for their configurations."""
import json
import os

import pytest

import make_plan_fixtures as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("name,g,tin,tout", M.CONFIGS)
def test_plan_fixture_matches_planner(name, g, tin, tout):
    with open(os.path.join(ROOT, "oracle", "plans", name)) as f:
        committed = json.load(f)
    assert committed == M.build(name, g, tin, tout)
