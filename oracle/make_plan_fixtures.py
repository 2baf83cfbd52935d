"""Writes the block lists the CPU oracle walks for the timed CPU baseline.

The oracle's literal block walk (dfft_oracle.execute_literal) follows a
plan's topology chain and per-rank block list.  For the timed CPU legs of
bench.py those come from the JSON files under oracle/plans/ instead of the
library, so that the CPU baseline loads nothing of the product.  The files
hold the planner's output for the bench's topology, which the tests pin
against the reference's own topology tables (tests/test_planner_golden.py)
and compare with the files (tests/test_plan_fixtures.py).

Run after a planner change:  python oracle/make_plan_fixtures.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# (file name, global extents, in topology, out topology): the pencil of the
# bench workload at the CPU sample sizes (256^3, and 128^3 / 64^3 when many
# timed steps must fit the reference arm's time) and at the workload size
CONFIGS = [("c2c_64_pencil_441_144.json", (64, 64, 64), (4, 4, 1), (1, 4, 4)),
           ("c2c_128_pencil_441_144.json", (128, 128, 128), (4, 4, 1), (1, 4, 4)),
           ("c2c_256_pencil_441_144.json", (256, 256, 256), (4, 4, 1), (1, 4, 4)),
           ("c2c_512_pencil_441_144.json", (512, 512, 512), (4, 4, 1), (1, 4, 4))]


def plan_info_of(plan, norm="backward"):
    chain, trans, layouts = plan.topology_chain()
    return dict(in_extents=list(plan.in_extents), out_extents=list(plan.out_extents), axes=list(plan.axes),
                in_topology=list(plan.in_topology), out_topology=list(plan.out_topology),
                real_input=bool(plan.real_input), norm=norm, layout_right=plan.layout == "right",
                pencil=plan.name() == "PencilPlan", chain=[list(t) for t in chain],
                chain_layouts=list(layouts), blocks=[plan.block_infos(r) for r in range(plan.nprocs)])


def _plain(x):
    if isinstance(x, dict):
        return {k: _plain(v) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [_plain(v) for v in x]
    if hasattr(x, "item"):
        return x.item()
    return x


def build(name, g, tin, tout):
    sys.path.insert(0, os.path.join(ROOT, "distributed-fft-for-kokkos_b200"))
    import dfft
    p = dfft.Plan(g, g, (0, 1, 2), tin, tout, analyze_only=True)
    return _plain(dict(name=name, generator="oracle/make_plan_fixtures.py", plan=plan_info_of(p)))


def main():
    for name, g, tin, tout in CONFIGS:
        with open(os.path.join(HERE, "plans", name), "w") as f:
            json.dump(build(name, g, tin, tout), f)
        print("wrote", name)


if __name__ == "__main__":
    main()
