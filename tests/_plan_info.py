"""Builds the oracle's plan description from a dfft.Plan (host queries only)."""
import numpy as np


def plan_info(plan, norm="backward"):
    chain, trans, layouts = plan.topology_chain()
    P = plan.nprocs
    return dict(
        in_extents=plan.in_extents, out_extents=plan.out_extents, axes=plan.axes,
        in_topology=plan.in_topology, out_topology=plan.out_topology, real_input=plan.real_input,
        norm=norm, layout_right=plan.layout == "right", pencil=plan.name() == "PencilPlan",
        chain=chain, chain_layouts=layouts, blocks=[plan.block_infos(r) for r in range(P)])
