"""Extract the known-answer tables of get_all_slab_topologies and
get_all_pencil_topologies from the reference's unit test source
(distributed/unit_test/Test_Topologies.cpp) into topology_tables.json.

The tables are read as text: every ``test_get_all_{slab,pencil}_topologies*``
function declares its topologies symbolically (``nprocs``, ``np0``), its axes,
and a list of rows ``{in, out, axes, [trans_axes, layouts,] expected chain}``.
The JSON keeps the symbols; the tests evaluate them for nprocs = 2..6 exactly
as the reference's ``INSTANTIATE_TEST_SUITE_P(..., Values(1, 2, 3, 4, 5, 6))``
does (nprocs = 1 is the throwing branch).

Run (only where the reference source is present):
    python tests/golden/extract_topology_tables.py /path/to/reference
"""
import json
import os
import re
import sys

FN_RE = re.compile(r"void (test_get_all_(slab|pencil)_topologies\w+)\(std::size_t nprocs\) \{")


def split_functions(src):
    out = []
    for m in FN_RE.finditer(src):
        start = m.end()
        nxt = src.find("\nvoid ", start)
        nxt2 = src.find("\nTEST", start)
        ends = [e for e in (nxt, nxt2) if e >= 0]
        end = min(ends) if ends else len(src)
        out.append((m.group(1), m.group(2), src[start:end]))
    return out


def parse_list(s):
    s = s.strip()
    return [x.strip() for x in s.split(",") if x.strip()] if s else []


def parse_defs(body, kinds):
    defs = {}
    for kind in kinds:
        for m in re.finditer(kind + r"\s+((?:\w+\{[^}]*\}\s*,?\s*)+);", body):
            for dm in re.finditer(r"(\w+)\{([^}]*)\}", m.group(1)):
                defs[dm.group(1)] = dict(type=kind, values=parse_list(dm.group(2)))
    return defs


def main(ref_root):
    path = os.path.join(ref_root, "distributed", "unit_test", "Test_Topologies.cpp")
    src = open(path).read()
    tables = []
    for name, kind, body in split_functions(src):
        np0 = re.search(r"std::size_t np0 = (\d+);", body)
        topos = parse_defs(body, ["topo_type", "topo_r_type", "topo_l_type"])
        axes = {k: v["values"] for k, v in parse_defs(body, ["axes_type"]).items()}
        topo_defs = {}
        for k, v in topos.items():
            layout = "left" if v["type"] == "topo_l_type" else "right"
            topo_defs[k] = dict(values=v["values"], layout=layout)
        else_part = body[body.find("} else {"):]
        rows = []
        if kind == "slab":
            for m in re.finditer(r"\{(topo\d+),\s*(topo\d+),\s*(axes\d+),\s*vec_topo_type\{([^}]*)\}\}", else_part):
                rows.append(dict(inp=m.group(1), out=m.group(2), axes=m.group(3), chain=parse_list(m.group(4))))
        else:
            pat = (r"\{(topo\d+),\s*(topo\d+),\s*(axes\d+),\s*vec_axis_type\{([^}]*)\},\s*"
                   r"vec_layout_type\{([^}]*)\},\s*vec_topo_type\{([^}]*)\}\}")
            for m in re.finditer(pat, else_part):
                chain = [c.replace("ref_", "") for c in parse_list(m.group(6))]
                rows.append(dict(inp=m.group(1), out=m.group(2), axes=m.group(3),
                                 trans_axes=[int(x) for x in parse_list(m.group(4))],
                                 layouts=[int(x) for x in parse_list(m.group(5))], chain=chain))
        line = src[:src.find("void " + name + "(")].count("\n") + 1
        tables.append(dict(function=name, kind=kind, source=f"distributed/unit_test/Test_Topologies.cpp:{line}",
                           np0=int(np0.group(1)) if np0 else None, topologies=topo_defs, axes=axes, rows=rows))
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "topology_tables.json")
    with open(out, "w") as f:
        json.dump(dict(generator="tests/golden/extract_topology_tables.py", tables=tables), f, indent=1)
    for t in tables:
        print(t["function"], len(t["rows"]), "rows")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: extract_topology_tables.py <path to the reference checkout>")
    main(sys.argv[1])
