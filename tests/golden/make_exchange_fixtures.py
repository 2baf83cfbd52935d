"""Golden vectors of the reference's own unit tests for the data-movement layer.

The reference checks pack, unpack, all2all and TransBlock with index-valued
inputs whose expected buffers its tests build with host loops of their own
(a formulation independent of the Pack / Unpack functors they test).  The
reference cannot be built here (Kokkos, kokkos-fft, MPI and googletest are
absent), so this script restates those test constructions, each citing the
test file and lines it follows (paths relative to the reference's
``distributed/unit_test/``), and writes their inputs and expected outputs:

  exchange_fixtures.npz / exchange_fixtures.json
    pack      Test_Pack.cpp:101-240 (2D, gn = (8, 7)), :252-573 (3D, gn = (8, 7, 5));
              nprocs 1..4, every rank, every axis order, LayoutRight and LayoutLeft
    unpack    Test_Unpack.cpp:41-181 (2D), :198-520 (3D); same parameters
    all2all   Test_All2All.cpp:110-194 (world, (16, 15)), :304-397 (row), :495-590
              (column communicator of a 2 x 2 Cartesian grid)
    transblock Test_TransBlock.cpp:53-163 (2D, (11, 10)), :165-660 (3D, (8, 7, 5),
              row / column communicators), index-valued instead of random data
  layout_tables.json
    explicit known answers extracted as text: permute_map_by_axes tables
    (Test_Mapping.cpp:18-205), rank_to_coord tables (Test_MPI_Extents.cpp:164-290)

Arrays are stored flattened in the memory order of their layout (C order for
LayoutRight, Fortran order for LayoutLeft) as int16 (every value is a small
index).  Run (only where the reference source is present; the index-valued
constructions need no reference file, the explicit tables are read from it):

    python tests/golden/make_exchange_fixtures.py <path to the reference checkout>
"""
import itertools
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORDERS3 = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]  # Test_Pack.cpp:266-271


def distribute_extents(n, r, p):
    """Test_Utils.hpp:74-79: (start, length) of bin r of n over p."""
    base, rem = divmod(n, p)
    return r * base + min(r, rem), base + (1 if r < rem else 0)


def merge_topology(tin, tout):
    """Element-wise merge of two topologies that differ in at most two
    entries (KokkosFFT_Distributed_ContainerAnalyses.hpp:182-229 as used by
    compute_buffer_extents): the non-one value wherever one of them has it."""
    return tuple(max(a, b) for a, b in zip(tin, tout))


def diff_topology(merged, tin):
    """ContainerAnalyses.hpp:240-258: the value that merged adds to tin (1 if none)."""
    diffs = [m for m, a in zip(merged, tin) if m != a]
    return diffs[0] if diffs else 1


def buffer_extents(gext, tin, tout, right):
    """compute_buffer_extents<Layout> (KokkosFFT_Distributed_Extents.hpp:35-61),
    pinned by the explicit values of Test_Extents.cpp:20-60."""
    merged = merge_topology(tin, tout)
    p0 = diff_topology(merged, tin)
    ext = [(n - 1) // m + 1 for n, m in zip(gext, merged)]
    return tuple([p0] + ext) if right else tuple(ext + [p0])


def rank_to_coord(topo, r, right=True):
    """KokkosFFT_Distributed_MPI_Extents.hpp:492-529: row-major coordinates of
    rank r over the topology (LayoutRight), column-major for LayoutLeft."""
    dims = range(len(topo) - 1, -1, -1) if right else range(len(topo))
    c = [0] * len(topo)
    for k in dims:
        c[k] = r % topo[k]
        r //= topo[k]
    return tuple(c)


def local_block(gext, topo, r, right=True):
    """(starts, extents) of rank r's block (compute_local_extents_and_starts)."""
    c = rank_to_coord(topo, r, right)
    se = [distribute_extents(n, ci, t) for n, ci, t in zip(gext, c, topo)]
    return tuple(s for s, _ in se), tuple(e for _, e in se)


def flat(a, right):
    """Memory image of a logical array in the view's layout."""
    return np.asarray(a).ravel(order="C" if right else "F").astype(np.int16)


class Store:
    def __init__(self):
        self.arrays = {}
        self.cases = []

    def add(self, name, a, right):
        key = f"a{len(self.arrays)}"
        self.arrays[key] = flat(a, right)
        return key

    def case(self, **kw):
        self.cases.append(kw)


# ---------------------------------------------------------------------------
# pack / unpack (one rank's view <-> its buffer)
# ---------------------------------------------------------------------------
def _buffer_ref(bext, right, fill):
    """Loop over a buffer of extents bext as the tests do: p is the last index
    for LayoutLeft and the first for LayoutRight (Test_Pack.cpp:189-197),
    `fill(p, idx)` returns the value or None (left at zero)."""
    buf = np.zeros(bext, dtype=np.int64)
    for full in itertools.product(*[range(e) for e in bext]):
        if right:
            p, idx = full[0], full[1:]
        else:
            p, idx = full[-1], full[:-1]
        v = fill(p, idx)
        if v is not None:
            buf[full] = v
    return buf


def pack_unpack_2d(st, right, nprocs, rank, order):
    """Test_Pack.cpp:101-240 and Test_Unpack.cpp:41-181 (gn = (8, 7))."""
    gn0, gn1 = 8, 7
    n0s, n0l = distribute_extents(gn0, rank, nprocs)
    n1s, n1l = distribute_extents(gn1, rank, nprocs)
    gext, t0, t1 = (gn0, gn1), (1, nprocs), (nprocs, 1)
    src_map = (0, 1) if order == 0 else (1, 0)
    gu = np.array([[i1 + i0 * gn1 for i1 in range(gn1)] for i0 in range(gn0)])
    u_t0, u_t1 = gu[:, n1s:n1s + n1l], gu[n0s:n0s + n0l, :]
    bext = buffer_extents(gext, t0, t1, right)

    def fill_t0(p, idx):
        i0t, i1t = idx
        start0, length0 = distribute_extents(gn0, p, nprocs)
        gi0 = i0t + start0
        if gi0 < gn0 and i0t < length0 and i1t < u_t0.shape[1]:
            return u_t0[gi0, i1t]
        return None

    def fill_t1(p, idx):
        i0t, i1t = idx
        start1, length1 = distribute_extents(gn1, p, nprocs)
        gi1 = i1t + start1
        if gi1 < gn1 and i1t < length1 and i0t < u_t1.shape[0]:
            return u_t1[i0t, gi1]
        return None

    for u, fill, axis, tag in ((u_t0, fill_t0, 0, "t0"), (u_t1, fill_t1, 1, "t1")):
        u_p = np.transpose(u, src_map)
        buf = _buffer_ref(bext, right, fill)
        st.case(kind="pack_unpack", dim=2, tag=tag, layout="right" if right else "left", nprocs=nprocs, rank=rank,
                map=list(src_map), axis=axis, view_extents=list(u_p.shape), buffer_extents=list(bext),
                view=st.add("view", u_p, right), buffer=st.add("buffer", buf, right),
                pack_source="Test_Pack.cpp:101-240", unpack_source="Test_Unpack.cpp:41-181")


def pack_unpack_3d(st, right, nprocs, rank, order):
    """Test_Pack.cpp:252-573 and Test_Unpack.cpp:198-520 (gn = (8, 7, 5))."""
    gn = (8, 7, 5)
    gn0, gn1, gn2 = gn
    (n0s, n0l), (n1s, n1l), (n2s, n2l) = [distribute_extents(n, rank, nprocs) for n in gn]
    t0, t1, t2 = (1, 1, nprocs), (1, nprocs, 1), (nprocs, 1, 1)
    src_map = ORDERS3[order]
    gu = np.arange(gn0 * gn1 * gn2).reshape(gn)  # i2 + i1 gn2 + i0 gn2 gn1 (Test_Pack.cpp:352-358)
    u_t0, u_t1, u_t2 = gu[:, :, n2s:n2s + n2l], gu[:, n1s:n1s + n1l, :], gu[n0s:n0s + n0l, :, :]

    def filler(split, u, gidx):
        # value of the reference loop: merge index `split` with bin p, the
        # other index must fall inside the source view along `gidx` (the
        # axis split in the source topology)
        def fill(p, idx):
            it = list(idx)
            start, length = distribute_extents(gn[split], p, nprocs)
            g = it[split] + start
            if g < gn[split] and it[split] < length and it[gidx] < u.shape[gidx]:
                src = list(it)
                src[split] = g
                return u[tuple(src)]
            return None
        return fill

    # (view, topology pair, split axis, axis split in the source) as the six
    # pack calls of Test_Pack.cpp:487-492 / unpack calls of Test_Unpack.cpp:443-448
    cases = [("t01", u_t0, (t0, t1), 1, 2), ("t02", u_t0, (t0, t2), 0, 2),
             ("t10", u_t1, (t0, t1), 2, 1), ("t12", u_t1, (t1, t2), 0, 1),
             ("t20", u_t2, (t0, t2), 2, 0), ("t21", u_t2, (t1, t2), 1, 0)]
    for tag, u, (ta, tb), axis, gidx in cases:
        bext = buffer_extents(gn, ta, tb, right)
        buf = _buffer_ref(bext, right, filler(axis, u, gidx))
        u_p = np.transpose(u, src_map)
        st.case(kind="pack_unpack", dim=3, tag=tag, layout="right" if right else "left", nprocs=nprocs, rank=rank,
                map=list(src_map), axis=axis, view_extents=list(u_p.shape), buffer_extents=list(bext),
                view=st.add("view", u_p, right), buffer=st.add("buffer", buf, right),
                pack_source="Test_Pack.cpp:252-573", unpack_source="Test_Unpack.cpp:198-520")


# ---------------------------------------------------------------------------
# all2all (every rank's send buffer -> every rank's recv buffer)
# ---------------------------------------------------------------------------
def all2all_world(st, right, nprocs):
    """Test_All2All.cpp:110-194: (16, 15) split over all ranks; the value of
    send(i0, i1, i2) on `rank` and of the expected recv are explicit formulas."""
    n0, n1 = 16, 15
    n0l, n1l = (n0 - 1) // nprocs + 1, (n1 - 1) // nprocs + 1
    shape = (n0l, n1l, nprocs) if not right else (nprocs, n0l, n1l)
    size = n0l * n1l * nprocs
    sends, refs = [], []
    for rank in range(nprocs):
        s = np.zeros(shape, dtype=np.int64)
        r = np.zeros(shape, dtype=np.int64)
        for i0, i1, i2 in itertools.product(*[range(e) for e in shape]):
            if not right:
                s[i0, i1, i2] = rank * size + i0 + i1 * shape[0] + i2 * shape[0] * shape[1]
                r[i0, i1, i2] = i2 * size + i0 + i1 * shape[0] + rank * shape[0] * shape[1]
            else:
                s[i0, i1, i2] = rank * size + i2 + i1 * shape[2] + i0 * shape[2] * shape[1]
                r[i0, i1, i2] = i0 * size + i2 + i1 * shape[2] + rank * shape[2] * shape[1]
        sends.append(flat(s, right))
        refs.append(flat(r, right))
    st.case(kind="all2all", source="Test_All2All.cpp:110-194", layout="right" if right else "left", nprocs=nprocs,
            buffer_extents=list(shape), comm_axis=-1, cart_topology=None,
            send=st.add("send", np.concatenate(sends), True), expected=st.add("recv", np.concatenate(refs), True))


def all2all_cart(st, right, npx, npy, row):
    """Test_All2All.cpp:304-397 (row communicator: MPI_Cart_sub keeps dim 0)
    and :495-590 (column communicator: keeps dim 1) on an 8 x 8 array over a
    npx x npy Cartesian grid (MPI_Cart_create without reordering)."""
    n0, n1 = 8, 8
    P = npx * npy
    if row:
        n0l, n1l, pc = n0 // npx, n1 // (npx * npy), npx
    else:
        n0l, n1l, pc = n0 // (npx * npy), (n1 - 1) // npy + 1, npy
    shape = (n0l, n1l, pc) if not right else (pc, n0l, n1l)
    sends, refs = [], []
    for rank in range(P):
        rx, ry = rank // npy, rank % npy
        s = np.zeros(shape, dtype=np.int64)
        r = np.zeros(shape, dtype=np.int64)
        for i0, i1, i2 in itertools.product(*[range(e) for e in shape]):
            if row and not right:
                v = (ry * (n1 // npy) + i1) + (rx * (n0 // npx) + i0) * n1 + i2 * shape[2]
                vt = i1 + rx * shape[1] + ry * (n1 // npy) + i0 * n1 + i2 * (n0 // npx) * n1
            elif row:
                v = (ry * (n1 // npy) + i2) + (rx * (n0 // npx) + i1) * n1 + i0 * shape[0]
                vt = i2 + rx * shape[0] + ry * (n1 // npy) + i1 * n1 + i0 * (n0 // npx) * n1
            elif not right:
                v = (ry * shape[1] + i1) + (rx * (n0 // npx) + i0) * n1 + i2 * shape[2] * n1
                vt = i1 + (i0 + ry * shape[0]) * n1 + (i2 + rx * n1) * (n0 // npx)
            else:
                v = (ry * shape[2] + i2) + (rx * (n0 // npx) + i1) * n1 + i0 * shape[0] * n1
                vt = i2 + (i1 + ry * shape[0]) * n1 + (i0 + rx * n1) * (n0 // npx)
            s[i0, i1, i2] = v
            r[i0, i1, i2] = vt
        sends.append(flat(s, right))
        refs.append(flat(r, right))
    st.case(kind="all2all", source="Test_All2All.cpp:304-397" if row else "Test_All2All.cpp:495-590",
            layout="right" if right else "left", nprocs=P, buffer_extents=list(shape), comm_axis=0 if row else 1,
            cart_topology=[npx, npy], send=st.add("send", np.concatenate(sends), True),
            expected=st.add("recv", np.concatenate(refs), True))


# ---------------------------------------------------------------------------
# TransBlock (every rank's block in one topology -> its block in another)
# ---------------------------------------------------------------------------
def _blocks(gu, topo, topo_right, vmap, right):
    """Every rank's block of gu in `topo` (rank order of topo_right),
    permuted by vmap, each flattened in the view layout, concatenated."""
    out = []
    for r in range(int(np.prod(topo))):
        s, e = local_block(gu.shape, topo, r, topo_right)
        sub = gu[tuple(slice(a, a + b) for a, b in zip(s, e))]
        out.append(flat(np.transpose(sub, vmap), right))
    return np.concatenate(out)


def trans_block_case(st, source, gext, tin, tin_right, tout, tout_right, src_map, src_axis, dst_map, dst_axis,
                     comm_axis, cart, right):
    gu = np.arange(int(np.prod(gext))).reshape(gext)
    st.case(kind="trans_block", source=source, layout="right" if right else "left", global_extents=list(gext),
            in_topology=list(tin), in_topology_layout="right" if tin_right else "left", out_topology=list(tout),
            out_topology_layout="right" if tout_right else "left", src_map=list(src_map), src_axis=src_axis,
            dst_map=list(dst_map), dst_axis=dst_axis, comm_axis=comm_axis,
            cart_topology=list(cart) if cart is not None else None,
            buffer_extents=list(buffer_extents(gext, tin, tout, right)),
            input=st.add("in", _blocks(gu, tin, tin_right, src_map, right), True),
            expected=st.add("out", _blocks(gu, tout, tout_right, dst_map, right), True))


def trans_block_2d(st, right, nprocs):
    """Test_TransBlock.cpp:53-163: (11, 10), topology {1, P} -> {P, 1} over
    MPI_COMM_WORLD, TransBlock(buffer_01, map01, 0, map01 or map10, 1)."""
    for dst_map in ((0, 1), (1, 0)):
        trans_block_case(st, "Test_TransBlock.cpp:53-163", (11, 10), (1, nprocs), True, (nprocs, 1), True, (0, 1), 0,
                         dst_map, 1, -1, None, right)


def trans_block_3d(st, right, npx, npy):
    """Test_TransBlock.cpp:165-660: (8, 7, 5); topology0 {1, npx, npy},
    topology1 {npx, 1, npy}, topology2 {npx, npy, 1} (LayoutRight) and
    topology3 {npy, npx, 1} (LayoutLeft); the Cartesian communicator is built
    over the non-one entries of topology0, row_comm keeps dim 0, col_comm dim 1:
      trans_block_0_1(row_comm): TransBlock(buffer_01, map012, 0, map, 1)
      trans_block_0_3(col_comm): TransBlock(buffer_03, map012, 0, map, 2)
      trans_block_1_2(col_comm): TransBlock(buffer_12, map012, 1, map, 2)
    for every destination map."""
    gext = (8, 7, 5)
    t0, t1, t2, t3 = (1, npx, npy), (npx, 1, npy), (npx, npy, 1), (npy, npx, 1)
    for dst_map in ORDERS3:
        trans_block_case(st, "Test_TransBlock.cpp:421-490", gext, t0, True, t1, True, (0, 1, 2), 0, dst_map, 1, 0, t0,
                         right)
        trans_block_case(st, "Test_TransBlock.cpp:493-574", gext, t0, True, t3, False, (0, 1, 2), 0, dst_map, 2, 1,
                         t0, right)
        trans_block_case(st, "Test_TransBlock.cpp:576-658", gext, t1, True, t2, True, (0, 1, 2), 1, dst_map, 2, 1, t0,
                         right)


# ---------------------------------------------------------------------------
# explicit known-answer tables, read as text
# ---------------------------------------------------------------------------
def _ints(s):
    return [int(x) for x in re.findall(r"\d+", s)]


def extract_mapping(src):
    """permute_map_by_axes tables of Test_Mapping.cpp: per function, the
    LayoutLeft branch and the else (LayoutRight) branch assign
    ref_dst_map_<src>_axis<a> = {...}."""
    rows = []
    for fn in re.finditer(r"void (test_permute_map_by_axes\w+)\(\) \{(.*?)\n\}", src, flags=re.S):
        body = fn.group(2)
        cut = body.index("} else {")
        for layout, part in (("left", body[:cut]), ("right", body[cut:])):
            for m in re.finditer(r"ref_dst_map_(\d+)_axis(\d) = \{([^}]*)\}", part):
                rows.append(dict(layout=layout, src_map=[int(c) for c in m.group(1)], axis=int(m.group(2)),
                                 expected=_ints(m.group(3))))
    line = src[:src.index("void test_permute_map_by_axes2D_View2D")].count("\n") + 1
    return dict(source=f"Test_Mapping.cpp:{line}", rows=rows)


def extract_rank_to_coord(src):
    """rank_to_coord tables of Test_MPI_Extents.cpp: topologies declared as
    topologyN{...}, expected coordinates as ref_coordN_rankR{...} (LayoutRight)
    with the LayoutLeft overrides ref_coordN_rankR = {...}."""
    start = src.index("void test_rank_to_coord()")
    body = src[start:src.index("\n}\n", start)]
    topos = {m.group(1): _ints(m.group(2)) for m in re.finditer(r"\b(topology\d(?:_\d)?)\{([^}]*)\}", body)}
    right = {m.group(1): _ints(m.group(2)) for m in re.finditer(r"\b(ref_coord\w+?)\{([^}]*)\}", body)}
    left = dict(right)
    lb = body[body.index("is_same_v<LayoutType, Kokkos::LayoutLeft>"):]
    lb = lb[:lb.index("\n  }\n")]
    for m in re.finditer(r"\b(ref_coord\w+?) = \{([^}]*)\}", lb):
        left[m.group(1)] = _ints(m.group(2))
    rows = []
    for name, coord in right.items():
        m = re.fullmatch(r"ref_coord(\d(?:_\d)?)_rank(\d+)", name)
        topo = topos["topology" + m.group(1)]
        rows.append(dict(layout="right", topology=topo, rank=int(m.group(2)), expected=coord))
        rows.append(dict(layout="left", topology=topo, rank=int(m.group(2)), expected=left[name]))
    line = src[:start].count("\n") + 1
    return dict(source=f"Test_MPI_Extents.cpp:{line}", rows=rows)


def main(ref):
    st = Store()
    for right in (True, False):
        for nprocs in range(1, 5):  # m_max_nprocs = 4 (Test_Pack.cpp:21)
            for rank in range(nprocs):
                for order in range(2):
                    pack_unpack_2d(st, right, nprocs, rank, order)
                for order in range(6):
                    pack_unpack_3d(st, right, nprocs, rank, order)
        for nprocs in range(1, 7):
            all2all_world(st, right, nprocs)
            trans_block_2d(st, right, nprocs)
        for row in (True, False):
            all2all_cart(st, right, 2, 2, row)  # the tests run on perfect squares > 1
        for npx, npy in ((2, 2), (2, 3), (3, 2)):
            trans_block_3d(st, right, npx, npy)
    np.savez_compressed(os.path.join(HERE, "exchange_fixtures.npz"), **st.arrays)
    with open(os.path.join(HERE, "exchange_fixtures.json"), "w") as f:
        json.dump(dict(generator="tests/golden/make_exchange_fixtures.py", cases=st.cases), f)
    ut = os.path.join(ref, "distributed", "unit_test")
    tables = dict(generator="tests/golden/make_exchange_fixtures.py",
                  permute_map_by_axes=extract_mapping(open(os.path.join(ut, "Test_Mapping.cpp")).read()),
                  rank_to_coord=extract_rank_to_coord(open(os.path.join(ut, "Test_MPI_Extents.cpp")).read()))
    with open(os.path.join(HERE, "layout_tables.json"), "w") as f:
        json.dump(tables, f, indent=1)
    kinds = {}
    for c in st.cases:
        kinds[c["kind"]] = kinds.get(c["kind"], 0) + 1
    print(kinds, len(st.arrays), "arrays;", len(tables["permute_map_by_axes"]["rows"]), "map rows,",
          len(tables["rank_to_coord"]["rows"]), "coord rows")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_exchange_fixtures.py <path to the reference checkout>")
    main(sys.argv[1])
