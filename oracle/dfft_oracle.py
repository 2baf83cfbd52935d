"""CPU oracle for the distributed 3D FFT execute path (test infrastructure).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module, and only as the checker or as the timed CPU
baseline; the library itself never calls it.

It restates, in numpy, the reference algorithm of the path (file references
relative to the reference's ``distributed/src/``):

* ``bin_mapping``        KokkosFFT_Distributed_PackUnpack.hpp:40-46
* ``merge_indices``      KokkosFFT_Distributed_PackUnpack.hpp:62-73
* ``pack``               KokkosFFT_Distributed_PackUnpack.hpp:85-251 (Pack functor, zero fill)
* ``unpack``             KokkosFFT_Distributed_PackUnpack.hpp:258-420 (Unpack functor, skip padding)
* ``all2all``            KokkosFFT_Distributed_MPI_All2All.hpp:23-58 (MPI_Alltoall over the
                         communicator; pencil row / column communicators from
                         KokkosFFT_Distributed_PencilPlan.hpp:32-71)
* ``rank_to_coord``      KokkosFFT_Distributed_MPI_Extents.hpp:492-523
* ``local_extents``      KokkosFFT_Distributed_MPI_Extents.hpp:202-233
* ``buffer_extents``     KokkosFFT_Distributed_Extents.hpp:35-61 with merge/diff_topology
                         (KokkosFFT_Distributed_ContainerAnalyses.hpp:182-258)
* ``permute_map_by_axes`` KokkosFFT_Distributed_Mapping.hpp:39-100
* ``execute_literal``    the block walk of SlabInternalPlan<3> / PencilInternalPlan<3>
                         (KokkosFFT_Distributed_SlabPlan.hpp:963-1264,
                         KokkosFFT_Distributed_PencilPlan.hpp:1201-1599): local transpose to the
                         first block's map, per-block batched FFT over the innermost axes
                         (R2C on the innermost axis of the first FFT block), TransBlock
                         pack -> all2all -> unpack, final local transpose, normalize.

The local FFTs of the reference live in kokkos-fft (un-vendored submodule,
``>= 1.0.0``; FFTW on the host, cuFFT on CUDA) and are the unnormalised DFT
X_k = sum_j x_j exp(-2 pi i jk/n); here they are numpy's pocketfft in float64
(``global_fft`` / ``global_ifft`` give the global transform the reference's
tests compare against), cross-checked by ``naive_dftn`` on small shapes.

The block list and topology chain that the walk follows are the ones the
caller passes in (the planner's output, which the tests pin separately
against the reference's own topology tables).
"""
import numpy as np


# ---------------------------------------------------------------------------
# index math
# ---------------------------------------------------------------------------
def bin_mapping(n, nbins, ibin):
    """(start, length) of bin ``ibin`` of [0, n) split in ``nbins`` (first n%nbins bins one larger)."""
    base, rem = divmod(n, nbins)
    length = base + (1 if ibin < rem else 0)
    start = ibin * base + min(ibin, rem)
    return start, length


def merge_indices(idx, start, extent, axis, merged_axis):
    if axis == merged_axis:
        return -1 if idx >= extent else idx + start
    return idx


def rank_to_coord(topology, rank, layout_right=True):
    total = int(np.prod(topology))
    if rank >= total:
        raise ValueError("rank must be less than topology size.")
    coord = [0] * len(topology)
    r = rank
    order = range(len(topology) - 1, -1, -1) if layout_right else range(len(topology))
    for i in order:
        coord[i] = r % topology[i]
        r //= topology[i]
    return tuple(coord)


def local_extents(extents, topology, rank, layout_right=True, mapping=None):
    coords = rank_to_coord(topology, rank, layout_right)
    loc = []
    for n, t, c in zip(extents, topology, coords):
        loc.append(n // t + (1 if c < n % t else 0) if t > 1 else n)
    if mapping is not None:
        loc = [loc[m] for m in mapping]
    return tuple(loc)


def local_starts(extents, topology, rank, layout_right=True):
    coords = rank_to_coord(topology, rank, layout_right)
    return tuple(bin_mapping(n, t, c)[0] if t > 1 else 0 for n, t, c in zip(extents, topology, coords))


def merge_topology(a, b):
    if int(np.prod(a)) == 1:
        return tuple(a)
    diff = [i for i in range(len(a)) if a[i] != b[i]]
    if len(diff) != 2:
        raise ValueError("Input and output topologies must differ exactly two positions")
    return tuple(max(x, y) for x, y in zip(a, b))


def diff_topology(a, b):
    if int(np.prod(a)) == 1 and int(np.prod(b)) == 1:
        return 1
    diff = [i for i in range(len(a)) if a[i] != b[i]]
    if len(diff) != 1:
        raise ValueError("Input and output topologies must differ at exactly one position.")
    return max(a[diff[0]], b[diff[0]])


def buffer_extents(extents, in_topology, out_topology, layout_right=True):
    merged = merge_topology(in_topology, out_topology)
    p0 = diff_topology(merged, in_topology)
    body = tuple((n - 1) // m + 1 for n, m in zip(extents, merged))
    return (p0,) + body if layout_right else body + (p0,)


def permute_map_by_axes(src_map, axes, layout_right=True):
    axes = list(axes)
    if layout_right:
        out = [s for s in src_map if s not in axes] + axes
    else:
        ar = axes[::-1]
        out = ar + [s for s in src_map if s not in ar]
    return tuple(out[:len(src_map)])


def get_map_axes(rank, axes, layout_right=True):
    return permute_map_by_axes(tuple(range(rank)), axes, layout_right)


# ---------------------------------------------------------------------------
# pack / unpack / all2all on one rank's local array (logical numpy arrays,
# dims in the order of the block's map)
# ---------------------------------------------------------------------------
def pack(src, src_map, axis, buf_ext, layout_right=True):
    """Send buffer of one rank: Pack functor, KokkosFFT_Distributed_PackUnpack.hpp:148-250.

    ``src`` holds the rank's local data with dim i = logical axis src_map[i];
    ``buf_ext`` is the reference buffer shape ((P, b0..) for LayoutRight,
    (b0.., P) for LayoutLeft) with the b's in logical axis order."""
    D = src.ndim
    src_map = list(src_map)
    merged_size = src.shape[src_map.index(axis)]
    if layout_right:
        P, body = buf_ext[0], buf_ext[1:]
    else:
        P, body = buf_ext[-1], buf_ext[:-1]
    out = np.zeros((P,) + tuple(body), dtype=src.dtype)
    grids = np.indices(body)
    for p in range(P):
        start, length = bin_mapping(merged_size, P, p)
        sidx = []
        for k in range(D):
            if k == axis:
                sidx.append(np.where(grids[k] >= length, -1, grids[k] + start))
            else:
                sidx.append(grids[k])
        valid = np.ones(body, dtype=bool)
        for i in range(D):
            si = sidx[src_map[i]]
            valid &= (si < src.shape[i]) & (si != -1)
        gather = tuple(np.where(valid, sidx[src_map[i]], 0) for i in range(D))
        vals = src[gather]
        out[p] = np.where(valid, vals, np.zeros((), dtype=src.dtype))
    return out if layout_right else np.moveaxis(out, 0, -1)


def unpack(recv, dst_map, axis, dst_shape, dtype=None, layout_right=True, dst=None):
    """Local array of one rank from its recv buffer: Unpack functor,
    KokkosFFT_Distributed_PackUnpack.hpp:320-419.  ``dst_shape`` is the shape of
    the rank's output block in the order of ``dst_map``."""
    if not layout_right:
        recv = np.moveaxis(recv, -1, 0)
    P, body = recv.shape[0], recv.shape[1:]
    D = len(body)
    dst_map = list(dst_map)
    merged_size = dst_shape[dst_map.index(axis)]
    if dst is None:
        dst = np.zeros(dst_shape, dtype=dtype or recv.dtype)
    grids = np.indices(body)
    for p in range(P):
        start, length = bin_mapping(merged_size, P, p)
        didx = []
        for k in range(D):
            if k == axis:
                didx.append(np.where(grids[k] >= length, -1, grids[k] + start))
            else:
                didx.append(grids[k])
        valid = np.ones(body, dtype=bool)
        for i in range(D):
            di = didx[dst_map[i]]
            valid &= (di < dst_shape[i]) & (di != -1)
        target = tuple(didx[dst_map[i]][valid] for i in range(D))
        dst[target] = recv[p][valid]
    return dst


def exchange_groups(in_topology, nprocs, comm_axis, pencil):
    """For every world rank: (sub-rank, world ranks of its group by sub-rank).

    Slab: the whole communicator.  Pencil: MPI_Cart_create over the non-one
    entries of the input topology (row-major, reorder = 0) and MPI_Cart_sub
    keeping dim 0 (row_comm, comm_axis 0) or dim 1 (col_comm, comm_axis 1)."""
    out = []
    if not pencil:
        for r in range(nprocs):
            out.append((r, list(range(nprocs))))
        return out
    dims = [t for t in in_topology if t > 1]
    t0, t1 = dims
    for r in range(nprocs):
        c0, c1 = divmod(r, t1)
        if comm_axis == 0:
            out.append((c0, [j * t1 + c1 for j in range(t0)]))
        else:
            out.append((c1, [c0 * t1 + j for j in range(t1)]))
    return out


def all2all(sends, groups, layout_right=True):
    """recv_r[j] = send_{g_r[j]}[s(r)]  (MPI_Alltoall with equal counts)."""
    recvs = []
    for r, (sub, members) in enumerate(groups):
        parts = []
        for j, src in enumerate(members):
            s = sends[src]
            parts.append(s[sub] if layout_right else s[..., sub])
        recvs.append(np.stack(parts, axis=0 if layout_right else -1))
    return recvs


# ---------------------------------------------------------------------------
# global transforms
# ---------------------------------------------------------------------------
def global_fft(x, axes, real_input, norm="backward", workers=None):
    """Global forward transform the reference's tests compare against
    (KokkosFFT::rfftn / fftn with the given normalisation; "none" scales by 1
    in both directions).  FP64 pocketfft: numpy's, or scipy's (the same
    library, multi-threaded) when `workers` is given for large grids."""
    x = np.asarray(x)
    npn = "backward" if norm == "none" else norm
    if workers is not None:
        import scipy.fft as sf
        if real_input:
            return sf.rfftn(x.astype(np.float64), axes=axes, norm=npn, workers=workers)
        return sf.fftn(x.astype(np.complex128), axes=axes, norm=npn, workers=workers)
    if real_input:
        return np.fft.rfftn(x.astype(np.float64), axes=axes, norm=npn)
    return np.fft.fftn(x.astype(np.complex128), axes=axes, norm=npn)


def global_ifft(X, axes, real_input, real_shape=None, norm="backward", workers=None):
    X = np.asarray(X).astype(np.complex128)
    npn = "forward" if norm == "none" else norm  # "forward" leaves the inverse unscaled
    if workers is not None:
        import scipy.fft as sf
        if real_input:
            return sf.irfftn(X, s=[real_shape[a] for a in axes], axes=axes, norm=npn, workers=workers)
        return sf.ifftn(X, axes=axes, norm=npn, workers=workers)
    if real_input:
        s = [real_shape[a] for a in axes]
        return np.fft.irfftn(X, s=s, axes=axes, norm=npn)
    return np.fft.ifftn(X, axes=axes, norm=npn)


def naive_dftn(x, axes, sign=-1):
    """Unnormalised multi-dimensional DFT by direct summation (small shapes)."""
    y = np.asarray(x).astype(np.complex128)
    for a in axes:
        n = y.shape[a]
        k = np.arange(n)
        W = np.exp(sign * 2j * np.pi * np.outer(k, k) / n)
        y = np.moveaxis(np.tensordot(W, np.moveaxis(y, a, 0), axes=(1, 0)), 0, a)
    return y


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


# ---------------------------------------------------------------------------
# literal execution of the reference block sequence with virtual ranks
# ---------------------------------------------------------------------------
def _local_fft(x, fft_dim, first_fft, real_input, forward, layout_right, real_len=None, workers=None):
    D = x.ndim
    dims = list(range(D - fft_dim, D)) if layout_right else list(range(fft_dim))[::-1]
    # the last entry of `axes` is transformed as the real one: make it the
    # innermost (unit-stride) dim
    if workers:
        import scipy.fft as F  # pocketfft with a thread pool
        kw = dict(workers=workers)
    else:
        F, kw = np.fft, {}
    if forward:
        if first_fft and real_input:
            return F.rfftn(x, axes=dims, **kw)
        return F.fftn(x, axes=dims, **kw)
    if first_fft and real_input:
        s = [x.shape[d] for d in dims]
        s[-1] = real_len
        return F.irfftn(x, s=s, axes=dims, **kw) * np.prod(s)
    return F.ifftn(x, axes=dims, **kw) * np.prod([x.shape[d] for d in dims])


def execute_literal(x_global, plan_info, forward=True, record=None, workers=None):
    """Run the reference block walk on the host.

    ``plan_info``: dict with keys in_extents, out_extents, axes, in_topology,
    out_topology, real_input, norm, layout_right, pencil, chain (topologies),
    chain_layouts, blocks (block list of every rank: list over ranks of lists
    of dicts like Plan.block_infos).  ``x_global`` is the global input (forward)
    or global spectrum (backward).  Returns the global result; when ``record``
    is a dict, the per-rank pack inputs, send / recv buffers and unpack outputs
    of every transpose block are stored in it by block index."""
    pi = plan_info
    D = len(pi["in_extents"])
    P = int(np.prod(pi["in_topology"]))
    real = pi["real_input"]
    right = pi["layout_right"]
    blocks = pi["blocks"]
    nb = len(blocks[0])
    chain = [tuple(t) for t in pi["chain"]]
    flags = pi["chain_layouts"]
    gin, gout = tuple(pi["in_extents"]), tuple(pi["out_extents"])
    ident = tuple(range(D))
    topo_index = []
    t = 0
    for b in blocks[0]:
        topo_index.append(t)
        if b["block_type"] == "Transpose":
            t += 1

    def box(gext, topo, flag, r):
        st = local_starts(gext, topo, r, flag)
        ex = local_extents(gext, topo, r, flag)
        return tuple(slice(s, s + e) for s, e in zip(st, ex))

    fft_ext = [max(gin[a], gout[a]) for a in pi["axes"]]
    N = float(np.prod(fft_ext))
    norm = pi.get("norm", "backward")
    if forward:
        scale = {"backward": 1.0, "forward": 1.0 / N, "ortho": 1.0 / np.sqrt(N), "none": 1.0}[norm]
        # per-rank local arrays in the input topology, logical order
        loc = [np.array(x_global[box(gin, pi["in_topology"], pi.get("in_right", True), r)]) for r in range(P)]
        cur_map = ident
        n_fft = 0
        for i, b in enumerate(blocks[0]):
            k = topo_index[i]
            if b["block_type"] == "FFT":
                if tuple(b["in_map"]) != cur_map:
                    loc = [np.ascontiguousarray(np.transpose(np.transpose(l, np.argsort(cur_map)), b["in_map"]))
                           for l in loc]
                    cur_map = tuple(b["in_map"])
                loc = [_local_fft(l, b["fft_dim"], n_fft == 0, real, True, right, workers=workers) for l in loc]
                n_fft += 1
            else:
                pencil = pi["pencil"]
                groups = exchange_groups(pi["in_topology"], P, b["comm_axis"], pencil)
                bext = blocks[0][i]["buffer_extents"]
                sends = [pack(loc[r], b["in_map"], b["in_axis"], bext, right) for r in range(P)]
                recvs = all2all(sends, groups, right)
                outs = []
                for r in range(P):
                    shape = tuple(blocks[r][i]["out_extents"])
                    outs.append(unpack(recvs[r], b["out_map"], b["out_axis"], shape, dtype=loc[r].dtype,
                                       layout_right=right))
                if record is not None:
                    record[i] = dict(pack_in=loc, send=sends, recv=recvs, unpack_out=outs)
                loc = outs
                cur_map = tuple(b["out_map"])
        # final local transpose to the natural order
        loc = [np.transpose(l, np.argsort(cur_map)) for l in loc]
        out = np.zeros(gout, dtype=np.result_type(loc[0].dtype, np.complex64))
        fl = flags[-1] if pi["pencil"] else True
        for r in range(P):
            out[box(gout, pi["out_topology"], pi.get("out_right", fl), r)] = loc[r]
        return out * scale
    # backward
    scale = {"backward": 1.0 / N, "forward": 1.0, "ortho": 1.0 / np.sqrt(N), "none": 1.0}[norm]
    loc = [np.array(x_global[box(gout, pi["out_topology"], pi.get("out_right", True), r)]) for r in range(P)]
    cur_map = ident
    for ii in range(nb - 1, -1, -1):
        b = blocks[0][ii]
        if b["block_type"] == "FFT":
            if tuple(b["in_map"]) != cur_map:
                loc = [np.ascontiguousarray(np.transpose(np.transpose(l, np.argsort(cur_map)), b["in_map"]))
                       for l in loc]
                cur_map = tuple(b["in_map"])
            first = b["block_idx"] == 0
            real_len = None
            if first and real:
                inner = b["in_map"][-1] if right else b["in_map"][0]
                real_len = gin[inner]
            loc = [_local_fft(l, b["fft_dim"], first, real, False, right, real_len, workers=workers) for l in loc]
        else:
            pencil = pi["pencil"]
            groups = exchange_groups(pi["in_topology"], P, b["comm_axis"], pencil)
            bext = b["buffer_extents"]
            sends = [pack(loc[r], b["out_map"], b["out_axis"], bext, right) for r in range(P)]
            recvs = all2all(sends, groups, right)
            outs = []
            for r in range(P):
                shape = tuple(blocks[r][ii]["in_extents"])
                outs.append(unpack(recvs[r], b["in_map"], b["in_axis"], shape, dtype=loc[r].dtype,
                                   layout_right=right))
            if record is not None:
                record[ii] = dict(pack_in=loc, send=sends, recv=recvs, unpack_out=outs)
            loc = outs
            cur_map = tuple(b["in_map"])
    loc = [np.transpose(l, np.argsort(cur_map)) for l in loc]
    out = np.zeros(gin, dtype=loc[0].dtype)
    for r in range(P):
        out[box(gin, pi["in_topology"], pi.get("in_right", True), r)] = loc[r]
    return out * scale
