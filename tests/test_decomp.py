"""CPU: the host-side plumbing of the domain-decomposed path, with gloo ranks.

The library cuts the lattice into t slabs, one per process and GPU
(QPHIX_init with machsize {1,1,1,P}).  Without a second GPU here, the parts
that do not need one run as 2 and 3 gloo processes on CPU:
  * the slab of a global MILC raw array is a slice of each parity block,
    and the slices gather back to the global array;
  * the face exchange in the library's order (send the first three
    t-slices to the previous rank, receive the next rank's into the forward
    ghost, send the last three to the next rank, receive the previous
    rank's into the backward ghost -- nccl_exchange in csrc/comm.cu), with
    the library's face layout (k_halo_pack), gives every rank exactly the
    periodic window t = -3 .. Lt+2 of the global field: with two ranks both
    neighbours are the same process, so the pairing of the four messages
    matters;
  * a dot product summed over the ranks (the allreduce after each split
    reduction) equals the global one.
The device side (pack kernel, ghost reads, interior/boundary split) runs on
one GPU in the loopback tests of test_gpu_halo.py.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _field(dims, seed):
    V = int(np.prod(dims))
    return np.random.default_rng(seed).standard_normal(V * 6)


def _rank_main(rank, world, port, dims, q):
    import sys

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import __graft_entry__ as entry

    entry.load_package()
    from milc_qphix_b200 import decomp

    dist.init_process_group("gloo", rank=rank, world_size=world, init_method=f"tcp://127.0.0.1:{port}")
    try:
        out = {}
        glob = _field(dims, 7)
        other = _field(dims, 8)
        ldims = decomp.slab_dims(dims, world)
        loc = decomp.scatter(dims, glob, world, rank, 6)
        lo2 = decomp.scatter(dims, other, world, rank, 6)
        out["local_len"] = loc.size
        prev, nxt = (rank - 1) % world, (rank + 1) % world
        ok = True
        for parity in ("even", "odd"):
            back, fwd = decomp.pack_faces(ldims, loc, parity)
            tb = torch.from_numpy(np.ascontiguousarray(back).view(np.float64).copy())
            tf = torch.from_numpy(np.ascontiguousarray(fwd).view(np.float64).copy())
            gfwd = torch.empty_like(tb)
            gback = torch.empty_like(tf)
            reqs = [dist.isend(tb, prev), dist.irecv(gfwd, nxt), dist.isend(tf, nxt), dist.irecv(gback, prev)]
            for r in reqs:
                r.wait()
            gb = gback.numpy().view(np.complex128).reshape(3, -1)
            gf = gfwd.numpy().view(np.complex128).reshape(3, -1)
            ext = decomp.extend(ldims, loc, parity, gb, gf)
            want = decomp.periodic_window(dims, glob, world, rank, parity)
            ok &= bool(np.array_equal(ext, want))
        out["halo_ok"] = ok
        # a dot product of the even parity blocks, summed over the ranks
        Vl = int(np.prod(ldims))
        d = torch.tensor([float(loc[: 3 * Vl] @ lo2[: 3 * Vl])], dtype=torch.float64)
        dist.all_reduce(d)
        V = int(np.prod(dims))
        out["dot"] = (float(d.item()), float(glob[: 3 * V] @ other[: 3 * V]))
        # every rank's part, gathered, is the global array
        parts = [None] * world
        dist.all_gather_object(parts, loc)
        out["gather_ok"] = bool(np.array_equal(decomp.gather(dims, parts, 6), glob))
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,dims", [(2, (8, 4, 4, 8)), (3, (4, 4, 8, 12))])
def test_slab_exchange_and_sums(world, dims):
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, dims, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    V = int(np.prod(dims))
    for r in range(world):
        assert res[r]["local_len"] * world == V * 6
        assert res[r]["halo_ok"], r
        assert res[r]["gather_ok"], r
        got, want = res[r]["dot"]
        assert abs(got - want) <= 1e-12 * abs(want)


def test_scatter_links_is_a_slice_of_each_parity_block():
    import __graft_entry__ as entry

    entry.load_package()
    from milc_qphix_b200 import decomp

    dims = (4, 4, 4, 8)
    V = int(np.prod(dims))
    raw = np.arange(V * 72, dtype=np.float64)
    parts = [decomp.scatter(dims, raw, 2, r, 72) for r in range(2)]
    st = 2 * 4 * 4
    assert np.array_equal(parts[1][: st * 4 * 72], raw[st * 4 * 72: st * 8 * 72])
    assert np.array_equal(decomp.gather(dims, parts, 72), raw)
    with pytest.raises(ValueError):
        decomp.slab_dims((4, 4, 4, 8), 3)
