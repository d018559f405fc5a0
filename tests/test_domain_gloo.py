"""Domain decomposition in t-slabs (rhmc_b200/domain.py) with the gloo backend, world size 2, on
CPU: each rank owns half of the time slices of a 4x4x4x8 lattice, exchanges its link ghost slice
once and one spinor face each way per half-Dslash, and all-reduces its FP64 dot products.  The
local half-Dslash on each rank's extended lattice is the oracle's (lib/Action/fermionmatrix.cc:
8-97 restated), so what is tested is the decomposition: ghost exchange, the slab's parity and index
maps, and the global reductions.  Against the single-domain oracle: both half-Dslash and M^dag M
agree to 1e-14, the multi-shift CG (inverter.cc:142-339 recurrences) to 1e-9 with the same
iteration count to within one.  Not run on several GPUs here (one GPU per job on this pool)."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


DIMS = (4, 4, 4, 8)
MASS = 0.1
SHIFTS = [0.003, 0.05, 0.7, 9.0]


def _rank_main(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "rhmc-on-gpu_b200"))
    sys.path.insert(0, os.path.join(root, "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import torch
    import torch.distributed as dist
    import oracle
    from rhmc_b200 import domain as D
    from rhmc_b200 import fields as F
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        u = F.random_links(DIMS, seed=1001)
        x = F.random_spinor(DIMS, seed=2002)
        slab = D.TSlab(DIMS, rank, world)
        # links: interior from the global field, ghost slice by exchange
        u_full = slab.links_from_global(u)
        u_ext = torch.from_numpy(slab.links_from_global(u, ghosts=False))
        op0 = D.DDOperator(slab, MASS, None, dist)
        op0.exchange_link_ghosts(u_ext)
        links_ok = bool(np.array_equal(u_ext.numpy(), u_full))
        orc_loc = oracle.Oracle(slab.dims_ext)
        ue = u_ext.numpy()

        # the oracle library keeps one lattice geometry at a time: re-initialise before each use
        def local_dslash(p_ext, out, inp):
            orc_loc._reinit()
            f = orc_loc.deo if p_ext == 0 else orc_loc.doe
            out[:] = torch.from_numpy(f(ue, inp.numpy()))

        op = D.DDOperator(slab, MASS, local_dslash, dist)
        orc = oracle.Oracle(DIMS)
        a, b = slab.local_slice()
        xl = torch.from_numpy(x[a:b].copy())
        doe = op.dslash(1, xl).numpy()
        deo = op.dslash(0, xl).numpy()  # x read as an odd field: D_eo of it
        mdm = op.mdagm(xl, 0.37).numpy()
        halo = op.halo_bytes
        xs, it = D.multishift_cg(op, xl, SHIFTS, 1e-10)
        orc._reinit()
        err_doe = np.abs(doe - orc.doe(u, x)[a:b]).max()
        err_deo = np.abs(deo - orc.deo(u, x)[a:b]).max()
        err_mdagm = np.abs(mdm - orc.mdagm(u, x, MASS, 0.37)[a:b]).max()
        xr, itr = orc.msolve(u, x, MASS, np.array(SHIFTS), 1e-10)
        err_ms = max(np.linalg.norm(xs[i].numpy() - xr[i][a:b]) / np.linalg.norm(xr[i][a:b]) for i in range(len(SHIFTS)))
        q.put((rank, links_ok, err_doe, err_deo, err_mdagm, halo, it, int(itr), err_ms))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_tslab_decomposition_two_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=280) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    face_bytes = (4 * 4 * 4 // 2) * 3 * 16
    for rank, links_ok, e1, e2, e3, halo, it, itr, ems in res:
        assert links_ok, rank
        assert e1 < 1e-14 and e2 < 1e-14 and e3 < 1e-13, (rank, e1, e2, e3)
        assert halo == 4 * 2 * face_bytes  # 4 half-Dslash, one face each way
        assert abs(it - itr) <= 1, (it, itr)
        assert ems < 1e-9, ems


def test_tslab_geometry():
    import torch
    from rhmc_b200 import domain as D
    s = D.TSlab((4, 4, 4, 8), 1, 2)
    assert (s.nt_loc, s.t0, s.face, s.Vh_loc, s.Vh_ext) == (4, 4, 32, 128, 192)
    assert s.local_slice() == (128, 256) and s.interior() == (32, 160)
    assert s.ext_parity(0) == 1
    with pytest.raises(ValueError):
        D.TSlab((4, 4, 4, 6), 0, 2)  # 3 slices per rank: parity would not be preserved
    e = s.extend(torch.ones(128, 3, dtype=torch.complex128))
    assert e.shape == (192, 3) and float(e[:32].abs().sum()) == 0.0 and float(e[32:160].abs().sum()) == 384.0
