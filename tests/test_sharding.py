"""Multi-GPU partition logic on CPU ranks (gloo, world size 2).

The sharded path splits the output inlines over the ranks, each rank migrating
its slab from the traces of its aperture halo; the demigration partials are
summed over the ranks and CGLS all-reduces its image-space inner products.  Here
the operator pair is the FP64 oracle (restricted to a slab's columns and halo
traces), so the tests check the partition and the communication, not a kernel:
slabs gathered from two ranks equal the one-process image, and two-rank CGLS
follows the one-process iterates.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import pstm_fp64 as O
from seisproc_b200 import sharding as S


def _survey(seed=5, n_tr=160, n_s=96, n_il=7, n_xl=4):
    rs = np.random.RandomState(seed)
    mx = rs.uniform(-150, 300, n_tr)
    my = rs.uniform(-100, 150, n_tr)
    off = rs.uniform(0, 250, n_tr)
    az = rs.uniform(0, 2 * np.pi, n_tr)
    sx, sy = mx - 0.5 * off * np.cos(az), my - 0.5 * off * np.sin(az)
    rx, ry = mx + 0.5 * off * np.cos(az), my + 0.5 * off * np.sin(az)
    g = dict(n_il=n_il, n_xl=n_xl, origin_x=0.0, origin_y=0.0, il_dx=25.0, il_dy=5.0,
             xl_dx=-4.0, xl_dy=20.0, n_times=80, dt_ms=4.0, n_s=n_s, aperture=180.0,
             angle=60.0, v=1800.0)
    # data in the range of the operator: demigration of a random image
    cx, cy = _cols(g, 0, n_il)
    m_true = rs.standard_normal((g["n_times"], n_il * n_xl))
    d = O.demigrate_fp64(m_true, n_s, sx, sy, rx, ry, cx, cy, _t_ms(g), g["v"], g["dt_ms"], 0.0,
                         g["aperture"], g["angle"])
    return sx, sy, rx, ry, d, g


def _cols(g, il0, il1):
    il = np.arange(il0, il1)[:, None]
    xl = np.arange(g["n_xl"])[None, :]
    x = g["origin_x"] + il * g["il_dx"] + xl * g["xl_dx"]
    y = g["origin_y"] + il * g["il_dy"] + xl * g["xl_dy"]
    return x.ravel(), y.ravel()


def _t_ms(g):
    return np.arange(g["n_times"]) * g["dt_ms"]


def _slab_ops(sx, sy, rx, ry, g, il0, il1):
    """(L_partial, L^T) of one slab with the FP64 oracle, torch float64 in/out."""
    box = S.slab_bbox(g["origin_x"], g["origin_y"], g["il_dx"], g["il_dy"], g["xl_dx"],
                      g["xl_dy"], g["n_xl"], il0, il1)
    halo = S.halo_traces(sx, sy, rx, ry, box, g["aperture"])
    cx, cy = _cols(g, il0, il1)
    t = _t_ms(g)
    n_t, w, n_xl = g["n_times"], il1 - il0, g["n_xl"]

    def L(m):
        part = O.demigrate_fp64(m.numpy().reshape(n_t, -1), g["n_s"], sx[halo], sy[halo],
                                rx[halo], ry[halo], cx, cy, t, g["v"], g["dt_ms"], 0.0,
                                g["aperture"], g["angle"])
        out = np.zeros((g["n_s"], sx.shape[0]))
        out[:, halo] = part
        return torch.from_numpy(out)

    def Lt(r):
        img, _ = O.migrate_fp64(r.numpy()[:, halo], sx[halo], sy[halo], rx[halo], ry[halo], cx,
                                cy, t, g["v"], g["dt_ms"], 0.0, g["aperture"], g["angle"])
        return torch.from_numpy(img.reshape(n_t, w, n_xl))

    return L, Lt, halo


def test_inline_slabs_cover_once():
    for n_il, world in [(7, 2), (200, 8), (5, 5), (9, 4)]:
        sl = S.inline_slabs(n_il, world)
        assert sl[0][0] == 0 and sl[-1][1] == n_il
        assert all(a[1] == b[0] for a, b in zip(sl, sl[1:]))
        sizes = [b - a for a, b in sl]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        S.inline_slabs(0, 2)


def test_halo_holds_every_contributing_trace():
    sx, sy, rx, ry, _, g = _survey(seed=11, n_tr=2000)
    for il0, il1 in S.inline_slabs(g["n_il"], 3):
        box = S.slab_bbox(g["origin_x"], g["origin_y"], g["il_dx"], g["il_dy"], g["xl_dx"],
                          g["xl_dy"], g["n_xl"], il0, il1)
        halo = set(S.halo_traces(sx, sy, rx, ry, box, g["aperture"]).tolist())
        cx, cy = _cols(g, il0, il1)
        for x, y in zip(cx, cy):
            need = np.nonzero((np.hypot(sx - x, sy - y) < g["aperture"])
                              & (np.hypot(rx - x, ry - y) < g["aperture"]))[0]
            assert set(need.tolist()) <= halo
        assert len(halo) < sx.shape[0]  # the culling drops far traces


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sx, sy, rx, ry, d, g = _survey()
        slabs = S.inline_slabs(g["n_il"], world)
        il0, il1 = slabs[rank]
        L, Lt, _ = _slab_ops(sx, sy, rx, ry, g, il0, il1)
        local = Lt(torch.from_numpy(d))
        full = S.gather_slabs(local, slabs)
        m, hist = S.distributed_cgls(L, Lt, torch.from_numpy(d),
                                     (g["n_times"], il1 - il0, g["n_xl"]), n_iter=3)
        m_full = S.gather_slabs(m, slabs)
        if rank == 0:
            np.savez(os.path.join(out_dir, "two_rank.npz"), image=full.numpy(),
                     m=m_full.numpy(), res=np.array([h[1] for h in hist]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_and_cgls_match_one_process(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    got = np.load(tmp_path / "two_rank.npz")
    sx, sy, rx, ry, d, g = _survey()
    L, Lt, halo = _slab_ops(sx, sy, rx, ry, g, 0, g["n_il"])
    full = Lt(torch.from_numpy(d)).numpy()
    assert np.allclose(got["image"], full, rtol=1e-12, atol=1e-12 * np.abs(full).max())
    m1, hist1 = S.distributed_cgls(L, Lt, torch.from_numpy(d),
                                   (g["n_times"], g["n_il"], g["n_xl"]), n_iter=3)
    res1 = np.array([h[1] for h in hist1])
    assert np.allclose(got["res"], res1, rtol=1e-9)
    assert np.linalg.norm(got["m"] - m1.numpy()) <= 1e-9 * np.linalg.norm(m1.numpy())
    assert res1[-1] < 0.8  # the iterations reduce the misfit
