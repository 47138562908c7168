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


# --- bench.py's sharded mode (one survey, inline slabs over the ranks) -------

def _bench_rank_main(rank, world, port, out_dir):
    """One CPU rank of bench.py's sharded mode: the partition of one survey and
    the whole-job aggregation (slowest rank's time, all ranks' pairs); the
    rank's pairs come from the FP64 pair counter on its slab's columns."""
    import json
    import sys
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
        import bench
        from seisproc_b200 import synthetic
        s = synthetic.survey_3d(n_traces=3000, seed=9, n_samples=60, extent=900.0,
                                max_offset=700.0, n_il=9, n_xl=5, spacing=25.0,
                                n_diffractors=3, aperture=300.0, lateral_velocity=False)
        slabs, halos = bench.shard_partition(s, world)
        il0, il1 = slabs[rank]
        halo = halos[rank]
        il = np.arange(il0, il1)[:, None]
        xl = np.arange(s.n_xl)[None, :]
        cx = (s.origin_x + il * s.il_spacing + 0 * xl).ravel()
        cy = (s.origin_y + 0 * il + xl * s.xl_spacing).ravel()
        t_ms = np.arange(s.n_times) * s.dt_ms
        pairs_halo = O.count_pairs_fp64(s.source_x[halo], s.source_y[halo], s.receiver_x[halo],
                                        s.receiver_y[halo], cx, cy, t_ms, 2000.0,
                                        s.max_aperture_m, s.max_angle_deg)
        pairs_all = O.count_pairs_fp64(s.source_x, s.source_y, s.receiver_x, s.receiver_y, cx,
                                       cy, t_ms, 2000.0, s.max_aperture_m, s.max_angle_deg)
        ms, total = bench.shard_aggregate(10.0 + rank, float(pairs_halo), torch.device("cpu"))
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"slabs": slabs, "halo": int(halo.size), "n": s.n_traces,
                       "pairs_halo": float(pairs_halo), "pairs_all": float(pairs_all),
                       "ms": ms, "total": total}, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_bench_sharded_partition_and_aggregate_two_ranks(tmp_path):
    """bench.py --gpus 2 (sharded mode) on two gloo ranks: the slabs tile the
    inlines, each halo holds every pair of its slab (the culling loses none),
    and the whole-job figures are the slowest rank's time and the sum of the
    ranks' pairs, identical on both ranks."""
    import json
    world = 2
    mp.start_processes(_bench_rank_main, args=(world, _free_port(), str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    r = [json.load(open(tmp_path / f"rank{i}.json")) for i in range(world)]
    assert r[0]["slabs"] == r[1]["slabs"] == [[0, 5], [5, 9]]
    for x in r:
        assert x["pairs_halo"] == x["pairs_all"] > 0
        assert x["halo"] < x["n"]
    assert r[0]["ms"] == r[1]["ms"] == 11.0
    assert r[0]["total"] == r[1]["total"] == r[0]["pairs_halo"] + r[1]["pairs_halo"]
