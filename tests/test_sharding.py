"""Multi-GPU sharding logic on CPU: the work-balanced partition, and a
world-size-2 gloo run of the sharded adjoint whose alignment all-reduce must
equal the single-process gradient (host build of the core, double)."""
import ctypes as C
import os
import socket
from pathlib import Path

import numpy as np
import pytest

from detray_b200 import abi, geometry, sharding, tracks
from tests import adjoint_host as ah

REPO = Path(__file__).resolve().parent.parent


def test_partition_covers_and_balances():
    rng = np.random.default_rng(1)
    w = rng.exponential(1.0, 10_001) ** 3
    for world in (1, 2, 3, 8, 16):
        parts = sharding.partition(w, world)
        assert len(parts) == world
        assert parts[0][0] == 0 and parts[-1][1] == len(w)
        for (a, b), (c, d) in zip(parts, parts[1:]):
            assert b == c and a <= b
        sums = [w[a:b].sum() for a, b in parts]
        assert max(sums) <= w.sum() / world + w.max() + 1e-9
    assert sharding.partition(np.zeros(0), 4) == [(0, 0)] * 4
    assert sharding.partition(np.ones(3), 8)[-1] == (3, 3)


def test_work_estimate_loopers_and_exits():
    trk = tracks.toy_tracks(2000, seed=3, pt_range=(0.1, 100.0))
    w = sharding.work_estimate(trk, path_limit=5000.0)
    pt = np.hypot(trk[4], trk[5]) / np.abs(trk[7])
    assert (w <= 5000.0).all() and (w > 0).all()
    # low-pT central tracks loop to the limit; stiff ones leave early
    central = np.abs(trk[6]) < 0.3
    assert np.median(w[(pt < 0.2) & central]) > 4 * np.median(w[(pt > 10) & central])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    lib = C.CDLL(str(REPO / "tests" / "native" / "libcore_host.so"))
    lib.core_host_last_error.restype = C.c_char_p
    tables = geometry.load_geometry("toy_4brl_7edc")
    cfg = abi.make_config(max_records=32, search_window=(3, 3))
    trk = tracks.toy_tracks(400, seed=77)
    local, (lo, hi) = sharding.shard(trk, rank, world)
    res, tape = ah.forward(lib, tables, cfg, local)
    full_w = np.random.default_rng(5).normal(size=(6, cfg.max_records, 400))
    W = full_w[:, :, lo:hi] * ah.transported_mask(res, cfg.max_records)
    gfree, galign = ah.backward(lib, tables, cfg, local, res, tape, W)
    loss = float((W * np.nan_to_num(res["rec_bound"])).sum())
    ga, lt = sharding.allreduce_alignment(torch.from_numpy(galign),
                                          torch.tensor(loss, dtype=torch.float64))
    np.savez(Path(out_dir) / f"rank{rank}.npz", lo=lo, hi=hi, gfree=gfree,
             galign=ga.numpy(), loss=float(lt))
    dist.destroy_process_group()


def test_two_rank_adjoint_allreduce_matches_single_process(core_host, tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)),
             nprocs=world, join=True)
    tables = geometry.load_geometry("toy_4brl_7edc")
    cfg = abi.make_config(max_records=32, search_window=(3, 3))
    trk = tracks.toy_tracks(400, seed=77)
    res, tape = ah.forward(core_host, tables, cfg, trk)
    W = (np.random.default_rng(5).normal(size=(6, cfg.max_records, 400))
         * ah.transported_mask(res, cfg.max_records))
    gfree, galign = ah.backward(core_host, tables, cfg, trk, res, tape, W)
    loss = float((W * np.nan_to_num(res["rec_bound"])).sum())
    parts = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    assert parts[0]["hi"] == parts[1]["lo"] and parts[1]["hi"] == 400
    assert 0 < parts[0]["hi"] < 400
    for p in parts:
        np.testing.assert_allclose(p["galign"], galign, rtol=1e-10, atol=1e-12)
        assert float(p["loss"]) == pytest.approx(loss, rel=1e-12)
        lo, hi = int(p["lo"]), int(p["hi"])
        np.testing.assert_array_equal(p["gfree"], gfree[:, lo:hi])
