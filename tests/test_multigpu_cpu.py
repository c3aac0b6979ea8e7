"""The multi-rank host path on CPU: world size 2 over gloo, one process per rank.

Query shards: each rank evaluates its pixel tiles of one iteration's queries (the oracle stands in
for the device evaluation, which needs a GPU) over the whole photon and beam records, and one
all-reduce (sum) of the framebuffers must give the serial image of the iteration.

Whole iterations: each rank runs its round-robin share of the iterations, and
``multi.combine_framebuffers`` must give the reference's final framebuffer: the mean over renderers
of each renderer's mean over its iterations (``SmallUPBP.cxx:143-176``, ``Renderer.hxx:55-61``).
"""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CFG = "cube16x512"


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _image(iteration: int) -> np.ndarray:
    from oracle import port
    from smallupbp_b200 import workload as W

    w = W.generate(W.config(CFG), iteration=iteration)
    return port.run(w)["image"].astype(np.float64)


def _rank_main(rank, world, port, total, out_dir):
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    from smallupbp_b200 import multi

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    its = multi.split_iterations(total, rank, world)
    acc = None
    for it in its:
        img = _image(it)
        acc = img if acc is None else acc + img
    shape = _image_shape()
    t = torch.from_numpy(acc.reshape(-1) if acc is not None else np.zeros(int(np.prod(shape))))
    multi.combine_framebuffers(t, len(its))
    slow = multi.max_over_ranks(10.0 * (rank + 1), "cpu")
    units = multi.sum_over_ranks(len(its), "cpu")
    np.save(os.path.join(out_dir, "rank%d.npy" % rank), t.numpy())
    np.save(os.path.join(out_dir, "rank%d_stats.npy" % rank), np.array([slow, units]))
    dist.destroy_process_group()


def _shard_rank_main(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist
    from oracle import port as oport
    from smallupbp_b200 import multi
    from smallupbp_b200 import workload as W

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    cfg = W.config(CFG)
    w = multi.shard_workload(W.generate(cfg, iteration=0), cfg.width, rank, world, tile=4)
    t = torch.from_numpy(oport.run(w)["image"].astype(np.float64).reshape(-1))
    dist.all_reduce(t)
    units = multi.sum_over_ranks(len(w["sq_path_length"]) + len(w["pq_path_length"]), "cpu")
    np.save(os.path.join(out_dir, "shard%d.npy" % rank), t.numpy())
    np.save(os.path.join(out_dir, "shard%d_units.npy" % rank), np.array([units]))
    dist.destroy_process_group()


def test_query_shards_partition_the_queries():
    from smallupbp_b200 import multi
    from smallupbp_b200 import workload as W

    cfg = W.config(CFG)
    w = W.generate(cfg, iteration=0)
    for world in (1, 2, 3, 8):
        for key in ("sq_pixel", "pq_pixel"):
            parts = [multi.query_shard(w[key], cfg.width, r, world, tile=4) for r in range(world)]
            allq = np.sort(np.concatenate(parts))
            np.testing.assert_array_equal(allq, np.arange(len(w[key])))
            if world > 1 and key == "sq_pixel":
                sizes = np.array([len(p) for p in parts])
                assert sizes.min() > 0.5 * sizes.mean(), sizes
    s = multi.shard_workload(w, cfg.width, 1, 2, tile=4)
    assert len(s["sq_origin"]) == len(s["sq_pixel"]) < len(w["sq_pixel"])
    assert s["seg_dist_min"] is w["seg_dist_min"] and s["beam_origin"] is w["beam_origin"]
    with pytest.raises(ValueError):
        multi.query_shard(w["sq_pixel"], cfg.width, 2, 2)


def test_two_query_shards_sum_to_the_serial_image(tmp_path):
    from oracle import port as oport
    from smallupbp_b200 import workload as W

    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    w = W.generate(W.config(CFG), iteration=0)
    want = oport.run(w)["image"].astype(np.float64).reshape(-1)
    assert np.abs(want).max() > 0
    for r in range(2):
        got = np.load(os.path.join(tmp_path, "shard%d.npy" % r))
        np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-7 * np.abs(want).max())
        units = np.load(os.path.join(tmp_path, "shard%d_units.npy" % r))[0]
        assert units == len(w["sq_path_length"]) + len(w["pq_path_length"])


def _image_shape():
    from smallupbp_b200 import workload as W

    c = W.config(CFG)
    return (c.width * c.height, 3)


def _launch(world, total, tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, total, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    return [np.load(os.path.join(tmp_path, "rank%d.npy" % r)) for r in range(world)], \
           [np.load(os.path.join(tmp_path, "rank%d_stats.npy" % r)) for r in range(world)]


def test_rank_iteration_assignment():
    from smallupbp_b200 import multi

    assert multi.rank_iterations(1, 4, 3) == [1, 5, 9]
    assert multi.split_iterations(5, 0, 2) == [0, 2, 4]
    assert multi.split_iterations(5, 1, 2) == [1, 3]
    everything = sorted(i for r in range(3) for i in multi.split_iterations(10, r, 3))
    assert everything == list(range(10))
    with pytest.raises(ValueError):
        multi.rank_iterations(2, 2, 1)


def test_two_ranks_combine_to_the_serial_framebuffer(tmp_path):
    total = 4
    imgs, stats = _launch(2, total, tmp_path)
    # ranks: {0, 2} and {1, 3}; each renderer's mean, then the mean over renderers
    per = [_image(i) for i in range(total)]
    want = (((per[0] + per[2]) / 2 + (per[1] + per[3]) / 2) / 2).reshape(-1)
    assert np.abs(want).max() > 0
    for img in imgs:
        # the framebuffers are FP32 sums: compared at FP32 precision
        np.testing.assert_allclose(img, want, rtol=1e-6, atol=1e-12)
    for s in stats:
        assert s[0] == 20.0          # max over ranks
        assert s[1] == total         # units over ranks


def test_rank_without_iterations_does_not_count(tmp_path):
    imgs, _ = _launch(2, 1, tmp_path)  # rank 1 runs nothing, as an unused renderer
    want = _image(0).reshape(-1)
    for img in imgs:
        np.testing.assert_allclose(img, want, rtol=1e-6, atol=1e-12)
