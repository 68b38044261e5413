"""The multi-GPU sharding logic (sidr/dist.py) with world_size 2 on the CPU
(gloo): contiguous rule shards, the fitness all_gather, max-over-ranks
timing, and two ranks stepping the same GP in lockstep from gathered
fitness."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from sidr import dist as D


def test_shard_range_covers_every_rule_once():
    for P in (0, 1, 7, 1024, 1025):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                lo, hi = D.shard_range(P, r, world)
                seen.extend(range(lo, hi))
            assert seen == list(range(P))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from sidr import gp
        from sidr.workload import MENU29
        sess = gp.Session(MENU29, 7, population=37)

        def fake_eval(idx):
            # a deterministic stand-in for the evaluator: depends on the rule only
            pk = sess.packed()
            return [float(pk.lengths[i] * 3 + (pk.ops[pk.offsets[i]] % 5)) for i in idx]

        history = []
        for g in range(3):
            f = D.sharded_fitness(fake_eval, 37)
            history.append(f)
            sess.step(f)
        t = D.max_over_ranks(float(rank + 1) * 0.5)
        np.save(os.path.join(out_dir, f"r{rank}.npy"),
                np.concatenate([np.concatenate(history), [t], [len(sess.text())]]))
        with open(os.path.join(out_dir, f"pop{rank}.txt"), "w") as fh:
            fh.write("\n".join(sess.text()))
    finally:
        dist.destroy_process_group()


def test_two_ranks_stay_in_lockstep(tmp_path):
    port = _free_port()
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    a = np.load(tmp_path / "r0.npy")
    b = np.load(tmp_path / "r1.npy")
    assert np.array_equal(a, b)
    assert a[-2] == 1.0  # max over ranks of 0.5, 1.0
    assert (tmp_path / "pop0.txt").read_text() == (tmp_path / "pop1.txt").read_text()
    # the gathered fitness equals the unsharded computation
    from sidr import gp
    from sidr.workload import MENU29
    sess = gp.Session(MENU29, 7, population=37)
    for g in range(3):
        pk = sess.packed()
        f = np.array([float(pk.lengths[i] * 3 + (pk.ops[pk.offsets[i]] % 5)) for i in range(37)])
        assert np.array_equal(f, a[37 * g:37 * (g + 1)])
        sess.step(f)


def _gp_worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import sidr
        from sidr import workload
        w = workload.gp_generation(P=1, S=1)
        ctx = sidr.Context(w.sd, sidr.zstats(w.sd))
        sess, best = D.sharded_gp(ctx, workload.MENU29, w.mask, seed=2, generations=3,
                                  population=48, train_samples=8)
        np.save(os.path.join(out_dir, f"best{rank}.npy"), best)
        with open(os.path.join(out_dir, f"gp{rank}.txt"), "w") as fh:
            fh.write("\n".join(sess.text()))
        ctx.close()
    finally:
        dist.destroy_process_group()


import pytest  # noqa: E402

from conftest import cuda_available  # noqa: E402


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA device")
def test_sharded_gp_matches_the_seed_batched_driver(tmp_path):
    """The GP with rule shards over two ranks (both on this run's one GPU,
    gloo between them) evolves exactly as the seed-batched driver does in one
    process: same best train fitness every generation, same population."""
    port = _free_port()
    mp.spawn(_gp_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    b0, b1 = np.load(tmp_path / "best0.npy"), np.load(tmp_path / "best1.npy")
    assert np.array_equal(b0, b1)
    assert (tmp_path / "gp0.txt").read_text() == (tmp_path / "gp1.txt").read_text()
    import sidr
    from sidr import gp, workload
    w = workload.gp_generation(P=1, S=1)
    ctx = sidr.Context(w.sd, sidr.zstats(w.sd))
    res = gp.run_batched(ctx, workload.MENU29, w.mask, 1, first_seed=2, population=48,
                         generations=3, train_samples=8, test_samples=4)
    ctx.close()
    assert np.array_equal(res.best_train[:, 0], b0)
