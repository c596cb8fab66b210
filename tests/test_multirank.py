"""Multi-rank host logic on the CPU: two `gloo` ranks (127.0.0.1) run the same
code that `bench.py` and a sharded verify run under torchrun with one process
per GPU.  Each rank verifies its share of a seeded corpus (with the oracle
standing in for the per-rank GPU verifier, since this test runs without a
GPU), the verdict bytes are gathered in rank order, and the reductions used
for the benchmark's max-over-ranks time and summed item count are checked."""
import os
import socket

import numpy as np
import pytest

from ultrafastsecp256k1_b200.shard import shard_range


def test_shard_ranges_cover_exactly():
    for total in (0, 1, 7, 1000, 1 << 20):
        for world in (1, 2, 3, 8):
            spans = [shard_range(total, world, r) for r in range(world)]
            assert sum(n for _, n in spans) == total
            pos = 0
            for lo, n in spans:
                assert lo == pos
                pos += n
            assert max(n for _, n in spans) - min(n for _, n in spans) <= 1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, result_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    from conftest import schnorr_corpus
    from oracle import Oracle
    from ultrafastsecp256k1_b200.shard import Ranks, verify_sharded
    oracle = Oracle()
    oracle.set_threads(1)
    ranks = Ranks.from_env(device="cpu", backend="gloo", timeout_s=60)
    m, x, s = schnorr_corpus(oracle, 301, seed=5, tamper=0.1)       # odd count: ragged shares
    got = verify_sharded(oracle.schnorr_verify_batch, m, x, s, ranks)
    t_max = ranks.max(float(rank + 1) * 0.25)
    n_sum = ranks.sum(float(shard_range(301, world, rank)[1]))
    ranks.barrier()
    np.save(os.path.join(result_dir, f"r{rank}.npy"), np.concatenate([got, [int(t_max * 100), int(n_sum)]]))
    ranks.close()


def test_two_gloo_ranks_shard_and_gather(tmp_path, oracle):
    import torch.multiprocessing as mp
    from conftest import schnorr_corpus
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    m, x, s = schnorr_corpus(oracle, 301, seed=5, tamper=0.1)
    want = oracle.schnorr_verify_batch(m, x, s)
    for r in range(world):
        res = np.load(tmp_path / f"r{r}.npy")
        assert (res[:301] == want).all()
        assert res[301] == 50 and res[302] == 301          # max of 0.25, 0.5 -> 0.5; shares sum to 301
