"""One process per GPU: rank bookkeeping, reductions over ranks and sharded verify.

Verification shards by item with no exchange on the data path: each rank
verifies its own index range; the only collectives are the timing / count
reductions of a benchmark and, for a sharded call, one gather of the verdict
bytes (1 byte per item) at the end.

    ranks = Ranks.from_env(device="cuda")     # RANK / WORLD_SIZE / LOCAL_RANK from torchrun
    lo, n = shard_range(total, ranks.world, ranks.rank)
    verdicts = verify_sharded(verify_fn, msgs, pubs, sigs, ranks)

`verify_fn(msgs, pubs, sigs) -> uint8 verdicts` is any per-rank verifier, e.g.
GpuContext(local_rank).schnorr_verify_batch.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np


def shard_range(total: int, world: int, rank: int) -> tuple[int, int]:
    """(first item, item count) of `rank`'s contiguous share; shares differ by at most one."""
    base, extra = divmod(total, world)
    lo = rank * base + min(rank, extra)
    return lo, base + (1 if rank < extra else 0)


@dataclass
class Ranks:
    world: int = 1
    rank: int = 0
    local: int = 0
    device: str = "cpu"          # where reduction tensors live: "cuda" for NCCL, "cpu" for gloo

    @classmethod
    def from_env(cls, device: str = "cuda", backend: str | None = None, timeout_s: int = 180) -> "Ranks":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        local = int(os.environ.get("LOCAL_RANK", "0"))
        r = cls(world, rank, local, device)
        if world > 1:
            import torch
            import torch.distributed as dist
            from datetime import timedelta
            if not dist.is_initialized():
                be = backend or ("nccl" if device == "cuda" else "gloo")
                kw = {"timeout": timedelta(seconds=timeout_s)}
                if be == "nccl":
                    kw["device_id"] = torch.device("cuda", local)
                dist.init_process_group(be, **kw)
        return r

    def _reduce(self, v: float, op) -> float:
        if self.world == 1:
            return v
        import torch
        import torch.distributed as dist
        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=op)
        return float(t.item())

    def barrier(self) -> None:
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max(self, v: float) -> float:
        import torch.distributed as dist
        return self._reduce(v, dist.ReduceOp.MAX) if self.world > 1 else v

    def sum(self, v: float) -> float:
        import torch.distributed as dist
        return self._reduce(v, dist.ReduceOp.SUM) if self.world > 1 else v

    def gather_bytes(self, local: np.ndarray, total: int) -> np.ndarray:
        """Concatenate every rank's contiguous uint8 share (rank order) on every rank."""
        if self.world == 1:
            return local
        import torch
        import torch.distributed as dist
        width = shard_range(total, self.world, 0)[1]
        buf = torch.zeros(width, dtype=torch.uint8, device=self.device)
        buf[:len(local)] = torch.from_numpy(np.ascontiguousarray(local)).to(self.device)
        parts = [torch.zeros_like(buf) for _ in range(self.world)]
        dist.all_gather(parts, buf)
        out = [p[:shard_range(total, self.world, r)[1]].cpu().numpy() for r, p in enumerate(parts)]
        return np.concatenate(out)

    def close(self) -> None:
        if self.world > 1:
            import torch.distributed as dist
            if dist.is_initialized():
                dist.destroy_process_group()


def verify_sharded(verify_fn, msgs, pubs, sigs, ranks: Ranks) -> np.ndarray:
    """Every rank verifies its share of the items; all ranks return all verdicts."""
    total = len(msgs)
    lo, n = shard_range(total, ranks.world, ranks.rank)
    mine = np.asarray(verify_fn(msgs[lo:lo + n], pubs[lo:lo + n], sigs[lo:lo + n]), np.uint8) if n else \
        np.zeros(0, np.uint8)
    return ranks.gather_bytes(mine, total)
