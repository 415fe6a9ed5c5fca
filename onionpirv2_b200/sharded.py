"""One database split by candidate rows across the ranks of a
torch.distributed process group (one rank per GPU).

Rank r holds row shard r of G = world size (RowShardServer,
opir_server_create_row_shard): the rows that feed the level-1 MUX positions
s with s mod G == r. Every rank expands each query itself (the expansion and
the selectors are the same on every shard), scans its rows and runs its MUX
levels, leaving one partial ciphertext per query. The one exchange of the
path is a gather of those G partials (one ciphertext per query and rank,
32 KiB under CONFIG_N2048_K1_COMP) to the root rank, which runs the last
log2 G MUX levels and the modulus switch. The responses equal
PirServer::make_query's (src/server.cpp:895-947) bit for bit.

The reference has no multi-GPU form; this module only orchestrates the C ABI
calls and the collective. `engine` exists so that the orchestration can be
exercised without a GPU; the default is the CUDA implementation.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np
import torch
import torch.distributed as dist

from .server import PirParams, RowShardServer


class ShardedServer:
    """make_query over a row-sharded database. Call every method on every
    rank of `group` in the same order (the query calls are collective);
    results are returned on `root` only (None elsewhere)."""

    def __init__(self, params: PirParams, group=None, root: int = 0, device: int | None = None,
                 engine=None):
        self.params = params
        self.group = group
        self.root = root
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.device = torch.cuda.current_device() if device is None and engine is None else device
        self.engine = engine if engine is not None else RowShardServer(
            params, self.rank, self.world, device=self.device)

    # ---- database and keys (local to each rank's shard)
    def load_data(self, logical_num_pt: int, source):
        self.engine.load_data(logical_num_pt, source)

    def load_data_seeded(self, logical_num_pt: int, seed: int):
        self.engine.load_data_seeded(logical_num_pt, seed)

    def set_client_keys(self, client_id: int, bv_keys: np.ndarray, gsw_key: np.ndarray):
        self.engine.set_client_keys(client_id, bv_keys, gsw_key)

    # ---- queries
    def _gather(self, t: torch.Tensor) -> list[torch.Tensor] | None:
        bucket = [torch.empty_like(t) for _ in range(self.world)] if self.rank == self.root else None
        dist.gather(t, bucket, dst=self.root, group=self.group)
        return bucket

    def make_query_batch(self, client_ids: Sequence[int], queries: np.ndarray) -> np.ndarray | None:
        """Host buffers: every rank passes the same client ids and queries;
        the root returns the (n, 2, N) responses."""
        partials = self.engine.make_query_shard_batch(client_ids, queries)
        t = torch.from_numpy(np.ascontiguousarray(partials).view(np.int64))
        if dist.get_backend(self.group) == "nccl":
            t = t.to(torch.device("cuda", torch.cuda.current_device()))
        bucket = self._gather(t)
        if bucket is None:
            return None
        stacked = torch.stack(bucket).cpu().numpy().view(np.uint64)
        return self.engine.combine_shards(client_ids, stacked)

    def make_query_batch_device(self, client_ids: Sequence[int], d_queries: torch.Tensor,
                                d_responses: torch.Tensor | None = None) -> torch.Tensor | None:
        """Device buffers on this rank's GPU, on torch's current stream:
        d_queries (n,) + ct_shape int64; the root returns (n, 2, N) int64
        responses (written into d_responses when given)."""
        n = len(client_ids)
        stream = torch.cuda.current_stream().cuda_stream
        partial = torch.empty((n,) + self.params.ct_shape, dtype=torch.int64, device=d_queries.device)
        self.engine.make_query_shard_batch_device(client_ids, d_queries.data_ptr(),
                                                  partial.data_ptr(), stream)
        bucket = self._gather(partial)
        if bucket is None:
            return None
        stacked = torch.stack(bucket)
        if d_responses is None:
            d_responses = torch.empty((n, 2, self.params.N), dtype=torch.int64,
                                      device=d_queries.device)
        self.engine.combine_shards_device(client_ids, stacked.data_ptr(), d_responses.data_ptr(),
                                          stream)
        return d_responses
