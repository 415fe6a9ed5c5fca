// Row sharding of the candidate rows (opir_shard.h).
#include "opir_shard.h"

#include <stdexcept>
#include <string>

namespace opir {

RowShard row_shard(uint64_t other, uint32_t num_dims, uint32_t shard, uint32_t num_shards) {
  if (num_dims < 2)
    throw std::invalid_argument("row shards need a layout with further dimensions (num_dims >= 2)");
  const uint32_t h = num_dims - 1;
  if (h > 31) throw std::invalid_argument("row shards: selector tree too high");
  if (other > (1ull << h) || 2 * other < (1ull << h))
    throw std::invalid_argument("row shards: candidate count outside (2^(h-1), 2^h]");
  if (num_shards == 0 || (num_shards & (num_shards - 1)) != 0)
    throw std::invalid_argument("row shards: the shard count must be a power of two");
  uint32_t k = 0;
  while ((1u << k) < num_shards) ++k;
  if (k > h - 1)
    throw std::invalid_argument("row shards: more shards (" + std::to_string(num_shards) +
                                ") than level-1 positions (" + std::to_string(1ull << (h - 1)) +
                                ")");
  if (shard >= num_shards) throw std::invalid_argument("row shards: shard index out of range");
  RowShard r;
  r.shard = shard;
  r.num_shards = num_shards;
  r.tree_h = h - k;
  const uint64_t last = 2 * other - (1ull << h);  // rows paired at level 0
  const uint64_t offset = other - last;            // rows carried over at level 0
  const uint64_t perfect = 1ull << (h - 1);
  for (uint64_t s = shard; s < perfect; s += num_shards) {
    if (s < offset) {
      r.rows.push_back(static_cast<uint32_t>(s));
    } else {
      r.rows.push_back(static_cast<uint32_t>(2 * s - offset));
      r.rows.push_back(static_cast<uint32_t>(2 * s - offset + 1));
    }
  }
  return r;
}

}  // namespace opir
