// Row sharding of one database across G = 2^k GPUs.
//
// evaluate_other_dim (src/server.cpp:599-649) reduces the `other` candidate
// rows with a MUX tree of height h = num_dims - 1: level 0 pairs rows
// (offset + 2i, offset + 2i + 1) into position offset + i and carries rows
// below offset = 2^h - other over unchanged, so level 1 sees 2^(h-1)
// positions s, position s fed by row s (s < offset) or by rows
// 2s - offset and 2s - offset + 1; every level a >= 1 pairs positions i and
// i + 2^(h-a-1), the top bit of the remaining index.
//
// Shard g owns the level-1 positions s with s mod G == g and the rows that
// feed them. Its levels 0 .. h-k-1 then pair only positions it owns: the
// shard is itself a layout of height h - k whose rows are its rows in
// increasing s (the unpaired ones first, as in the full layout), answered
// by the same kernels with the global selectors 0 .. h-k-1. What is left on
// shard g is the full tree's level-(h-k) position g; the last k levels pair
// those G ciphertexts (one per shard) and run wherever they are gathered.
#pragma once

#include <algorithm>
#include <cstdint>
#include <vector>

namespace opir {

struct RowShard {
  uint32_t shard = 0, num_shards = 1;
  uint32_t tree_h = 0;            // MUX levels answered on the shard: h - log2 G
  std::vector<uint32_t> rows;     // local row -> global candidate row
};

// Throws std::invalid_argument unless G is a power of two with
// 1 <= G <= 2^(h-1) (every shard keeps at least one level-1 position),
// shard < G and the layout has a MUX tree (num_dims >= 2,
// 2^(h-1) <= other <= 2^h).
RowShard row_shard(uint64_t other, uint32_t num_dims, uint32_t shard, uint32_t num_shards);

// For the local plaintexts [pb, pe) of a handle whose rows are `rows`
// (empty = the identity), calls fill(b, e, dst) once per run of database
// plaintexts [b, e) below `logical` that sit at consecutive local positions;
// dst points at the run's first plaintext in `host` (ncoef coefficients per
// plaintext, host indexed from pb).
template <typename T, typename Fill>
void fill_runs(const std::vector<uint32_t> &rows, uint64_t n0, uint64_t logical, uint64_t pb,
               uint64_t pe, T *host, Fill &&fill, uint64_t ncoef) {
  if (rows.empty()) {
    const uint64_t e = std::min(pe, logical);
    if (pb < e) fill(pb, e, host);
    return;
  }
  for (uint64_t pt = pb; pt < pe;) {
    const uint64_t r = pt / n0, k = pt % n0;
    const uint64_t seg = std::min<uint64_t>(pe, (r + 1) * n0) - pt;
    const uint64_t gb = static_cast<uint64_t>(rows[r]) * n0 + k;
    const uint64_t ge = std::min(gb + seg, logical);
    if (gb < ge) fill(gb, ge, host + (pt - pb) * ncoef);
    pt += seg;
  }
}

}  // namespace opir
