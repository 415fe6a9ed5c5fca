// Tensor-core (tcgen05) first-dimension scan over byte-plane operands.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace opir {

struct TcScanArgs {
  uint32_t k_tiles;         // ceil(n0p / 128)
  uint32_t other;           // rows per level (candidates)
  uint32_t m_tiles;         // ceil(other / 128)
  uint32_t ncols;           // real output columns (2 x batch)
  uint32_t ntile;           // query columns per tile: 16, 32 or 64
  uint32_t col_tiles;       // ceil(ncols / ntile)
  uint32_t zcount;          // residues x levels
  uint32_t levels_per_res;  // N
  uint32_t q[2];
  uint64_t mu[2];           // floor(2^64 / q)
  uint32_t w[2][7];         // 2^(8 s) mod q
  uint32_t *cmat;           // [z][row][ncols] u32
  uint32_t *err;            // error bits (0 = ok)
};

// 3-D byte tensor [planes][rows][k_bytes] for TMA (128B swizzle, boxes of
// 128 bytes x box_rows rows); rows past `rows` read as zero.
void make_plane_map(CUtensorMap *map, const uint8_t *base, uint64_t k_bytes, uint64_t rows,
                    uint64_t planes, uint32_t box_rows);
size_t scan_tc_smem(uint32_t ntile);
void launch_scan_tc(const CUtensorMap &mapA, const CUtensorMap &mapQ, const TcScanArgs &args,
                    int sm_count, cudaStream_t st);

}  // namespace opir
