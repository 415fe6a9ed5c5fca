// Tensor-core (tcgen05) first-dimension scan over byte-plane operands.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace opir {

struct TcScanArgs {
  uint32_t k_tiles;         // ceil(n0p / kt)
  uint32_t kt;              // K bytes per pipeline stage: 128 or 64 (= swizzle width)
  uint32_t stages;          // pipeline stages (2 .. scan_tc_max_stages)
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
  uint32_t *cmat;           // [z][column][row] u32
  uint32_t *err;            // error bits (0 = ok)
  long long wait_cycles;    // limit of each pipeline wait (clock cycles)
};

// 3-D byte tensor [planes][rows][k_bytes] for TMA (box_k-byte swizzle, boxes
// of box_k bytes x box_rows rows, box_k = 128 or 64); rows past `rows` read
// as zero.
void make_plane_map(CUtensorMap *map, const uint8_t *base, uint64_t k_bytes, uint64_t rows,
                    uint64_t planes, uint32_t box_rows, uint32_t box_k);
size_t scan_tc_smem(uint32_t ntile, uint32_t kt, uint32_t stages);
// Most pipeline stages that fit the shared memory of one block.
uint32_t scan_tc_max_stages(uint32_t ntile, uint32_t kt);
void launch_scan_tc(const CUtensorMap &mapA, const CUtensorMap &mapQ, const TcScanArgs &args,
                    int sm_count, cudaStream_t st);

// Recombination-rate probe (the scan epilogue's arithmetic on register
// values, `classes` = 5 or 7 shift classes): blocks of 256 threads that fill
// `sms` SMs, and a launch of `iters` iterations into sink (blocks x 256 u32).
// Returns the outputs the launch finishes.
uint32_t recombine_rate_blocks(int sms, int classes);
uint64_t launch_recombine_rate(uint32_t *sink, uint32_t blocks, uint32_t iters, int classes,
                               cudaStream_t st);

}  // namespace opir
