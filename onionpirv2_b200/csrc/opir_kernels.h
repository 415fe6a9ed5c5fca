// Host-callable launchers for the sm_100a kernels of the OnionPIRv2 server
// path. All launches are asynchronous on the given stream.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "opir_device.cuh"

namespace opir {

// Shape of one make_query call (derived from PirParams).
struct Shape {
  uint32_t n0;          // fst_dim_sz
  uint32_t other;       // other_dim_sz
  uint32_t num_dims;
  uint32_t h;           // expansion height
  uint32_t useful;      // n0 + l_ep (num_dims - 1)
  uint32_t l_ep, l_key, l_ks;
  uint32_t base_ep, base_key, base_ks;
  uint32_t n0p;         // n0 rounded up to 16 (byte-plane row length)
  uint32_t gadget;      // 0: CONFIG_N2048_K1_COMP gadgets, 1: CONFIG_N2048_K2_MP gadgets
  uint64_t num_pt;
  // cluster width per expansion level d / MUX level a (1, 2, 4 or 8 CTAs
  // per key switch or MUX); 0 = the default rule (split while the level has
  // fewer CTAs than the GPU has slots). Set by the handle's autotuner.
  uint8_t split_exp[16];
  uint8_t split_mux[32];
};

// Number of heap nodes processed at expansion level d (nodes whose leftmost
// leaf is below `useful`, src/server.cpp:786-792).
inline uint32_t expand_nodes(const Shape &s, uint32_t d) {
  const uint64_t span = 1ull << (s.h - d);
  return static_cast<uint32_t>((s.useful + span - 1) / span);
}

// u64 (mod q) arrays -> residue pairs. in: n_items x per_item polys x N u64
// (contiguous); out: item i at out + i * out_item_stride u32 words, each item
// per_item x 2 x N u32.
void launch_split_u64(const DevParams &P, const uint64_t *in, uint32_t *out,
                      uint64_t n_items, uint64_t per_item, uint64_t out_item_stride,
                      cudaStream_t st);
// residue pairs -> u64 (mod q); the inverse of launch_split_u64.
void launch_compose_u64(const DevParams &P, const uint32_t *in, uint64_t in_item_stride,
                        uint64_t *out, uint64_t n_items, uint64_t per_item,
                        cudaStream_t st);

// Database preprocessing (src/server.cpp:80-171): plaintexts [pt][N] (u16,
// or generated from `seed` when coeffs == nullptr) -> NTT -> residues ->
// byte planes db8[((res N + level) 4 + plane) other + row][n0p] with
// pt = row n0 + k. Covers plaintexts [pt_begin, pt_end); rows >= logical are
// zero. Padding bytes (k >= n0) are never written: the buffer starts zeroed.
// row_map (device, one entry per row of s; null = identity) names the
// database row stored at each row of a row shard: generated coefficients and
// the logical bound use the database index row_map[pt / n0] n0 + pt % n0.
void launch_db_preprocess(const DevParams &P, const Shape &s, const uint16_t *coeffs,
                          uint64_t coeff_pt_begin, uint64_t seed, uint64_t t,
                          uint64_t logical, uint64_t pt_begin, uint64_t pt_end,
                          const uint32_t *row_map, uint8_t *db8, cudaStream_t st);

// One expansion level d over `batch` queries. in: batch x in_stride cts,
// out: batch x out_stride cts. bv_level[b] points at the (galois level d) key
// block of query b: L_KS x [b|a] x 2 residues x N u32, NTT form.
// ntt_nodes > 0 (the last level only): the children of nodes below ntt_nodes
// are written in NTT form (canonical, the layout k_fst_ntt writes), the
// others in coefficient form; the level then runs one CTA per key switch.
void launch_expand_level(const DevParams &P, const Shape &s, uint32_t d,
                         const uint32_t *in, uint64_t in_stride, uint32_t *out,
                         uint64_t out_stride, const uint32_t *const *bv_keys,
                         uint64_t bv_level_stride, uint32_t batch, cudaStream_t st,
                         uint32_t ntt_nodes = 0);

// Selector completion (src/server.cpp:823-855, src/gsw.cpp:317-357).
// leaves: batch x leaf_stride cts; gsw[b]: 2 L_KEY rows x 2 polys x 2 res x N;
// sel: batch x (num_dims-1) x 2 L_EP rows x 2 x 2 x N (NTT form).
void launch_selectors(const DevParams &P, const Shape &s, const uint32_t *leaves,
                      uint64_t leaf_stride, const uint32_t *const *gsw_keys,
                      uint32_t *sel, uint32_t batch, cudaStream_t st);

// Twiddles with index < 64 (value and Shoup companion, forward and inverse)
// and {N^-1, Shoup, iw[1] N^-1, Shoup} of both residues, copied to the
// kernels' constant memory on the current device. Once per device; later
// calls are no-ops. Throws if q differs from the moduli the kernels are
// compiled for.
void upload_ntt_constants(const uint32_t q[2], const uint32_t *const fw[2],
                          const uint32_t *const fw_sh[2], const uint32_t *const iw[2],
                          const uint32_t *const iw_sh[2], const uint32_t nscale[2][4]);

// First-dimension query matrix (src/server.cpp:332-346 + 264-304): NTT of the
// first n0 leaves of each query, written as byte planes
// qb[((res N + level) 4 + plane) 2 batch + column][n0p], column = 2 b + poly.
void launch_fst_prep(const DevParams &P, const Shape &s, const uint32_t *leaves,
                     uint64_t leaf_stride, uint32_t *ntt, uint64_t ntt_stride, uint8_t *qb,
                     uint32_t batch, cudaStream_t st);
// The byte-plane transpose alone, for leaves already in NTT form (the last
// expansion level's NTT-form children).
void launch_fst_pack(const Shape &s, const uint32_t *ntt, uint64_t ntt_stride, uint8_t *qb,
                     uint32_t batch, cudaStream_t st);

// First-dimension scan on CUDA cores (matrix.cpp:240-350): per residue and
// NTT level, C[res][l][c][r] = sum_k A[r][k] Q[k][c] mod q_res, c < 2 batch,
// with A and Q rebuilt from their byte planes (the tensor-core form writes
// the same [res x level][column][row] layout).
void launch_scan(const DevParams &P, const Shape &s, const uint8_t *db8,
                 const uint8_t *qb, uint32_t *cmat, uint32_t batch,
                 cudaStream_t st);

// Gather + INTT of the scan output into candidate ciphertexts
// (src/server.cpp:529-597). mid: batch x mid_stride cts (coefficient form).
void launch_scan_epilogue(const DevParams &P, const Shape &s, const uint32_t *cmat,
                          uint32_t *mid, uint64_t mid_stride, uint32_t batch,
                          cudaStream_t st);

// One MUX level of evaluate_other_dim (src/server.cpp:599-722) in a selector
// tree of height tree_h (num_dims - 1 for a whole layout, less on a row
// shard), selector slot `level` of each query's set:
// level 0: pairs (offset + 2i, offset + 2i + 1) -> out[offset + i], and
//          out[0, offset) = in[0, offset), offset = 2^tree_h - s.other;
// level a >= 1: pairs (i, i + half) -> out[i], i < half = 2^(tree_h-a-1).
void launch_mux_level(const DevParams &P, const Shape &s, uint32_t level, uint32_t tree_h,
                      const uint32_t *in, uint32_t *out, uint64_t mid_stride,
                      const uint32_t *sel, uint32_t batch, cudaStream_t st);

// Modulus switch (src/server.cpp:1025-1043) + response bit packing
// (src/server.cpp:950-1009). ct: batch x ct_stride cts; resp: batch x 2N u64;
// bytes: batch x resp_bytes (may be nullptr).
void launch_modswitch(const DevParams &P, const uint32_t *ct, uint64_t ct_stride,
                      uint64_t *resp, uint8_t *bytes, uint32_t resp_bytes,
                      uint32_t batch, cudaStream_t st);

// Kernel launches issued so far by this library (all launchers count).
uint64_t launch_count();
// Adjusts the launch counter (kernels launched outside opir_kernels.cu, or
// replayed from a CUDA graph).
void note_launches(int64_t delta);

// Butterfly-rate probe: `blocks` x 256 threads, each running `iters`
// iterations of three register-resident forward radix-8 passes; sink holds
// blocks x 256 u32. Returns the butterflies the launch performs.
// Blocks of 256 threads that fill `sms` SMs with the probe (its occupancy).
uint32_t bfly_rate_blocks(int sms);
uint64_t launch_bfly_rate(uint32_t *sink, uint32_t blocks, uint32_t iters, cudaStream_t st);

}  // namespace opir
