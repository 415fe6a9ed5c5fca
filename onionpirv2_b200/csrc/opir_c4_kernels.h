// Launchers of the CONFIG_N4096_K2_MP kernels (opir_c4_kernels.cu).
//
// Device layouts (u64 words, canonical residues):
//   ciphertext : [c0 limb0 (N)][c0 limb1 (N)][c1 limb0 (N)][c1 limb1 (N)]
//                (rlwe.h:17-31 with K = 2), kCtWords = 4 N words
//   database   : db8[(z 8 + plane)][row][n0p] bytes, z = limb N + NTT level:
//                byte `plane` of the reference's db[level * num_pt + pt],
//                pt = row n0 + col (server.cpp:172-194), rows padded to
//                n0p = n0 rounded up to 16
//   BV keys    : per client [level < h][row < L_KS][b (2N)][a (2N)]
//                [b' (2N)][a' (2N)], NTT form, w' = floor(w 2^64 / q_limb)
//                the Shoup companion of w (kRowWords per row)
//   RGSW key   : per client [row < 2 L_KEY][c0][c1][c0'][c1'], NTT form
//   selectors  : [query][dim < num_dims-1][row < 2 L_EP][c0][c1][c0'][c1']
//   query mat  : qm[z][col < 2 B][k < n0] u64, col = 2 query + poly, then
//                qb[(z 8 + plane)][col][n0p] bytes
//   cmat       : [z][col][row] u64
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace opir4 {

constexpr int kN = 4096;
constexpr uint64_t kQ0 = 1152921504606830593ull;  // 2^60 - 2^14 + 1
constexpr uint64_t kQ1 = 1152921504606748673ull;  // 2^60 - 2^16 - 2^15 + 1
constexpr int kCtWords = 4 * kN;  // u64 words per ciphertext (2 polys x 2 limbs)
constexpr int kRowWords = 8 * kN; // a key / RGSW row: ciphertext + Shoup companions

// Full twiddle tables in global memory, (w, floor(w 2^64 / q)) pairs per limb
struct Tables {
  const ulonglong2 *fwt[2], *iwt[2];
  const ulonglong2 *pwt[2];  // (psi^m, floor(psi^m 2^64 / q)) for m < 2N
};

struct Dev4 {
  uint64_t q0inv, q0inv_sh;        // q0^-1 mod q1 and its Shoup companion
  Tables T;
  uint64_t small_q;
  uint32_t small_q_width;
};

struct Shape4 {
  uint32_t n0, n0p, other, num_dims, h, useful, l_ep;
  uint64_t num_pt;
};

uint64_t launch_count();
// Adjusts the launch counter (a launch made outside opir_c4_kernels.cu, or
// kernels replayed from a CUDA graph).
void note_launches(int64_t delta);

void upload_constants(const uint64_t *const fw[2], const uint64_t *const fw_sh[2],
                      const uint64_t *const iw[2], const uint64_t *const iw_sh[2],
                      const uint64_t ninv[2][2], const uint64_t w1ninv[2][2]);

// Nodes of expansion level d that lead to a useful leaf (server.cpp:794-809).
uint32_t expand_nodes(const Shape4 &s, uint32_t d);

// server.cpp:80-203: plaintexts [pt_begin, pt_end) -> NTT per limb -> db.
// coeffs (device, u64 < t) holds plaintexts from coeff_pt_begin on; null
// generates coefficient(pt, c) = mix64(seed + (pt N + c + 1) golden) % t.
// row_map (device, one entry per row of s; null = identity) names the
// database row stored at each row of a row shard: generated coefficients and
// the logical bound use the database index row_map[pt / n0] n0 + pt % n0.
void launch_db_preprocess(const Dev4 &P, const Shape4 &s, const uint64_t *coeffs,
                          uint64_t coeff_pt_begin, uint64_t seed, uint64_t t, uint64_t logical,
                          uint64_t pt_begin, uint64_t pt_end, const uint32_t *row_map,
                          uint8_t *db8, cudaStream_t st);
// One expansion level for `batch` queries; bv_keys: device array of per-query
// key pointers.
// ntt_nodes > 0 (the last level only): the children of nodes below
// ntt_nodes (the first-dimension leaves) are written in NTT form, canonical,
// in the ciphertext layout; the other nodes' children in coefficient form.
void launch_expand_level(const Dev4 &P, const Shape4 &s, uint32_t d, const uint64_t *in,
                         uint64_t in_stride, uint64_t *out, uint64_t out_stride,
                         const uint64_t *const *bv_keys, uint64_t bv_level_stride, uint32_t batch,
                         cudaStream_t st, uint32_t ntt_nodes = 0);
void launch_selectors(const Dev4 &P, const Shape4 &s, const uint64_t *leaves, uint64_t leaf_stride,
                      const uint64_t *const *gsw_keys, uint64_t *sel, uint32_t batch,
                      cudaStream_t st);
void launch_fst_ntt(const Dev4 &P, const Shape4 &s, const uint64_t *leaves, uint64_t leaf_stride,
                    uint64_t *qm, uint32_t batch, cudaStream_t st);
void launch_fst_pack(const Shape4 &s, const uint64_t *qm, uint8_t *qb, uint32_t batch,
                     cudaStream_t st);
// The same byte planes from NTT-form leaves in the ciphertext layout
// (leaves: batch x leaf_stride ciphertexts, the last expansion level's
// NTT-form children).
void launch_fst_pack_leaves(const Shape4 &s, const uint64_t *leaves, uint64_t leaf_stride,
                            uint8_t *qb, uint32_t batch, cudaStream_t st);
void launch_epilogue(const Dev4 &P, const Shape4 &s, const uint64_t *cmat, uint64_t *mid,
                     uint64_t mid_stride, uint32_t batch, cudaStream_t st);
// One MUX level in a selector tree of height tree_h (num_dims - 1 for a
// whole layout, less on a row shard); level 0 carries the unpaired prefix
// 2^tree_h - s.other, level a >= 1 pairs (i, i + 2^(tree_h-a-1)).
void launch_mux_level(const Dev4 &P, const Shape4 &s, uint32_t level, uint32_t tree_h,
                      const uint64_t *in, uint64_t *out, uint64_t mid_stride, const uint64_t *sel,
                      uint32_t batch, cudaStream_t st);
// Modulus switch + (optional) bit packing of `batch` results; resp: 2N u64 per query.
void launch_modswitch(const Dev4 &P, const uint64_t *ct, uint64_t ct_stride, uint64_t *resp,
                      uint8_t *bytes, uint32_t resp_bytes, uint32_t batch, cudaStream_t st);

// Tensor-core scan (opir_c4_scan_tc.cu): cmat = db8 . qb per z, mod q_limb.
struct Tc4Args {
  uint32_t k_tiles;    // ceil(n0p / 64)
  uint32_t stages;     // pipeline stages (2 .. scan_tc4_max_stages)
  uint32_t other;      // rows per level
  uint32_t m_tiles;    // ceil(other / 128)
  uint32_t ncols;      // output columns (2 x batch)
  uint32_t ntile;      // columns per tile: 16 or 32
  uint32_t col_tiles;  // ceil(ncols / ntile)
  uint32_t zcount;     // 2 N (limbs x levels)
  uint64_t *cmat;      // [z][col][row]
  uint32_t *err;       // error bits (0 = ok)
  uint32_t *progress;  // per-CTA item counters (>= grid entries) or null
  long long wait_cycles;  // limit of each pipeline wait (clock cycles)
};
size_t scan_tc4_smem(uint32_t ntile, uint32_t stages);
uint32_t scan_tc4_max_stages(uint32_t ntile);
void launch_scan_tc4(const CUtensorMap &mapA, const CUtensorMap &mapQ, const Tc4Args &args,
                     int sm_count, cudaStream_t st);

// Butterfly-rate probe of the two-limb NTT (as opir::launch_bfly_rate);
// sink holds blocks x 256 u64. Returns the butterflies the launch performs.
// Blocks of 256 threads that fill `sms` SMs with the probe (its occupancy).
uint32_t bfly_rate_blocks(int sms);
uint64_t launch_bfly_rate(uint64_t *sink, uint32_t blocks, uint32_t iters, cudaStream_t st);

}  // namespace opir4
