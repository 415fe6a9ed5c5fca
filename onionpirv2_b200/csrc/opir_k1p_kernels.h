// Launchers of the CONFIG_N2048_K1 kernels (opir_k1p_kernels.cu): the
// reference's default parameter set (includes/database_constants.h:61-76),
// N = 2048 with one real 60-bit NTT prime q = 2^60 - 2^14 + 1
// (generate_ntt_friendly_primes({60}, 2048)), PlainMod 14, SmallQWidth 22,
// L_EP 5 (base 2^12), L_KEY 8 (base 2^8), L_KS 8 (base 2^8), all balanced
// digits of the centred value in [-B/2, B/2) (gsw.cpp:252-295,
// bv_keyswitch.cpp:20-40, 296-367).
//
// Device layouts (u64 words, canonical values mod q):
//   ciphertext : [c0 (N)][c1 (N)] (rlwe.h:17-31 with K = 1), kCtWords = 2N
//   database   : db8[(z 8 + plane)][row][n0p] bytes, z = NTT level < N: byte
//                `plane` of the reference's db[level * num_pt + pt],
//                pt = row n0 + col (server.cpp:172-194), rows padded to
//                n0p = n0 rounded up to 16
//   BV keys    : per client [level < h][row < L_KS][b (N)][a (N)][b' (N)]
//                [a' (N)], NTT form, w' = floor(w 2^64 / q) the Shoup
//                companion of w (kRowWords per row)
//   RGSW key   : per client [row < 2 L_KEY][c0][c1][c0'][c1'], NTT form
//   selectors  : [query][dim < num_dims-1][row < 2 L_EP][c0][c1][c0'][c1']
//   query mat  : qm[col < 2 B][k < n0][z < N] u64, col = 2 query + poly, then
//                qb[(z 8 + plane)][col][n0p] bytes
//   cmat       : [z][col][row] u64 (the 64-bit-limb scan's output layout)
// Launches are counted with the CONFIG_N4096_K2_MP kernels' (opir4).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "opir_c4_kernels.h"

namespace opir1 {

constexpr int kN = 2048;
constexpr uint64_t kQ = 1152921504606830593ull;  // 2^60 - 2^14 + 1
constexpr int kCtWords = 2 * kN;   // u64 words per ciphertext
constexpr int kRowWords = 4 * kN;  // a key / RGSW row: ciphertext + Shoup companions
constexpr int kLEp = 5, kBaseEp = 12, kLKey = 8, kBaseKey = 8, kLKs = 8, kBaseKs = 8;

struct Dev1 {
  const ulonglong2 *fwt, *iwt;  // (w, floor(w 2^64 / q)), bit-reversed order
  uint64_t small_q;
  uint32_t small_q_width;
  const ulonglong2 *pwt;        // (psi^m, floor(psi^m 2^64 / q)) for m < 2N
};

// the layout fields the kernels read (the two-limb set's shape struct)
using Shape1 = opir4::Shape4;
static_assert(kQ == opir4::kQ0, "the scan reduces CONFIG_N2048_K1 levels mod limb 0's prime");

// Twiddles with index < 64 and {N^-1, iw[1] N^-1} (value, Shoup) to the
// kernels' constant memory of the current device (once per device).
void upload_constants(const uint64_t *fw, const uint64_t *fw_sh, const uint64_t *iw,
                      const uint64_t *iw_sh, const uint64_t ninv[2], const uint64_t w1ninv[2]);

// server.cpp:80-203: plaintexts [pt_begin, pt_end) -> NTT mod q -> db8.
// coeffs (device, u64 < t) holds plaintexts from coeff_pt_begin on; null
// generates coefficient(pt, c) = mix64(seed + (pt N + c + 1) golden) % t.
void launch_db_preprocess(const Dev1 &P, const Shape1 &s, const uint64_t *coeffs,
                          uint64_t coeff_pt_begin, uint64_t seed, uint64_t t, uint64_t logical,
                          uint64_t pt_begin, uint64_t pt_end, uint8_t *db8, cudaStream_t st);
void launch_expand_level(const Dev1 &P, const Shape1 &s, uint32_t d, const uint64_t *in,
                         uint64_t in_stride, uint64_t *out, uint64_t out_stride,
                         const uint64_t *const *bv_keys, uint64_t bv_level_stride, uint32_t batch,
                         cudaStream_t st, uint32_t ntt_nodes = 0);
void launch_selectors(const Dev1 &P, const Shape1 &s, const uint64_t *leaves, uint64_t leaf_stride,
                      const uint64_t *const *gsw_keys, uint64_t *sel, uint32_t batch,
                      cudaStream_t st);
void launch_fst_ntt(const Dev1 &P, const Shape1 &s, const uint64_t *leaves, uint64_t leaf_stride,
                    uint64_t *qm, uint32_t batch, cudaStream_t st);
void launch_fst_pack(const Shape1 &s, const uint64_t *qm, uint8_t *qb, uint32_t batch,
                     cudaStream_t st);
// The same byte planes from NTT-form leaves in the ciphertext layout (the
// last expansion level's NTT-form children; batch x leaf_stride cts).
void launch_fst_pack_leaves(const Shape1 &s, const uint64_t *leaves, uint64_t leaf_stride,
                            uint8_t *qb, uint32_t batch, cudaStream_t st);
void launch_epilogue(const Dev1 &P, const Shape1 &s, const uint64_t *cmat, uint64_t *mid,
                     uint64_t mid_stride, uint32_t batch, cudaStream_t st);
// One MUX level of a selector tree of height tree_h: level 0 carries the
// unpaired prefix 2^tree_h - s.other, level a >= 1 pairs
// (i, i + 2^(tree_h-a-1)).
void launch_mux_level(const Dev1 &P, const Shape1 &s, uint32_t level, uint32_t tree_h,
                      const uint64_t *in, uint64_t *out, uint64_t mid_stride, const uint64_t *sel,
                      uint32_t batch, cudaStream_t st);
// Modulus switch + (optional) bit packing; resp: 2N u64 per query.
void launch_modswitch(const Dev1 &P, const uint64_t *ct, uint64_t ct_stride, uint64_t *resp,
                      uint8_t *bytes, uint32_t resp_bytes, uint32_t batch, cudaStream_t st);

}  // namespace opir1
