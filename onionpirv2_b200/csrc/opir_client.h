// Host helpers of the client kernels (opir_client.cu) that the server also
// uses: the reference's forward negacyclic NTT on u64 polynomials.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/onionpir_b200.h"

namespace opir {

// root^BitRev(k) for k < N, per limb ([K][N]): the logical q with its CRT
// root when K = 1, each RNS limb with its own root when K = 2.
std::vector<uint64_t> forward_twiddles(const opir_params &p);

// In-place forward NTT (Cooley-Tukey from natural order, bit-reversed output,
// canonical values) of `count` polynomials of N u64 each, the limb of
// polynomial i being i % K; d_fw holds forward_twiddles(p) on the device.
void forward_ntt_polys(uint64_t *d_polys, uint64_t count, const opir_params &p,
                       const uint64_t *d_fw, cudaStream_t st);

}  // namespace opir
