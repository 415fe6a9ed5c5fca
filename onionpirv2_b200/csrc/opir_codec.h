// Wire codec for queries and client keys: seed-compressed, as the
// reference's communication model assumes (includes/pir.h:115-139: a 32-byte
// seed stands for every uniformly random polynomial) but does not implement.
//
// Every uniform polynomial (the query's c1, the `a` of each BV key row, the
// c1 of each RGSW row) is Expand(seed, domain, index): the ChaCha20 block
// function (RFC 8439) keyed by the seed, nonce = domain (u32 LE) || index
// (u64 LE), block counter from 0, read as little-endian u64 words; limb k of
// the polynomial takes, coefficient by coefficient, the next word whose low
// bit_length(q_k) bits are below q_k (rejection sampling, limb-major). The
// other polynomial of each ciphertext is packed at bit_length(q_k) bits per
// coefficient, LSB first, limb-major.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

namespace opir::codec {

// RFC 8439 section 2.3: 16 output words of the block function.
void chacha20_block(const uint32_t key[8], uint32_t counter, const uint32_t nonce[3],
                    uint32_t out[16]);

// Expand(seed, domain, index) into K = mods.size() limbs of n coefficients.
void expand_uniform(const uint8_t seed[32], uint32_t domain, uint64_t index,
                    const std::vector<uint64_t> &mods, uint32_t n, uint64_t *out);

// Bit width of a modulus (bits needed for values below it).
uint32_t width_of(uint64_t q);

// LSB-first packing of `count` values of `width` bits; returns bytes written
// (ceil(count width / 8)). unpack reads the same layout.
size_t pack_bits(const uint64_t *v, size_t count, uint32_t width, uint8_t *out);
void unpack_bits(const uint8_t *in, size_t count, uint32_t width, uint64_t *v);

}  // namespace opir::codec
