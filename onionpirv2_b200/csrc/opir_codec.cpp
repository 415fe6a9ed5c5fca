// Wire codec primitives (opir_codec.h): the ChaCha20 block function of
// RFC 8439 section 2.3, uniform expansion by rejection sampling, and
// LSB-first bit packing.
#include "opir_codec.h"

#include <algorithm>
#include <cstring>
#include <stdexcept>

namespace opir::codec {

namespace {

inline uint32_t rotl(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

inline void quarter(uint32_t &a, uint32_t &b, uint32_t &c, uint32_t &d) {
  a += b; d ^= a; d = rotl(d, 16);
  c += d; b ^= c; b = rotl(b, 12);
  a += b; d ^= a; d = rotl(d, 8);
  c += d; b ^= c; b = rotl(b, 7);
}

inline uint32_t load32(const uint8_t *p) {
  return static_cast<uint32_t>(p[0]) | static_cast<uint32_t>(p[1]) << 8 |
         static_cast<uint32_t>(p[2]) << 16 | static_cast<uint32_t>(p[3]) << 24;
}

// Little-endian u64 words of the keystream of one (seed, domain, index).
class Stream {
 public:
  Stream(const uint8_t seed[32], uint32_t domain, uint64_t index) {
    for (int i = 0; i < 8; ++i) key_[i] = load32(seed + 4 * i);
    nonce_[0] = domain;
    nonce_[1] = static_cast<uint32_t>(index);
    nonce_[2] = static_cast<uint32_t>(index >> 32);
  }
  uint64_t next() {
    if (pos_ == 8) {
      if (counter_ == 0xFFFFFFFFu) throw std::runtime_error("codec: keystream exhausted");
      chacha20_block(key_, counter_++, nonce_, block_);
      pos_ = 0;
    }
    const uint64_t w = static_cast<uint64_t>(block_[2 * pos_]) |
                       static_cast<uint64_t>(block_[2 * pos_ + 1]) << 32;
    ++pos_;
    return w;
  }

 private:
  uint32_t key_[8], nonce_[3], block_[16];
  uint32_t counter_ = 0;
  int pos_ = 8;
};

}  // namespace

void chacha20_block(const uint32_t key[8], uint32_t counter, const uint32_t nonce[3],
                    uint32_t out[16]) {
  uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                    key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7],
                    counter, nonce[0], nonce[1], nonce[2]};
  uint32_t x[16];
  std::memcpy(x, s, sizeof(x));
  for (int r = 0; r < 10; ++r) {  // 20 rounds: column then diagonal
    quarter(x[0], x[4], x[8], x[12]);
    quarter(x[1], x[5], x[9], x[13]);
    quarter(x[2], x[6], x[10], x[14]);
    quarter(x[3], x[7], x[11], x[15]);
    quarter(x[0], x[5], x[10], x[15]);
    quarter(x[1], x[6], x[11], x[12]);
    quarter(x[2], x[7], x[8], x[13]);
    quarter(x[3], x[4], x[9], x[14]);
  }
  for (int i = 0; i < 16; ++i) out[i] = x[i] + s[i];
}

uint32_t width_of(uint64_t q) {
  uint32_t w = 0;
  while (w < 64 && (q - 1) >> w) ++w;
  return w;
}

void expand_uniform(const uint8_t seed[32], uint32_t domain, uint64_t index,
                    const std::vector<uint64_t> &mods, uint32_t n, uint64_t *out) {
  Stream st(seed, domain, index);
  for (size_t k = 0; k < mods.size(); ++k) {
    const uint64_t q = mods[k];
    const uint32_t w = width_of(q);
    const uint64_t mask = w == 64 ? ~0ull : (1ull << w) - 1;
    for (uint32_t j = 0; j < n; ++j) {
      uint64_t v;
      do v = st.next() & mask; while (v >= q);
      out[k * n + j] = v;
    }
  }
}

size_t pack_bits(const uint64_t *v, size_t count, uint32_t width, uint8_t *out) {
  const size_t bytes = (count * width + 7) / 8;
  std::memset(out, 0, bytes);
  size_t bit = 0;
  for (size_t i = 0; i < count; ++i) {
    const uint64_t x = width == 64 ? v[i] : v[i] & ((1ull << width) - 1);
    for (uint32_t b = 0; b < width;) {
      const size_t byte = bit / 8;
      const uint32_t off = bit % 8, take = std::min<uint32_t>(8 - off, width - b);
      out[byte] |= static_cast<uint8_t>(((x >> b) & ((1u << take) - 1)) << off);
      b += take;
      bit += take;
    }
  }
  return bytes;
}

void unpack_bits(const uint8_t *in, size_t count, uint32_t width, uint64_t *v) {
  size_t bit = 0;
  for (size_t i = 0; i < count; ++i) {
    uint64_t x = 0;
    for (uint32_t b = 0; b < width;) {
      const size_t byte = bit / 8;
      const uint32_t off = bit % 8, take = std::min<uint32_t>(8 - off, width - b);
      x |= static_cast<uint64_t>((in[byte] >> off) & ((1u << take) - 1)) << b;
      b += take;
      bit += take;
    }
    v[i] = x;
  }
}

}  // namespace opir::codec
