// Host-side generator of the reference's initial noise: Julia's
// rand(MersenneTwister(seed), n, n) (core_shell.jl:32).
//
// The stream is defined outside the reference, by Julia 1.12's Random standard
// library and the dSFMT library it calls; this file restates both published
// algorithms:
//   * seeding: the seed's 32-bit words (least significant first) are hashed
//     with SHA2-256 (FIPS 180-4) over their little-endian bytes, and the digest,
//     read as eight little-endian 32-bit words, keys dSFMT's init_by_array;
//   * dSFMT-19937 (Saito & Matsumoto): init_by_array over the 768 32-bit state
//     words, the mask that puts the state in [1, 2), period certification, and
//     the 128-bit recursion with its "lung" word;
//   * rand on a fresh generator: the first count outputs in memory order, each
//     in [1, 2) minus 1.
// No GPU is involved; esc_julia_rand is plain host code.
#include <cstdint>
#include <cstring>
#include <vector>

#include "esc.h"

namespace {

// ---------------------------------------------------------------- SHA2-256
const uint32_t kSha256K[64] = {
    0x428a2f98u, 0x71374491u, 0xb5c0fbcfu, 0xe9b5dba5u, 0x3956c25bu, 0x59f111f1u, 0x923f82a4u, 0xab1c5ed5u,
    0xd807aa98u, 0x12835b01u, 0x243185beu, 0x550c7dc3u, 0x72be5d74u, 0x80deb1feu, 0x9bdc06a7u, 0xc19bf174u,
    0xe49b69c1u, 0xefbe4786u, 0x0fc19dc6u, 0x240ca1ccu, 0x2de92c6fu, 0x4a7484aau, 0x5cb0a9dcu, 0x76f988dau,
    0x983e5152u, 0xa831c66du, 0xb00327c8u, 0xbf597fc7u, 0xc6e00bf3u, 0xd5a79147u, 0x06ca6351u, 0x14292967u,
    0x27b70a85u, 0x2e1b2138u, 0x4d2c6dfcu, 0x53380d13u, 0x650a7354u, 0x766a0abbu, 0x81c2c92eu, 0x92722c85u,
    0xa2bfe8a1u, 0xa81a664bu, 0xc24b8b70u, 0xc76c51a3u, 0xd192e819u, 0xd6990624u, 0xf40e3585u, 0x106aa070u,
    0x19a4c116u, 0x1e376c08u, 0x2748774cu, 0x34b0bcb5u, 0x391c0cb3u, 0x4ed8aa4au, 0x5b9cca4fu, 0x682e6ff3u,
    0x748f82eeu, 0x78a5636fu, 0x84c87814u, 0x8cc70208u, 0x90befffau, 0xa4506cebu, 0xbef9a3f7u, 0xc67178f2u};

inline uint32_t rotr(uint32_t x, int r) { return (x >> r) | (x << (32 - r)); }

void sha256_block(uint32_t h[8], const uint8_t blk[64]) {
  uint32_t w[64];
  for (int t = 0; t < 16; ++t)
    w[t] = (uint32_t)blk[4 * t] << 24 | (uint32_t)blk[4 * t + 1] << 16 | (uint32_t)blk[4 * t + 2] << 8 |
           (uint32_t)blk[4 * t + 3];
  for (int t = 16; t < 64; ++t) {
    const uint32_t s0 = rotr(w[t - 15], 7) ^ rotr(w[t - 15], 18) ^ (w[t - 15] >> 3);
    const uint32_t s1 = rotr(w[t - 2], 17) ^ rotr(w[t - 2], 19) ^ (w[t - 2] >> 10);
    w[t] = w[t - 16] + s0 + w[t - 7] + s1;
  }
  uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], k = h[7];
  for (int t = 0; t < 64; ++t) {
    const uint32_t t1 = k + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) + kSha256K[t] + w[t];
    const uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
    k = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
  }
  h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += k;
}

// SHA2-256 of len bytes; digest in 32 bytes (big-endian words, the standard byte order).
void sha256(const uint8_t *msg, size_t len, uint8_t out[32]) {
  uint32_t h[8] = {0x6a09e667u, 0xbb67ae85u, 0x3c6ef372u, 0xa54ff53au,
                   0x510e527fu, 0x9b05688cu, 0x1f83d9abu, 0x5be0cd19u};
  size_t off = 0;
  for (; off + 64 <= len; off += 64) sha256_block(h, msg + off);
  uint8_t tail[128] = {0};
  const size_t rest = len - off;
  std::memcpy(tail, msg + off, rest);
  tail[rest] = 0x80;
  const size_t tl = rest + 9 <= 64 ? 64 : 128;
  const uint64_t bits = (uint64_t)len * 8;
  for (int i = 0; i < 8; ++i) tail[tl - 1 - i] = (uint8_t)(bits >> (8 * i));
  sha256_block(h, tail);
  if (tl == 128) sha256_block(h, tail + 64);
  for (int i = 0; i < 8; ++i)
    for (int b = 0; b < 4; ++b) out[4 * i + b] = (uint8_t)(h[i] >> (24 - 8 * b));
}

// ---------------------------------------------------------------- dSFMT-19937
constexpr int kN = 191;        // 128-bit words of state
constexpr int kPos1 = 117;
constexpr int kSl1 = 19;
constexpr int kSr = 12;
constexpr uint64_t kMsk1 = 0x000ffafffffffb3fULL, kMsk2 = 0x000ffdfffc90fffdULL;
constexpr uint64_t kFix1 = 0x90014964b32f4329ULL, kFix2 = 0x3b8d12ac548a7c7aULL;
constexpr uint64_t kPcv1 = 0x3d84e1ac0dc82880ULL, kPcv2 = 0x0000000000000001ULL;
constexpr uint64_t kLow = 0x000fffffffffffffULL, kHigh = 0x3ff0000000000000ULL;

inline uint32_t ini1(uint32_t x) { return (x ^ (x >> 27)) * 1664525u; }
inline uint32_t ini2(uint32_t x) { return (x ^ (x >> 27)) * 1566083941u; }

// init_by_array: st receives 2*(kN+1) 64-bit words (the state, then the lung).
void dsfmt_init(const uint32_t *key, int klen, uint64_t st[2 * (kN + 1)]) {
  const int size = (kN + 1) * 4, lag = 11, mid = (size - lag) / 2;
  std::vector<uint32_t> s(size, 0x8b8b8b8bu);
  int count = klen + 1 > size ? klen + 1 : size;
  uint32_t r = ini1(s[0] ^ s[mid] ^ s[size - 1]);
  s[mid] += r;
  r += (uint32_t)klen;
  s[(mid + lag) % size] += r;
  s[0] = r;
  --count;
  int i = 1;
  for (int j = 0; j < count; ++j) {
    r = ini1(s[i] ^ s[(i + mid) % size] ^ s[(i + size - 1) % size]);
    s[(i + mid) % size] += r;
    r += (j < klen ? key[j] : 0u) + (uint32_t)i;
    s[(i + mid + lag) % size] += r;
    s[i] = r;
    i = (i + 1) % size;
  }
  for (int j = 0; j < size; ++j) {
    r = ini2(s[i] + s[(i + mid) % size] + s[(i + size - 1) % size]);
    s[(i + mid) % size] ^= r;
    r -= (uint32_t)i;
    s[(i + mid + lag) % size] ^= r;
    s[i] = r;
    i = (i + 1) % size;
  }
  for (int k = 0; k < 2 * (kN + 1); ++k) st[k] = (uint64_t)s[2 * k] | (uint64_t)s[2 * k + 1] << 32;
  for (int k = 0; k < 2 * kN; ++k) st[k] = (st[k] & kLow) | kHigh;
  uint64_t inner = ((st[2 * kN] ^ kFix1) & kPcv1) ^ ((st[2 * kN + 1] ^ kFix2) & kPcv2);
  for (int sh = 32; sh > 0; sh >>= 1) inner ^= inner >> sh;
  if ((inner & 1) != 1) st[2 * kN + 1] ^= 1;
}

}  // namespace

extern "C" esc_status esc_julia_rand(uint64_t seed, double *out, int64_t count) {
  if (count < 0 || (count > 0 && !out)) return ESC_EINVAL;
  // key = SHA2-256 over the little-endian 32-bit words of the seed
  uint8_t bytes[8];
  int nb = 0;
  do {
    const uint32_t w = (uint32_t)(seed & 0xffffffffu);
    for (int b = 0; b < 4; ++b) bytes[nb++] = (uint8_t)(w >> (8 * b));
    seed >>= 32;
  } while (seed != 0);
  uint8_t dig[32];
  sha256(bytes, (size_t)nb, dig);
  uint32_t key[8];
  for (int i = 0; i < 8; ++i)
    key[i] = (uint32_t)dig[4 * i] | (uint32_t)dig[4 * i + 1] << 8 | (uint32_t)dig[4 * i + 2] << 16 |
             (uint32_t)dig[4 * i + 3] << 24;
  uint64_t st[2 * (kN + 1)];
  dsfmt_init(key, 8, st);

  // The stream x_0, x_1, ... of 128-bit outputs follows the state words:
  // x_i = rec(x_{i-N}, x_{i-N+POS1}, lung), with x_{-N..-1} the state.  A ring of
  // the last N outputs is all the recursion reads.
  std::vector<uint64_t> ring(2 * kN);
  std::memcpy(ring.data(), st, sizeof(uint64_t) * 2 * kN);
  uint64_t l0 = st[2 * kN], l1 = st[2 * kN + 1];
  const int64_t nw = (count + 1) / 2;
  for (int64_t i = 0; i < nw; ++i) {
    const int ia = (int)(i % kN);                  // x_{i-N}: overwritten by x_i
    const int ib = (int)((i + kPos1) % kN);        // x_{i-N+POS1}
    const uint64_t a0 = ring[2 * ia], a1 = ring[2 * ia + 1];
    const uint64_t b0 = ring[2 * ib], b1 = ring[2 * ib + 1];
    const uint64_t n0 = (a0 << kSl1) ^ (l1 >> 32) ^ (l1 << 32) ^ b0;
    const uint64_t n1 = (a1 << kSl1) ^ (l0 >> 32) ^ (l0 << 32) ^ b1;
    l0 = n0;
    l1 = n1;
    const uint64_t r0 = (l0 >> kSr) ^ (l0 & kMsk1) ^ a0;
    const uint64_t r1 = (l1 >> kSr) ^ (l1 & kMsk2) ^ a1;
    ring[2 * ia] = r0;
    ring[2 * ia + 1] = r1;
    double d0, d1;
    std::memcpy(&d0, &r0, 8);
    std::memcpy(&d1, &r1, 8);
    out[2 * i] = d0 - 1.0;
    if (2 * i + 1 < count) out[2 * i + 1] = d1 - 1.0;
  }
  return ESC_OK;
}
