// SHA-256 (FIPS 180-4) for the RLC row consumers: the host data root over
// every encoded row (src/benchmarks/utils.rs:51-59) and the per-column
// coefficient hashes on the device (src/zoda/rlc.rs:48-65).
//
// The round constants are derived from their definition rather than typed
// in: H0[i] is the first 32 fractional bits of sqrt(prime_i) and K[i] those of
// cbrt(prime_i), for the first 8 and 64 primes, computed exactly with integer
// square and cube roots of prime * 2^64 and prime * 2^96.
#pragma once
#include <cstddef>
#include <cstdint>

namespace zb {
namespace sha {

struct Consts {
    uint32_t k[64];
    uint32_t h0[8];
};

// The first 64 primes' constants (host only; computed once).
const Consts& consts();

__host__ __device__ __forceinline__ uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

// One compression of the 64-byte big-endian block w[0..16) into h[0..8).
__host__ __device__ inline void compress(uint32_t h[8], const uint32_t blk[16], const uint32_t* k) {
    uint32_t w[64];
    for (int i = 0; i < 16; i++) w[i] = blk[i];
    for (int i = 16; i < 64; i++) {
        const uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
        const uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
        w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
    for (int i = 0; i < 64; i++) {
        const uint32_t S1 = rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25);
        const uint32_t ch = (e & f) ^ (~e & g);
        const uint32_t t1 = hh + S1 + ch + k[i] + w[i];
        const uint32_t S0 = rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22);
        const uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
        const uint32_t t2 = S0 + mj;
        hh = g;
        g = f;
        f = e;
        e = d + t1;
        d = c;
        c = b;
        b = a;
        a = t1 + t2;
    }
    h[0] += a;
    h[1] += b;
    h[2] += c;
    h[3] += d;
    h[4] += e;
    h[5] += f;
    h[6] += g;
    h[7] += hh;
}

// Streaming host hasher.
class Hasher {
   public:
    Hasher();
    void update(const void* data, size_t len);
    void final(uint8_t out[32]);
    // State after the whole 64-byte blocks seen so far, and the bytes pending.
    const uint32_t* state() const { return h_; }
    size_t pending() const { return n_; }
    const uint8_t* pending_bytes() const { return buf_; }
    uint64_t length() const { return len_; }

   private:
    uint32_t h_[8];
    uint8_t buf_[64];
    size_t n_ = 0;
    uint64_t len_ = 0;
};

}  // namespace sha
}  // namespace zb
