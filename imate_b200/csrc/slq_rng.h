// Host side of the probe generator.
//
// Parity mode reproduces the reference's Rademacher stream bit for bit: the
// single-thread estimator draws probe g from words [g*W, (g+1)*W) of one
// xoshiro256** stream (W = n/64 + 1, random_array_generator.cpp:63-165), the
// stream being SplitMix64(seed) jumped once (random_number_generator.cpp:
// 120-137).  To generate those words in parallel on the device, each thread
// starts from a state advanced by k draws.  xoshiro256's state update is
// linear over GF(2), so advancing by k equals applying q(T) with
// q(x) = x^k mod P(x), P the characteristic polynomial of the update; q(T)s is
// evaluated as sum_i q_i T^i s with 256 ordinary steps, the same evaluation
// the published jump() uses for k = 2^128.  P is recovered once by
// Berlekamp-Massey from a state-bit sequence and checked against the
// published jump polynomial.

#ifndef SLQ_RNG_H_
#define SLQ_RNG_H_

#include <cstdint>
#include <vector>

namespace slq {

struct Poly256 {  // GF(2) polynomial of degree < 256, bit i = coeff of x^i
    uint64_t w[4];
};

// One xoshiro256** draw (Blackman & Vigna), advancing s.
inline uint64_t xoshiro_next(uint64_t* s)
{
    const uint64_t x = s[1] * 5;
    const uint64_t result = ((x << 7) | (x >> 57)) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = (s[3] << 45) | (s[3] >> 19);
    return result;
}

// Stream state of the single-thread reference estimator for `seed` (>= 0).
void stream_state(int64_t seed, uint64_t* state);

// x^k mod P.
Poly256 jump_poly(uint64_t k);

// (a * b) mod P.
Poly256 poly_mulmod(const Poly256& a, const Poly256& b);

// state <- q(T) state.
void apply_poly(const Poly256& q, uint64_t* state);

// state <- T^k state.
void jump_ahead(uint64_t* state, uint64_t k);

// True if the recovered P reproduces the published 2^128 jump polynomial.
bool self_check();

}  // namespace slq

#endif  // SLQ_RNG_H_
