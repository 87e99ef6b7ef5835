// Host side of the probe generator: characteristic polynomial of the
// xoshiro256 state update, GF(2) polynomial arithmetic modulo it, and
// jump-ahead.  See slq_rng.h.

#include "slq_rng.h"

#include <cstring>
#include <mutex>

namespace slq {

namespace {

// P(x) = x^256 + low(x); low holds coefficients 0..255.
Poly256 g_low;
bool g_ready = false;
std::once_flag g_once;

inline bool bit(const Poly256& p, int i) { return (p.w[i >> 6] >> (i & 63)) & 1ULL; }

// p <- p * x mod P
inline void mulx(Poly256& p)
{
    const bool carry = (p.w[3] >> 63) & 1ULL;
    p.w[3] = (p.w[3] << 1) | (p.w[2] >> 63);
    p.w[2] = (p.w[2] << 1) | (p.w[1] >> 63);
    p.w[1] = (p.w[1] << 1) | (p.w[0] >> 63);
    p.w[0] = p.w[0] << 1;
    if (carry)
        for (int k = 0; k < 4; ++k) p.w[k] ^= g_low.w[k];
}

// Berlekamp-Massey over GF(2) on the sequence of bit 0 of state word 0.
void find_characteristic_polynomial()
{
    const int N = 512;
    uint64_t s[4] = {0x9e3779b97f4a7c15ULL, 0xbf58476d1ce4e5b9ULL,
                     0x94d049bb133111ebULL, 0x2545f4914f6cdd1dULL};
    std::vector<uint8_t> seq(N);
    for (int t = 0; t < N; ++t)
    {
        seq[t] = static_cast<uint8_t>(s[0] & 1ULL);
        xoshiro_next(s);
    }
    // connection polynomial C(x) = 1 + c1 x + ... + cL x^L
    std::vector<uint8_t> C(N + 1, 0), B(N + 1, 0), T;
    C[0] = B[0] = 1;
    int L = 0, m = 1;
    for (int n = 0; n < N; ++n)
    {
        uint8_t d = seq[n];
        for (int i = 1; i <= L; ++i) d ^= C[i] & seq[n - i];
        if (d == 0)
        {
            ++m;
        }
        else if (2 * L <= n)
        {
            T = C;
            for (int i = 0; i + m <= N; ++i) C[i + m] ^= B[i];
            L = n + 1 - L;
            B = T;
            m = 1;
        }
        else
        {
            for (int i = 0; i + m <= N; ++i) C[i + m] ^= B[i];
            ++m;
        }
    }
    // characteristic polynomial P(x) = x^L C(1/x): coefficient of x^(L-i)
    // is c_i.  For xoshiro256 L = 256 (checked by self_check()).
    std::memset(&g_low, 0, sizeof(g_low));
    for (int i = 1; i <= L && i <= 256; ++i)
        if (C[i])
        {
            int e = L - i;
            g_low.w[e >> 6] |= 1ULL << (e & 63);
        }
    g_ready = (L == 256);
}

void ensure_ready()
{
    std::call_once(g_once, find_characteristic_polynomial);
}

inline uint64_t splitmix_next(uint64_t* st)
{
    uint64_t z = (*st += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

}  // namespace

Poly256 poly_mulmod(const Poly256& a, const Poly256& b)
{
    ensure_ready();
    Poly256 r = {{0, 0, 0, 0}};
    for (int i = 255; i >= 0; --i)
    {
        mulx(r);
        if (bit(b, i))
            for (int k = 0; k < 4; ++k) r.w[k] ^= a.w[k];
    }
    return r;
}

Poly256 jump_poly(uint64_t k)
{
    ensure_ready();
    Poly256 result = {{1, 0, 0, 0}};  // x^0
    Poly256 base = {{2, 0, 0, 0}};    // x^1
    while (k)
    {
        if (k & 1ULL) result = poly_mulmod(result, base);
        k >>= 1;
        if (k) base = poly_mulmod(base, base);
    }
    return result;
}

void apply_poly(const Poly256& q, uint64_t* state)
{
    uint64_t acc[4] = {0, 0, 0, 0};
    for (int i = 0; i < 256; ++i)
    {
        if (bit(q, i))
            for (int k = 0; k < 4; ++k) acc[k] ^= state[k];
        xoshiro_next(state);
    }
    std::memcpy(state, acc, sizeof(acc));
}

void jump_ahead(uint64_t* state, uint64_t k)
{
    if (k == 0) return;
    if (k < 512)
    {
        for (uint64_t i = 0; i < k; ++i) xoshiro_next(state);
        return;
    }
    apply_poly(jump_poly(k), state);
}

void stream_state(int64_t seed, uint64_t* state)
{
    // split_mix_64.cpp:28-48 and xoshiro_256_star_star.cpp constructor,
    // then one jump (random_number_generator.cpp:132-135 for thread 0).
    uint64_t s = static_cast<uint64_t>(seed);
    uint64_t st = (s << 32) | s;
    for (int i = 0; i < 4; ++i) state[i] = splitmix_next(&st);
    // x^(2^128) mod P: 128 squarings of x
    Poly256 q = {{2, 0, 0, 0}};
    for (int i = 0; i < 128; ++i) q = poly_mulmod(q, q);
    apply_poly(q, state);
}

bool self_check()
{
    ensure_ready();
    if (!g_ready) return false;
    Poly256 q = {{2, 0, 0, 0}};
    for (int i = 0; i < 128; ++i) q = poly_mulmod(q, q);
    // published xoshiro256 jump polynomial (coefficients of x^0..x^255)
    static const uint64_t J[4] = {0x180ec6d33cfd0abaULL, 0xd5a61266f0c9392cULL,
                                  0xa9582618e03fc9aaULL, 0x39abdc4529b1661cULL};
    for (int k = 0; k < 4; ++k)
        if (q.w[k] != J[k]) return false;
    return true;
}

}  // namespace slq
