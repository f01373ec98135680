// ORACLE — test infrastructure only.  Nothing in the product library links or
// includes this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg use the oracle, and only to compare results against (or to time it).
//
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11), restated from the
// paper.  The reference draws from one sequential boost::random::mt19937
// stream (ABM-3d/ABM-3d-cpp/include/simulation.hpp:1173); no reference test
// pins that stream, so the oracle and the CUDA path share this counter-based
// policy instead and are compared bit for bit under it.
#pragma once
#include <cstdint>
#include <cmath>

namespace oracle {

struct Philox4 { uint32_t v[4]; };

inline void philox_mulhilo(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo)
{
    uint64_t p = static_cast<uint64_t>(a) * static_cast<uint64_t>(b);
    hi = static_cast<uint32_t>(p >> 32);
    lo = static_cast<uint32_t>(p);
}

inline Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                             uint32_t k0, uint32_t k1)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    uint32_t x0 = c0, x1 = c1, x2 = c2, x3 = c3;
    for (int r = 0; r < 10; ++r)
    {
        uint32_t hi0, lo0, hi1, lo1;
        philox_mulhilo(M0, x0, hi0, lo0);
        philox_mulhilo(M1, x2, hi1, lo1);
        uint32_t y0 = hi1 ^ x1 ^ k0;
        uint32_t y1 = lo1;
        uint32_t y2 = hi0 ^ x3 ^ k1;
        uint32_t y3 = lo0;
        x0 = y0; x1 = y1; x2 = y2; x3 = y3;
        k0 += W0; k1 += W1;
    }
    Philox4 out = {{x0, x1, x2, x3}};
    return out;
}

// 52 random bits -> (bits + 0.5) * 2^-52, exactly representable, in (0, 1).
inline double philox_u01(uint32_t hi, uint32_t lo)
{
    uint64_t bits = ((static_cast<uint64_t>(hi) << 32) | lo) >> 12;
    return (static_cast<double>(bits) + 0.5) * (1.0 / 4503599627370496.0);
}

// Purposes, mixed into the second key word so the noise and division
// streams never overlap.
const uint32_t RNG_PURPOSE_NOISE = 0x4E6F6973u;
const uint32_t RNG_PURPOSE_DIVIDE = 0x44697669u;
const uint32_t RNG_PURPOSE_SWITCH = 0x53776974u;

inline void rng_key(uint64_t seed, uint32_t purpose, uint32_t& k0, uint32_t& k1)
{
    k0 = static_cast<uint32_t>(seed);
    k1 = static_cast<uint32_t>(seed >> 32) ^ purpose;
}

// One uniform for (a, b, c, d).
inline double rng_uniform(uint64_t seed, uint32_t purpose, uint32_t a, uint32_t b,
                          uint32_t c, uint32_t d)
{
    uint32_t k0, k1;
    rng_key(seed, purpose, k0, k1);
    Philox4 x = philox4x32_10(a, b, c, d, k0, k1);
    return philox_u01(x.v[0], x.v[1]);
}

}   // namespace oracle
