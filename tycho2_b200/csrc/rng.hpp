// Seeded pseudo-random numbers for the synthetic problems (mesh jitter,
// lognormal cross sections, batch/serving draws): xoshiro256** seeded through
// splitmix64.  Deterministic across platforms; no library state.
#pragma once

#include <cmath>
#include <cstdint>

namespace tycho {

class Rng {
public:
    explicit Rng(uint64_t seed)
    {
        uint64_t z = seed;
        for (auto &w : s_) w = splitmix(z);
    }
    uint64_t next()
    {
        const uint64_t r = rotl(s_[1] * 5, 7) * 9;
        const uint64_t t = s_[1] << 17;
        s_[2] ^= s_[0]; s_[3] ^= s_[1]; s_[1] ^= s_[2]; s_[0] ^= s_[3];
        s_[2] ^= t; s_[3] = rotl(s_[3], 45);
        return r;
    }
    // Uniform in [0, 1) with 53 random bits.
    double uniform() { return (next() >> 11) * 0x1.0p-53; }
    // Standard normal (Box-Muller, one value per call).
    double normal()
    {
        double u1 = uniform(), u2 = uniform();
        return std::sqrt(-2.0 * std::log1p(-u1)) * std::cos(6.283185307179586 * u2);
    }
    // Integer in [lo, hi].
    int64_t range(int64_t lo, int64_t hi) { return lo + (int64_t)(next() % (uint64_t)(hi - lo + 1)); }

private:
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    static uint64_t splitmix(uint64_t &x)
    {
        uint64_t z = (x += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    uint64_t s_[4];
};

}  // namespace tycho
