// The uniform random stream of the reference's initialisation, drawn fast and bit for bit.
//
// The reference draws std::uniform_real_distribution<double>(0.0, 1.0) from std::mt19937_64
// (src/CAinitialize.cpp:1464-1465, 1603-1604, 1844-1845). With libstdc++ each draw is
// generate_canonical<double, 53> of one 64-bit output x: x converted to double (round to nearest),
// divided by 2^64 (exact: a power of two) and, when that rounds up to 1, replaced by the largest
// double below 1; the distribution then multiplies by (b - a) = 1 and adds a = 0, both exact.
// uniform01() restates that value. libstdc++ evaluates it through long-double logarithms on every
// draw, which made the 1.35e8 draws of a 512^3 problem take over a second.
//
// Mt64 is the published MT19937-64 generator (M. Matsumoto and T. Nishimura; the parameters of
// std::mt19937_64 in the C++ standard, [rand.predef]): seeded as std::mt19937_64(seed) it yields
// the same outputs in the same order. It keeps a block of 312 tempered outputs, refilled by one
// twist of the state, so a caller can scan a block for outputs below an integer threshold
// (scan_below) instead of converting every draw.
#pragma once

#include <cstdint>

namespace exaca {

// One twist of the 312-word state and the tempering of all 312 new words into out; returns the
// smallest of them. Compiled for AVX-512, AVX2 and the baseline instruction set; the loader picks
// the best one the host supports.
uint64_t mt64_twist_temper(uint64_t *s, uint64_t *out);

class Mt64 {
  public:
    static constexpr int kN = 312, kM = 156;

    explicit Mt64(uint64_t seed) {
        s_[0] = seed;
        for (int i = 1; i < kN; i++)
            s_[i] = 6364136223846793005ull * (s_[i - 1] ^ (s_[i - 1] >> 62)) + (uint64_t)i;
        pos_ = kN;
    }

    uint64_t next() {
        if (pos_ == kN)
            refill();
        return out_[pos_++];
    }

    // Draws `count` outputs and calls hit(t) for the t-th of them (0-based) when it is below x_lim.
    template <class F> void scan_below(uint64_t count, uint64_t x_lim, F &&hit) {
        uint64_t t = 0;
        while (t < count) {
            if (pos_ == kN)
                refill();
            const int take = (int)((uint64_t)(kN - pos_) < count - t ? (uint64_t)(kN - pos_) : count - t);
            const uint64_t *o = out_ + pos_;
            uint64_t mn = block_min_;
            if (take < kN) {
                mn = ~0ull;
                for (int k = 0; k < take; k++)
                    mn = o[k] < mn ? o[k] : mn;
            }
            if (mn < x_lim)
                for (int k = 0; k < take; k++)
                    if (o[k] < x_lim)
                        hit(t + (uint64_t)k);
            pos_ += take;
            t += (uint64_t)take;
        }
    }

  private:
    void refill() {
        block_min_ = mt64_twist_temper(s_, out_);
        pos_ = 0;
    }

    uint64_t s_[kN];
    uint64_t out_[kN];
    uint64_t block_min_ = 0;
    int pos_;
};

// std::uniform_real_distribution<double>(0, 1) of the output x (libstdc++, see above)
inline double uniform01(uint64_t x) {
    const double u = (double)x * 0x1p-64;
    return u < 1.0 ? u : 0x1.fffffffffffffp-1;
}

// For 0 < p <= 0.5: the smallest output x with uniform01(x) >= p, so that a draw is below p exactly
// when its output is below this limit (uniform01 is non-decreasing in x).
inline uint64_t uniform01_limit(double p) {
    uint64_t lo = 0, hi = 1ull << 63; // uniform01(0) = 0 < p <= 0.5 = uniform01(2^63)
    while (hi - lo > 1) {
        const uint64_t mid = lo + (hi - lo) / 2;
        if (uniform01(mid) < p)
            lo = mid;
        else
            hi = mid;
    }
    return hi;
}

} // namespace exaca
