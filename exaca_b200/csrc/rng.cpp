// MT19937-64 block refill of rng.hpp, in its own translation unit: it is built with -O3 (the
// vectoriser's full cost model) for the baseline instruction set, AVX2 and AVX-512 (whose unsigned
// 64-bit minimum halves the refill's time on hosts that have it).
#include "rng.hpp"

namespace exaca {

__attribute__((target_clones("avx512f", "avx2", "default"))) uint64_t mt64_twist_temper(uint64_t *s, uint64_t *out) {
    constexpr int kN = Mt64::kN, kM = Mt64::kM;
    constexpr uint64_t kUpper = 0xffffffff80000000ull, kLower = 0x7fffffffull, kA = 0xb5026f5aa96619e9ull;
    for (int i = 0; i < kN - kM; i++) {
        const uint64_t y = (s[i] & kUpper) | (s[i + 1] & kLower);
        s[i] = s[i + kM] ^ (y >> 1) ^ ((uint64_t)0 - (y & 1ull) & kA);
    }
    for (int i = kN - kM; i < kN - 1; i++) {
        const uint64_t y = (s[i] & kUpper) | (s[i + 1] & kLower);
        s[i] = s[i + kM - kN] ^ (y >> 1) ^ ((uint64_t)0 - (y & 1ull) & kA);
    }
    {
        const uint64_t y = (s[kN - 1] & kUpper) | (s[0] & kLower);
        s[kN - 1] = s[kM - 1] ^ (y >> 1) ^ ((uint64_t)0 - (y & 1ull) & kA);
    }
    uint64_t mn = ~0ull;
    for (int i = 0; i < kN; i++) {
        uint64_t z = s[i];
        z ^= (z >> 29) & 0x5555555555555555ull;
        z ^= (z << 17) & 0x71d67fffeda60000ull;
        z ^= (z << 37) & 0xfff7eee000000000ull;
        z ^= z >> 43;
        out[i] = z;
        mn = z < mn ? z : mn;
    }
    return mn;
}

} // namespace exaca
