// Shared host-side helpers of libbcg: per-thread error message, status codes.
#pragma once
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include "bcg.h"

namespace bcg {

// Records a formatted message for bcg_last_error() and returns code.
int set_error(int code, const char *fmt, ...)
#if defined(__GNUC__)
    __attribute__((format(printf, 2, 3)))
#endif
    ;

void clear_error();

// splitmix64 (Steele, Lea, Flood 2014): the one PRNG of every generator.
inline uint64_t splitmix64(uint64_t &state) {
    uint64_t z = (state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Uniform double in [0, 1) from the top 53 bits.
inline double u01(uint64_t &state) {
    return (double)(splitmix64(state) >> 11) * (1.0 / 9007199254740992.0);
}

// Uniform integer in [0, range) (Lemire's multiply-high reduction).
inline uint64_t below(uint64_t &state, uint64_t range) {
    return (uint64_t)(((unsigned __int128)splitmix64(state) * range) >> 64);
}

// Independent stream for chunk `idx` of a generator seeded with `seed`.
inline uint64_t stream_seed(uint64_t seed, uint64_t idx) {
    uint64_t s = seed ^ (0xD1B54A32D192ED03ull * (idx + 1));
    return splitmix64(s);
}

}  // namespace bcg
