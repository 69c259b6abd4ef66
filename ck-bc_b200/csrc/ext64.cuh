// Extended-range non-negative numbers in 64 bits, for shortest-path counts
// that overflow uint64 and double (a 2048 x 2048 grid has counts near 2^4088).
//
// Encoding: 0 is 0; otherwise bits 63..48 hold a biased exponent E (1..65535)
// and bits 47..0 the fraction f of a 49-bit significand M = 2^48 + f, value
// M * 2^(E - kExtBias) with kExtBias = 32768 + 48: values from about 2^-32815
// to 2^32816, 49 significant bits.  As unsigned integers the encodings order
// like the values, so 0 tests and comparisons need no decoding.  Every
// operation rounds to nearest, ties to even, on the 49-bit significand.
#pragma once
#include <stdint.h>

namespace bcg {

constexpr int kExtBias = 32768 + 48;
constexpr unsigned long long kExtOne = 0x8000000000000000ull;  // 1.0: E = 32768, f = 0
constexpr unsigned long long kExtFrac = (1ull << 48) - 1;

__host__ __device__ __forceinline__ unsigned long long ext_pack(int e, unsigned long long m) {
    // m in [2^48, 2^49); an exponent outside the encodable range saturates
    if (e < 1) return 0ull;
    if (e > 65535) return ~0ull;
    return ((unsigned long long)e << 48) | (m & kExtFrac);
}

// s in [2^59, 2^61) stands for the value s * 2^(e - kExtBias - 11) (with more
// nonzero bits below s when `sticky`); rounds it to a 49-bit significand.
__host__ __device__ __forceinline__ unsigned long long ext_round(unsigned long long s, bool sticky, int e) {
    if (s >= (1ull << 60)) {
        sticky |= (s & 1ull) != 0;
        s >>= 1;
        ++e;
    }
    unsigned long long m = s >> 11;
    const unsigned long long rb = s & 0x7FFull;
    if (rb > 0x400ull || (rb == 0x400ull && (sticky || (m & 1ull)))) {
        ++m;
        if (m == (1ull << 49)) {
            m >>= 1;
            ++e;
        }
    }
    return ext_pack(e, m);
}

__host__ __device__ __forceinline__ unsigned long long ext_add(unsigned long long a, unsigned long long b) {
    if (!a) return b;
    if (!b) return a;
    if (a < b) {
        const unsigned long long t = a;
        a = b;
        b = t;
    }
    const int ea = (int)(a >> 48), eb = (int)(b >> 48);
    const int d = ea - eb;
    const unsigned long long A = ((a & kExtFrac) | (1ull << 48)) << 11;
    const unsigned long long B = ((b & kExtFrac) | (1ull << 48)) << 11;
    unsigned long long bs;
    bool sticky;
    if (d == 0) {
        bs = B;
        sticky = false;
    } else if (d < 64) {
        bs = B >> d;
        sticky = (B << (64 - d)) != 0;
    } else {
        bs = 0;
        sticky = true;
    }
    return ext_round(A + bs, sticky, ea);
}

__host__ __device__ __forceinline__ unsigned long long ext_mul(unsigned long long a, unsigned long long b) {
    if (!a || !b) return 0ull;
    const unsigned long long ma = (a & kExtFrac) | (1ull << 48), mb = (b & kExtFrac) | (1ull << 48);
#ifdef __CUDA_ARCH__
    const unsigned long long hi = __umul64hi(ma, mb), lo = ma * mb;
#else
    const unsigned __int128 p = (unsigned __int128)ma * mb;
    const unsigned long long hi = (unsigned long long)(p >> 64), lo = (unsigned long long)p;
#endif
    // p = ma * mb in [2^96, 2^98), value p * 2^(ea + eb - 2 bias); s = p >> 37 in
    // [2^59, 2^61) stands for s * 2^(e - bias - 11) (ext_round's scaling), so
    // e - bias - 11 = 37 + ea + eb - 2 bias, i.e. e = ea + eb - bias + 48
    const unsigned long long s = (hi << 27) | (lo >> 37);
    const bool sticky = (lo & ((1ull << 37) - 1)) != 0;
    return ext_round(s, sticky, (int)(a >> 48) + (int)(b >> 48) - kExtBias + 48);
}

// x > 0 finite double -> extended value x * 2^k.
__host__ __device__ __forceinline__ unsigned long long ext_from_double(double x, int k = 0) {
    if (!(x > 0.0)) return 0ull;
    int q;
    const double m = frexp(x, &q);  // x = m * 2^q, m in [0.5, 1)
    // 53-bit integer significand D = m * 2^53, x * 2^k = D * 2^(q - 53 + k);
    // s = D * 2^8 in [2^60, 2^61) stands for s * 2^(e - bias - 11), so
    // e = q + k - 50 + bias
    const unsigned long long D = (unsigned long long)ldexp(m, 53);
    return ext_round(D << 8, false, q + k - 50 + kExtBias);
}

// Extended value -> double (inf / 0 outside the double range).
__host__ __device__ __forceinline__ double ext_to_double(unsigned long long a) {
    if (!a) return 0.0;
    const unsigned long long m = (a & kExtFrac) | (1ull << 48);
    return ldexp((double)m, (int)(a >> 48) - kExtBias);
}

// num / value(a) for a double num > 0 and a != 0, as an extended value.
__host__ __device__ __forceinline__ unsigned long long ext_div(double num, unsigned long long a) {
    const unsigned long long m = (a & kExtFrac) | (1ull << 48);
    return ext_from_double(num / (double)m, kExtBias - (int)(a >> 48));
}

}  // namespace bcg
