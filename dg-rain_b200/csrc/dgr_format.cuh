/*
 * Fixed-point decimal formatting of doubles with 15 fractional digits, as C's
 * printf("%1.15f") prints them (2DCode/time_evolution.c:284-306, 363-386 write every state
 * value that way): the exact binary value rounded to 15 decimals, ties to even (the
 * round-to-nearest mode), a leading '-' for every value with the sign bit set (also when
 * it rounds to zero), "nan" / "inf" with their sign.  Integer arithmetic only, so the
 * device and the host produce the same bytes.
 *
 * For |v| < 2^63: v = i + f with i = floor(|v|) (an exact integer) and f = |v| - i (exact);
 * f = m 2^-k with an integer m < 2^53, so f 10^15 = m 10^15 / 2^k is rounded exactly in
 * 128-bit integers (m 10^15 < 2^103).  Larger magnitudes are not formatted (return -1).
 */
#pragma once

#include <stdint.h>
#include <string.h>

#ifndef DGR_HD
#ifdef __CUDACC__
#define DGR_HD __host__ __device__ __forceinline__
#else
#define DGR_HD inline
#endif
#endif

namespace dgr {

constexpr int F15_MAX = 1 + 19 + 1 + 15; /* sign, integer digits of a value < 2^63, '.', fraction */

DGR_HD int f15_put_u64(uint64_t x, char *out)
{
    char tmp[20];
    int n = 0;
    do {
        tmp[n++] = (char)('0' + (int)(x % 10));
        x /= 10;
    } while (x);
    for (int j = 0; j < n; ++j) out[j] = tmp[n - 1 - j];
    return n;
}

/* writes the characters of printf("%1.15f", v) to out (no terminator); returns their
 * count, or -1 for |v| >= 2^63 */
DGR_HD int format_f15(double v, char *out)
{
    uint64_t bits;
    memcpy(&bits, &v, 8);
    const bool neg = (bits >> 63) != 0;
    const int ex = (int)((bits >> 52) & 0x7ff);
    int n = 0;
    if (ex == 0x7ff) {
        if (neg) out[n++] = '-';
        const bool nan = (bits & 0xfffffffffffffull) != 0;
        out[n++] = nan ? 'n' : 'i';
        out[n++] = nan ? 'a' : 'n';
        out[n++] = nan ? 'n' : 'f';
        return n;
    }
    const double a = neg ? -v : v;
    if (!(a < 9223372036854775808.0)) return -1;
    uint64_t ip = (uint64_t)a;
    const double f = a - (double)ip; /* exact: the fraction bits of a */
    uint64_t q = 0;
    if (f != 0.0) {
        uint64_t fb;
        memcpy(&fb, &f, 8);
        const int fe = (int)((fb >> 52) & 0x7ff);
        const uint64_t mf = fe ? ((fb & 0xfffffffffffffull) | (1ull << 52)) : (fb & 0xfffffffffffffull);
        const int k = fe ? 1075 - fe : 1074; /* f = mf 2^-k, k > 52 since f < 1 */
        if (k < 128) {
            const unsigned __int128 P = (unsigned __int128)mf * 1000000000000000ull;
            const unsigned __int128 one = 1;
            q = (uint64_t)(P >> k);
            const unsigned __int128 rem = P & ((one << k) - 1);
            const unsigned __int128 half = one << (k - 1);
            if (rem > half || (rem == half && (q & 1))) ++q;
        } /* else f 10^15 < 2^-25: rounds to 0 */
    }
    if (q == 1000000000000000ull) {
        ++ip;
        q = 0;
    }
    if (neg) out[n++] = '-';
    n += f15_put_u64(ip, out + n);
    out[n++] = '.';
    for (int j = 14; j >= 0; --j) {
        out[n + j] = (char)('0' + (int)(q % 10));
        q /= 10;
    }
    return n + 15;
}

}  // namespace dgr
