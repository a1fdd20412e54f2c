/*
 * Test harness: div_rcp of dg-rain_b200/csrc/dgr_device.cuh (a / b through a shared
 * reciprocal and Markstein's correction) compiled for the host and compared with the host's
 * IEEE division, bit for bit, on seeded random operands and on hard cases.  Not part of
 * the library.
 */
#include <cstdint>
#include <cstring>

#include "../dg-rain_b200/csrc/dgr_device.cuh"

namespace {

uint64_t mix(uint64_t x)
{ /* splitmix64 */
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

double make(uint64_t mant, int exp2, int neg)
{
    uint64_t u = ((uint64_t)(exp2 + 1023) << 52) | (mant & ((1ull << 52) - 1));
    if (neg) u |= 1ull << 63;
    double d;
    memcpy(&d, &u, 8);
    return d;
}

uint64_t bits(double d)
{
    uint64_t u;
    memcpy(&u, &d, 8);
    return u;
}

}  // namespace

/* n seeded cases of each kind; returns mismatches (results that are not bit-equal to a / b
 * wherever div_rcp reports itself valid) and counts the valid cases in *valid. */
extern "C" long long dgr_t_div_rcp(long long n, unsigned long long seed, long long *valid)
{
    long long bad = 0, nvalid = 0;
    for (long long i = 0; i < n; ++i) {
        const uint64_t r1 = mix(seed ^ (2 * (uint64_t)i)), r2 = mix(seed ^ (2 * (uint64_t)i + 1));
        const int kind = (int)(r1 & 7);
        double b = make(r2 >> 12, (int)((r2 >> 3) % 201) - 100, (int)(r2 & 1));
        double a;
        switch (kind) {
        case 0: /* anything in the valid range */
            a = make(r1 >> 12, (int)((r1 >> 3) % 1801) - 900, (int)((r1 >> 2) & 1));
            break;
        case 1: /* quotients with few significant bits: exact divisions */
            a = b * (double)(int64_t)((r1 >> 20) % 4096 - 2048);
            break;
        case 2: /* near exact quotients: q b plus or minus a few ulps */
        {
            const double q = make(r1 >> 12, (int)((r1 >> 3) % 41) - 20, 0);
            a = q * b;
            uint64_t u = bits(a) + ((r1 >> 8) % 5) - 2;
            memcpy(&a, &u, 8);
            break;
        }
        case 3: /* divisor with an all-ones or a one-bit mantissa */
            b = make((r2 & 2) ? ((1ull << 52) - 1) : 1ull, (int)((r2 >> 3) % 201) - 100, (int)(r2 & 1));
            a = make(r1 >> 12, (int)((r1 >> 3) % 201) - 100, (int)((r1 >> 2) & 1));
            break;
        case 4: /* quotient near a power of two */
        {
            const double p2 = make(0, (int)((r1 >> 3) % 81) - 40, (int)((r1 >> 2) & 1));
            a = p2 * b;
            uint64_t u = bits(a) + ((r1 >> 8) % 9) - 4;
            memcpy(&a, &u, 8);
            break;
        }
        case 5: /* the edges of the valid range */
            a = make(r1 >> 12, ((r1 >> 3) & 1) ? 900 : -900, (int)((r1 >> 2) & 1));
            b = make(r2 >> 12, ((r2 >> 3) & 1) ? 100 : -100, (int)(r2 & 1));
            break;
        case 6: /* zeros of both signs */
            a = ((r1 >> 3) & 1) ? -0.0 : 0.0;
            break;
        default: /* operands of the RT0 fit's size: numerators ~1e-12..1e4, determinants ~1e-3..1e3 */
            a = make(r1 >> 12, (int)((r1 >> 3) % 56) - 40, (int)((r1 >> 2) & 1));
            b = make(r2 >> 12, (int)((r2 >> 3) % 21) - 10, (int)(r2 & 1));
        }
        bool ok = dgr::rcp_divisor_ok(b);
        const double q = dgr::div_rcp(a, b, 1.0 / b, ok);
        if (!ok) continue;
        ++nvalid;
        if (bits(q) != bits(a / b)) ++bad;
    }
    *valid = nvalid;
    return bad;
}
