/*
 * Test harness: the library's fixed-point formatter (dgr_format.cuh) compiled as host code
 * and compared with the C library's printf("%1.15f") on the given values.  Not part of the
 * library.
 */
#include <stdio.h>
#include <string.h>

#include "../dg-rain_b200/csrc/dgr_format.cuh"

extern "C" long long dgr_t_format_mismatches(const double *v, long long n, long long *first_bad)
{
    long long bad = 0;
    *first_bad = -1;
    char a[64], b[64];
    for (long long i = 0; i < n; ++i) {
        const int la = dgr::format_f15(v[i], a);
        if (la < 0) continue; /* not formatted by the library (|v| >= 2^63) */
        a[la] = 0;
        snprintf(b, sizeof b, "%1.15f", v[i]);
        if (strcmp(a, b) != 0) {
            if (*first_bad < 0) *first_bad = i;
            ++bad;
        }
    }
    return bad;
}
