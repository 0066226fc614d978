/* Host restatement of the device's correctly rounded division by a run
 * constant (xdiv_flag in csrc/nicr_physics.h) and an exhaustive-style check
 * of it against IEEE division (x86-64 SSE2 double: correctly rounded).
 *
 * The method: the host stores y = RN(1/b) and the double-word reciprocal
 * zh = RD(1/b), zl = RN(1/b - zh) >= 0, the latter two scaled by 2^128. For
 * b > 0 with 2^-60 <= b <= 2^60 and any numerator a:
 *     as = a * 2^128                       exact for |a| < 2^895, subnormals included
 *     q0 = RN(a*zh' + RN(a*zl'))           within (1/2 + 2^-51) ulp of as/b
 *     e  = RN(q0*b - as)                   exact (q0 within one ulp; as/b >= 2^-1006)
 *     qs = RN(q0 - e*y)                    = RN(as/b) (Markstein's correction theorem,
 *                                           IBM J. Res. Dev. 34(1), 1990)
 *     q  = qs * 2^-128                     exact when a/b is normal or zero
 * (the double-word reciprocal of a divisor known in advance: Brisebarre,
 * Muller, Raina, IEEE Trans. Comput. 53(8), 2004). Zeros keep their sign
 * (zl >= 0, e formed as q0*b - as). The result is flagged, and the IEEE
 * division taken, when qs is nonzero below 2^-894 (a subnormal quotient,
 * which the final scaling would round a second time), infinite or NaN
 * (infinite, NaN or huge numerators), or the divisor is out of range.
 *
 * Cases: random numerators over the whole exponent range, subnormals among
 * them, numerators whose quotient lies within ~2^-102 relative of a rounding
 * midpoint (built with integer arithmetic, below) and their neighbours,
 * signed zeros, infinities and NaN; divisors with random mantissas, mantissas
 * of all ones, powers of two, near sqrt(2), above 1, and the grid spacings
 * and time steps of the solver's configurations.
 *
 * Usage: division_check <cases per divisor> <seed>; prints
 * "checked N mismatches M fallbacks F near-midpoint H" and exits 1 on any
 * mismatch. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    double b, y, zh, zl;
    unsigned erange, gate;
} divc;

static divc make(double b) {
    divc d;
    d.b = b;
    d.y = 1.0 / b;
    double zh = d.y;
    double rem = fma(-zh, b, 1.0); /* exact: zh within one ulp of 1/b */
    if (rem < 0) {
        zh = nextafter(zh, 0.0);
        rem = fma(-zh, b, 1.0);
    }
    d.zh = ldexp(zh, 128);
    d.zl = ldexp(rem / b, 128);
    const int fast = isnormal(b) && b > 0 && b >= ldexp(1.0, -60) && b <= ldexp(1.0, 60);
    d.gate = fast ? 0u : 1u;
    d.erange = 0;
    return d;
}

static uint64_t bits(double x) {
    uint64_t u;
    memcpy(&u, &x, 8);
    return u;
}
static double from_bits(uint64_t u) {
    double x;
    memcpy(&x, &u, 8);
    return x;
}

/* the device sequence; *fallback set when the result is flagged */
static double xdiv(double a, const divc* d, int* fallback) {
    const double as = a * 0x1p128;
    const double t = a * d->zl;
    const double q0 = fma(a, d->zh, t);
    const double e = fma(q0, d->b, -as);
    const double qs = fma(-e, d->y, q0);
    const unsigned u = (unsigned)(bits(qs) >> 32) & 0x7FFFFFFFu;
    const int bad = (u - 1u) < 0x080FFFFFu || u >= 0x7FF00000u || d->gate;
    *fallback = bad;
    return bad ? a / d->b : qs * 0x1p-128;
}

static uint64_t s = 0x243F6A8885A308D3ull;
static uint64_t rnd(void) {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return s;
}

static long long checked = 0, mism = 0, fallbacks = 0;

static void one(double a, const divc* d) {
    int fb;
    const double q = xdiv(a, d, &fb), w = a / d->b;
    ++checked;
    fallbacks += fb;
    if (bits(q) != bits(w) && !(isnan(q) && isnan(w))) {
        if (mism < 10)
            printf("MISMATCH a=%a b=%a got %a want %a\n", a, d->b, q, w);
        ++mism;
    }
}

/* numerators whose quotient by b lies within ~2^-102 relative of a rounding
 * midpoint: with b = B * 2^k (B odd), take M = delta / B mod 2^54 for a small
 * odd delta, kept when it has 54 bits (M odd, 2^53 <= M < 2^54); then
 * B * M = A * 2^54 + delta with A < B <= 2^53, and a = A (scaled) gives
 * a / b = (M - delta / B) * 2^-54 (scaled): next to M * 2^-54, a midpoint of
 * the 53-bit grid, closer than the double-word reciprocal alone resolves. */
static uint64_t inverse_mod_2_54(uint64_t b) {
    uint64_t x = b; /* Newton's iteration for the inverse of an odd b modulo 2^64 */
    for (int i = 0; i < 6; ++i) x *= 2 - b * x;
    return x & ((1ull << 54) - 1);
}
static long long hard = 0;
static void near_midpoints(const divc* d, int n) {
    int eb;
    uint64_t B = (uint64_t)ldexp(frexp(d->b, &eb), 53);
    if (B == 0) return;
    while (!(B & 1)) B >>= 1;
    const uint64_t inv = inverse_mod_2_54(B), mask = (1ull << 54) - 1;
    for (int i = 0; i < n; ++i) {
        const long long delta = ((long long)(rnd() % 32) - 16) | 1;   /* odd, -15 .. 15 */
        const uint64_t M = ((uint64_t)delta * inv) & mask;
        if (!(M >> 53)) continue;
        const __int128 num = (__int128)((unsigned __int128)B * M) - delta;
        if (num <= 0 || (num & ((((__int128)1) << 54) - 1)) != 0) continue;
        const uint64_t A = (uint64_t)(num >> 54);
        const double a = ldexp((double)A, (int)(rnd() % 2000) - 1100);
        ++hard;
        one(a, d);
        one(-a, d);
        one(nextafter(a, INFINITY), d);
        one(nextafter(a, -INFINITY), d);
    }
}

static void run_divisor(double b, long long n) {
    const divc d = make(b);
    for (long long i = 0; i < n; ++i) {
        const uint64_t r = rnd();
        double a;
        switch (i & 7) {
        case 0: /* any finite bit pattern */
            a = from_bits(r);
            if (!isfinite(a)) continue;
            break;
        case 1: /* typical field values */
            a = ldexp((double)(r >> 11) * 0x1p-53, (int)(rnd() % 60) - 50);
            break;
        case 2: /* differences of nearby values: few significant bits */
            a = ldexp((double)(r >> 40), (int)(rnd() % 200) - 100);
            break;
        case 3: /* subnormals */
            a = from_bits(r & 0x000FFFFFFFFFFFFFull);
            break;
        default: /* every exponent */
            a = ldexp(1.0 + (double)(r >> 12) * 0x1p-52, (int)(rnd() % 2100) - 1075);
            break;
        }
        if (r & 1) a = -a;
        one(a, &d);
    }
    near_midpoints(&d, (int)(n / 16));
    const double specials[] = {0.0, -0.0, 0x1p-1074, -0x1p-1074, 0x1p-1022, 0x1.fffffffffffffp-1023,
                               0x1p-900, 0x1p-901, 0x1.fffffffffffffp+900, 0x1p+901, 0x1.fffffffffffffp+1023,
                               INFINITY, -INFINITY, 1.0, -1.0, 3.0, 0.1};
    for (unsigned k = 0; k < sizeof specials / sizeof specials[0]; ++k) one(specials[k], &d);
    one(NAN, &d);
}

int main(int argc, char** argv) {
    const long long n = argc > 1 ? atoll(argv[1]) : 200000;
    s ^= argc > 2 ? strtoull(argv[2], 0, 10) * 0x9E3779B97F4A7C15ull : 0;
    /* grid spacings, their squares and time steps of the solver's configurations */
    const double fixed[] = {5e-9, 5e-9 * 5e-9, 1e-8, 1e-8 * 1e-8, 2.5e-9, 2.5e-9 * 2.5e-9, 1e-12, 5e-13, 2e-12,
                            1e-9, 1e-9 * 1e-9, 1.0, 2.0, 0.5, 3.0, 0x1.fffffffffffffp+0, 0x1.6a09e667f3bcdp+0,
                            0x1.6a09e667f3bccp+0, 0x1.0000000000001p+0, 0x1p-60, 0x1.fffffffffffffp+59, 7.0};
    for (unsigned k = 0; k < sizeof fixed / sizeof fixed[0]; ++k) run_divisor(fixed[k], n);
    for (int k = 0; k < 48; ++k) { /* random mantissas, all ones and near 1 */
        const int e = (int)(rnd() % 121) - 60;
        double m;
        if (k % 3 == 0) m = 2.0 - ldexp(1.0, -(int)(rnd() % 52) - 1);
        else if (k % 3 == 1) m = 1.0 + ldexp((double)(rnd() >> 44), -52);
        else m = 1.0 + (double)(rnd() >> 12) * 0x1p-52;
        run_divisor(ldexp(m, e), n);
    }
    for (int k = 0; k < 4096; ++k) { /* many divisors, near-midpoint numerators only */
        const divc d = make(ldexp(1.0 + (double)(rnd() >> 12) * 0x1p-52, (int)(rnd() % 121) - 60));
        near_midpoints(&d, (int)(n / 4096 + 64));
    }
    run_divisor(-3.0, n / 8); /* not guarded: the IEEE division throughout */
    run_divisor(0x1p-70, n / 8);
    run_divisor(0x1.8p+40, n / 4); /* large divisors: subnormal quotients */
    run_divisor(0x1.fffffffffffffp+59, n / 4);
    printf("checked %lld mismatches %lld fallbacks %lld near-midpoint %lld\n", checked, mism, fallbacks, hard);
    return mism ? 1 : 0;
}
