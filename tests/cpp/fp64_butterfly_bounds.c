/* CPU check of the FP64 butterfly schedule with signed twiddles (FpArT<true>
 * in csrc/ntt.cuh): rounds of K <= 4 radix-2 stages, one normalisation at the
 * end of a round; forward (CT) multiplies by the M1 product in every stage,
 * inverse (GS) by M1 in its first three stages and M2 in the fourth.
 * Every operation is the kernel's IEEE double operation (fma correctly
 * rounded, no contraction), so the check is bit-exact to the device. Each
 * product's input magnitude precondition (M1: |y| < 2^52, M2: |y| < 2^53)
 * and every value's magnitude (< 2^53) is asserted, and every output is
 * compared with exact 128-bit modular arithmetic, on random inputs and on
 * adversarial ones (values at +-q/2, twiddles at +-(q-1)/2).
 * Usage: fp64_butterfly_bounds <trials per modulus>; exit 0 when clean. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

typedef unsigned __int128 u128;
static const double M1 = 6755399441055744.0, M2 = 13510798882111488.0;
static const double TWO52 = 4503599627370496.0, TWO53 = 9007199254740992.0;
static double q, qinv;
static uint64_t Q;
static long violations, mismatches;
static double max_val;

static void bound(double v, double lim) {
    double a = fabs(v);
    if (a > max_val) max_val = a;
    if (a >= lim) violations++;
}
static double norm(double z) { double k = fma(z, qinv, M1) - M1; return fma(-k, q, z); }
static double mulq(double y, double w, int even) {
    bound(y, even ? TWO53 : TWO52);
    double M = even ? M2 : M1;
    double h = y * w, l = fma(y, w, -h), k = fma(h, qinv, M) - M;
    return fma(-k, q, h) + l;
}
static uint64_t rnd64(void) { return ((uint64_t)rand() << 42) ^ ((uint64_t)rand() << 21) ^ (uint64_t)rand(); }
static uint64_t mm(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a * b) % Q); }
static double sgn(uint64_t w) { return w > Q / 2 ? -(double)(Q - w) : (double)w; }
static uint64_t canon(double z) {   /* FpAr::out on a normalised value */
    double c = z < 0.0 ? z + q : z;
    return (uint64_t)c;
}

static void round_check(int K, int inverse, int adv) {
    const int n = 1 << K;
    uint64_t x[16], e[16], w[16];
    double v[16];
    for (int u = 0; u < n; ++u) {
        x[u] = (adv & 1) ? (Q / 2 + (uint64_t)(rand() % 3)) % Q : rnd64() % Q;
        if ((adv & 1) && (rand() & 1)) x[u] = Q - x[u];
        v[u] = norm((double)x[u]);
        bound(v[u], 0.5 * q + 1.5);
        e[u] = x[u];
    }
    for (int u = 0; u < 16; ++u)
        w[u] = (adv & 2) ? ((rand() & 1) ? Q / 2 - (uint64_t)(rand() % 4) : Q / 2 + 1 + (uint64_t)(rand() % 4))
                         : rnd64() % Q;
    if (!inverse) {
        for (int L = 0; L < K; ++L) {
            int half = 1 << (K - 1 - L);
            for (int g = 0; g < (1 << L); ++g) {
                uint64_t wi = w[((1 << L) + g) & 15];
                for (int o = 0; o < half; ++o) {
                    int a = g * 2 * half + o, b = a + half;
                    double r = mulq(v[b], sgn(wi), 0), xx = v[a];
                    v[a] = xx + r;
                    v[b] = xx - r;
                    bound(v[a], TWO53);
                    bound(v[b], TWO53);
                    uint64_t er = mm(e[b], wi), ea = e[a];
                    e[a] = (ea + er) % Q;
                    e[b] = (ea + Q - er) % Q;
                }
            }
        }
    } else {
        for (int L = K - 1; L >= 0; --L) {
            int half = 1 << (K - 1 - L), even = (K - 1 - L) >= 3;
            for (int g = 0; g < (1 << L); ++g) {
                uint64_t wi = w[((1 << L) + g) & 15];
                for (int o = 0; o < half; ++o) {
                    int a = g * 2 * half + o, b = a + half;
                    double xx = v[a], yy = v[b];
                    v[a] = xx + yy;
                    v[b] = mulq(xx - yy, sgn(wi), even);
                    bound(v[a], TWO53);
                    bound(v[b], TWO53);
                    uint64_t ea = e[a], eb = e[b];
                    e[a] = (ea + eb) % Q;
                    e[b] = mm((ea + Q - eb) % Q, wi);
                }
            }
        }
    }
    for (int u = 0; u < n; ++u) {
        double z = norm(v[u]);
        bound(z, 0.5 * q + 1.5);
        if (canon(z) != e[u]) mismatches++;
    }
}

int main(int argc, char** argv) {
    /* the largest primes below 2^50 that are 1 mod 2^10 (n = 2^9, the worst
     * case of the bounds) and 1 mod 2^17 (n = 2^16), the first 1 mod 2^17
     * prime above 2^49, and a 30-bit NTT prime */
    const uint64_t mods[] = {1125899906826241ull, 1125899903827969ull, 562949955125249ull, 1073872897ull};
    const long trials = argc > 1 ? atol(argv[1]) : 100000;
    srand(12345);
    for (int m = 0; m < 4; ++m) {
        Q = mods[m];
        q = (double)Q;
        qinv = 1.0 / q;
        max_val = 0;
        for (long t = 0; t < trials; ++t)
            for (int K = 1; K <= 4; ++K) {
                round_check(K, 0, (int)(t & 3));
                round_check(K, 1, (int)(t & 3));
            }
        printf("q=%llu: max |value| / q = %.4f\n", (unsigned long long)Q, max_val / q);
    }
    printf("violations=%ld mismatches=%ld\n", violations, mismatches);
    return (violations || mismatches) ? 1 : 0;
}
