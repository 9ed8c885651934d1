/*
 * fbb_oracle.c -- CPU ORACLE for the fractional-Brownian-bridge centerline generator
 * (test infrastructure only; only tests/, smoke() and bench.py's baseline leg load it).
 *
 * The reference generator is FBB_with_parameters.m:76-126, which draws fBm with
 * MATLAB's closed `wfbm` (Wavelet Toolbox, not vendored) and MATLAB's randn/rand
 * streams.  Neither is reproducible here, so generator parity is UNPINNED against
 * the reference; it is checked statistically (S2(r) ~ r^{2H}, the reference's own
 * check at FBB_with_parameters.m:150-166) and bit-for-bit against this oracle's
 * random stream.
 *
 * Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3", SC'11), restated from the paper.  Gaussians by the
 * Box-Muller transform on 53-bit uniforms.  The counter layout is the project's own:
 *   ctr = {index, tube, stream, 0}, key = {seed_lo, seed_hi}
 *   stream 0,1,2 : Gaussian pair (Za, Zb) for coordinate 0,1,2 at circulant index `index`
 *   stream 3     : uniform shift for coordinate `index` (0..2)
 *   stream 4     : circulation sign (index 0)
 */
#include <math.h>
#include <stdint.h>

#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

static void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)PHILOX_M0 * c[0];
        const uint64_t p1 = (uint64_t)PHILOX_M1 * c[2];
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
        k0 += PHILOX_W0;
        k1 += PHILOX_W1;
    }
}

/* the bare block function on an arbitrary counter and key (for the published KAT vectors) */
void orc_philox_raw(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    philox4x32_10(c, key[0], key[1]);
    out[0] = c[0]; out[1] = c[1]; out[2] = c[2]; out[3] = c[3];
}

void orc_philox(uint64_t seed, uint32_t index, uint32_t tube, uint32_t stream, uint32_t out[4])
{
    uint32_t c[4] = {index, tube, stream, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    out[0] = c[0]; out[1] = c[1]; out[2] = c[2]; out[3] = c[3];
}

/* 53-bit uniform in (0,1) from two words */
static inline double u53(uint32_t hi, uint32_t lo)
{
    return ((double)(hi >> 5) * 67108864.0 + (double)(lo >> 6) + 0.5) * (1.0 / 9007199254740992.0);
}

/* n Gaussian pairs for (tube, coord): za[k] + i zb[k], k = 0..n-1 */
void orc_fbb_gauss(uint64_t seed, uint32_t tube, uint32_t coord, int n, double *za, double *zb)
{
    const double two_pi = 6.28318530717958647692;
    for (int k = 0; k < n; ++k) {
        uint32_t w[4];
        orc_philox(seed, (uint32_t)k, tube, coord, w);
        const double a = u53(w[0], w[1]), b = u53(w[2], w[3]);
        const double r = sqrt(-2.0 * log(a));
        za[k] = r * cos(two_pi * b);
        zb[k] = r * sin(two_pi * b);
    }
}

/* uniform shift in [0,1) for coordinate co and circulation sign (+1/-1) of a tube */
double orc_fbb_shift(uint64_t seed, uint32_t tube, uint32_t coord)
{
    uint32_t w[4];
    orc_philox(seed, coord, tube, 3u, w);
    return ((double)(w[0] >> 5) * 67108864.0 + (double)(w[1] >> 6)) * (1.0 / 9007199254740992.0);
}

int orc_fbb_sign(uint64_t seed, uint32_t tube)
{
    uint32_t w[4];
    orc_philox(seed, 0u, tube, 4u, w);
    return (w[0] & 1u) ? -1 : 1;
}
