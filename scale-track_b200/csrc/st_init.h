/*
 * st_init.h -- parcel initialisation clustered along a Hilbert curve, compiled unchanged for
 * the device (st_init.cu) and the host (the CPU oracle), so both produce the same parcels.
 *
 * Follows the reference's initWithHilbert! (A:559-638; A = run/icoJuliaParcelFoam/cavity3D/
 * asyncParallelTracking.jl): cloud c of nc draws each parcel's Hilbert index uniformly from
 * its own segment [round(c 2^30 / nc), round((c+1) 2^30 / nc)] of a 1024^3 curve, so every
 * cloud fills a compact region; the curve point (p_x, p_y, p_z) in [0, 1024)^3 selects the
 * cell (N_a p_a) div 1024 on each axis, and the parcel sits at a uniformly random point of
 * that cell; velocities start at zero; diameters are uniform in [d_min, d_max) (the
 * reference draws 5e-3 + 5e-3 U).  Differences from the reference, which are this project's:
 *   - random numbers come from a counter-based generator (the SplitMix64 output function of
 *     Steele, Lea and Flood, "Fast splittable pseudorandom number generators", OOPSLA 2014,
 *     applied to a key made of seed, cloud, parcel and draw), so any parcel can be generated
 *     by any thread without a shared state;
 *   - the Hilbert decode is Skilling's transpose-to-axes algorithm ("Programming the Hilbert
 *     curve", AIP Conf. Proc. 707, 2004) instead of libhilbert's hilbert_i2c (A:546-557),
 *     which is not part of the reference's sources;
 *   - the in-cell offset is scaled by 0.99999 and a coordinate that rounds onto the upper
 *     wall is moved one representable value inwards, instead of scaling the absolute
 *     position by 0.99999 (A:622-630), which only keeps parcels inside for a zero origin.
 */
#ifndef ST_INIT_H
#define ST_INIT_H

#include <stdint.h>
#include <math.h>
#include <string.h>

#if defined(__CUDACC__)
#define ST_IHD __host__ __device__ __forceinline__
#else
#define ST_IHD static inline
#endif

/* SplitMix64 output function of x + golden gamma */
ST_IHD uint64_t st_mix64(uint64_t x)
{
    uint64_t z = x + 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

/* Uniform double in [0, 1) for draw k of parcel j of cloud c (53 random bits). */
ST_IHD double st_uniform(uint64_t seed, uint32_t c, uint64_t j, uint32_t k)
{
    const uint64_t key = st_mix64(seed ^ ((uint64_t)c << 32)) ^ (j * 8u + k);
    return (double)(st_mix64(key) >> 11) * 1.1102230246251565e-16; /* 2^-53 */
}

/* Point p[3] in [0, 2^bits)^3 of Hilbert index h (3 bits per level, most significant
 * level first): the index is split into the "transpose" form, then Gray-decoded and
 * untwisted level by level (Skilling 2004). */
ST_IHD void st_hilbert3(uint64_t h, int bits, uint32_t p[3])
{
    uint32_t X[3] = {0u, 0u, 0u};
    for (int lev = 0; lev < bits; ++lev)
        for (int i = 0; i < 3; ++i) {
            const int src = 3 * bits - 1 - (3 * lev + i);       /* bit of h, MSB first */
            X[i] |= (uint32_t)((h >> src) & 1u) << (bits - 1 - lev);
        }
    const uint32_t N = 2u << (bits - 1);
    uint32_t t = X[2] >> 1;                                     /* Gray decode */
    X[2] ^= X[1];
    X[1] ^= X[0];
    X[0] ^= t;
    for (uint32_t Q = 2; Q != N; Q <<= 1) {                     /* undo excess work */
        const uint32_t P = Q - 1;
        for (int i = 2; i >= 0; --i) {
            if (X[i] & Q) {
                X[0] ^= P;
            } else {
                t = (X[0] ^ X[i]) & P;
                X[0] ^= t;
                X[i] ^= t;
            }
        }
    }
    p[0] = X[0];
    p[1] = X[1];
    p[2] = X[2];
}

/* Segment of cloud c of nc on a curve of 2^(3 bits) points: [lo, hi], both inclusive,
 * c 2^(3 bits) / nc rounded half up (A:600-601 rounds the same quotients). */
ST_IHD void st_hilbert_segment(int c, int nc, int bits, uint64_t& lo, uint64_t& hi)
{
    const uint64_t L = (uint64_t)1 << (3 * bits);
    lo = (2 * (uint64_t)c * L + (uint64_t)nc) / (2 * (uint64_t)nc);
    hi = (2 * (uint64_t)(c + 1) * L + (uint64_t)nc) / (2 * (uint64_t)nc);
}

/* nextafter(v, -inf) on the IEEE bit patterns (the same on host and device, no math
 * library): zeros step to the negative smallest subnormal, +inf to the largest finite value,
 * -inf and NaN stay. */
ST_IHD float st_next_down(float v)
{
    if (v != v || v == -INFINITY) return v;
    uint32_t b;
    memcpy(&b, &v, sizeof b);
    b = (v == 0.0f) ? 0x80000001u : (v > 0.0f ? b - 1u : b + 1u);
    memcpy(&v, &b, sizeof b);
    return v;
}
ST_IHD double st_next_down(double v)
{
    if (v != v || v == -(double)INFINITY) return v;
    uint64_t b;
    memcpy(&b, &v, sizeof b);
    b = (v == 0.0) ? 0x8000000000000001ull : (v > 0.0 ? b - 1u : b + 1u);
    memcpy(&v, &b, sizeof b);
    return v;
}

/* v, or the largest value of type P below `ending` when v is not below it. */
template <class P>
ST_IHD P st_below(P v, double ending)
{
    for (int it = 0; it < 4 && !((double)v < ending); ++it) v = st_next_down(v);
    return v;
}

/* Parcel j of cloud c: position (in P) and diameter (in double, rounded by the caller). */
template <class P>
ST_IHD void st_init_parcel(uint64_t seed, int c, int nc, uint64_t j, const int32_t N[3],
                           const double origin[3], const double ending[3], P xyz[3], double& d,
                           double d_min, double d_max)
{
    const int bits = 10;                                        /* A:589 nHilbert */
    uint64_t lo, hi;
    st_hilbert_segment(c, nc, bits, lo, hi);
    uint64_t span = hi - lo + 1;
    uint64_t h = lo + (uint64_t)(st_uniform(seed, (uint32_t)c, j, 0) * (double)span);
    if (h > hi) h = hi;
    if (h >= ((uint64_t)1 << (3 * bits))) h = ((uint64_t)1 << (3 * bits)) - 1;
    uint32_t p[3];
    st_hilbert3(h, bits, p);
    for (int a = 0; a < 3; ++a) {
        const int64_t cell = ((int64_t)N[a] * (int64_t)p[a]) >> bits;   /* A:622-630 */
        const double delta = (ending[a] - origin[a]) / (double)N[a];
        const double u = st_uniform(seed, (uint32_t)c, j, 1 + a) * 0.99999;
        xyz[a] = st_below<P>((P)(origin[a] + delta * ((double)cell + u)), ending[a]);
    }
    d = d_min + (d_max - d_min) * st_uniform(seed, (uint32_t)c, j, 4);
}

#endif /* ST_INIT_H */
