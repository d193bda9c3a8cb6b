/* C restatement of the reference MSM path — TEST INFRASTRUCTURE ONLY.
 *
 * The oracle: only tests, the smoke check and the benchmark's CPU-baseline
 * leg load this library, as the checker of the CUDA product.  It restates
 * the reference's CPU Pippenger for BN254 (NeonFieldOps/bn254_msm.c:1145-1187)
 * and BLS12-381 G1 (NeonFieldOps/bls12_381_ops.c:1141-1165) in portable C
 * (64-bit limbs, unsigned __int128, OpenMP threads), plus the helpers the
 * tests need: Montgomery Fr -> integer (bn254_msm.c:1537-1552), Jacobian ->
 * affine (bn254_msm.c:1502-1514) and k*G base generation.
 *
 * Layouts are the reference's: affine points NL x u64 x then y, Montgomery,
 * identity = all zero; Jacobian X, Y, Z; scalars 8 x u32 little endian.
 * curve: 0 = BN254, 1 = BLS12-381, 2 = BLS12-377 (the BLS12-381 code with its
 * own constants; the reference's twin is NeonFieldOps/bls12_377_ops.c:1476).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

typedef struct { uint64_t p[4]; uint64_t inv; uint64_t one[4]; } bn_params;
typedef struct { uint64_t p[6]; uint64_t inv; uint64_t one[6]; } bl_params;

/* Constants computed from the curve moduli: inv = -p^-1 mod 2^64, one = 2^(64 NL) mod p */
static const bn_params BN = {
    {0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
    0x87d20782e4866389ULL,
    {0xd35d438dc58f0d9dULL, 0x0a78eb28f5c70b3dULL, 0x666ea36f7879462cULL, 0x0e0a77c19a07df2fULL}};
/* BLS12-377 (same 6-limb code as BLS12-381, y^2 = x^3 + 1) */
static const bl_params B7 = {
    {0x8508c00000000001ULL, 0x170b5d4430000000ULL, 0x1ef3622fba094800ULL, 0x1a22d9f300f5138fULL,
     0xc63b05c06ca1493bULL, 0x01ae3a4617c510eaULL},
    0x8508bfffffffffffULL,
    {0x02cdffffffffff68ULL, 0x51409f837fffffb1ULL, 0x9f7db3a98a7d3ff2ULL, 0x7b4e97b76e7c6305ULL,
     0x4cf495bf803c84e8ULL, 0x008d6661e2fdf49aULL}};
static const bl_params BL = {
    {0xb9feffffffffaaabULL, 0x1eabfffeb153ffffULL, 0x6730d2a0f6b0f624ULL, 0x64774b84f38512bfULL,
     0x4b1ba7b6434bacd7ULL, 0x1a0111ea397fe69aULL},
    0x89f3fffcfffcfffdULL,
    {0x760900000002fffdULL, 0xebf4000bc40c0002ULL, 0x5f48985753c758baULL, 0x77ce585370525745ULL,
     0x5c071a97a256ec6dULL, 0x15f65ec3fa80e493ULL}};

#define NL 4
#define FN(x) bn_##x
#include "cmsm_impl.h"
#undef NL
#undef FN

#define NL 6
#define FN(x) bl_##x
#include "cmsm_impl.h"
#undef NL
#undef FN

/* Fr moduli and Montgomery constants (R = 2^256 for both curves' Fr) */
static const uint64_t FR_BN[4] = {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL,
                                  0xb85045b68181585dULL, 0x30644e72e131a029ULL};
static const uint64_t FR_BL[4] = {0xffffffff00000001ULL, 0x53bda402fffe5bfeULL,
                                  0x3339d80809a1d805ULL, 0x73eda753299d7d48ULL};
static const uint64_t FR_B7[4] = {0x0a11800000000001ULL, 0x59aa76fed0000001ULL,
                                  0x60b44d1e5c37b001ULL, 0x12ab655e9a2ca556ULL};

/* the 6-limb parameter set of curve 1 (BLS12-381) or 2 (BLS12-377) */
static const bl_params *bl_of(int curve) { return curve == 2 ? &B7 : &BL; }

static uint64_t neg_inv64(uint64_t p0) {
    uint64_t x = 1;
    for (int i = 0; i < 6; i++) x *= 2 - p0 * x; /* Newton: x = p0^-1 mod 2^64 */
    return (uint64_t)0 - x;
}

/* Montgomery reduce of a 4-limb value (multiply by 1 in Montgomery form) */
static void fr_from_mont(const uint64_t *q, const uint64_t *a, uint64_t *r) {
    uint64_t inv = neg_inv64(q[0]);
    uint64_t t[5] = {a[0], a[1], a[2], a[3], 0};
    for (int i = 0; i < 4; i++) {
        uint64_t m = t[0] * inv;
        u128 c = (u128)m * q[0] + t[0];
        c >>= 64;
        for (int j = 1; j < 4; j++) {
            c += (u128)m * q[j] + t[j];
            t[j - 1] = (uint64_t)c;
            c >>= 64;
        }
        c += t[4];
        t[3] = (uint64_t)c;
        t[4] = (uint64_t)(c >> 64);
    }
    int ge = t[4] != 0;
    if (!ge) {
        ge = 1;
        for (int i = 3; i >= 0; i--) {
            if (t[i] > q[i]) break;
            if (t[i] < q[i]) { ge = 0; break; }
        }
    }
    if (ge) {
        u128 bw = 0;
        for (int i = 0; i < 4; i++) {
            u128 d = (u128)t[i] - q[i] - bw;
            t[i] = (uint64_t)d;
            bw = (d >> 64) & 1;
        }
    }
    memcpy(r, t, 32);
}

int cm_threads = 0;

static int nthreads(void) {
    if (cm_threads > 0) return cm_threads;
#ifdef _OPENMP
    extern int omp_get_max_threads(void);
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void cm_set_threads(int t) { cm_threads = t; }

/* MSM, result as affine (identity = zeros).  Returns 0. */
int cm_msm(int curve, const uint64_t *points, const uint32_t *scalars, long n, uint64_t *out_affine) {
    if (curve == 0) {
        bn_jac r;
        bn_pippenger(&BN, (const bn_aff *)points, scalars, n, &r, nthreads());
        bn_to_affine(&BN, &r, (bn_aff *)out_affine);
    } else {
        bl_jac r;
        bl_pippenger(bl_of(curve), (const bl_aff *)points, scalars, n, &r, nthreads());
        bl_to_affine(bl_of(curve), &r, (bl_aff *)out_affine);
    }
    return 0;
}

/* Jacobian (X,Y,Z Montgomery) -> affine */
void cm_jacobian_to_affine(int curve, const uint64_t *jac, uint64_t *aff) {
    if (curve == 0) bn_to_affine(&BN, (const bn_jac *)jac, (bn_aff *)aff);
    else bl_to_affine(bl_of(curve), (const bl_jac *)jac, (bl_aff *)aff);
}

/* out[i] = k[i] * G for the given affine generator, as affine points */
void cm_fixed_base_mul(int curve, const uint64_t *gen_affine, const uint32_t *ks, long n, uint64_t *out) {
    #pragma omp parallel for schedule(static) num_threads(nthreads())
    for (long i = 0; i < n; i++) {
        if (curve == 0) {
            bn_jac r;
            bn_scalar_mul(&BN, (const bn_aff *)gen_affine, ks + 8 * i, &r);
            bn_to_affine(&BN, &r, (bn_aff *)(out + 8 * i));
        } else {
            bl_jac r;
            bl_scalar_mul(bl_of(curve), (const bl_aff *)gen_affine, ks + 8 * i, &r);
            bl_to_affine(bl_of(curve), &r, (bl_aff *)(out + 12 * i));
        }
    }
}

/* Montgomery Fr (4 x u64) -> integer (4 x u64 == 8 x u32 LE) */
void cm_fr_from_mont(int curve, const uint64_t *mont, uint64_t *out, long n) {
    const uint64_t *q = curve == 0 ? FR_BN : curve == 1 ? FR_BL : FR_B7;
    #pragma omp parallel for schedule(static) num_threads(nthreads())
    for (long i = 0; i < n; i++) fr_from_mont(q, mont + 4 * i, out + 4 * i);
}

/* r = a + b for affine inputs (identity = zeros); helper for partial-sum checks */
void cm_affine_add(int curve, const uint64_t *a, const uint64_t *b, uint64_t *r) {
    if (curve == 0) {
        bn_jac A, R;
        bn_set_id(&BN, &A);
        bn_add_aff(&BN, &A, (const bn_aff *)a, &A);
        bn_add_aff(&BN, &A, (const bn_aff *)b, &R);
        bn_to_affine(&BN, &R, (bn_aff *)r);
    } else {
        const bl_params *P = bl_of(curve);
        bl_jac A, R;
        bl_set_id(P, &A);
        bl_add_aff(P, &A, (const bl_aff *)a, &A);
        bl_add_aff(P, &A, (const bl_aff *)b, &R);
        bl_to_affine(P, &R, (bl_aff *)r);
    }
}

/* ---------------------------------------------------------------- inputs
 * The seeded counter-based generator of the synthetic inputs, restated for
 * the host (the same words as the Python restatement's draw_word, so host
 * and device inputs of one seed are the same bytes):
 *   word = splitmix64(splitmix64(seed*FNV + stream*golden ^ (index*8 + w)) ^ attempt*C)
 * uniform values below r by masked rejection (64 attempts, then 1). */
static uint64_t sm64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static uint64_t draw_word(uint64_t seed, uint64_t stream, uint64_t index, uint64_t attempt, uint64_t w) {
    uint64_t ctr = seed * 0x100000001B3ULL + stream * 0x9E3779B1ULL;
    ctr = sm64(ctr ^ (index * 8 + w));
    return sm64(ctr ^ (attempt * 0xD1B54A32D192ED03ULL));
}

static int lt4(const uint64_t *a, const uint64_t *b) {
    for (int i = 3; i >= 0; i--) {
        if (a[i] < b[i]) return 1;
        if (a[i] > b[i]) return 0;
    }
    return 0;
}

static void uniform_below_r(const uint64_t *r, uint64_t seed, uint64_t stream, uint64_t index, int lo,
                            uint64_t *out) {
    int nbits = 256;
    while (nbits > 0 && !((r[(nbits - 1) / 64] >> ((nbits - 1) % 64)) & 1)) nbits--;
    for (uint64_t att = 0; att < 64; att++) {
        uint64_t v[4];
        for (int w = 0; w < 4; w++) v[w] = draw_word(seed, stream, index, att, w);
        if (nbits < 256) v[3] &= (nbits - 192) >= 64 ? ~0ULL : ((1ULL << (nbits - 192)) - 1);
        int nz = (v[0] | v[1] | v[2] | v[3]) != 0;
        if (lt4(v, r) && (!lo || nz)) { memcpy(out, v, 32); return; }
    }
    out[0] = 1; out[1] = out[2] = out[3] = 0;
}

/* s * 2^256 mod r by 256 modular doublings (s < r) */
static void fr_to_mont_slow(const uint64_t *r, const uint64_t *s, uint64_t *out) {
    uint64_t v[4];
    memcpy(v, s, 32);
    for (int k = 0; k < 256; k++) {
        uint64_t top = v[3] >> 63;
        for (int i = 3; i > 0; i--) v[i] = (v[i] << 1) | (v[i - 1] >> 63);
        v[0] <<= 1;
        if (top || !lt4(v, r)) {
            u128 bw = 0;
            for (int i = 0; i < 4; i++) {
                u128 d = (u128)v[i] - r[i] - bw;
                v[i] = (uint64_t)d;
                bw = (d >> 64) & 1;
            }
        }
    }
    memcpy(out, v, 32);
}

enum { ST_BASE_K = 1, ST_SCALAR = 2, ST_KIND = 3 };

/* n scalars of element indices index0.. : dist 0 uniform in Fr, 1 witness-like
 * (40% 0, 20% 1, 25% below 2^32, 15% uniform); fmt 0 integer, 1 Montgomery. */
void cm_gen_scalars(int curve, uint64_t seed, uint64_t index0, long n, int dist, int fmt, uint64_t *out) {
    const uint64_t *q = curve == 0 ? FR_BN : curve == 1 ? FR_BL : FR_B7;
    #pragma omp parallel for schedule(static) num_threads(nthreads())
    for (long i = 0; i < n; i++) {
        uint64_t gi = index0 + (uint64_t)i, s[4] = {0, 0, 0, 0};
        if (dist == 0) {
            uniform_below_r(q, seed, ST_SCALAR, gi, 0, s);
        } else {
            uint64_t u = draw_word(seed, ST_KIND, gi, 0, 0) % 100;
            if (u < 40) {
            } else if (u < 60) {
                s[0] = 1;
            } else if (u < 85) {
                s[0] = draw_word(seed, ST_SCALAR, gi, 0, 0) & 0xFFFFFFFFULL;
            } else {
                uniform_below_r(q, seed, ST_SCALAR, gi, 0, s);
            }
        }
        if (fmt == 1) fr_to_mont_slow(q, s, s);
        memcpy(out + 4 * i, s, 32);
    }
}

/* n bases P_i = k_i * G, k_i uniform in [1, r) (element indices index0..),
 * affine Montgomery in the reference layout; 16-bit comb.  Returns 0, or -1
 * when the comb table cannot be allocated. */
int cm_gen_bases(int curve, const uint64_t *gen_affine, uint64_t seed, uint64_t index0, long n, uint64_t *out) {
    const uint64_t *q = curve == 0 ? FR_BN : curve == 1 ? FR_BL : FR_B7;
    uint64_t *ks = (uint64_t *)malloc(32 * (size_t)(n > 0 ? n : 1));
    if (!ks) return -1;
    #pragma omp parallel for schedule(static) num_threads(nthreads())
    for (long i = 0; i < n; i++) uniform_below_r(q, seed, ST_BASE_K, index0 + (uint64_t)i, 1, ks + 4 * i);
    int rc = 0;
    if (curve == 0) {
        bn_aff *tab = bn_comb_table(&BN, (const bn_aff *)gen_affine, nthreads());
        if (!tab) rc = -1;
        else bn_comb_mul(&BN, tab, (const uint32_t *)ks, n, (bn_aff *)out, nthreads());
        free(tab);
    } else {
        const bl_params *P = bl_of(curve);
        bl_aff *tab = bl_comb_table(P, (const bl_aff *)gen_affine, nthreads());
        if (!tab) rc = -1;
        else bl_comb_mul(P, tab, (const uint32_t *)ks, n, (bl_aff *)out, nthreads());
        free(tab);
    }
    free(ks);
    return rc;
}

/* ---------------------------------------------------------------- GLV bound
 * The largest bit length of |k1|, |k2| over n scalars k uniform in [0, r)
 * (seeded generator, stream ST_SCALAR) for the Babai split
 *   c_j = (k * g_j + 2^255) >> 256,  k1 = k - c1 a1 - c2 a2,  k2 = -c1 b1 - c2 b2
 * (the device's decomposition and the Python restatement's glv_split).
 * Constants are 256-bit two's complement (4 x u64 little endian); all
 * arithmetic is exact: k * g as a 512-bit product, the rest modulo 2^256,
 * which holds every true value here (|c_j a_i| < 2^255). */
typedef struct { uint64_t w[4]; } i256;

static int i256_neg_p(const i256 *a) { return (int)(a->w[3] >> 63); }

static i256 i256_negate(i256 a) {
    u128 c = 1;
    for (int i = 0; i < 4; i++) {
        c += (u128)(~a.w[i]);
        a.w[i] = (uint64_t)c;
        c >>= 64;
    }
    return a;
}

static i256 i256_add(i256 a, const i256 *b) {
    u128 c = 0;
    for (int i = 0; i < 4; i++) {
        c += (u128)a.w[i] + b->w[i];
        a.w[i] = (uint64_t)c;
        c >>= 64;
    }
    return a;
}

static i256 i256_mul_lo(const i256 *a, const i256 *b) { /* a * b mod 2^256 */
    uint64_t t[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
        u128 c = 0;
        for (int j = 0; i + j < 4; j++) {
            c += (u128)a->w[i] * b->w[j] + t[i + j];
            t[i + j] = (uint64_t)c;
            c >>= 64;
        }
    }
    i256 r;
    memcpy(r.w, t, 32);
    return r;
}

/* floor((k * g + 2^255) / 2^256) for k >= 0, g signed */
static i256 babai_c(const uint64_t *k, i256 g) {
    int neg = i256_neg_p(&g);
    if (neg) g = i256_negate(g);
    uint64_t p[8] = {0};
    for (int i = 0; i < 4; i++) {
        u128 c = 0;
        for (int j = 0; j < 4; j++) {
            c += (u128)k[i] * g.w[j] + p[i + j];
            p[i + j] = (uint64_t)c;
            c >>= 64;
        }
        p[i + 4] = (uint64_t)c;
    }
    i256 hi;
    if (!neg) { /* (P + 2^255) >> 256 */
        u128 c = (u128)p[3] + (1ULL << 63);
        c >>= 64;
        for (int i = 0; i < 4; i++) {
            c += p[4 + i];
            hi.w[i] = (uint64_t)c;
            c >>= 64;
        }
        return hi;
    }
    /* floor((2^255 - P) / 2^256) = -ceil((P - 2^255) / 2^256) */
    uint64_t q[8];
    u128 bw = 0;
    for (int i = 0; i < 8; i++) {
        u128 d = (u128)p[i] - (i == 3 ? (1ULL << 63) : 0) - bw;
        q[i] = (uint64_t)d;
        bw = (d >> 64) & 1;
    }
    if (bw) { /* P < 2^255: the quotient is 0 */
        memset(hi.w, 0, 32);
        return hi;
    }
    int frac = (q[0] | q[1] | q[2] | q[3]) != 0;
    for (int i = 0; i < 4; i++) hi.w[i] = q[4 + i];
    if (frac) {
        i256 one = {{1, 0, 0, 0}};
        hi = i256_add(hi, &one);
    }
    return i256_negate(hi);
}

static int bits_of_abs(i256 v) {
    if (i256_neg_p(&v)) v = i256_negate(v);
    for (int i = 3; i >= 0; i--)
        if (v.w[i]) return 64 * i + 64 - __builtin_clzll(v.w[i]);
    return 0;
}

/* consts: g1, g2, a1, a2, b1, b2 (6 x 4 u64).  Returns the largest bit length
 * of |k1|, |k2| over n seeded scalars and the m extra scalars in `extra`. */
int cm_glv_max_bits(int curve, const uint64_t *consts, uint64_t seed, long n, const uint64_t *extra, long m) {
    const uint64_t *q = curve == 0 ? FR_BN : curve == 1 ? FR_BL : FR_B7;
    i256 g1, g2, a1, a2, b1, b2;
    memcpy(g1.w, consts, 32);
    memcpy(g2.w, consts + 4, 32);
    memcpy(a1.w, consts + 8, 32);
    memcpy(a2.w, consts + 12, 32);
    memcpy(b1.w, consts + 16, 32);
    memcpy(b2.w, consts + 20, 32);
    int best = 0;
    #pragma omp parallel for schedule(static) reduction(max : best) num_threads(nthreads())
    for (long i = 0; i < n + m; i++) {
        uint64_t k[4];
        if (i < n) uniform_below_r(q, seed, ST_SCALAR, (uint64_t)i, 0, k);
        else memcpy(k, extra + 4 * (i - n), 32);
        i256 c1 = babai_c(k, g1), c2 = babai_c(k, g2);
        i256 kk;
        memcpy(kk.w, k, 32);
        i256 t1 = i256_negate(i256_mul_lo(&c1, &a1)), t2 = i256_negate(i256_mul_lo(&c2, &a2));
        i256 k1 = i256_add(i256_add(kk, &t1), &t2);
        i256 u1 = i256_negate(i256_mul_lo(&c1, &b1)), u2 = i256_negate(i256_mul_lo(&c2, &b2));
        i256 k2 = i256_add(u1, &u2);
        int b = bits_of_abs(k1);
        int b2v = bits_of_abs(k2);
        if (b2v > b) b = b2v;
        if (b > best) best = b;
    }
    return best;
}
