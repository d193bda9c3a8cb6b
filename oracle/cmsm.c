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
