/* Field / curve / Pippenger template for the C oracle (TEST INFRASTRUCTURE).
 *
 * Included twice by cmsm.c with NL = 4 (BN254 Fp, 4x64-bit limbs) and NL = 6
 * (BLS12-381 Fp, 6x64-bit limbs).  FN(x) names the instantiation.  The
 * arithmetic follows the reference C kernels it restates:
 *   - CIOS Montgomery multiply        bn254_msm.c:38-154, bls12_381_ops.c:479-521
 *   - Jacobian dbl / add / mixed add  bn254_msm.c:373-533, bls12_381_ops.c:789-944
 *   - batch to affine (Montgomery's trick, Fermat inverse) bn254_msm.c:544-599
 *   - per-window worker: bucket accumulate, running sum   bn254_msm.c:647-698
 *   - window sizing, Horner combine    bn254_msm.c:621-631, 1145-1187
 * Written from the published algorithms (Koc-Acar-Kaliski CIOS; the
 * "add-2007-bl" / "dbl-2009-l" Jacobian formulas), not copied.
 */

typedef struct { uint64_t x[NL], y[NL], z[NL]; } FN(jac);
typedef struct { uint64_t x[NL], y[NL]; } FN(aff);

static inline int FN(is_zero)(const uint64_t *a) {
    uint64_t t = 0;
    for (int i = 0; i < NL; i++) t |= a[i];
    return t == 0;
}

static inline int FN(eq)(const uint64_t *a, const uint64_t *b) {
    uint64_t t = 0;
    for (int i = 0; i < NL; i++) t |= a[i] ^ b[i];
    return t == 0;
}

static inline int FN(geq_p)(const uint64_t *a, const FN(params) *P) {
    for (int i = NL - 1; i >= 0; i--) {
        if (a[i] > P->p[i]) return 1;
        if (a[i] < P->p[i]) return 0;
    }
    return 1;
}

static inline void FN(sub_p)(uint64_t *a, const FN(params) *P) {
    u128 bw = 0;
    for (int i = 0; i < NL; i++) {
        u128 d = (u128)a[i] - P->p[i] - bw;
        a[i] = (uint64_t)d;
        bw = (d >> 64) & 1;
    }
}

static inline void FN(add)(const FN(params) *P, const uint64_t *a, const uint64_t *b, uint64_t *r) {
    u128 c = 0;
    uint64_t t[NL];
    for (int i = 0; i < NL; i++) {
        c += (u128)a[i] + b[i];
        t[i] = (uint64_t)c;
        c >>= 64;
    }
    if (c || FN(geq_p)(t, P)) FN(sub_p)(t, P);
    memcpy(r, t, sizeof t);
}

static inline void FN(sub)(const FN(params) *P, const uint64_t *a, const uint64_t *b, uint64_t *r) {
    u128 bw = 0;
    uint64_t t[NL];
    for (int i = 0; i < NL; i++) {
        u128 d = (u128)a[i] - b[i] - bw;
        t[i] = (uint64_t)d;
        bw = (d >> 64) & 1;
    }
    if (bw) {
        u128 c = 0;
        for (int i = 0; i < NL; i++) {
            c += (u128)t[i] + P->p[i];
            t[i] = (uint64_t)c;
            c >>= 64;
        }
    }
    memcpy(r, t, sizeof t);
}

/* CIOS Montgomery product a*b/2^(64 NL) mod p */
static inline void FN(mul)(const FN(params) *P, const uint64_t *a, const uint64_t *b, uint64_t *r) {
    uint64_t t[NL + 2];
    memset(t, 0, sizeof t);
    for (int i = 0; i < NL; i++) {
        u128 c = 0;
        for (int j = 0; j < NL; j++) {
            c += (u128)a[j] * b[i] + t[j];
            t[j] = (uint64_t)c;
            c >>= 64;
        }
        c += t[NL];
        t[NL] = (uint64_t)c;
        t[NL + 1] = (uint64_t)(c >> 64);
        uint64_t m = t[0] * P->inv;
        c = (u128)m * P->p[0] + t[0];
        c >>= 64;
        for (int j = 1; j < NL; j++) {
            c += (u128)m * P->p[j] + t[j];
            t[j - 1] = (uint64_t)c;
            c >>= 64;
        }
        c += t[NL];
        t[NL - 1] = (uint64_t)c;
        t[NL] = t[NL + 1] + (uint64_t)(c >> 64);
    }
    if (t[NL] || FN(geq_p)(t, P)) FN(sub_p)(t, P);
    memcpy(r, t, NL * 8);
}

static void FN(inv)(const FN(params) *P, const uint64_t *a, uint64_t *r) {
    /* Fermat: a^(p-2), square-and-multiply over the bits of p-2 */
    uint64_t e[NL], acc[NL];
    memcpy(e, P->p, sizeof e);
    e[0] -= 2; /* p is odd and > 2: no borrow */
    memcpy(acc, P->one, sizeof acc);
    for (int i = NL * 64 - 1; i >= 0; i--) {
        FN(mul)(P, acc, acc, acc);
        if ((e[i / 64] >> (i % 64)) & 1) FN(mul)(P, acc, a, acc);
    }
    memcpy(r, acc, sizeof acc);
}

static inline void FN(set_id)(const FN(params) *P, FN(jac) *R) {
    memcpy(R->x, P->one, NL * 8);
    memcpy(R->y, P->one, NL * 8);
    memset(R->z, 0, NL * 8);
}

static inline int FN(jac_is_id)(const FN(jac) *A) { return FN(is_zero)(A->z); }

/* dbl-2009-l (a = 0) */
static void FN(dbl)(const FN(params) *P, const FN(jac) *A, FN(jac) *R) {
    if (FN(jac_is_id)(A) || FN(is_zero)(A->y)) { FN(set_id)(P, R); return; }
    uint64_t a[NL], b[NL], c[NL], d[NL], e[NL], f[NL], t[NL];
    FN(mul)(P, A->x, A->x, a);
    FN(mul)(P, A->y, A->y, b);
    FN(mul)(P, b, b, c);
    FN(add)(P, A->x, b, t);
    FN(mul)(P, t, t, t);
    FN(sub)(P, t, a, t);
    FN(sub)(P, t, c, t);
    FN(add)(P, t, t, d);
    FN(add)(P, a, a, e);
    FN(add)(P, e, a, e);
    FN(mul)(P, e, e, f);
    FN(jac) o;
    FN(sub)(P, f, d, o.x);
    FN(sub)(P, o.x, d, o.x);
    FN(sub)(P, d, o.x, t);
    FN(mul)(P, e, t, o.y);
    FN(add)(P, c, c, c);
    FN(add)(P, c, c, c);
    FN(add)(P, c, c, c);
    FN(sub)(P, o.y, c, o.y);
    FN(mul)(P, A->y, A->z, o.z);
    FN(add)(P, o.z, o.z, o.z);
    *R = o;
}

/* add-2007-bl with the equal / opposite cases made explicit */
static void FN(addj)(const FN(params) *P, const FN(jac) *A, const FN(jac) *B, FN(jac) *R) {
    if (FN(jac_is_id)(A)) { *R = *B; return; }
    if (FN(jac_is_id)(B)) { *R = *A; return; }
    uint64_t z1z1[NL], z2z2[NL], u1[NL], u2[NL], s1[NL], s2[NL], t[NL];
    FN(mul)(P, A->z, A->z, z1z1);
    FN(mul)(P, B->z, B->z, z2z2);
    FN(mul)(P, A->x, z2z2, u1);
    FN(mul)(P, B->x, z1z1, u2);
    FN(mul)(P, B->z, z2z2, t);
    FN(mul)(P, A->y, t, s1);
    FN(mul)(P, A->z, z1z1, t);
    FN(mul)(P, B->y, t, s2);
    if (FN(eq)(u1, u2)) {
        if (FN(eq)(s1, s2)) { FN(dbl)(P, A, R); return; }
        FN(set_id)(P, R);
        return;
    }
    uint64_t h[NL], i[NL], j[NL], rr[NL], v[NL];
    FN(sub)(P, u2, u1, h);
    FN(add)(P, h, h, i);
    FN(mul)(P, i, i, i);
    FN(mul)(P, h, i, j);
    FN(sub)(P, s2, s1, rr);
    FN(add)(P, rr, rr, rr);
    FN(mul)(P, u1, i, v);
    FN(jac) o;
    FN(mul)(P, rr, rr, o.x);
    FN(sub)(P, o.x, j, o.x);
    FN(sub)(P, o.x, v, o.x);
    FN(sub)(P, o.x, v, o.x);
    FN(sub)(P, v, o.x, t);
    FN(mul)(P, rr, t, o.y);
    FN(mul)(P, s1, j, t);
    FN(add)(P, t, t, t);
    FN(sub)(P, o.y, t, o.y);
    FN(add)(P, A->z, B->z, t);
    FN(mul)(P, t, t, t);
    FN(sub)(P, t, z1z1, t);
    FN(sub)(P, t, z2z2, t);
    FN(mul)(P, t, h, o.z);
    *R = o;
}

static void FN(add_aff)(const FN(params) *P, const FN(jac) *A, const FN(aff) *Q, FN(jac) *R) {
    FN(jac) B;
    if (FN(is_zero)(Q->x) && FN(is_zero)(Q->y)) { *R = *A; return; }
    memcpy(B.x, Q->x, NL * 8);
    memcpy(B.y, Q->y, NL * 8);
    memcpy(B.z, P->one, NL * 8);
    FN(addj)(P, A, &B, R);
}

static void FN(to_affine)(const FN(params) *P, const FN(jac) *A, FN(aff) *Q) {
    if (FN(jac_is_id)(A)) { memset(Q, 0, sizeof *Q); return; }
    uint64_t zi[NL], zi2[NL], zi3[NL];
    FN(inv)(P, A->z, zi);
    FN(mul)(P, zi, zi, zi2);
    FN(mul)(P, zi2, zi, zi3);
    FN(mul)(P, A->x, zi2, Q->x);
    FN(mul)(P, A->y, zi3, Q->y);
}

static inline uint32_t FN(window)(const uint32_t *s, int w, int wb) {
    int bit = w * wb, word = bit / 32, sh = bit % 32;
    uint64_t v = s[word];
    if (word + 1 < 8) v |= (uint64_t)s[word + 1] << 32;
    return (uint32_t)((v >> sh) & ((1u << wb) - 1));
}

/* Unsigned-window Pippenger; scalars are 8x u32 integers (any value < 2^256). */
static void FN(pippenger)(const FN(params) *P, const FN(aff) *pts, const uint32_t *sc, long n,
                          FN(jac) *out, int threads) {
    if (n <= 0) { FN(set_id)(P, out); return; }
    int wb = n <= 4 ? 3 : n <= 32 ? 5 : n <= 256 ? 8 : n <= 2048 ? 10 : n <= 8192 ? 11
           : n <= 32768 ? 13 : n <= 131072 ? 14 : n <= 524288 ? 15 : 16;
    int nw = (256 + wb - 1) / wb;
    long nb = (1L << wb) - 1;
    FN(jac) *wres = (FN(jac) *)malloc(sizeof(FN(jac)) * nw);
    #pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (int w = 0; w < nw; w++) {
        FN(jac) *bk = (FN(jac) *)malloc(sizeof(FN(jac)) * (nb + 1));
        for (long b = 0; b <= nb; b++) FN(set_id)(P, &bk[b]);
        for (long i = 0; i < n; i++) {
            uint32_t d = FN(window)(sc + 8 * i, w, wb);
            if (d) FN(add_aff)(P, &bk[d], &pts[i], &bk[d]);
        }
        FN(jac) run, tot;
        FN(set_id)(P, &run);
        FN(set_id)(P, &tot);
        for (long b = nb; b >= 1; b--) {
            FN(addj)(P, &run, &bk[b], &run);
            FN(addj)(P, &tot, &run, &tot);
        }
        wres[w] = tot;
        free(bk);
    }
    FN(jac) acc = wres[nw - 1];
    for (int w = nw - 2; w >= 0; w--) {
        for (int s = 0; s < wb; s++) FN(dbl)(P, &acc, &acc);
        FN(addj)(P, &acc, &wres[w], &acc);
    }
    *out = acc;
    free(wres);
}

/* r = k * G by 4-bit fixed windows (k an integer, 8x u32) */
static void FN(scalar_mul)(const FN(params) *P, const FN(aff) *G, const uint32_t *k, FN(jac) *out) {
    FN(jac) tab[16];
    FN(set_id)(P, &tab[0]);
    for (int i = 1; i < 16; i++) FN(add_aff)(P, &tab[i - 1], G, &tab[i]);
    FN(jac) acc;
    FN(set_id)(P, &acc);
    for (int nib = 63; nib >= 0; nib--) {
        for (int s = 0; s < 4; s++) FN(dbl)(P, &acc, &acc);
        uint32_t d = (k[nib / 8] >> (4 * (nib % 8))) & 15;
        if (d) FN(addj)(P, &acc, &tab[d], &acc);
    }
    *out = acc;
}

/* Jacobian -> affine for m points with one inversion (Montgomery's trick:
 * prefix products of the Z, one Fermat inverse, then back-substitution);
 * identities (Z = 0) become the all-zero affine point.  bn254_msm.c:544-599
 * batch-normalises the same way. */
static void FN(batch_to_affine)(const FN(params) *P, const FN(jac) *in, FN(aff) *out, long m, uint64_t *pre) {
    uint64_t acc[NL];
    memcpy(acc, P->one, sizeof acc);
    for (long i = 0; i < m; i++) {
        memcpy(pre + i * NL, acc, sizeof acc);
        if (!FN(jac_is_id)(&in[i])) FN(mul)(P, acc, in[i].z, acc);
    }
    uint64_t inv[NL];
    FN(inv)(P, acc, inv);
    for (long i = m - 1; i >= 0; i--) {
        if (FN(jac_is_id)(&in[i])) { memset(&out[i], 0, sizeof out[i]); continue; }
        uint64_t zi[NL], zi2[NL], zi3[NL];
        FN(mul)(P, inv, pre + i * NL, zi);     /* 1 / Z_i */
        FN(mul)(P, inv, in[i].z, inv);         /* drop Z_i from the running inverse */
        FN(mul)(P, zi, zi, zi2);
        FN(mul)(P, zi2, zi, zi3);
        FN(mul)(P, in[i].x, zi2, out[i].x);
        FN(mul)(P, in[i].y, zi3, out[i].y);
    }
}

/* Fixed-base comb of 16 rows of 16-bit digits: tab[j * 65536 + d] = d * 2^(16 j) * G
 * (affine, d = 0 is the zero point).  Rows are built in parallel. */
#define FN_COMB_ROWS 16
#define FN_COMB_SPAN 65536L
static FN(aff) *FN(comb_table)(const FN(params) *P, const FN(aff) *G, int threads) {
    FN(aff) *tab = (FN(aff) *)malloc(sizeof(FN(aff)) * FN_COMB_ROWS * FN_COMB_SPAN);
    if (!tab) return NULL;
    #pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (int j = 0; j < FN_COMB_ROWS; j++) {
        FN(jac) b;
        FN(set_id)(P, &b);
        FN(add_aff)(P, &b, G, &b);
        for (int s = 0; s < 16 * j; s++) FN(dbl)(P, &b, &b);
        FN(aff) ba;
        FN(to_affine)(P, &b, &ba);
        FN(jac) *row = (FN(jac) *)malloc(sizeof(FN(jac)) * FN_COMB_SPAN);
        uint64_t *pre = (uint64_t *)malloc(8 * NL * FN_COMB_SPAN);
        FN(set_id)(P, &row[0]);
        for (long d = 1; d < FN_COMB_SPAN; d++) FN(add_aff)(P, &row[d - 1], &ba, &row[d]);
        FN(batch_to_affine)(P, row, tab + j * FN_COMB_SPAN, FN_COMB_SPAN, pre);
        free(pre);
        free(row);
    }
    return tab;
}

/* out[i] = k_i * G (affine) for integer scalars k_i < 2^256 (8x u32): 16 comb
 * additions per point, then one batch inversion per block of points. */
static void FN(comb_mul)(const FN(params) *P, const FN(aff) *tab, const uint32_t *ks, long n, FN(aff) *out,
                         int threads) {
    const long BLK = 1024;
    #pragma omp parallel num_threads(threads)
    {
        FN(jac) *acc = (FN(jac) *)malloc(sizeof(FN(jac)) * BLK);
        uint64_t *pre = (uint64_t *)malloc(8 * NL * BLK);
        #pragma omp for schedule(dynamic, 1)
        for (long b0 = 0; b0 < n; b0 += BLK) {
            long m = n - b0 < BLK ? n - b0 : BLK;
            for (long i = 0; i < m; i++) {
                const uint32_t *k = ks + 8 * (b0 + i);
                FN(set_id)(P, &acc[i]);
                for (int j = 0; j < FN_COMB_ROWS; j++) {
                    uint32_t d = (k[j / 2] >> (16 * (j % 2))) & 0xffffu;
                    if (d) FN(add_aff)(P, &acc[i], &tab[j * FN_COMB_SPAN + d], &acc[i]);
                }
            }
            FN(batch_to_affine)(P, acc, out + b0, m, pre);
        }
        free(pre);
        free(acc);
    }
}
#undef FN_COMB_ROWS
#undef FN_COMB_SPAN
