// Plain data shared by the host engine and the kernels.
#pragma once
#include "curve.cuh"

namespace zkmsm {

template <class Fp_, class Fr_, class Glv_, class Gen_>
struct CurveCfg {
    using Fp = Fp_;
    using Fr = Fr_;
    using Glv = Glv_;
    using Gen = Gen_;
};
using Bn254 = CurveCfg<Bn254Fp, Bn254Fr, Bn254Glv, Bn254Gen>;
using Bls381 = CurveCfg<Bls381Fp, Bls381Fr, Bls381Glv, Bls381Gen>;
using Bls377 = CurveCfg<Bls377Fp, Bls377Fr, Bls377Glv, Bls377Gen>;
// BN254 G2: Fp2 coordinates, the same scalar field; GLV with the
// endomorphism psi (eigenvalue p mod r) instead of phi
using Bn254G2 = CurveCfg<Fp2Of<Bn254Fp>, Bn254Fr, Bn254G2Glv, Bn254G2Gen>;

// One MSM of a batch, as the kernels see it.
struct MsmDesc {
    uint64_t scalar_off;  // index of its first scalar in the scalar array
    uint32_t n;           // number of (base, scalar) pairs
    uint32_t base_off;    // index of its first base in the base table
    uint32_t c;           // window bits
    uint32_t nwin;        // number of windows
    uint32_t glv;         // 1: split scalars with the endomorphism
    uint32_t bucket_off;  // first global bucket id
    uint32_t fmt;         // 0: integer scalars, 1: Montgomery-form Fr
    uint32_t win_off;     // first window-sum slot
    // Shift-table MSMs (bases 2^(c*w)*P_i precomputed for every window w):
    // the base index of window w's digit is base_off + i + w*wstep and all
    // windows share one bucket set (nred = 1 window sum, no doublings in the
    // combine).  wstep = 0: ordinary windows, nred = nwin.
    uint32_t wstep;
    uint32_t nred;        // window sums (bucket sets) of this MSM
    // Window widths: windows [0, nlo) are c bits wide, windows [nlo, nwin)
    // c + 1 bits (the bits + 1 bits a signed recoding covers, split as evenly
    // as the window count allows); nlo = nwin: every window c bits.
    uint32_t nlo;
};

// Most window sums one MSM may have: the window combine holds two per lane
// of one warp.
constexpr uint32_t MAX_WINDOWS = 64;

// Width, first scalar bit and first bucket (relative to bucket_off) of
// window w of an MSM: windows below nlo have 2^(c-1) buckets, the others 2^c.
__host__ __device__ inline uint32_t win_width(const MsmDesc& d, uint32_t w) { return d.c + (w >= d.nlo ? 1u : 0u); }
__host__ __device__ inline uint32_t win_bit(const MsmDesc& d, uint32_t w) {
    return w * d.c + (w > d.nlo ? w - d.nlo : 0u);
}
__host__ __device__ inline uint32_t win_bucket(const MsmDesc& d, uint32_t w) {
    return (w + (w > d.nlo ? w - d.nlo : 0u)) << (d.c - 1);
}

// Sorted-entry value: base index (30 bits) | endo << 30 | negate << 31
constexpr uint32_t VAL_IDX_MASK = 0x3fffffffu;

// Radix sort of the entries (k_radix_digits / k_radix_hist /
// k_radix_scatter): digit-extraction block size and its shared buffer of
// entries, entries per sort tile and threads per sort block, and the widest
// digit (2^8 bins; one bin per sort thread).
constexpr uint32_t SORT_DTHREADS = 256;
constexpr uint32_t SORT_DBUF = 4096;
constexpr uint32_t SORT_ETILE = 4096;
constexpr uint32_t SORT_ETHREADS = 256;
constexpr uint32_t SORT_MAX_BINS = 256;

// MSD radix sort of large entry sets (k_msd_count / k_msd_scatter): entries
// per tile (staged whole in shared memory), threads per tile block, widest
// digit per pass (2^12 bins), and the smallest entry bound sorted this way
// (smaller batches take the LSD sort above, whose 4096-entry tiles keep more
// blocks busy).
constexpr uint32_t MSD_TILE = 24576;
constexpr uint32_t MSD_THREADS = 1024;
constexpr uint32_t MSD_MAX_BITS = 12;
constexpr uint64_t MSD_MIN_ENTRIES = 1ull << 21;
// Tiles per scatter group: pass 1 splits its tiles over one group per SM,
// each counted in MSD_COUNT_PARTS parts (two count blocks fit an SM); pass 2
// cuts each segment into chunks of at most MSD_CHUNK_TILES tiles.
constexpr uint32_t MSD_COUNT_PARTS = 2;
constexpr uint32_t MSD_CHUNK_TILES = 8;

// Scalar profile for the window-layout choice (k_scalar_profile): bins of
// the bit length (0..288) of a prepared scalar half, and sampled scalars.
constexpr uint32_t PROFILE_BINS = 320;
constexpr uint32_t PROFILE_SAMPLES = 4096;

// Bucket-reduction levels with at most this many output nodes run the
// inline-product kernel (few threads: latency-bound).
constexpr uint32_t RED_INLINE_MAX_NODES = 32768;

struct RedTask {
    uint32_t in_off;   // first child node
    uint32_t n_in;     // children
    uint32_t out_off;  // first parent node (prefix sum of parents per task)
    uint32_t n_out;
};

}  // namespace zkmsm
