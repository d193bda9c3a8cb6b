// BN254 G1 MSM entry point that allocates no device memory.
//
// Who needs it: callers that may not call cudaMalloc on their hot path.
// Typical cases are a host framework that has already reserved nearly all of
// HBM for its own pool (so a library cudaMalloc fails or fragments it), a
// latency-critical prover loop that forbids allocation after start-up
// because cudaMalloc/cudaFree can synchronise the whole device, and code that
// enqueues work from inside a stream it does not want stalled by an
// allocation.  They pass device inputs and a device output and get the MSM
// without any allocation by this library.
//
// How: all scratch (bucket counts, sorted entries, buckets, partial sums,
// reduction nodes, the endomorphism image of the bases, the launch tables)
// lives in one file-scope __device__ array g_scratch of SCRATCH_BYTES
// (7,572,224 bytes),
// which every GPU that loads the library holds until the process exits.
// Host code cannot use the array's name as a device address, so the first
// call on each device (with that device current) looks its address up with
// cudaGetSymbolAddress and caches it; make that first call before any stream
// capture.  The cached address belongs to the device's context: after a
// cudaDeviceReset of that device in the same process it is stale, so do not
// call this entry point again after such a reset.  The call's own launch
// tables (MSM descriptor, reduction tasks) are written into the array by a
// one-thread kernel from by-value arguments, so the call reads no host memory
// after it returns.  Limits: n <= N_MAX (8192), fixed window width 10 with
// GLV.  Every call shares the one array and it keeps the last call's
// contents: the parts that must start at zero are cleared on each call, and
// two calls whose GPU work overlaps (different streams, or different host
// threads) race on it -- serialise them.  Calls queued one after another on
// one stream are ordered by the stream and need nothing more.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/zkmsm.h"
#include "msm_kernels.cuh"

namespace zkmsm {
void set_error(const std::string& s);  // per-thread error text (capi.cu)

namespace noalloc {

using C = Bn254;
using P = Bn254Fp;

constexpr uint32_t N_MAX = 8192;
constexpr uint32_t CB = 10;                                            // window bits
constexpr uint32_t NWIN = (Bn254Glv::HALF_BITS + 1 + CB - 1) / CB;     // 13 signed windows
constexpr uint32_t BPW = 1u << (CB - 1);                               // buckets per window
constexpr uint32_t NB = NWIN * BPW;                                    // 6656 buckets
constexpr uint64_t E_MAX = 2ull * N_MAX * NWIN;                        // sorted entries
constexpr uint32_t K1 = 16, KJ = 16;                                   // chunk lengths
constexpr uint32_t T1_MAX = (uint32_t)((E_MAX + K1 - 1) / K1);
constexpr uint32_t M2_MAX = 2 * T1_MAX;                                // level-1 partials
constexpr uint32_t M3_MAX = 2 * ((M2_MAX + KJ - 1) / KJ);              // level-2 partials
constexpr uint32_t RED_L = 8, RED_LOG2L = 3;
constexpr uint32_t RED_NODES0 = NWIN * (BPW / RED_L);                  // 832
constexpr int RED_LEVELS = 3;                                          // 512 -> 64 -> 8 -> 1
constexpr int MAX_ACC_LEVELS = 16;
constexpr size_t XS = sizeof(Xyzz<P>);

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// byte offsets inside the scratch array
constexpr size_t OFF_COUNTS = 0;
constexpr size_t OFF_CURSOR = align256(OFF_COUNTS + (NB + 1) * 4);
constexpr size_t OFF_ENTS = align256(OFF_CURSOR + (NB + 1) * 4);
constexpr size_t OFF_BUCKETS = align256(OFF_ENTS + E_MAX * 8);
constexpr size_t OFF_CNT = align256(OFF_BUCKETS + NB * XS);
constexpr size_t OFF_TILES = align256(OFF_CNT + T1_MAX * 4);
constexpr size_t OFF_TOTALS = align256(OFF_TILES + 4096);
constexpr size_t OFF_PK0 = align256(OFF_TOTALS + 64 * 4);
constexpr size_t OFF_PV0 = align256(OFF_PK0 + M2_MAX * 4);
constexpr size_t OFF_PK1 = align256(OFF_PV0 + M2_MAX * XS);
constexpr size_t OFF_PV1 = align256(OFF_PK1 + M3_MAX * 4);
constexpr size_t OFF_RS0 = align256(OFF_PV1 + M3_MAX * XS);
constexpr size_t OFF_RW0 = align256(OFF_RS0 + RED_NODES0 * XS);
constexpr size_t OFF_RS1 = align256(OFF_RW0 + RED_NODES0 * XS);
constexpr size_t OFF_RW1 = align256(OFF_RS1 + RED_NODES0 * XS);
constexpr size_t OFF_PHI = align256(OFF_RW1 + RED_NODES0 * XS);
constexpr size_t OFF_DESC = align256(OFF_PHI + (size_t)N_MAX * 2 * P::N * 4);
constexpr size_t OFF_TASKS = align256(OFF_DESC + sizeof(MsmDesc));
constexpr size_t SCRATCH_BYTES = align256(OFF_TASKS + RED_LEVELS * NWIN * sizeof(RedTask));
static_assert(SCRATCH_BYTES < (16u << 20), "scratch must stay modest");
static_assert((T1_MAX + 2047) / 2048 * 4 <= 4096, "scan tile sums fit their slot");

static __device__ __align__(256) unsigned char g_scratch[SCRATCH_BYTES];

static std::mutex g_mu;
static unsigned char* g_addr[64];

// The launch tables of one call, built on the device from by-value
// arguments: the MSM descriptor (one MSM, window width CB, GLV) and the
// reduction tasks (RED_LEVELS levels of NWIN windows, L = RED_L).
static __global__ void k_noalloc_tables(MsmDesc* __restrict__ desc, RedTask* __restrict__ tasks, uint32_t n,
                                        uint32_t fmt) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    MsmDesc d{};
    d.scalar_off = 0;
    d.n = n;
    d.base_off = 0;
    d.c = CB;
    d.nwin = NWIN;
    d.glv = 1;
    d.bucket_off = 0;
    d.fmt = fmt;
    d.win_off = 0;
    d.wstep = 0;
    d.nred = NWIN;
    d.nlo = NWIN;
    *desc = d;
    uint32_t nin = BPW;
    for (int l = 0; l < RED_LEVELS; l++) {
        const uint32_t nout = (nin + RED_L - 1) / RED_L;
        for (uint32_t w = 0; w < NWIN; w++) {
            RedTask t;
            t.in_off = l == 0 ? w * BPW : w * nin;
            t.n_in = nin;
            t.out_off = w * nout;
            t.n_out = nout;
            tasks[l * NWIN + w] = t;
        }
        nin = nout;
    }
}

static void scan(unsigned char* base, uint32_t* d, uint32_t n, uint32_t* d_total, uint32_t* copy, cudaStream_t s) {
    uint32_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (tiles == 0) tiles = 1;
    uint32_t* ts = reinterpret_cast<uint32_t*>(base + OFF_TILES);
    k_scan_tiles<<<tiles, SCAN_THREADS, 0, s>>>(d, n, d, ts);
    k_scan_sums<<<1, SCAN_THREADS, 0, s>>>(ts, tiles, d_total);
    k_scan_add<<<tiles, SCAN_THREADS, 0, s>>>(d, n, ts, copy);
}

}  // namespace noalloc
}  // namespace zkmsm

using namespace zkmsm;
using namespace zkmsm::noalloc;

extern "C" ZkMetalStatus zkmsm_bn254_msm_noalloc(const void* d_points, const void* d_scalars, int fmt,
                                                 uint32_t n_points, void* d_result, void* stream) {
    if (!d_points || !d_scalars || !d_result) {
        set_error("zkmsm_bn254_msm_noalloc: null device pointer");
        return ZKMETAL_ERR_INVALID_INPUT;
    }
    if (n_points == 0) {
        set_error("zkmsm_bn254_msm_noalloc: n_points is 0");
        return ZKMETAL_ERR_INVALID_INPUT;
    }
    if (fmt != ZKMSM_SCALAR_INT && fmt != ZKMSM_SCALAR_MONT) {
        set_error("zkmsm_bn254_msm_noalloc: scalar_fmt must be 0 (integer) or 1 (Montgomery)");
        return ZKMETAL_ERR_INVALID_INPUT;
    }
    if (n_points > N_MAX) {
        set_error("zkmsm_bn254_msm_noalloc: n_points exceeds the allocation-free limit of 8192");
        return ZKMETAL_ERR_INVALID_INPUT;
    }
    // a launch error left pending by the caller's own work would otherwise be
    // reported below as this call's: refuse, and leave it pending for them
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
        set_error(std::string("zkmsm_bn254_msm_noalloc: a CUDA error was pending before the call: ") +
                  cudaGetErrorString(pending));
        return ZKMETAL_ERR_GPU_ERROR;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0;
    cudaError_t de = cudaGetDevice(&dev);
    if (de != cudaSuccess || dev < 0 || dev >= 64) {
        if (de != cudaSuccess) cudaGetLastError();
        set_error(std::string("zkmsm_bn254_msm_noalloc: no usable current device: ") +
                  (de != cudaSuccess ? cudaGetErrorString(de) : "device index out of range"));
        return ZKMETAL_ERR_NO_GPU;
    }
    unsigned char* base;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_addr[dev]) {
            void* ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
            if (e != cudaSuccess || !ptr) {
                cudaGetLastError();
                set_error(std::string("zkmsm_bn254_msm_noalloc: cudaGetSymbolAddress failed: ") +
                          cudaGetErrorString(e));
                return ZKMETAL_ERR_GPU_ERROR;
            }
            g_addr[dev] = static_cast<unsigned char*>(ptr);
        }
        base = g_addr[dev];
    }
    const uint32_t n = n_points;
    uint32_t accK[MAX_ACC_LEVELS], accT[MAX_ACC_LEVELS];
    int nacc = 0;
    uint64_t M = 2ull * n * NWIN;
    uint32_t K = K1;
    while (nacc < MAX_ACC_LEVELS) {
        uint64_t T = (M + K - 1) / K;
        if (T == 0) T = 1;
        accK[nacc] = K;
        accT[nacc] = (uint32_t)T;
        nacc++;
        if (T <= 1) break;
        M = 2 * T;
        K = KJ;
    }
    k_noalloc_tables<<<1, 32, 0, s>>>(reinterpret_cast<MsmDesc*>(base + OFF_DESC),
                                      reinterpret_cast<RedTask*>(base + OFF_TASKS), n, (uint32_t)fmt);
    cudaError_t me = cudaMemsetAsync(base + OFF_COUNTS, 0, (NB + 1) * 4, s);
    if (me == cudaSuccess) me = cudaMemsetAsync(base + OFF_BUCKETS, 0, NB * XS, s);
    if (me != cudaSuccess) {
        cudaGetLastError();
        set_error(std::string("zkmsm_bn254_msm_noalloc: clearing the scratch failed: ") + cudaGetErrorString(me));
        return ZKMETAL_ERR_GPU_ERROR;
    }

    const uint32_t* pts = static_cast<const uint32_t*>(d_points);
    const uint32_t* sc = static_cast<const uint32_t*>(d_scalars);
    uint32_t* phi = reinterpret_cast<uint32_t*>(base + OFF_PHI);
    uint32_t* counts = reinterpret_cast<uint32_t*>(base + OFF_COUNTS);
    uint32_t* cursor = reinterpret_cast<uint32_t*>(base + OFF_CURSOR);
    uint2* ents = reinterpret_cast<uint2*>(base + OFF_ENTS);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(base + OFF_CNT);
    uint32_t* tot = reinterpret_cast<uint32_t*>(base + OFF_TOTALS);
    Xyzz<P>* buckets = reinterpret_cast<Xyzz<P>*>(base + OFF_BUCKETS);
    uint32_t* pk[2] = {reinterpret_cast<uint32_t*>(base + OFF_PK0), reinterpret_cast<uint32_t*>(base + OFF_PK1)};
    Xyzz<P>* pv[2] = {reinterpret_cast<Xyzz<P>*>(base + OFF_PV0), reinterpret_cast<Xyzz<P>*>(base + OFF_PV1)};
    Xyzz<P>* rS[2] = {reinterpret_cast<Xyzz<P>*>(base + OFF_RS0), reinterpret_cast<Xyzz<P>*>(base + OFF_RS1)};
    Xyzz<P>* rW[2] = {reinterpret_cast<Xyzz<P>*>(base + OFF_RW0), reinterpret_cast<Xyzz<P>*>(base + OFF_RW1)};
    const MsmDesc* dd = reinterpret_cast<const MsmDesc*>(base + OFF_DESC);
    const RedTask* dt = reinterpret_cast<const RedTask*>(base + OFF_TASKS);

    k_endo<C><<<(n + 255) / 256, 256, 0, s>>>(pts, n, phi);
    k_digit_hist<C><<<(n + 255) / 256, 256, 0, s>>>(sc, dd, 1, n, counts);
    scan(base, counts, NB, tot + 0, cursor, s);
    k_digit_scatter<C><<<(n + 255) / 256, 256, 0, s>>>(sc, dd, 1, n, cursor, ents);
    const uint32_t* lk = reinterpret_cast<const uint32_t*>(ents);
    uint32_t ks = 2;
    int cur = 0;
    for (int l = 0; l < nacc; l++) {
        uint32_t Kl = accK[l], Tl = accT[l];
        k_chunk_count<<<(Tl + 255) / 256, 256, 0, s>>>(lk, ks, tot + l, Kl, Tl, cnt);
        scan(base, cnt, Tl, tot + l + 1, nullptr, s);
        if (l == 0)
            k_acc_l1<C><<<(Tl + AccLaunch<C>::THREADS - 1) / AccLaunch<C>::THREADS, AccLaunch<C>::THREADS, 0, s>>>(ents, tot + l, Kl, pts, phi, cnt, buckets, pk[cur],
                                                          pv[cur]);
        else
            k_acc_lj<C, false><<<(Tl + 255) / 256, 256, 0, s>>>(lk, pv[cur ^ 1], tot + l, Kl, cnt, buckets, pk[cur],
                                                               pv[cur]);
        lk = pk[cur];
        ks = 1;
        cur ^= 1;
    }
    const Xyzz<P>* inS = buckets;
    const Xyzz<P>* inW = nullptr;
    uint32_t nodes = BPW;
    for (int l = 0; l < RED_LEVELS; l++) {
        nodes = (nodes + RED_L - 1) / RED_L;
        uint32_t nout = nodes * NWIN;
        k_reduce_level<C, false><<<(nout + 127) / 128, 128, 0, s>>>(inS, inW, dt + l * NWIN, NWIN, nout, RED_L,
                                                             (uint32_t)l * RED_LOG2L, rS[l & 1], rW[l & 1]);
        inS = rS[l & 1];
        inW = rW[l & 1];
    }
    k_combine<C><<<1, 32 * COMBINE_WARPS, 0, s>>>(inS, inW, dd, 1, static_cast<uint32_t*>(d_result));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("zkmsm_bn254_msm_noalloc: launch failed: ") + cudaGetErrorString(e));
        return ZKMETAL_ERR_GPU_ERROR;
    }
    return ZKMETAL_SUCCESS;
}
