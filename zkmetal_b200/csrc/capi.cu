// C ABI (include/zkmsm.h): the zkMetal-ffi compatible MSM entry points and
// the new device-resident / batched entry points.  Argument checks, status
// codes and the count == 0 convention follow the reference FFI
// (Sources/zkMetal-ffi/zkMetal_ffi.swift:302-379, 1048-1300).
#include <cuda_runtime.h>

#include <cstdio>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <type_traits>

#include "../../include/zkmsm.h"
#include "engine.cuh"

namespace zkmsm {

static thread_local std::string g_last_error;
void set_error(const std::string& s) { g_last_error = s; }

// bytes of one coordinate (a BN254 G2 coordinate is an Fp2 element: 64 B)
static int fp_bytes(int curve) { return curve == ZKMSM_BN254 ? 32 : curve == ZKMSM_BN254_G2 ? 64 : 48; }

static bool curve_ok(int curve) {
    return curve == ZKMSM_BN254 || curve == ZKMSM_BLS12_381 || curve == ZKMSM_BLS12_377 || curve == ZKMSM_BN254_G2;
}

// Calls f(C{}) with the curve configuration of a curve id (checked by
// curve_ok before).
template <class F>
static void with_curve(int curve, F&& f) {
    switch (curve) {
        case ZKMSM_BN254: f(Bn254{}); break;
        case ZKMSM_BLS12_381: f(Bls381{}); break;
        case ZKMSM_BLS12_377: f(Bls377{}); break;
        case ZKMSM_BN254_G2: f(Bn254G2{}); break;
        default: throw std::invalid_argument("unknown curve id");
    }
}

// A window setting: 0 (automatic), a width 2..24, or a two-width layout
// c | nlo << 16 (nlo >= 1 windows of c = 2..22 bits, then c + 1-bit windows).
static bool window_setting_ok(int w) {
    if (w < 0) return false;
    if (w < 65536) return w != 1 && w <= 24;
    const int c = w & 0xffff, nlo = w >> 16;
    return c >= 2 && c <= 22 && nlo >= 1 && nlo <= 256;
}

// Map exceptions to reference status codes.
template <class F>
static ZkMetalStatus guarded(F&& f) {
    try {
        g_last_error.clear();
        return f();
    } catch (const CudaError& e) {
        set_error(std::string(e.where) + ": " + cudaGetErrorString(e.code));
        cudaGetLastError();  // clear a sticky non-fatal error state where possible
        if (e.code == cudaErrorMemoryAllocation) return ZKMETAL_ERR_ALLOC_FAILED;
        if (e.code == cudaErrorNoDevice || e.code == cudaErrorInsufficientDriver) return ZKMETAL_ERR_NO_GPU;
        return ZKMETAL_ERR_GPU_ERROR;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return ZKMETAL_ERR_ALLOC_FAILED;
    } catch (const std::exception& e) {
        set_error(e.what());
        return ZKMETAL_ERR_GPU_ERROR;
    }
}

static bool have_gpu() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return false;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, 0) != cudaSuccess) return false;
    return prop.major == 10;
}

// Copy host data to a device buffer of the engine's workspace.
static void h2d(Engine& e, DevBuf& buf, const void* src, size_t bytes) {
    buf.ensure(bytes + 16);
    if (bytes) ZK_CUDA(cudaMemcpyAsync(buf.p, src, bytes, cudaMemcpyHostToDevice, e.stream));
}

// Host-buffer MSMs of at least two stripes of f points (engine setting
// zkmsm_engine_set_stripe: f = 2^stripe_log2; by default half of n's next
// power of two from 2^22 points, and 2^20 for BN254 G1 from 2^21) are
// streamed: the
// point range is cut into stripes that start at f/4 points and grow by 1.6x
// up to f (a short first stripe exposes little of the copy before work
// starts; a stripe's compute, ~3 ns per BN254 point, covers the copy of the
// next, 1.6x longer one at ~1.8 ns per point); stripe s is copied on the
// engine's copy stream while stripe s-1 is
// sorted and accumulated on the compute stream.  Every stripe uses one
// window layout and fills its own bucket array; the arrays are then added
// bucket by bucket and reduced once, so the result is the same point as the
// unstriped MSM.
template <class C>
static std::vector<std::pair<uint32_t, uint32_t>> stripe_ranges(const Engine& e, uint32_t n) {
    std::vector<std::pair<uint32_t, uint32_t>> r;
    int lg = e.stripe_log2;
    if (lg < 0) {  // automatic
        // below the threshold the exposed copy is shorter than what striping
        // adds (a smaller stripe's extra windows, the fold).  BN254 G1 drop-in
        // calls: 2^19 points 4.6 ms unstriped, 5.6 ms striped; 2^21 12.2 vs
        // 11.8 ms.  BLS12-381 2^21: 21.9 unstriped, 24.8 ms striped.
        const uint32_t min_n = std::is_same<C, Bn254>::value ? (1u << 21) : (1u << 22);
        if (n < min_n) return r;
        if (n < (1u << 22)) {
            lg = 20;
        } else {
            lg = 0;
            while ((1ull << lg) < n) lg++;
            lg -= 1;
        }
    }
    if (lg < 2 || lg > 30 || (n >> lg) < 1) return r;
    const uint32_t f = 1u << lg;
    uint32_t off = 0, len = std::max(f / 4, 1u);
    while (off < n) {
        uint32_t cnt = std::min(len, n - off);
        if (r.size() == 15) cnt = n - off;  // at most 16 stripes
        r.push_back({off, cnt});
        off += cnt;
        len = (uint32_t)std::min<uint64_t>(f, (uint64_t)len * 8 / 5 + 1);
    }
    return r;
}

template <class C>
static void msm_host_striped(Engine& e, const uint8_t* points, const uint8_t* scalars, uint32_t n, int fmt,
                             uint32_t scalar_bits, const std::vector<std::pair<uint32_t, uint32_t>>& rg,
                             uint8_t* out) {
    using P = typename C::Fp;
    const size_t pb = (size_t)2 * P::N * 4, xs = (size_t)4 * P::N * 4;  // bytes per point, per XYZZ bucket
    const uint32_t S = (uint32_t)rg.size();
    // every stripe takes the window layout (width c, and nlo windows of c
    // bits before the c + 1-bit ones when the widths differ) of the largest
    // stripe: each stripe fills its own bucket array, so the layout of the
    // whole n (2^24: 8.4M buckets) would cost a gigabyte per stripe to fill
    // and fold (BN254 2^24 from host buffers: 59.2 ms, against 57.0 ms with
    // the 2^23 layout of 1.2M buckets)
    uint32_t fmax = 0;
    for (auto& q : rg) fmax = std::max(fmax, q.second);
    const MsmDesc d0 = e.get_plan<C>({fmax}, {0}, fmt, scalar_bits).descs[0];
    const uint32_t layout = d0.c | (d0.nlo < d0.nwin ? d0.nlo << 16 : 0u);
    // one plan per distinct stripe length; a lookup may evict the cache, so
    // all are fetched a second time before any is used
    std::map<uint32_t, Plan*> plans;
    for (int pass = 0; pass < 2; pass++)
        for (auto& q : rg) plans[q.second] = &e.get_plan<C>({q.second}, {0}, fmt, scalar_bits, layout);
    const Plan& p0 = *plans[rg[0].second];
    const bool glv = p0.descs[0].glv;
    const size_t nb = p0.nbuckets;
    for (auto& kv : plans)
        if (kv.second->nbuckets != nb) throw std::runtime_error("stripe bucket layouts differ");
    bool grew = e.w_points.ensure((size_t)n * pb + 16);
    grew |= e.w_scalars.ensure((size_t)n * 32 + 16);
    if (glv) grew |= e.w_phi.ensure((size_t)n * pb + 16);
    if (grew) e.drop_graphs();
    for (auto& kv : plans) e.ensure_workspace<C>(*kv.second);
    e.w_stripe_buckets.ensure(S * nb * xs + 16);
    // events: [s] stripe s's scalars copied, [S] buffers allocated,
    // [S + 1 + s] stripe s's bases copied
    e.ensure_copy_resources(2 * S + 1);
    // buffers (re)allocated in the compute stream's order: the copies wait for that
    ZK_CUDA(cudaEventRecord(e.copy_events[S], e.stream));
    ZK_CUDA(cudaStreamWaitEvent(e.copy_stream, e.copy_events[S], 0));
    uint8_t* dp = static_cast<uint8_t*>(e.w_points.p);
    uint8_t* ds = static_cast<uint8_t*>(e.w_scalars.p);
    uint8_t* dphi = glv ? static_cast<uint8_t*>(e.w_phi.p) : dp;
    uint8_t* bk = static_cast<uint8_t*>(e.w_stripe_buckets.p);
    for (uint32_t s = 0; s < S; s++) {
        const size_t off = rg[s].first;
        const uint32_t cnt = rg[s].second;
        e.copy_h2d(ds + off * 32, scalars + off * 32, (size_t)cnt * 32, e.copy_stream);
        ZK_CUDA(cudaEventRecord(e.copy_events[s], e.copy_stream));
        e.copy_h2d(dp + off * pb, points + off * pb, (size_t)cnt * pb, e.copy_stream);
        ZK_CUDA(cudaEventRecord(e.copy_events[S + 1 + s], e.copy_stream));
        // the stripe's sort needs only its scalars; its bases are waited
        // for after the sort, before the endomorphism and the accumulation
        ZK_CUDA(cudaStreamWaitEvent(e.stream, e.copy_events[s], 0));
        const uint32_t* sp = reinterpret_cast<const uint32_t*>(dp + off * pb);
        uint32_t* sphi = reinterpret_cast<uint32_t*>(dphi + off * pb);
        Engine::BasesWait bw;
        bw.ready = e.copy_events[S + 1 + s];
        bw.phi_n = glv ? cnt : 0;
        bw.phi_out = glv ? sphi : nullptr;
        e.enqueue<C>(*plans[cnt], sp, sphi, reinterpret_cast<const uint32_t*>(ds + off * 32), nullptr,
                     Engine::ENQ_ACC_ONLY, bk + s * nb * xs, &bw);
    }
    e.fold_buckets<C>(bk, (uint32_t)nb, S);
    e.enqueue_reduce<C>(p0, bk, e.w_results.as<uint32_t>());
    ZK_CUDA(cudaMemcpyAsync(out, e.w_results.p, 3 * P::N * 4, cudaMemcpyDeviceToHost, e.stream));
    ZK_CUDA(cudaStreamSynchronize(e.stream));
}

// host-buffer MSMs up to this many points run as a replayed CUDA graph
constexpr uint32_t SMALL_GRAPH_POINTS = 1u << 16;

template <class C>
static ZkMetalStatus msm_host(Engine& e, const uint8_t* points, const uint8_t* scalars, uint32_t n, int fmt,
                              uint32_t scalar_bits, uint8_t* rx, uint8_t* ry, uint8_t* rz) {
    using P = typename C::Fp;
    const int fb = P::N * 4;
    if (n == 0 || !points || !scalars || !rx || !ry || !rz) return ZKMETAL_ERR_INVALID_INPUT;
    const auto rg = stripe_ranges<C>(e, n);
    if (rg.size() > 1) {
        uint8_t out[3 * 4 * MAX_COORD_WORDS];
        msm_host_striped<C>(e, points, scalars, n, fmt, scalar_bits, rg, out);
        memcpy(rx, out, fb);
        memcpy(ry, out + fb, fb);
        memcpy(rz, out + 2 * fb, fb);
        return ZKMETAL_SUCCESS;
    }
    uint8_t out[3 * 4 * MAX_COORD_WORDS];
    if (n <= SMALL_GRAPH_POINTS) {
        // small MSMs are a chain of ~30 short launches: replay them as one
        // CUDA graph (captured on the second call of a shape; the buffers
        // are the engine's own, so later calls of the same size replay it)
        h2d(e, e.w_points, points, (size_t)n * 2 * fb);
        h2d(e, e.w_scalars, scalars, (size_t)n * 32);
        Plan& pl = e.get_plan<C>({n}, {0}, fmt, scalar_bits);
        const bool glv = pl.descs[0].glv;
        if (glv) {
            e.w_phi.ensure((size_t)n * 2 * fb + 16);
            e.make_phi<C>(e.w_points.as<uint32_t>(), n, e.w_phi.as<uint32_t>());
        }
        const uint32_t* phi = glv ? e.w_phi.as<uint32_t>() : e.w_points.as<uint32_t>();
        e.run_device_graph<C>(pl, e.w_points.as<uint32_t>(), phi, e.w_scalars.as<uint32_t>(), out);
    } else {
        // the scalars go first on the engine stream and the bases on the
        // copy stream: the scalar preparation and sort, which read only the
        // scalars, run while the bases arrive
        Plan* pl = &e.get_plan<C>({n}, {0}, fmt, scalar_bits);
        const bool glv = pl->descs[0].glv;
        bool grew = e.w_points.ensure((size_t)n * 2 * fb + 16);
        grew |= e.w_scalars.ensure((size_t)n * 32 + 16);
        if (glv) grew |= e.w_phi.ensure((size_t)n * 2 * fb + 16);
        if (grew) e.drop_graphs();
        e.ensure_copy_resources(2);
        // buffers (re)allocated in the engine stream's order: the copy waits for that
        ZK_CUDA(cudaEventRecord(e.copy_events[0], e.stream));
        ZK_CUDA(cudaStreamWaitEvent(e.copy_stream, e.copy_events[0], 0));
        e.copy_h2d(e.w_scalars.p, scalars, (size_t)n * 32, e.stream);
        e.copy_h2d(e.w_points.p, points, (size_t)n * 2 * fb, e.copy_stream);
        ZK_CUDA(cudaEventRecord(e.copy_events[1], e.copy_stream));
        // window layout from a sample of the scalars (the bases keep arriving)
        if (!scalar_bits && glv) {
            const auto sl = e.sampled_layout<C>(e.w_scalars.as<uint32_t>(), n, fmt);
            if (sl.window) pl = &e.get_plan<C>({n}, {0}, fmt, 0, sl.window, {}, sl.entries);
        }
        e.ensure_workspace<C>(*pl);
        Engine::BasesWait bw;
        bw.ready = e.copy_events[1];
        bw.phi_n = glv ? n : 0;
        bw.phi_out = glv ? e.w_phi.as<uint32_t>() : nullptr;
        const uint32_t* phi = glv ? e.w_phi.as<uint32_t>() : e.w_points.as<uint32_t>();
        e.enqueue<C>(*pl, e.w_points.as<uint32_t>(), phi, e.w_scalars.as<uint32_t>(), e.w_results.as<uint32_t>(), 0,
                     nullptr, &bw);
        ZK_CUDA(cudaMemcpyAsync(out, e.w_results.p, 3 * P::N * 4, cudaMemcpyDeviceToHost, e.stream));
        ZK_CUDA(cudaStreamSynchronize(e.stream));
    }
    memcpy(rx, out, fb);
    memcpy(ry, out + fb, fb);
    memcpy(rz, out + 2 * fb, fb);
    return ZKMETAL_SUCCESS;
}

// small-scalar variants: zero-extend to 32 B (zkMetal_ffi.swift:1150-1190)
static ZkMetalStatus msm_small(Engine& e, const uint8_t* points, const uint8_t* scalars, uint32_t n, int width,
                               uint8_t* rx, uint8_t* ry, uint8_t* rz) {
    if (n == 0 || !points || !scalars) return ZKMETAL_ERR_INVALID_INPUT;
    std::vector<uint32_t> wide((size_t)n * 8, 0);
    for (uint32_t i = 0; i < n; i++) {
        uint32_t v = 0;
        for (int b = 0; b < width; b++) v |= (uint32_t)scalars[(size_t)i * width + b] << (8 * b);
        wide[(size_t)i * 8] = v;
    }
    return msm_host<Bn254>(e, points, reinterpret_cast<const uint8_t*>(wide.data()), n, ZKMSM_SCALAR_INT,
                           8 * width, rx, ry, rz);
}

template <class C>
static ZkMetalStatus msm_batch_host(Engine& e, const uint8_t* all_points, const uint8_t* all_scalars,
                                    const uint32_t* counts, uint32_t n_msms, int fmt, uint8_t* results) {
    using P = typename C::Fp;
    const int fb = P::N * 4;
    if (n_msms == 0 || !counts || !results) return ZKMETAL_ERR_INVALID_INPUT;
    std::vector<uint32_t> cnt(counts, counts + n_msms), boff(n_msms);
    uint64_t total = 0;
    for (uint32_t m = 0; m < n_msms; m++) {
        boff[m] = (uint32_t)total;
        total += cnt[m];
    }
    if (total >= (1ull << 30)) return ZKMETAL_ERR_INVALID_INPUT;
    if (total && (!all_points || !all_scalars)) return ZKMETAL_ERR_INVALID_INPUT;
    h2d(e, e.w_points, all_points, (size_t)total * 2 * fb);
    h2d(e, e.w_scalars, all_scalars, (size_t)total * 32);
    Plan& pl = e.get_plan<C>(cnt, boff, fmt);
    e.w_phi.ensure((size_t)total * 2 * fb + 16);
    e.make_phi<C>(e.w_points.as<uint32_t>(), total, e.w_phi.as<uint32_t>());
    std::vector<uint8_t> out((size_t)n_msms * 3 * fb);
    e.run_device<C>(pl, e.w_points.as<uint32_t>(), e.w_phi.as<uint32_t>(), e.w_scalars.as<uint32_t>(), out.data());
    for (uint32_t m = 0; m < n_msms; m++) {
        uint8_t* dst = results + (size_t)m * 3 * fb;
        if (cnt[m] == 0) memset(dst, 0, 3 * fb);
        else memcpy(dst, out.data() + (size_t)m * 3 * fb, 3 * fb);
    }
    return ZKMETAL_SUCCESS;
}

// Resident base table (commitment key).
struct Table {
    Engine* engine;
    int curve;
    uint64_t n;
    DevBuf points, phi;
    // window shifts (zkmsm_table_precompute): `points` then holds `copies`
    // copies of the n points, copy k = 2^(shift_bits*k) * P_i
    uint32_t shift_bits = 0, copies = 1;
    ShiftSpec shifts() const { return ShiftSpec{shift_bits, shift_bits ? (uint32_t)n : 0u}; }
};

bool table_view(ZkMsmTable t, TableView* out) {
    if (!t || !out) return false;
    Table* tb = static_cast<Table*>(t);
    out->curve = tb->curve;
    out->n = tb->n;
    out->points = tb->points.as<uint32_t>();
    out->phi = tb->phi.as<uint32_t>();
    out->shifts = tb->shifts();
    return true;
}

// Batches of host scalars from this many points on are run as two groups of
// consecutive MSMs with about the same number of points each: the second
// group's scalars are copied on the copy stream while the first group runs
// (the copy of a 24-MSM, 1.2e7-point batch is 7 ms at 55 GB/s).  Each group
// is its own batch plan over the same table, so the results are unchanged.
// Every group pays its own sort, reduction tail and combine: measured on
// that batch, two groups 45.2 ms against 46.2 ms for one, three groups no
// gain; a 2.4e6-point BLS12-381 batch in two groups lost 3 ms.
constexpr uint64_t BATCH_GROUP_MIN_POINTS = 1ull << 23;

template <class C>
static void batch_commit_grouped(Engine& e, const Table& t, const uint8_t* scalars, int fmt,
                                 const std::vector<uint32_t>& cnt, uint8_t* out) {
    using P = typename C::Fp;
    const uint32_t n_msms = (uint32_t)cnt.size();
    uint64_t total = 0;
    for (auto c : cnt) total += c;
    const uint32_t G = 2;
    // group g = MSMs [first[g], first[g + 1]), cut where the running count
    // passes g * total / G
    std::vector<uint32_t> first{0};
    uint64_t run = 0;
    for (uint32_t m = 0; m < n_msms && first.size() < G; m++) {
        run += cnt[m];
        if (run * G >= (uint64_t)first.size() * total && m + 1 < n_msms) first.push_back(m + 1);
    }
    first.push_back(n_msms);
    const uint32_t ng = (uint32_t)first.size() - 1;
    std::vector<uint64_t> soff(ng + 1, 0);
    for (uint32_t g = 0; g < ng; g++) {
        soff[g + 1] = soff[g];
        for (uint32_t m = first[g]; m < first[g + 1]; m++) soff[g + 1] += cnt[m];
    }
    if (e.w_scalars.ensure((size_t)total * 32 + 16)) e.drop_graphs();
    // plans; a lookup may evict the cache, so all are fetched twice
    std::vector<Plan*> plans(ng);
    for (int pass = 0; pass < 2; pass++)
        for (uint32_t g = 0; g < ng; g++) {
            std::vector<uint32_t> c(cnt.begin() + first[g], cnt.begin() + first[g + 1]), b(c.size(), 0);
            plans[g] = &e.get_plan<C>(c, b, fmt, 0, 0, t.shifts());
        }
    for (uint32_t g = 0; g < ng; g++) e.ensure_workspace<C>(*plans[g]);
    e.ensure_copy_resources(ng + 1);
    // buffers (re)allocated in the compute stream's order: the copies wait for that
    ZK_CUDA(cudaEventRecord(e.copy_events[ng], e.stream));
    ZK_CUDA(cudaStreamWaitEvent(e.copy_stream, e.copy_events[ng], 0));
    uint8_t* ds = static_cast<uint8_t*>(e.w_scalars.p);
    auto copy = [&](uint32_t g) {
        ZK_CUDA(cudaMemcpyAsync(ds + soff[g] * 32, scalars + soff[g] * 32, (soff[g + 1] - soff[g]) * 32,
                                cudaMemcpyHostToDevice, e.copy_stream));
        ZK_CUDA(cudaEventRecord(e.copy_events[g], e.copy_stream));
    };
    copy(0);
    for (uint32_t g = 0; g < ng; g++) {
        if (g + 1 < ng) copy(g + 1);  // in flight while group g runs
        ZK_CUDA(cudaStreamWaitEvent(e.stream, e.copy_events[g], 0));
        e.run_device_graph<C>(*plans[g], t.points.as<uint32_t>(), t.phi.as<uint32_t>(),
                              reinterpret_cast<const uint32_t*>(ds + soff[g] * 32),
                              out + (size_t)first[g] * 3 * P::N * 4);
    }
}

// lazily created shared engine for the _auto entry points (zkMetal_ffi.swift:22-35)
static std::mutex g_auto_mu;
static Engine* g_auto = nullptr;
static Engine& auto_engine() {
    if (!g_auto) g_auto = new Engine();
    return *g_auto;
}

// Autotuner: for each power-of-two size in [min_l2, max_l2], time the MSM at
// window widths around the cost model's choice on synthetic inputs (the
// library's generator) and keep the fastest; then, from 2^14 points, the tile
// schedule at that layout: the level-1 chunk length (half and twice the cost
// rule's), 128 instead of 256 threads per accumulation block, and a
// reduction tree of arity 4 or 16 instead of 8, one knob at a time.  The
// tables feed every later plan of this engine (MSMs are matched to the
// nearest power of two; a batch takes the schedule of its largest MSM).
// The reference's tuner covers window bits and threadgroup sizes
// (Tuning.swift:9-127).
template <class C>
static std::string autotune(Engine& e, int min_l2, int max_l2) {
    using P = typename C::Fp;
    const size_t fb = P::N * 4;
    const uint64_t nmax = 1ull << max_l2;
    DevBuf pts, phi, sc, res;
    pts.ensure(nmax * 2 * fb);
    phi.ensure(nmax * 2 * fb);
    sc.ensure(nmax * 32);
    res.ensure(3 * fb + 16);
    e.gen_bases<C>(0xA070u, 0, nmax, pts.as<uint32_t>());
    e.gen_scalars<C>(0xA070u, 0, nmax, 0, ZKMSM_SCALAR_MONT, sc.as<uint32_t>());
    e.make_phi<C>(pts.as<uint32_t>(), nmax, phi.as<uint32_t>());
    cudaEvent_t a, b;
    ZK_CUDA(cudaEventCreate(&a));
    ZK_CUDA(cudaEventCreate(&b));
    const int saved_w = e.tuning.window_bits;
    const bool saved_prof = e.profile;
    e.profile = false;
    // device time of one n-point MSM under the engine's current tuning
    auto time_plan = [&](uint32_t n) -> float {
        Plan& pl = e.get_plan<C>({n}, {0}, ZKMSM_SCALAR_MONT);
        e.ensure_workspace<C>(pl);
        e.enqueue<C>(pl, pts.as<uint32_t>(), phi.as<uint32_t>(), sc.as<uint32_t>(), res.as<uint32_t>());
        ZK_CUDA(cudaEventRecord(a, e.stream));
        const int reps = n >= (1u << 20) ? 2 : 4;
        for (int r = 0; r < reps; r++)
            e.enqueue<C>(pl, pts.as<uint32_t>(), phi.as<uint32_t>(), sc.as<uint32_t>(), res.as<uint32_t>());
        ZK_CUDA(cudaEventRecord(b, e.stream));
        ZK_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        ZK_CUDA(cudaEventElapsedTime(&ms, a, b));
        return ms / reps;
    };
    std::string rep = "{";
    for (int l2 = min_l2; l2 <= max_l2; l2++) {
        uint32_t n = 1u << l2;
        e.tuning.window_bits = 0;
        e.tuning.window_table.erase({CurveTraits<C>::id * 2 + 1, l2});
        e.tuning.sched_table.erase({CurveTraits<C>::id * 2 + 1, l2});
        e.tuning.version++;
        const MsmDesc d0 = e.get_plan<C>({n}, {0}, ZKMSM_SCALAR_MONT).descs[0];
        const int c0 = (int)d0.c;
        // candidates: equal windows of c0 - 2 .. c0 + 2 bits, and the
        // planner's two-width layout when it chose one (table value 0)
        const bool two_width = d0.nlo < d0.nwin;
        int best_c = c0;
        float best = 1e30f;
        std::string row;
        for (int c = two_width ? 0 : std::max(4, c0 - 2); c <= std::min(22, c0 + 2); c++) {
            if (c > 0 && c < std::max(4, c0 - 2)) continue;
            e.tuning.window_bits = c;
            const float ms = time_plan(n);
            row += (row.empty() ? "" : ",") + std::string("\"") + std::to_string(c) + "\":" + std::to_string(ms);
            if (ms < best) {
                best = ms;
                best_c = c;
            }
        }
        e.tuning.window_table[{CurveTraits<C>::id * 2 + 1, l2}] = best_c;
        e.tuning.window_bits = 0;
        e.tuning.version++;
        // then the tile schedule at that window layout, one knob at a time
        // (kept when it is at least 1% faster): level-1 chunk length, threads
        // per accumulation block, arity of the reduction tree
        Tuning::Schedule bs;
        std::string srow;
        if (l2 >= 14) {
            const std::pair<int, int> key{CurveTraits<C>::id * 2 + 1, l2};
            auto try_sched = [&](Tuning::Schedule cand, const char* name, int v) {
                e.tuning.sched_table[key] = cand;
                e.tuning.version++;
                const float ms = time_plan(n);
                srow += (srow.empty() ? "" : ",") + std::string("\"") + name + "=" + std::to_string(v) +
                        "\":" + std::to_string(ms);
                if (ms < best * 0.99f) {
                    best = ms;
                    bs = cand;
                }
            };
            for (int pct : {50, 200}) {
                Tuning::Schedule c = bs;
                c.chunk_pct = pct;
                try_sched(c, "chunk_pct", pct);
            }
            {
                Tuning::Schedule c = bs;
                c.acc_threads = 128;
                try_sched(c, "acc_threads", 128);
            }
            for (int L : {4, 16}) {
                Tuning::Schedule c = bs;
                c.red_L = L;
                try_sched(c, "red_L", L);
            }
            e.tuning.sched_table[key] = bs;
            e.tuning.version++;
        }
        rep += (l2 == min_l2 ? "" : ",") + std::string("\"") + std::to_string(l2) + "\":{\"best\":" +
               std::to_string(best_c) + ",\"model\":" + std::to_string(two_width ? 0 : c0) + ",\"ms\":{" + row +
               "},\"schedule\":{\"chunk_pct\":" + std::to_string(bs.chunk_pct) + ",\"acc_threads\":" +
               std::to_string(bs.acc_threads) + ",\"red_L\":" + std::to_string(bs.red_L) + ",\"ms\":{" + srow +
               "}},\"best_ms\":" + std::to_string(best) + "}";
    }
    rep += "}";
    e.tuning.window_bits = saved_w;
    e.tuning.version++;
    e.profile = saved_prof;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    ZK_CUDA(cudaStreamSynchronize(e.stream));
    return rep;
}

}  // namespace zkmsm

using namespace zkmsm;

extern "C" {

ZkMetalStatus zkmetal_msm_engine_create(ZkMetalMSMEngine* out) {
    if (!out) return ZKMETAL_ERR_INVALID_INPUT;
    if (!have_gpu()) {
        set_error("no compute-capability 10.x CUDA device");
        return ZKMETAL_ERR_NO_GPU;
    }
    return guarded([&] {
        *out = new Engine();
        return ZKMETAL_SUCCESS;
    });
}

void zkmetal_msm_engine_destroy(ZkMetalMSMEngine engine) { delete static_cast<Engine*>(engine); }

#define ENG(x) (*static_cast<Engine*>(x))

ZkMetalStatus zkmetal_bn254_msm(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars,
                                uint32_t n, uint8_t* rx, uint8_t* ry, uint8_t* rz) {
    if (!engine) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] { return msm_host<Bn254>(ENG(engine), points, scalars, n, ZKMSM_SCALAR_INT, 0, rx, ry, rz); });
}

ZkMetalStatus zkmetal_bn254_msm_fr(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars,
                                   uint32_t n, uint8_t* rx, uint8_t* ry, uint8_t* rz) {
    if (!engine) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] { return msm_host<Bn254>(ENG(engine), points, scalars, n, ZKMSM_SCALAR_MONT, 0, rx, ry, rz); });
}

ZkMetalStatus zkmetal_bn254_msm_auto(const uint8_t* points, const uint8_t* scalars, uint32_t n, uint8_t* rx,
                                     uint8_t* ry, uint8_t* rz) {
    if (!have_gpu()) return ZKMETAL_ERR_NO_GPU;
    std::lock_guard<std::mutex> lk(g_auto_mu);
    return guarded([&] { return msm_host<Bn254>(auto_engine(), points, scalars, n, ZKMSM_SCALAR_INT, 0, rx, ry, rz); });
}

#define SMALL_VARIANT(NAME, W)                                                                                \
    ZkMetalStatus NAME(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars, uint32_t n,    \
                       uint8_t* rx, uint8_t* ry, uint8_t* rz) {                                               \
        if (!engine) return ZKMETAL_ERR_INVALID_INPUT;                                                        \
        return guarded([&] { return msm_small(ENG(engine), points, scalars, n, W, rx, ry, rz); });          \
    }                                                                                                         \
    ZkMetalStatus NAME##_auto(const uint8_t* points, const uint8_t* scalars, uint32_t n, uint8_t* rx,         \
                              uint8_t* ry, uint8_t* rz) {                                                     \
        if (!have_gpu()) return ZKMETAL_ERR_NO_GPU;                                                           \
        std::lock_guard<std::mutex> lk(g_auto_mu);                                                            \
        return guarded([&] { return msm_small(auto_engine(), points, scalars, n, W, rx, ry, rz); });        \
    }

SMALL_VARIANT(zkmetal_bn254_msm_u8, 1)
SMALL_VARIANT(zkmetal_bn254_msm_u16, 2)
SMALL_VARIANT(zkmetal_bn254_msm_u32, 4)

ZkMetalStatus zkmetal_bn254_msm_batch(ZkMetalMSMEngine engine, const uint8_t* all_points, const uint8_t* all_scalars,
                                      const uint32_t* counts, uint32_t n_msms, uint8_t* results) {
    if (!engine) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] {
        return msm_batch_host<Bn254>(ENG(engine), all_points, all_scalars, counts, n_msms, ZKMSM_SCALAR_INT, results);
    });
}

ZkMetalStatus zkmetal_bn254_msm_batch_auto(const uint8_t* all_points, const uint8_t* all_scalars,
                                           const uint32_t* counts, uint32_t n_msms, uint8_t* results) {
    if (!have_gpu()) return ZKMETAL_ERR_NO_GPU;
    std::lock_guard<std::mutex> lk(g_auto_mu);
    return guarded([&] {
        return msm_batch_host<Bn254>(auto_engine(), all_points, all_scalars, counts, n_msms, ZKMSM_SCALAR_INT,
                                     results);
    });
}

ZkMetalStatus zkmsm_msm_batch(ZkMetalMSMEngine engine, int curve, const uint8_t* all_points,
                              const uint8_t* all_scalars, int fmt, const uint32_t* counts, uint32_t n_msms,
                              uint8_t* results) {
    if (!engine || !curve_ok(curve)) return ZKMETAL_ERR_INVALID_INPUT;
    if (fmt != ZKMSM_SCALAR_INT && fmt != ZKMSM_SCALAR_MONT) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] {
        ZkMetalStatus st = ZKMETAL_SUCCESS;
        with_curve(curve, [&](auto cv) {
            st = msm_batch_host<decltype(cv)>(ENG(engine), all_points, all_scalars, counts, n_msms, fmt, results);
        });
        return st;
    });
}

ZkMetalStatus zkmetal_bls12_381_g1_msm(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars,
                                       uint32_t n, uint8_t* rx, uint8_t* ry, uint8_t* rz) {
    if (!engine) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] { return msm_host<Bls381>(ENG(engine), points, scalars, n, ZKMSM_SCALAR_INT, 0, rx, ry, rz); });
}

ZkMetalStatus zkmetal_bls12_381_g1_msm_fr(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars,
                                          uint32_t n, uint8_t* rx, uint8_t* ry, uint8_t* rz) {
    if (!engine) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded(
        [&] { return msm_host<Bls381>(ENG(engine), points, scalars, n, ZKMSM_SCALAR_MONT, 0, rx, ry, rz); });
}

ZkMetalStatus zkmetal_bls12_381_g1_msm_batch(ZkMetalMSMEngine engine, const uint8_t* all_points,
                                             const uint8_t* all_scalars, const uint32_t* counts, uint32_t n_msms,
                                             uint8_t* results) {
    if (!engine) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] {
        return msm_batch_host<Bls381>(ENG(engine), all_points, all_scalars, counts, n_msms, ZKMSM_SCALAR_INT,
                                      results);
    });
}

ZkMetalStatus zkmetal_bls12_377_g1_msm(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars,
                                       uint32_t n, uint8_t* rx, uint8_t* ry, uint8_t* rz) {
    if (!engine) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] { return msm_host<Bls377>(ENG(engine), points, scalars, n, ZKMSM_SCALAR_INT, 0, rx, ry, rz); });
}

ZkMetalStatus zkmetal_bls12_377_g1_msm_fr(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars,
                                          uint32_t n, uint8_t* rx, uint8_t* ry, uint8_t* rz) {
    if (!engine) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded(
        [&] { return msm_host<Bls377>(ENG(engine), points, scalars, n, ZKMSM_SCALAR_MONT, 0, rx, ry, rz); });
}

ZkMetalStatus zkmetal_bls12_377_g1_msm_batch(ZkMetalMSMEngine engine, const uint8_t* all_points,
                                             const uint8_t* all_scalars, const uint32_t* counts, uint32_t n_msms,
                                             uint8_t* results) {
    if (!engine) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] {
        return msm_batch_host<Bls377>(ENG(engine), all_points, all_scalars, counts, n_msms, ZKMSM_SCALAR_INT,
                                      results);
    });
}

ZkMetalStatus zkmetal_bn254_g2_msm(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars,
                                   uint32_t n, uint8_t* rx, uint8_t* ry, uint8_t* rz) {
    if (!engine) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] { return msm_host<Bn254G2>(ENG(engine), points, scalars, n, ZKMSM_SCALAR_INT, 0, rx, ry, rz); });
}

ZkMetalStatus zkmetal_bn254_g2_msm_fr(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars,
                                      uint32_t n, uint8_t* rx, uint8_t* ry, uint8_t* rz) {
    if (!engine) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded(
        [&] { return msm_host<Bn254G2>(ENG(engine), points, scalars, n, ZKMSM_SCALAR_MONT, 0, rx, ry, rz); });
}

void zkmetal_set_shader_dir(const char*) {}

int32_t zkmetal_gpu_available(void) { return have_gpu() ? 1 : 0; }

const char* zkmetal_version(void) { return "zkmsm-b200 0.1.0"; }

const char* zkmsm_last_error(void) { return g_last_error.c_str(); }

ZkMetalStatus zkmsm_msm_device(ZkMetalMSMEngine engine, int curve, const void* d_points, const void* d_scalars,
                               int fmt, uint32_t n, uint8_t* result, void* stream) {
    if (!engine || !d_points || !d_scalars || !result || n == 0) return ZKMETAL_ERR_INVALID_INPUT;
    if (!curve_ok(curve)) return ZKMETAL_ERR_INVALID_INPUT;
    if (fmt != ZKMSM_SCALAR_INT && fmt != ZKMSM_SCALAR_MONT) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] {
        Engine& e = ENG(engine);
        cudaStream_t saved = e.stream;
        if (stream) e.stream = static_cast<cudaStream_t>(stream);
        struct Restore {
            Engine& e;
            cudaStream_t s;
            ~Restore() { e.stream = s; }
        } restore{e, saved};
        const uint32_t* pts = static_cast<const uint32_t*>(d_points);
        const uint32_t* sc = static_cast<const uint32_t*>(d_scalars);
        with_curve(curve, [&](auto cv) {
            using C = decltype(cv);
            const auto sl = e.sampled_layout<C>(sc, n, fmt);
            Plan& pl = e.get_plan<C>({n}, {0}, fmt, 0, sl.window, {}, sl.entries);
            e.w_phi.ensure((size_t)n * 2 * fp_bytes(curve) + 16);
            e.make_phi<C>(pts, n, e.w_phi.as<uint32_t>());
            e.run_device<C>(pl, pts, e.w_phi.as<uint32_t>(), sc, result);
        });
        return ZKMETAL_SUCCESS;
    });
}

ZkMetalStatus zkmsm_msm_device_async(ZkMetalMSMEngine engine, int curve, const void* d_points, const void* d_phi,
                                     const void* d_scalars, int fmt, uint32_t n, void* d_result, void* stream) {
    if (!engine || !d_points || !d_scalars || !d_result || n == 0 || n >= (1u << 30)) return ZKMETAL_ERR_INVALID_INPUT;
    if (!curve_ok(curve)) return ZKMETAL_ERR_INVALID_INPUT;
    if (fmt != ZKMSM_SCALAR_INT && fmt != ZKMSM_SCALAR_MONT) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] {
        Engine& e = ENG(engine);
        cudaStream_t saved = e.stream;
        if (stream) e.stream = static_cast<cudaStream_t>(stream);
        struct Restore {
            Engine& e;
            cudaStream_t s;
            ~Restore() { e.stream = s; }
        } restore{e, saved};
        const uint32_t* pts = static_cast<const uint32_t*>(d_points);
        const uint32_t* phi = static_cast<const uint32_t*>(d_phi);
        const uint32_t* sc = static_cast<const uint32_t*>(d_scalars);
        uint32_t* res = static_cast<uint32_t*>(d_result);
        with_curve(curve, [&](auto cv) {
            using C = decltype(cv);
            const auto sl = e.sampled_layout<C>(sc, n, fmt);
            Plan& pl = e.get_plan<C>({n}, {0}, fmt, 0, sl.window, {}, sl.entries);
            e.ensure_workspace<C>(pl);
            if (!phi) {
                e.w_phi.ensure((size_t)n * 2 * fp_bytes(curve) + 16);
                e.make_phi<C>(pts, n, e.w_phi.as<uint32_t>());
                phi = e.w_phi.as<uint32_t>();
            }
            e.enqueue<C>(pl, pts, phi, sc, res);
        });
        return ZKMETAL_SUCCESS;
    });
}

ZkMetalStatus zkmsm_table_create(ZkMetalMSMEngine engine, int curve, const void* points, uint64_t n,
                                 int on_device, ZkMsmTable* out) {
    if (!engine || !points || !out || n == 0 || n >= (1ull << 30)) return ZKMETAL_ERR_INVALID_INPUT;
    if (!curve_ok(curve)) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] {
        Engine& e = ENG(engine);
        std::unique_ptr<Table> t(new Table{&e, curve, n, {}, {}});
        size_t bytes = (size_t)n * 2 * fp_bytes(curve);
        t->points.alloc_exact(bytes);
        with_curve(curve, [&](auto cv) {
            if (CurveTraits<decltype(cv)>::glv) t->phi.alloc_exact(bytes);
        });
        ZK_CUDA(cudaMemcpyAsync(t->points.p, points, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                e.stream));
        with_curve(curve, [&](auto cv) {
            e.make_phi<decltype(cv)>(t->points.as<uint32_t>(), n, t->phi.as<uint32_t>());
        });
        ZK_CUDA(cudaStreamSynchronize(e.stream));
        *out = t.release();
        return ZKMETAL_SUCCESS;
    });
}

ZkMetalStatus zkmsm_table_precompute(ZkMsmTable table, int spacing_bits) {
    if (!table || spacing_bits < 0 || spacing_bits == 1 || spacing_bits > 24) return ZKMETAL_ERR_INVALID_INPUT;
    Table& t = *static_cast<Table*>(table);
    const uint32_t s = (uint32_t)spacing_bits;
    uint32_t fr_bits = 0;
    with_curve(t.curve, [&](auto cv) { fr_bits = CurveTraits<decltype(cv)>::fr_bits; });
    // a window's top digit may carry into bit fr_bits, so copies cover fr_bits + 1 bits
    const uint32_t copies = s ? (fr_bits + 1 + s - 1) / s : 1;
    if ((uint64_t)copies * t.n > VAL_IDX_MASK) {
        set_error("shift table index exceeds 30 bits: use a wider spacing");
        return ZKMETAL_ERR_INVALID_INPUT;
    }
    if (s == t.shift_bits) return ZKMETAL_SUCCESS;
    return guarded([&] {
        Engine& e = *t.engine;
        const size_t ab = (size_t)2 * fp_bytes(t.curve);
        DevBuf nb;
        nb.alloc_exact((size_t)copies * t.n * ab);
        ZK_CUDA(cudaMemcpyAsync(nb.p, t.points.p, (size_t)t.n * ab, cudaMemcpyDeviceToDevice, e.stream));
        with_curve(t.curve, [&](auto cv) { e.make_shifts<decltype(cv)>(nb.as<uint32_t>(), t.n, s, copies); });
        ZK_CUDA(cudaStreamSynchronize(e.stream));
        e.drop_graphs();  // graphs captured over the old table address
        std::swap(t.points.p, nb.p);
        std::swap(t.points.cap, nb.cap);
        t.shift_bits = s;
        t.copies = copies;
        return ZKMETAL_SUCCESS;
    });
}

int zkmsm_table_shift_bits(ZkMsmTable table) { return table ? (int)static_cast<Table*>(table)->shift_bits : -1; }

void zkmsm_table_destroy(ZkMsmTable table) { delete static_cast<Table*>(table); }

const void* zkmsm_table_device_points(ZkMsmTable table) {
    return table ? static_cast<Table*>(table)->points.p : nullptr;
}

ZkMetalStatus zkmsm_batch_commit(ZkMetalMSMEngine engine, ZkMsmTable table, const void* scalars, int on_device,
                                 int fmt, const uint32_t* counts, uint32_t n_msms, uint8_t* results) {
    if (!engine || !table || !scalars || !counts || !results || n_msms == 0) return ZKMETAL_ERR_INVALID_INPUT;
    if (fmt != ZKMSM_SCALAR_INT && fmt != ZKMSM_SCALAR_MONT) return ZKMETAL_ERR_INVALID_INPUT;
    Table& t = *static_cast<Table*>(table);
    uint64_t total = 0;
    for (uint32_t m = 0; m < n_msms; m++) {
        if (counts[m] > t.n) return ZKMETAL_ERR_INVALID_INPUT;
        total += counts[m];
    }
    return guarded([&] {
        Engine& e = ENG(engine);
        std::vector<uint32_t> cnt(counts, counts + n_msms), boff(n_msms, 0);
        int fb = fp_bytes(t.curve);
        std::vector<uint8_t> out((size_t)n_msms * 3 * fb);
        if (!on_device && n_msms >= 2 && total >= BATCH_GROUP_MIN_POINTS) {
            with_curve(t.curve, [&](auto cv) {
                batch_commit_grouped<decltype(cv)>(e, t, static_cast<const uint8_t*>(scalars), fmt, cnt,
                                                   out.data());
            });
            for (uint32_t m = 0; m < n_msms; m++) {
                uint8_t* dst = results + (size_t)m * 3 * fb;
                if (counts[m] == 0) memset(dst, 0, 3 * fb);
                else memcpy(dst, out.data() + (size_t)m * 3 * fb, 3 * fb);
            }
            return ZKMETAL_SUCCESS;
        }
        const uint32_t* sc = static_cast<const uint32_t*>(scalars);
        if (!on_device) {
            h2d(e, e.w_scalars, scalars, (size_t)total * 32);
            sc = e.w_scalars.as<uint32_t>();
        }
        with_curve(t.curve, [&](auto cv) {
            using C = decltype(cv);
            Plan& pl = e.get_plan<C>(cnt, boff, fmt, 0, 0, t.shifts());
            e.run_device_graph<C>(pl, t.points.as<uint32_t>(), t.phi.as<uint32_t>(), sc, out.data());
        });
        for (uint32_t m = 0; m < n_msms; m++) {
            uint8_t* dst = results + (size_t)m * 3 * fb;
            if (counts[m] == 0) memset(dst, 0, 3 * fb);
            else memcpy(dst, out.data() + (size_t)m * 3 * fb, 3 * fb);
        }
        return ZKMETAL_SUCCESS;
    });
}

ZkMetalStatus zkmsm_autotune(ZkMetalMSMEngine engine, int curve, int min_log2n, int max_log2n, char* report,
                             uint64_t report_len) {
    if (!engine || min_log2n < 4 || max_log2n > 26 || min_log2n > max_log2n) return ZKMETAL_ERR_INVALID_INPUT;
    if (!curve_ok(curve)) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] {
        std::string r;
        with_curve(curve, [&](auto cv) { r = autotune<decltype(cv)>(ENG(engine), min_log2n, max_log2n); });
        if (report && report_len) {
            size_t k = std::min<size_t>(r.size(), report_len - 1);
            memcpy(report, r.data(), k);
            report[k] = 0;
        }
        return ZKMETAL_SUCCESS;
    });
}

ZkMetalStatus zkmsm_tuning_save(ZkMetalMSMEngine engine, const char* path) {
    if (!engine || !path) return ZKMETAL_ERR_INVALID_INPUT;
    FILE* f = fopen(path, "w");
    if (!f) {
        set_error(std::string("cannot write ") + path);
        return ZKMETAL_ERR_INVALID_INPUT;
    }
    fprintf(f, "zkmsm-tuning 2\n");
    for (auto& kv : ENG(engine).tuning.window_table)
        fprintf(f, "w %d %d %d\n", kv.first.first, kv.first.second, kv.second);
    for (auto& kv : ENG(engine).tuning.sched_table)
        fprintf(f, "s %d %d %d %d %d\n", kv.first.first, kv.first.second, kv.second.chunk_pct, kv.second.acc_threads,
                kv.second.red_L);
    fclose(f);
    return ZKMETAL_SUCCESS;
}

ZkMetalStatus zkmsm_tuning_load(ZkMetalMSMEngine engine, const char* path) {
    if (!engine || !path) return ZKMETAL_ERR_INVALID_INPUT;
    FILE* f = fopen(path, "r");
    if (!f) {
        set_error(std::string("cannot read ") + path);
        return ZKMETAL_ERR_INVALID_INPUT;
    }
    char head[32] = {0};
    int ver = 0;
    if (fscanf(f, "%31s %d", head, &ver) != 2 || std::string(head) != "zkmsm-tuning" || (ver != 1 && ver != 2)) {
        fclose(f);
        set_error("not a zkmsm tuning file");
        return ZKMETAL_ERR_INVALID_INPUT;
    }
    Engine& e = ENG(engine);
    int k, l2, c;
    if (ver == 1) {  // window lines only: "k l2 c"
        while (fscanf(f, "%d %d %d", &k, &l2, &c) == 3)
            if (k >= 0 && k < 2 * NCURVES && l2 >= 0 && l2 < 40 && (c == 0 || (c >= 2 && c <= 24)))
                e.tuning.window_table[{k, l2}] = c;  // 0: the planner's own layout
    } else {  // "w k l2 c" and "s k l2 chunk_pct acc_threads red_L"
        char tag[4] = {0};
        while (fscanf(f, "%3s", tag) == 1) {
            if (tag[0] == 'w') {
                if (fscanf(f, "%d %d %d", &k, &l2, &c) != 3) break;
                if (k >= 0 && k < 2 * NCURVES && l2 >= 0 && l2 < 40 && (c == 0 || (c >= 2 && c <= 24)))
                    e.tuning.window_table[{k, l2}] = c;
            } else if (tag[0] == 's') {
                Tuning::Schedule sc;
                if (fscanf(f, "%d %d %d %d %d", &k, &l2, &sc.chunk_pct, &sc.acc_threads, &sc.red_L) != 5) break;
                const bool ok = sc.chunk_pct >= 0 && sc.chunk_pct <= 1000 &&
                                (sc.acc_threads == 0 || sc.acc_threads == 128 || sc.acc_threads == 256) &&
                                (sc.red_L == 0 || sc.red_L == 4 || sc.red_L == 8 || sc.red_L == 16);
                if (k >= 0 && k < 2 * NCURVES && l2 >= 0 && l2 < 40 && ok) e.tuning.sched_table[{k, l2}] = sc;
            } else {
                break;
            }
        }
    }
    fclose(f);
    e.tuning.version++;
    return ZKMETAL_SUCCESS;
}

ZkMetalStatus zkmsm_engine_set_tuning(ZkMetalMSMEngine engine, int window_bits, int chunk, int glv) {
    if (!engine || !window_setting_ok(window_bits) || chunk < 0 || chunk > 4096) return ZKMETAL_ERR_INVALID_INPUT;
    Engine& e = ENG(engine);
    e.tuning.window_bits = window_bits;
    e.tuning.chunk = chunk;
    e.tuning.glv = glv < 0 ? -1 : (glv ? 1 : 0);
    e.tuning.version++;
    return ZKMETAL_SUCCESS;
}

ZkMetalStatus zkmsm_engine_set_sampling(ZkMetalMSMEngine engine, int enable) {
    if (!engine || enable < 0 || enable > 1) return ZKMETAL_ERR_INVALID_INPUT;
    ENG(engine).scalar_sampling = enable;
    return ZKMETAL_SUCCESS;
}

ZkMetalStatus zkmsm_engine_set_stripe(ZkMetalMSMEngine engine, int stripe_log2) {
    if (!engine || stripe_log2 < -1 || stripe_log2 > 30) return ZKMETAL_ERR_INVALID_INPUT;
    ENG(engine).stripe_log2 = stripe_log2;
    return ZKMETAL_SUCCESS;
}

ZkMetalStatus zkmsm_gen_bases(ZkMetalMSMEngine engine, int curve, uint64_t seed, uint64_t index0, uint64_t n,
                              void* d_out) {
    if (!engine || !d_out || !curve_ok(curve)) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] {
        with_curve(curve, [&](auto cv) {
            ENG(engine).gen_bases<decltype(cv)>(seed, index0, n, static_cast<uint32_t*>(d_out));
        });
        return ZKMETAL_SUCCESS;
    });
}

ZkMetalStatus zkmsm_gen_scalars(ZkMetalMSMEngine engine, int curve, uint64_t seed, uint64_t index0, uint64_t n,
                                int dist, int fmt, void* d_out) {
    if (!engine || !d_out || !curve_ok(curve) || (dist != 0 && dist != 1) || (fmt != 0 && fmt != 1))
        return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] {
        with_curve(curve, [&](auto cv) {
            ENG(engine).gen_scalars<decltype(cv)>(seed, index0, n, dist, fmt, static_cast<uint32_t*>(d_out));
        });
        return ZKMETAL_SUCCESS;
    });
}

ZkMetalStatus zkmsm_engine_profile(ZkMetalMSMEngine engine, int enable) {
    if (!engine) return ZKMETAL_ERR_INVALID_INPUT;
    ENG(engine).profile = enable != 0;
    return ZKMETAL_SUCCESS;
}

ZkMetalStatus zkmsm_engine_phase_times(ZkMetalMSMEngine engine, double* ms5, uint64_t* calls, int reset) {
    if (!engine || !ms5) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] {
        Engine& e = ENG(engine);
        e.prof_collect();
        for (int i = 0; i < Engine::NPHASE; i++) ms5[i] = e.phase_ms[i];
        if (calls) *calls = e.phase_calls;
        if (reset) {
            for (int i = 0; i < Engine::NPHASE; i++) e.phase_ms[i] = 0;
            e.phase_calls = 0;
        }
        return ZKMETAL_SUCCESS;
    });
}

static ZkMetalStatus plan_json(int curve, const uint32_t* counts, uint32_t n_msms, int fmt, int window_bits,
                               int chunk, int glv, int scalar_bits, ShiftSpec sh, char* buf, uint64_t buflen) {
    if (!counts || !buf || n_msms == 0 || !window_setting_ok(window_bits)) return ZKMETAL_ERR_INVALID_INPUT;
    return guarded([&] {
        Tuning t;
        t.window_bits = window_bits;
        t.chunk = chunk;
        t.glv = glv;
        std::vector<uint32_t> cnt(counts, counts + n_msms), boff(n_msms, 0);
        Plan pl;
        with_curve(curve, [&](auto cv) {
            Engine::plan_shape<decltype(cv)>(pl, t, cnt, boff, fmt, scalar_bits, 0, sh);
        });
        std::string s = "{\"descs\":[";
        for (size_t i = 0; i < pl.descs.size(); i++) {
            auto& d = pl.descs[i];
            s += (i ? "," : "") + std::string("[") + std::to_string(d.scalar_off) + "," + std::to_string(d.n) + "," +
                 std::to_string(d.base_off) + "," + std::to_string(d.c) + "," + std::to_string(d.nwin) + "," +
                 std::to_string(d.glv) + "," + std::to_string(d.bucket_off) + "," + std::to_string(d.fmt) + "," +
                 std::to_string(d.win_off) + "," + std::to_string(d.wstep) + "," + std::to_string(d.nred) + "," +
                 std::to_string(d.nlo) + "]";
        }
        s += "],\"entry_bound\":" + std::to_string(pl.entry_bound) + ",\"nbuckets\":" + std::to_string(pl.nbuckets) +
             ",\"sort\":[" + std::to_string(pl.sort_maxd) + "," + std::to_string(pl.sort_spb) + "," +
             std::to_string(pl.sort_passes) + "," + std::to_string(pl.sort_bits) + "," +
             std::to_string(pl.sort_tiles) + "],\"msd\":[" + std::to_string(pl.msd_passes) + "," +
             std::to_string(pl.msd_bits1) + "," + std::to_string(pl.msd_bits2) + "," + std::to_string(pl.msd_tiles1) +
             "," + std::to_string(pl.msd_tiles2) + "," + std::to_string(pl.msd_groups1) + "," +
             std::to_string(pl.msd_chunks2) + "],\"acc\":[";
        for (size_t l = 0; l < pl.acc_K.size(); l++)
            s += (l ? "," : "") + std::string("[") + std::to_string(pl.acc_K[l]) + "," + std::to_string(pl.acc_T[l]) +
                 "," + std::to_string(pl.acc_Mbound[l]) + "]";
        s += "],\"red_L\":" + std::to_string(pl.red_L) + ",\"red_log2L\":" + std::to_string(pl.red_log2L) +
             ",\"red\":[";
        for (size_t l = 0; l < pl.red_tasks.size(); l++) {
            s += (l ? "," : "") + std::string("[");
            for (size_t k = 0; k < pl.red_tasks[l].size(); k++) {
                auto& tk = pl.red_tasks[l][k];
                s += (k ? "," : "") + std::string("[") + std::to_string(tk.in_off) + "," + std::to_string(tk.n_in) +
                     "," + std::to_string(tk.out_off) + "," + std::to_string(tk.n_out) + "]";
            }
            s += "]";
        }
        s += "]}";
        if (s.size() + 1 > buflen) return ZKMETAL_ERR_INVALID_INPUT;
        memcpy(buf, s.c_str(), s.size() + 1);
        return ZKMETAL_SUCCESS;
    });
}

ZkMetalStatus zkmsm_plan_describe(int curve, const uint32_t* counts, uint32_t n_msms, int fmt, int window_bits,
                                  int chunk, int glv, int scalar_bits, char* buf, uint64_t buflen) {
    return plan_json(curve, counts, n_msms, fmt, window_bits, chunk, glv, scalar_bits, ShiftSpec{}, buf, buflen);
}

ZkMetalStatus zkmsm_plan_describe_shift(int curve, const uint32_t* counts, uint32_t n_msms, int fmt,
                                        int window_bits, int shift_bits, uint32_t table_points, char* buf,
                                        uint64_t buflen) {
    if (shift_bits < 2 || shift_bits > 24) return ZKMETAL_ERR_INVALID_INPUT;
    return plan_json(curve, counts, n_msms, fmt, window_bits, 0, -1, 0,
                     ShiftSpec{(uint32_t)shift_bits, table_points}, buf, buflen);
}

uint64_t zkmsm_engine_launch_count(ZkMetalMSMEngine engine) { return engine ? ENG(engine).launches : 0; }

uint64_t zkmsm_engine_last_entries(ZkMetalMSMEngine engine) {
    if (!engine) return 0;
    Engine& e = ENG(engine);
    if (!e.w_totals.p) return 0;
    uint32_t v = 0;
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(&v, e.w_totals.p, sizeof v, cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return v;
}

void* zkmsm_device_alloc(uint64_t bytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void zkmsm_device_free(void* p) {
    if (p) cudaFree(p);
}

ZkMetalStatus zkmsm_memcpy_h2d(void* d_dst, const void* src, uint64_t bytes) {
    return guarded([&] {
        ZK_CUDA(cudaMemcpy(d_dst, src, bytes, cudaMemcpyHostToDevice));
        return ZKMETAL_SUCCESS;
    });
}

ZkMetalStatus zkmsm_memcpy_d2h(void* dst, const void* d_src, uint64_t bytes) {
    return guarded([&] {
        ZK_CUDA(cudaMemcpy(dst, d_src, bytes, cudaMemcpyDeviceToHost));
        return ZKMETAL_SUCCESS;
    });
}

ZkMetalStatus zkmsm_device_sync(void) {
    return guarded([&] {
        ZK_CUDA(cudaDeviceSynchronize());
        return ZKMETAL_SUCCESS;
    });
}

}  // extern "C"
