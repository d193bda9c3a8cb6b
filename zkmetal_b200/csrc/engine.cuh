// Host-side MSM engine: plans a batch of MSMs, owns the device workspace and
// issues the kernel pipeline on its stream.
//
// Replaces the orchestration of the reference's MetalMSM.msm
// (MSM/MSMEngine.swift:287-909) and BLS12381MSM.msm
// (MSM/BLS12381MSMEngine.swift:260-513): buffer caching (ensureBuffers,
// MSMEngine.swift:232-277) becomes a grow-only device workspace; window
// selection (MSMEngine.swift:356-373) becomes a per-MSM cost model
// (overridable, and refined by the autotuner); the CPU sort and CPU Horner
// become device kernels so a whole batch runs without host round trips.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "types.cuh"

namespace zkmsm {

void set_error(const std::string& s);

struct CudaError {
    cudaError_t code;
    std::string where;
};

#define ZK_CUDA(call)                                                       \
    do {                                                                    \
        cudaError_t e__ = (call);                                           \
        if (e__ != cudaSuccess) throw ::zkmsm::CudaError{e__, #call};       \
    } while (0)

// Grow-only device buffer.
// Device buffer that only grows.  Bound to an owner's stream variable `sp`
// (the engine's current stream, which follows a caller's stream during
// calls on it), it grows through the stream-ordered allocator: the old block
// returns to the device's memory pool once the work already issued on that
// stream is done, so growing one engine's workspace never waits for other
// engines' work the way cudaFree does, and the new block is ready for work
// issued on the same stream (other streams must wait on it).
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaStream_t* sp = nullptr;
    bool ensure(size_t bytes) {  // true when it had to reallocate
        if (bytes <= cap) return false;
        // growth is geometric (at least 1.5x): a buffer that keeps growing is
        // reallocated a logarithmic number of times
        size_t want = std::max(bytes + bytes / 8 + 256, cap + cap / 2);
        if (sp) {
            if (p) ZK_CUDA(cudaFreeAsync(p, *sp));
            p = nullptr;
            cap = 0;
            ZK_CUDA(cudaMallocAsync(&p, want, *sp));
        } else {
            if (p) cudaFree(p);
            p = nullptr;
            cap = 0;
            ZK_CUDA(cudaMalloc(&p, want));
        }
        cap = want;
        return true;
    }
    // exactly `bytes` (synchronous allocation, contents dropped): for
    // long-lived buffers such as resident tables, where growth slack would
    // waste gigabytes
    void alloc_exact(size_t bytes) {
        release();
        ZK_CUDA(cudaMalloc(&p, bytes));
        cap = bytes;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
};

// Host-to-device copies from pageable host memory.  The driver stages a
// pageable copy through its own small pinned buffers on one thread (about
// 10 GB/s here); a caller handing over plain arrays (a Swift [PointAffine],
// a numpy array) would wait that long.  The stager instead copies chunks
// into a ring of its own pinned buffers with several host threads and DMAs
// each chunk from there on the caller's stream, the next chunk's host copy
// running while the previous one is on the bus.  A buffer is refilled once
// its DMA has completed (event).  Calls return when the last chunk is
// queued, like a pageable cudaMemcpyAsync.
class HostStager {
   public:
    static constexpr size_t CHUNK = 32u << 20;
    static constexpr int SLOTS = 3;

    ~HostStager() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
        for (int i = 0; i < SLOTS; i++) {
            if (done_[i]) cudaEventDestroy(done_[i]);
            if (buf_[i]) cudaFreeHost(buf_[i]);
        }
    }

    // dst (device) <- src (pageable host), enqueued on stream s
    cudaError_t copy(void* dst, const void* src, size_t bytes, cudaStream_t s) {
        cudaError_t e = init();
        if (e != cudaSuccess) return e;
        const uint8_t* sp = static_cast<const uint8_t*>(src);
        uint8_t* dp = static_cast<uint8_t*>(dst);
        for (size_t off = 0; off < bytes; off += CHUNK) {
            const size_t len = std::min(CHUNK, bytes - off);
            const int k = next_++ % SLOTS;
            if ((e = cudaEventSynchronize(done_[k])) != cudaSuccess) return e;
            parallel_memcpy(buf_[k], sp + off, len);
            if ((e = cudaMemcpyAsync(dp + off, buf_[k], len, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
            if ((e = cudaEventRecord(done_[k], s)) != cudaSuccess) return e;
        }
        return cudaSuccess;
    }

    static bool pageable(const void* p) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
            cudaGetLastError();
            return true;
        }
        return a.type == cudaMemoryTypeUnregistered;
    }

   private:
    cudaError_t init() {
        if (buf_[0]) return cudaSuccess;
        for (int i = 0; i < SLOTS; i++) {
            cudaError_t e = cudaMallocHost(&buf_[i], CHUNK);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done_[i], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
        unsigned hw = std::thread::hardware_concurrency();
        const int nt = (int)std::max(1u, std::min(8u, hw / 2));
        for (int i = 0; i < nt; i++) workers_.emplace_back([this] { work(); });
        return cudaSuccess;
    }

    void work() {
        uint64_t seen = 0;
        for (;;) {
            std::function<void()> job;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || (gen_ != seen && taken_ < parts_); });
                if (stop_) return;
                const size_t i = taken_++;
                if (taken_ == parts_) seen = gen_;
                job = [this, i] { part(i); };
            }
            job();
            {
                std::lock_guard<std::mutex> lk(mu_);
                if (++finished_ == parts_) cv_done_.notify_all();
            }
        }
    }

    void part(size_t i) {
        const size_t per = (len_ + parts_ - 1) / parts_;
        const size_t a = std::min(len_, i * per), b = std::min(len_, a + per);
        if (b > a) memcpy(static_cast<uint8_t*>(dst_) + a, static_cast<const uint8_t*>(src_) + a, b - a);
    }

    void parallel_memcpy(void* dst, const void* src, size_t len) {
        std::unique_lock<std::mutex> lk(mu_);
        dst_ = dst;
        src_ = src;
        len_ = len;
        parts_ = workers_.size();
        taken_ = finished_ = 0;
        gen_++;
        cv_.notify_all();
        cv_done_.wait(lk, [&] { return finished_ == parts_; });
    }

    void* buf_[SLOTS] = {};
    cudaEvent_t done_[SLOTS] = {};
    uint64_t next_ = 0;
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, cv_done_;
    bool stop_ = false;
    uint64_t gen_ = 0;
    void* dst_ = nullptr;
    const void* src_ = nullptr;
    size_t len_ = 0, parts_ = 0, taken_ = 0, finished_ = 0;
};

// Curves with an engine instantiation// Curves with an engine instantiation (CurveTraits<C>::id = 0 .. NCURVES - 1);
// every per-curve array of the engine has this many entries.
constexpr int NCURVES = 4;
// widest coordinate of any curve, in 32-bit words (BN254 G2: two 8-word Fp)
constexpr int MAX_COORD_WORDS = 16;

struct Tuning {
    // 0: autotuned table if present, else cost model; 2..24: equal windows of
    // that width; c | nlo << 16: nlo windows of c bits, the rest c + 1 bits
    int window_bits = 0;
    int chunk = 0;        // level-1 chunk length, 0: automatic
    int glv = -1;         // -1: automatic (on), 0 off, 1 on
    // autotuned window width per (curve*2 + glv, nearest log2 n); filled by
    // zkmsm_autotune or zkmsm_tuning_load
    std::map<std::pair<int, int>, int> window_table;
    // autotuned schedule per (curve*2 + glv, nearest log2 n) of the largest
    // MSM of a plan: level-1 chunk length as a percentage of the cost
    // rule's (0: the rule's), threads per block of the level-1
    // accumulation (0: the curve's default), arity of the bucket-reduction
    // tree (0: 8)
    struct Schedule {
        int chunk_pct = 0, acc_threads = 0, red_L = 0;
    };
    std::map<std::pair<int, int>, Schedule> sched_table;
    uint64_t version = 0;  // bumped whenever the table changes
    // threads of the level-1 accumulation kernel resident at once on the
    // device, per curve (0: unknown; then chunks are not wave-aligned)
    uint32_t acc_wave[NCURVES] = {};
    // SMs of the device (the MSD sort's first pass runs one group per SM)
    uint32_t sms = 148;
};

// Host description of one batch run.
struct Plan {
    int curve = 0;
    std::vector<MsmDesc> descs;
    uint64_t total_scalars = 0;
    uint64_t entry_bound = 0;
    uint32_t nbuckets = 0;
    uint32_t nwin_total = 0;
    // radix sort of the entries (msm_kernels.cuh): at most sort_maxd digits
    // per scalar, sort_spb scalars per digit block, sort_passes passes of
    // sort_bits-bit digits over sort_tiles tiles of SORT_ETILE entries
    uint32_t sort_maxd = 0, sort_spb = 0, sort_passes = 0, sort_bits = 0, sort_tiles = 0;
    // MSD sort instead (msd_passes 1 or 2; 0: the LSD passes above): digit
    // widths of the passes (the first takes the top bits), tile-count
    // bounds of the passes (pass 2: one partial tile more per segment), the
    // scatter groups of pass 1 and the chunk-count bound of pass 2
    uint32_t msd_passes = 0, msd_bits1 = 0, msd_bits2 = 0, msd_tiles1 = 0, msd_tiles2 = 0;
    uint32_t msd_groups1 = 0, msd_chunks2 = 0;
    // segmented-sum levels: chunk length and chunk-count bound per level
    std::vector<uint32_t> acc_K, acc_T;
    std::vector<uint64_t> acc_Mbound;
    // bucket-reduction levels
    uint32_t red_L = 8, red_log2L = 3;
    // threads per block of the level-1 accumulation (0: the curve's default)
    uint32_t acc_threads = 0;
    std::vector<std::vector<RedTask>> red_tasks;
    std::vector<uint32_t> red_nout;
    // device copies of descs and reduction tasks (uploaded once per plan)
    DevBuf d_descs, d_tasks;
    std::vector<size_t> task_level_off;
    // calls of this plan through run_device_graph that found no captured graph
    mutable uint32_t graph_misses = 0;
    // forget the host-side shape (device tables are kept for reuse)
    void clear_host() {
        descs.clear();
        total_scalars = entry_bound = 0;
        nbuckets = nwin_total = 0;
        sort_maxd = sort_spb = sort_passes = sort_bits = sort_tiles = 0;
        msd_passes = msd_bits1 = msd_bits2 = msd_tiles1 = msd_tiles2 = 0;
        msd_groups1 = msd_chunks2 = 0;
        red_L = 8;
        red_log2L = 3;
        acc_threads = 0;
        acc_K.clear();
        acc_T.clear();
        acc_Mbound.clear();
        red_tasks.clear();
        red_nout.clear();
        task_level_off.clear();
        graph_misses = 0;
    }
};

// Words of the MSD sort's count rows (one row per tile, the larger pass; the
// slot rows are as large) and of its scan layout (one word per digit and group: pass-1 groups in
// MSD_COUNT_PARTS parts, pass-2 chunks).
inline uint64_t msd_rows_words(const Plan& pl) {
    return std::max<uint64_t>((uint64_t)(1u << pl.msd_bits1) * pl.msd_tiles1,
                              pl.msd_passes == 2 ? (uint64_t)(1u << pl.msd_bits2) * pl.msd_tiles2 : 0);
}
inline uint64_t msd_scan_words(const Plan& pl) {
    return std::max<uint64_t>((uint64_t)(1u << pl.msd_bits1) * pl.msd_groups1 * MSD_COUNT_PARTS,
                              pl.msd_passes == 2 ? (uint64_t)(1u << pl.msd_bits2) * pl.msd_chunks2 : 0);
}

// Nearest power-of-two exponent of n (n >= 1).
inline int nearest_log2(uint64_t n) {
    int l2 = 0;
    while ((1ull << (l2 + 1)) <= n) l2++;
    if (n - (1ull << l2) > (1ull << l2) / 2) l2++;
    return l2;
}

// Signed windows a half-scalar of `bits` bits needs at width c.
inline uint32_t windows_for(uint32_t bits, uint32_t c) { return (bits + 1 + c - 1) / c; }

// Relative cost of window width c for `entries_per_window` entries: mixed
// additions (one per nonzero digit) plus ~3 XYZZ additions per bucket in the
// reduction, plus a latency term for the reduction depth and Horner chain.
inline uint32_t choose_window(uint64_t entries_per_window, uint32_t bits) {
    double best = 1e300;
    uint32_t bc = 8;
    for (uint32_t c = 4; c <= 22; c++) {
        uint32_t w = windows_for(bits, c);
        double add = (double)entries_per_window * w;
        double red = 4.2 * (double)w * (double)(1u << (c - 1));
        double lat = 2.0e5 * (c + 6) + 4.0e4 * (double)w * c;  // serial tails, in madd units
        double cost = add + red + lat;
        if (cost < best) {
            best = cost;
            bc = c;
        }
    }
    return bc;
}

// Two-width window layout from LAYOUT_MIN_ENTRIES entries per window up:
// W windows cover the bits + 1 bits of the signed recoding as evenly as
// possible (nlo windows of c bits, W - nlo of c + 1), which for a given
// window count holds fewer buckets than equal windows whose last one is
// mostly empty.  Cost in units of one sorted entry: W per entry, 3 per
// bucket (the reduction: 0.51 ns per bucket against 0.171 ns per entry of
// the accumulation, BN254 at 2^24 on a B200) and the latency terms of
// choose_window.
constexpr uint64_t LAYOUT_MIN_ENTRIES = 1ull << 21;
struct WinLayout {
    uint32_t c, nlo, nwin;
};
inline WinLayout choose_layout(uint64_t entries_per_window, uint32_t bits) {
    const uint32_t cover = bits + 1;
    WinLayout best{cover, 1, 1};
    double best_cost = 1e300;
    for (uint32_t W = 1; W <= cover; W++) {
        const uint32_t c = cover / W, nhi = cover - W * c;
        if (c < 2) break;
        if (c + (nhi ? 1 : 0) > 22) continue;
        const double buckets = (double)(W - nhi) * (double)(1u << (c - 1)) + (double)nhi * (double)(1u << c);
        const double cost = (double)entries_per_window * W + 3.0 * buckets + 2.0e5 * (c + 6) + 4.0e4 * (double)W * c;
        if (cost < best_cost) {
            best_cost = cost;
            best = WinLayout{c, W - nhi, W};
        }
    }
    return best;
}

// Nonzero signed digits of one scalar half of bit length b under a layout:
// one per window that starts below bit b, and one more for the carry out of
// the top such window when b reaches that window's top bit (its digit is
// then above 2^(width-1) and is recoded with a carry into the next window).
inline double layout_digits(uint32_t b, uint32_t c, uint32_t nlo, uint32_t nwin) {
    uint32_t k = 0, end = 0;
    for (uint32_t w = 0; w < nwin; w++) {
        const uint32_t start = w * c + (w > nlo ? w - nlo : 0u);
        if (start < b) {
            k++;
            end = start + c + (w >= nlo ? 1u : 0u);
        }
    }
    if (k && k < nwin && b == end) k++;
    return (double)k;
}

// The window layout for an MSM of n scalars whose sampled half lengths are
// `hist` (k_scalar_profile; `halves` = sampled halves in total): the cost of
// choose_layout with the entry count taken from the sample instead of every
// digit being nonzero, over the two-width layouts and equal windows of 4..22
// bits.  Scalar sets with many zero, one or short values then get fewer,
// narrower buckets (BN254 witness-like scalars at 2^24: 7 windows of 19 bits
// rather than 6 of 21-22).  Returns c | nlo << 16 (nlo = 0: equal windows).
inline uint32_t choose_layout_sampled(const uint32_t* hist, uint64_t halves, uint64_t n, uint32_t bits,
                                      uint32_t halves_per_scalar, uint64_t* expected_entries = nullptr) {
    const uint32_t cover = bits + 1;
    double best_cost = 1e300, best_entries = 0;
    uint32_t best = 0;
    auto consider = [&](uint32_t c, uint32_t nlo, uint32_t nwin, double buckets) {
        double per_half = 0;
        for (uint32_t b = 0; b < PROFILE_BINS; b++)
            if (hist[b]) per_half += (double)hist[b] * layout_digits(b, c, nlo, nwin);
        const double entries = (double)n * halves_per_scalar * per_half / (double)std::max<uint64_t>(1, halves);
        const double cost = entries + 3.0 * buckets + 2.0e5 * (c + 6) + 4.0e4 * (double)nwin * c;
        if (cost < best_cost) {
            best_cost = cost;
            best_entries = entries;
            best = c | (nlo < nwin ? nlo << 16 : 0u);
        }
    };
    for (uint32_t W = 1; W <= cover; W++) {  // two-width layouts, as choose_layout
        const uint32_t c = cover / W, nhi = cover - W * c;
        if (c < 2) break;
        if (c + (nhi ? 1 : 0) > 22) continue;
        consider(c, W - nhi, W, (double)(W - nhi) * (double)(1u << (c - 1)) + (double)nhi * (double)(1u << c));
    }
    for (uint32_t c = 4; c <= 22; c++) {  // equal windows
        const uint32_t W = windows_for(bits, c);
        consider(c, W, W, (double)W * (double)(1u << (c - 1)));
    }
    if (expected_entries) *expected_entries = (uint64_t)best_entries;
    return best;
}

// Expected sorted entries of a sampled MSM, rounded to a power of 2^(1/8)
// (so that similar samples share one cached plan).
inline uint64_t quantize_entries(uint64_t e) {
    if (e < 16) return 16;
    const double q = std::round(std::log2((double)e) * 8.0) / 8.0;
    return (uint64_t)std::exp2(q);
}

// Window width for an MSM over a shift table with spacing s (copy k of the
// table holds 2^(s*k) * P_i): a multiple of s, at most 20.  All windows share
// one bucket set and there is no Horner chain.  Cost in units of one sorted
// entry (a mixed addition): n per window, 1.8 per bucket of the single set,
// and latency terms for the reduction depth (per window bit) and for the
// segmented-sum depth (log of the entries per bucket).  The coefficients are
// a least-squares fit of measured BN254 MSM times, n = 2^8..2^16 and
// c = 4..20 on a B200 (within 0.18 ms).
inline uint32_t choose_window_shift(uint64_t n, uint32_t bits, uint32_t s) {
    double best = 1e300;
    uint32_t bc = s;
    for (uint32_t c = s; c <= std::max<uint32_t>(s, 20); c += s) {
        const uint32_t w = windows_for(bits, c);
        const double add = (double)n * w;
        const double red = 1.8 * (double)(1u << (c - 1));
        const double per_bucket = (double)n * w / (double)(1u << (c - 1));
        const double lat = 5.5e5 * c + 3.06e5 * std::log2(per_bucket + 1.0);
        const double cost = add + red + lat;
        if (cost < best) {
            best = cost;
            bc = c;
        }
        if (c > bits) break;  // wider windows only add buckets
    }
    return bc;
}

// The same for an MSM inside a large batch over a shift table: the batch
// runs its MSMs side by side, so their fixed latencies overlap and what an
// MSM costs is its throughput -- n entries per window plus about three
// entries' worth per bucket (the reduction) -- minimised over widths that
// are multiples of s, at most 20.  Small MSMs then take wider windows than
// alone (2^12 points: 12 bits instead of 4, a third of the entries); in the
// 24-MSM batch of 2^12..2^22 points this cuts 176 M entries to 164 M.
inline uint32_t choose_window_shift_batch(uint64_t n, uint32_t bits, uint32_t s) {
    double best = 1e300;
    uint32_t bc = s;
    for (uint32_t c = s; c <= std::max<uint32_t>(s, 20); c += s) {
        const double cost = (double)n * windows_for(bits, c) + 3.0 * (double)(1u << (c - 1));
        if (cost < best) {
            best = cost;
            bc = c;
        }
        if (c > bits) break;
    }
    return bc;
}
// Batches over a shift table from this many points use the throughput rule.
constexpr uint64_t SHIFT_BATCH_MIN_POINTS = 1ull << 20;

// The precomputed window shifts of a resident base table: `copies` copies of
// its `points` points, copy k holding 2^(bits*k) * P_i (bits 0: none).
struct ShiftSpec {
    uint32_t bits = 0;
    uint32_t points = 0;
};

// Read-only view of a resident base table (capi.cu owns tables; the
// commitment server reads them through table_view).
struct TableView {
    int curve;
    uint64_t n;
    const uint32_t* points;
    const uint32_t* phi;
    ShiftSpec shifts;
};
bool table_view(void* table, TableView* out);

template <class C>
struct CurveTraits;
template <>
struct CurveTraits<Bn254> {
    static constexpr bool glv = true;  // endomorphism split available
    static constexpr int id = 0;
    static constexpr uint32_t half_bits = Bn254Glv::HALF_BITS;
    static constexpr uint32_t fr_bits = Bn254Fr::BITS;
};
template <>
struct CurveTraits<Bls381> {
    static constexpr bool glv = true;
    static constexpr int id = 1;
    static constexpr uint32_t half_bits = Bls381Glv::HALF_BITS;
    static constexpr uint32_t fr_bits = Bls381Fr::BITS;
};
template <>
struct CurveTraits<Bls377> {
    static constexpr bool glv = true;
    static constexpr int id = 2;
    static constexpr uint32_t half_bits = Bls377Glv::HALF_BITS;
    static constexpr uint32_t fr_bits = Bls377Fr::BITS;
};
template <>
struct CurveTraits<Bn254G2> {
    static constexpr bool glv = true;  // split with psi
    static constexpr int id = 3;
    static constexpr uint32_t half_bits = Bn254G2Glv::HALF_BITS;
    static constexpr uint32_t fr_bits = Bn254Fr::BITS;
};

class Engine {
   public:
    cudaStream_t stream = nullptr;
    Tuning tuning;
    int device = 0;
    uint64_t launches = 0;  // kernels launched by this engine (for reporting)
    uint64_t workspace_growths = 0;  // times ensure_workspace had to reallocate

    // Optional per-phase timing with CUDA events on the engine's stream:
    // phases 0 scalar prep + sort, 1 level-1 accumulation, 2 later
    // segmented-sum levels, 3 bucket reduction, 4 window combine.
    static constexpr int NPHASE = 5;
    bool profile = false;
    std::vector<std::vector<cudaEvent_t>> prof_pending;
    double phase_ms[NPHASE] = {0, 0, 0, 0, 0};
    uint64_t phase_calls = 0;
    // Sample the scalars of MSMs of at least 2^21 points and choose their
    // window layout from the sample (k_scalar_profile); 0 = layout from n
    // alone.  Sampling waits for the stream the call runs on.  (At 2^20
    // BN254 points it did not pay: witness-like scalars 2.93 -> 2.97 ms,
    // uniform 5.21 -> 5.30 ms for the wait; at 2^21 witness-like 4.35 ->
    // 4.04 ms, at 2^24 17.3 -> 14.6 ms.)
    int scalar_sampling = 1;
    static constexpr uint64_t SAMPLE_MIN_POINTS = 1ull << 21;
    std::vector<cudaEvent_t> prof_begin() {
        std::vector<cudaEvent_t> ev;
        if (!profile) return ev;
        ev.resize(NPHASE + 1);
        for (auto& x : ev) ZK_CUDA(cudaEventCreate(&x));
        return ev;
    }
    void prof_mark(std::vector<cudaEvent_t>& ev, int i) {
        if (!ev.empty()) ZK_CUDA(cudaEventRecord(ev[i], stream));
    }
    void prof_end(std::vector<cudaEvent_t>& ev) {
        if (!ev.empty()) prof_pending.push_back(std::move(ev));
    }
    // Wait for recorded calls and fold their phase times into phase_ms.
    void prof_collect() {
        for (auto& ev : prof_pending) {
            ZK_CUDA(cudaEventSynchronize(ev.back()));
            for (int p = 0; p < NPHASE; p++) {
                float ms = 0;
                ZK_CUDA(cudaEventElapsedTime(&ms, ev[p], ev[p + 1]));
                phase_ms[p] += ms;
            }
            for (auto& x : ev) cudaEventDestroy(x);
            phase_calls++;
        }
        prof_pending.clear();
    }

    // workspace
    DevBuf w_points, w_phi, w_scalars, w_counts, w_offsets, w_cursor, w_ents, w_buckets;
    DevBuf w_ents2, w_thist, w_stripe_buckets, w_seg;
    DevBuf w_cnt, w_pos, w_tiles, w_totals, w_pkeys[2], w_pvals[2], w_redS[2], w_redW[2];
    DevBuf w_results, w_comb, w_profile;
    uint32_t* h_profile = nullptr;  // pinned, PROFILE_BINS words
    bool comb_ready[NCURVES] = {};
    uint32_t* h_results = nullptr;  // pinned
    size_t h_results_cap = 0;

    // Workspace buffers grow on the engine stream; the device's default
    // memory pool keeps at least 4 GiB of freed blocks for reuse (a larger
    // setting, e.g. a server's reservation, is left as it is).
    void bind_workspace_stream() {
        DevBuf* bufs[] = {&w_points, &w_phi, &w_scalars, &w_counts, &w_offsets, &w_cursor, &w_ents, &w_buckets,
                          &w_ents2, &w_thist, &w_stripe_buckets, &w_seg, &w_cnt, &w_pos, &w_tiles, &w_totals,
                          &w_pkeys[0], &w_pkeys[1], &w_pvals[0], &w_pvals[1], &w_redS[0], &w_redS[1],
                          &w_redW[0], &w_redW[1], &w_results, &w_comb, &w_profile, &transient.d_descs,
                          &transient.d_tasks};
        for (DevBuf* b : bufs) b->sp = &stream;
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t keep = 4ull << 30, cur = 0;
            cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &cur);
            if (cur < keep) cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
    }

    Engine() {
        ZK_CUDA(cudaGetDevice(&device));
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0)
            tuning.sms = (uint32_t)sms;
        cudaGetLastError();
        ZK_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        bind_workspace_stream();
        tuning.acc_wave[0] = acc_resident_threads<Bn254>();
        tuning.acc_wave[1] = acc_resident_threads<Bls381>();
        tuning.acc_wave[2] = acc_resident_threads<Bls377>();
        tuning.acc_wave[3] = acc_resident_threads<Bn254G2>();
    }
    // Second stream and events for host-to-device copies that overlap the
    // compute stream (striped MSMs from host buffers).
    cudaStream_t copy_stream = nullptr;
    std::vector<cudaEvent_t> copy_events;
    // largest stripe of streamed host-buffer MSMs: 2^stripe_log2 points;
    // -1: automatic (half of n's next power of two, for n >= 2^22); 0: off
    int stripe_log2 = -1;
    void ensure_copy_resources(size_t n_events) {
        if (!copy_stream) ZK_CUDA(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
        while (copy_events.size() < n_events) {
            cudaEvent_t ev;
            ZK_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            copy_events.push_back(ev);
        }
    }
    // pageable host-to-device copies of the streamed host calls
    std::unique_ptr<HostStager> stager;
    // dst <- src on stream s: through the stager when src is pageable and
    // large, else one cudaMemcpyAsync
    void copy_h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
        if (bytes >= (8u << 20) && HostStager::pageable(src)) {
            if (!stager) stager.reset(new HostStager());
            ZK_CUDA(stager->copy(dst, src, bytes, s));
            return;
        }
        if (bytes) ZK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    }

    ~Engine() {
        stager.reset();
        drop_graphs();
        for (auto ev : copy_events) cudaEventDestroy(ev);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        if (stream) cudaStreamDestroy(stream);
        if (h_results) cudaFreeHost(h_results);
        if (h_profile) cudaFreeHost(h_profile);
    }

    // ------------------------------------------------------------ planning
    template <class C>
    void make_plan(Plan& pl, const std::vector<uint32_t>& counts, const std::vector<uint32_t>& base_offs,
                   int fmt, uint32_t scalar_bits, uint32_t window_override = 0, ShiftSpec sh = {},
                   uint64_t entries_hint = 0) const {
        plan_shape<C>(pl, tuning, counts, base_offs, fmt, scalar_bits, window_override, sh, entries_hint);
    }

    // Pure host planning (no device needed): window widths, bucket layout,
    // chunking of the segmented sums and the reduction tree.
    template <class C>
    // window_override > 0 fixes every MSM's window width (the stripes of one
    // striped MSM share one bucket layout).  `sh`: the bases are a shift
    // table; an MSM whose points lie in it uses the precomputed shifts (no
    // GLV, window width a multiple of sh.bits, one bucket set).
    // entries_hint: the expected number of sorted entries (from a scalar
    // sample; 0: unknown, every digit counted as nonzero): sizes the level-1
    // chunks for the entries there will be rather than for the bound.
    static void plan_shape(Plan& pl, const Tuning& tuning, const std::vector<uint32_t>& counts,
                           const std::vector<uint32_t>& base_offs, int fmt, uint32_t scalar_bits,
                           uint32_t window_override = 0, ShiftSpec sh = {}, uint64_t entries_hint = 0) {
        pl.curve = CurveTraits<C>::id;
        uint64_t soff = 0;
        uint32_t boff = 0, woff = 0;
        uint64_t batch_points = 0;
        for (auto c : counts) batch_points += c;
        const bool throughput_windows = counts.size() > 1 && batch_points >= SHIFT_BATCH_MIN_POINTS;
        for (size_t m = 0; m < counts.size(); m++) {
            MsmDesc d{};
            d.scalar_off = soff;
            d.n = counts[m];
            d.base_off = base_offs[m];
            d.fmt = fmt;
            bool small = scalar_bits > 0 && scalar_bits <= 64;
            if (sh.bits && d.n && (uint64_t)d.base_off + d.n <= sh.points) {
                const uint32_t bits = small ? scalar_bits : CurveTraits<C>::fr_bits;
                uint32_t c = window_override ? window_override & 0xffffu
                                             : tuning.window_bits > 0 ? (uint32_t)tuning.window_bits & 0xffffu
                                                                      : choose_window_shift(d.n, bits, sh.bits);
                if (!window_override && tuning.window_bits <= 0 && throughput_windows)
                    c = std::max(c, choose_window_shift_batch(d.n, bits, sh.bits));
                c = std::max<uint32_t>(1, (c + sh.bits - 1) / sh.bits) * sh.bits;
                d.glv = 0;
                d.c = c;
                d.nwin = windows_for(bits, c);
                d.nlo = d.nwin;
                d.wstep = (c / sh.bits) * sh.points;
                d.nred = 1;
                d.bucket_off = boff;
                d.win_off = woff;
                boff += 1u << (c - 1);
                woff += 1;
                pl.entry_bound += (uint64_t)d.n * d.nwin;
                soff += d.n;
                pl.descs.push_back(d);
                continue;
            }
            d.glv = (small || !CurveTraits<C>::glv) ? 0 : (tuning.glv == 0 ? 0 : 1);
            uint32_t bits = small ? scalar_bits : (d.glv ? CurveTraits<C>::half_bits : CurveTraits<C>::fr_bits);
            uint64_t epw = (uint64_t)d.n * (d.glv ? 2 : 1);
            // a window setting of 2^16 or more is a layout: c | nlo << 16
            const uint32_t tw = tuning.window_bits > 0 ? (uint32_t)tuning.window_bits : 0u;
            const uint32_t ov = window_override ? window_override : tw >> 16 ? tw : 0u;
            uint32_t c = tw ? tw & 0xffffu : choose_window(epw, bits);
            uint32_t nlo = 0;  // 0: every window c bits
            if (ov) {
                c = ov & 0xffffu;
                nlo = ov >> 16;
            } else if (tw == 0 && d.n) {
                auto it = small ? tuning.window_table.end()
                                : tuning.window_table.find({CurveTraits<C>::id * 2 + (int)d.glv, nearest_log2(d.n)});
                if (it != tuning.window_table.end() && it->second > 0) {
                    c = (uint32_t)it->second;
                } else if (epw >= LAYOUT_MIN_ENTRIES) {
                    const WinLayout lay = choose_layout(epw, bits);
                    c = lay.c;
                    nlo = lay.nlo < lay.nwin ? lay.nlo : 0;
                }
            }
            if (c > bits + 1) c = bits + 1 < 2 ? 2 : bits + 1;
            if (c < 2) c = 2;
            d.c = c;
            if (nlo && nlo * c < bits + 1) {
                // nlo windows of c bits, then c + 1-bit windows up to bits + 1
                d.nwin = d.n ? nlo + (bits + 1 - nlo * c + c) / (c + 1) : 0;
                d.nlo = std::min(nlo, d.nwin);
            } else {
                d.nwin = d.n ? windows_for(bits, c) : 0;
                d.nlo = d.nwin;
            }
            if (d.nwin > MAX_WINDOWS) {  // too narrow for the combine: widen
                while (windows_for(bits, c) > MAX_WINDOWS) c++;
                d.c = c;
                d.nwin = d.nlo = windows_for(bits, c);
            }
            d.wstep = 0;
            d.nred = d.nwin;
            d.bucket_off = boff;
            d.win_off = woff;
            boff += win_bucket(d, d.nwin);
            woff += d.nwin;
            pl.entry_bound += epw * d.nwin;
            soff += d.n;
            pl.descs.push_back(d);
        }
        pl.total_scalars = soff;
        pl.nbuckets = boff;
        pl.nwin_total = woff;
        {
            uint32_t maxd = 1;
            for (auto& d : pl.descs) maxd = std::max(maxd, (d.glv ? 2u : 1u) * d.nwin);
            // scalars per digit block: each warp owns a buffer slice of
            // SORT_DBUF / 8 entries; rounds of 256 scalars while a lane's
            // digits of all rounds fit its share of the slice, else fewer
            // lanes per warp (k_radix_digits)
            const uint32_t wslice = SORT_DBUF / (SORT_DTHREADS / 32);
            const uint32_t spb = maxd * 32 <= wslice ? SORT_DTHREADS * (wslice / (32 * maxd))
                                                     : (SORT_DTHREADS / 32) * std::max<uint32_t>(1, wslice / maxd);
            uint32_t kb = 0;
            while (kb < 32 && (1ull << kb) < (uint64_t)boff) kb++;
            uint32_t passes = (kb + 7) / 8;
            pl.sort_maxd = maxd;
            pl.sort_spb = std::max<uint32_t>(spb, 1);
            pl.sort_passes = passes;
            pl.sort_bits = passes ? (kb + passes - 1) / passes : 0;
            pl.sort_tiles = (uint32_t)std::max<uint64_t>((pl.entry_bound + SORT_ETILE - 1) / SORT_ETILE, 1);
            // large entry sets: MSD passes of up to 12 bits (two cover bucket
            // ids of up to 24 bits), the first pass over the top bits.  An odd
            // width gives the first pass the narrower digit: its scatter writes
            // runs all over the output, where fewer, longer runs pay (BN254
            // 2^24: 11 + 12 bits, prep+sort 4.25 ms, against 4.35 with 12 + 11),
            // while the second writes inside one segment
            if (pl.entry_bound >= MSD_MIN_ENTRIES && kb >= 1 && kb <= 2 * MSD_MAX_BITS) {
                pl.msd_passes = kb <= MSD_MAX_BITS ? 1 : 2;
                pl.msd_bits1 = pl.msd_passes == 1 ? kb : kb / 2;
                pl.msd_bits2 = kb - (pl.msd_passes == 1 ? kb : pl.msd_bits1);
                pl.msd_tiles1 = (uint32_t)((pl.entry_bound + MSD_TILE - 1) / MSD_TILE);
                pl.msd_tiles2 = pl.msd_passes == 2 ? pl.msd_tiles1 + (1u << pl.msd_bits1) : 0;
                pl.msd_groups1 = std::max<uint32_t>(1, std::min<uint32_t>(tuning.sms, pl.msd_tiles1));
                // sum over segments of ceil(tiles / chunk) <= tiles / chunk + segments
                pl.msd_chunks2 = pl.msd_passes == 2
                                         ? (pl.msd_tiles2 + MSD_CHUNK_TILES - 1) / MSD_CHUNK_TILES + (1u << pl.msd_bits1)
                                         : 0;
            }
        }
        // autotuned schedule of the plan's largest MSM, if any
        Tuning::Schedule sc;
        {
            const MsmDesc* big = nullptr;
            for (auto& d : pl.descs)
                if (!big || d.n > big->n) big = &d;
            if (big && big->n && !big->wstep) {
                auto it = tuning.sched_table.find({CurveTraits<C>::id * 2 + (int)big->glv, nearest_log2(big->n)});
                if (it != tuning.sched_table.end()) sc = it->second;
            }
        }
        pl.acc_threads = sc.acc_threads > 0 ? (uint32_t)sc.acc_threads : 0;
        if (sc.red_L == 4 || sc.red_L == 8 || sc.red_L == 16) {
            pl.red_L = (uint32_t)sc.red_L;
            pl.red_log2L = sc.red_L == 4 ? 2 : sc.red_L == 8 ? 3 : 4;
        }
        // segmented-sum levels
        uint64_t M = pl.entry_bound;
        uint32_t K1 = tuning.chunk > 0 ? (uint32_t)tuning.chunk : 0;
        if (!K1) {
            // long enough to hold about two average buckets and at least 192
            // entries (so few buckets are cut and the partial-sum levels stay
            // small: at 2^24 with ~24 entries per bucket, chunks of 192 beat
            // chunks of 48 by 0.9 ms), short enough to give at least 8 waves
            // of resident threads
            // (a hint within 10% of the bound is the bound: dense scalar sets
            // keep the plan they get without a sample)
            const uint64_t Me = entries_hint && entries_hint < M - M / 10 ? entries_hint : M;
            uint64_t waves8 = Me / (8ull * 148 * 512);
            uint64_t avg = pl.nbuckets ? Me / pl.nbuckets : 1;
            uint64_t k = std::min<uint64_t>(std::max<uint64_t>(8, waves8), std::max<uint64_t>(192, 2 * avg));
            K1 = (uint32_t)std::min<uint64_t>(k, 512);
            // then round the thread count to a whole number of waves of
            // resident threads: a last, nearly empty wave would run on an
            // almost idle device for a full chunk time
            const uint64_t W = tuning.acc_wave[CurveTraits<C>::id];
            if (W) {
                const double waves = (double)Me / ((double)K1 * (double)W);
                const uint64_t w = (uint64_t)(waves + 0.5);
                if (waves >= 1.0 && w >= 1) K1 = (uint32_t)std::max<uint64_t>(8, (Me + w * W - 1) / (w * W));
            }
            if (sc.chunk_pct > 0)
                K1 = (uint32_t)std::min<uint64_t>(4096, std::max<uint64_t>(8, (uint64_t)K1 * sc.chunk_pct / 100));
        }
        uint32_t K = K1;
        for (int lvl = 0; lvl < 40; lvl++) {
            uint64_t T = (M + K - 1) / K;
            if (T == 0) T = 1;
            pl.acc_K.push_back(K);
            pl.acc_T.push_back((uint32_t)T);
            pl.acc_Mbound.push_back(M);
            if (T <= 1) break;
            M = 2 * T;
            K = 16;
        }
        // reduction levels
        std::vector<RedTask> lvl0;
        uint32_t off = 0;
        for (auto& d : pl.descs) {
            for (uint32_t w = 0; w < d.nred; w++) {
                const uint32_t B = 1u << (win_width(d, w) - 1);
                RedTask t;
                t.in_off = d.bucket_off + win_bucket(d, w);
                t.n_in = B;
                t.out_off = off;
                t.n_out = (B + pl.red_L - 1) / pl.red_L;
                off += t.n_out;
                lvl0.push_back(t);
            }
        }
        pl.red_tasks.push_back(lvl0);
        pl.red_nout.push_back(off);
        while (true) {
            auto& prev = pl.red_tasks.back();
            bool done = true;
            for (auto& t : prev)
                if (t.n_out > 1) done = false;
            if (done) break;
            std::vector<RedTask> nx;
            uint32_t o = 0;
            for (auto& t : prev) {
                RedTask u;
                u.in_off = t.out_off;
                u.n_in = t.n_out;
                u.out_off = o;
                u.n_out = (u.n_in + pl.red_L - 1) / pl.red_L;
                o += u.n_out;
                nx.push_back(u);
            }
            pl.red_tasks.push_back(nx);
            pl.red_nout.push_back(o);
        }
    }

    // Plans are cached by shape, with their tables uploaded once, so that
    // repeated calls of the same shape issue no host-to-device copies.
    std::map<std::string, std::unique_ptr<Plan>> plan_cache;

    template <class C>
    Plan& get_plan(const std::vector<uint32_t>& counts, const std::vector<uint32_t>& base_offs, int fmt,
                   uint32_t scalar_bits = 0, uint32_t window_override = 0, ShiftSpec sh = {},
                   uint64_t entries_hint = 0) {
        std::string key;
        auto put = [&](uint64_t v) { key.append(reinterpret_cast<const char*>(&v), sizeof v); };
        put(CurveTraits<C>::id);
        put(fmt);
        put(scalar_bits);
        put(window_override);
        put(entries_hint);
        put((uint64_t)sh.bits << 32 | sh.points);
        put((uint64_t)(uint32_t)tuning.window_bits << 32 | (uint32_t)tuning.chunk);
        put((uint64_t)(int64_t)tuning.glv);
        put(tuning.version);
        for (auto c : counts) put(c);
        for (auto b : base_offs) put(b);
        auto it = plan_cache.find(key);
        if (it != plan_cache.end()) return *it->second;
        if (plan_cache.size() >= 256) {  // cudaFree in ~DevBuf waits for the device
            drop_graphs();                 // graphs are keyed by plan address
            plan_cache.clear();
        }
        std::unique_ptr<Plan> pl(new Plan());
        make_plan<C>(*pl, counts, base_offs, fmt, scalar_bits, window_override, sh, entries_hint);
        upload_plan(*pl, false);
        Plan& ref = *pl;
        plan_cache.emplace(key, std::move(pl));
        return ref;
    }

    // Device tables of a plan (MSM descriptors, reduction tasks); `async`
    // copies on the engine stream (the host vectors are pageable, so the
    // copy has left them when the call returns).
    void upload_plan(Plan& pl, bool async) {
        std::vector<RedTask> blob;
        pl.task_level_off.clear();
        for (auto& v : pl.red_tasks) {
            pl.task_level_off.push_back(blob.size());
            blob.insert(blob.end(), v.begin(), v.end());
        }
        pl.d_tasks.ensure((blob.size() + 1) * sizeof(RedTask));
        pl.d_descs.ensure((pl.descs.size() + 1) * sizeof(MsmDesc));
        if (async) {
            ZK_CUDA(cudaMemcpyAsync(pl.d_tasks.p, blob.data(), blob.size() * sizeof(RedTask), cudaMemcpyHostToDevice,
                                    stream));
            ZK_CUDA(cudaMemcpyAsync(pl.d_descs.p, pl.descs.data(), pl.descs.size() * sizeof(MsmDesc),
                                    cudaMemcpyHostToDevice, stream));
        } else {
            ZK_CUDA(cudaMemcpy(pl.d_tasks.p, blob.data(), blob.size() * sizeof(RedTask), cudaMemcpyHostToDevice));
            ZK_CUDA(cudaMemcpy(pl.d_descs.p, pl.descs.data(), pl.descs.size() * sizeof(MsmDesc),
                               cudaMemcpyHostToDevice));
        }
    }

    // An uncached plan for shapes that rarely repeat (served batches): built
    // again in place on every call, its device tables only grow, so steady
    // state serving neither allocates nor frees.  Valid until the next call.
    Plan transient;
    template <class C>
    Plan& transient_plan(const std::vector<uint32_t>& counts, const std::vector<uint32_t>& base_offs, int fmt,
                         ShiftSpec sh = {}) {
        transient.clear_host();
        make_plan<C>(transient, counts, base_offs, fmt, 0, 0, sh);
        upload_plan(transient, true);
        return transient;
    }

    template <class C>
    void ensure_workspace(const Plan& pl) {
        using P = typename C::Fp;
        const size_t xs = sizeof(Xyzz<P>);
        bool grew = false;
        grew |= w_counts.ensure(((size_t)pl.nbuckets + 1) * 4);
        grew |= w_cursor.ensure(((size_t)pl.nbuckets + 1) * 4);
        grew |= w_ents.ensure(pl.entry_bound * 8 + 16);
        uint64_t hsz = (uint64_t)(1u << pl.sort_bits) * pl.sort_tiles;
        if (pl.msd_passes) {
            // count and slot rows of every tile, then the scan layout of the groups
            hsz = 2 * msd_rows_words(pl) + msd_scan_words(pl);
            grew |= w_seg.ensure(((size_t)3 << pl.msd_bits1) * 4 + 64);
        }
        const uint64_t hwords = hsz;
        grew |= w_ents2.ensure(pl.entry_bound * 8 + 16);
        grew |= w_thist.ensure(hwords * 4 + 16);
        grew |= w_buckets.ensure((size_t)pl.nbuckets * xs + xs);
        uint64_t tmax = 1, m2 = 1, m3 = 1;
        for (size_t l = 0; l < pl.acc_T.size(); l++) tmax = std::max<uint64_t>(tmax, pl.acc_T[l]);
        if (pl.acc_Mbound.size() > 1) m2 = pl.acc_Mbound[1];
        for (size_t l = 2; l < pl.acc_Mbound.size(); l++) m3 = std::max<uint64_t>(m3, pl.acc_Mbound[l]);
        grew |= w_cnt.ensure(tmax * 4 + 16);
        grew |= w_pkeys[0].ensure(m2 * 4 + 16);
        grew |= w_pvals[0].ensure(m2 * xs + xs);
        grew |= w_pkeys[1].ensure(m3 * 4 + 16);
        grew |= w_pvals[1].ensure(m3 * xs + xs);
        if (w_totals.ensure(64 * 4)) {  // new memory holds anything: start the counters at zero
            grew = true;
            ZK_CUDA(cudaMemsetAsync(w_totals.p, 0, 64 * 4, stream));
        }
        size_t r0 = pl.red_nout.empty() ? 1 : pl.red_nout[0];
        for (int i = 0; i < 2; i++) {
            grew |= w_redS[i].ensure(r0 * xs + xs);
            grew |= w_redW[i].ensure(r0 * xs + xs);
        }
        grew |= w_results.ensure((pl.descs.size() + 1) * 3 * P::N * 4);
        // scan tile sums for the longest scanned array (no allocation inside enqueue)
        grew |= w_tiles.ensure(((std::max<uint64_t>(std::max<uint64_t>(pl.nbuckets, tmax), hsz) + 2047) / 2048 + 2) *
                               4);
        if (grew) {
            drop_graphs();  // captured graphs hold the old addresses
            workspace_growths++;
        }
    }

    // ------------------------------------------------------------ graphs
    // A batch shape that repeats is captured once into a CUDA graph and then
    // replayed with one launch.  Graphs are keyed by plan and buffer
    // addresses and dropped whenever the workspace is reallocated.
    struct GraphEntry {
        cudaGraphExec_t exec = nullptr;
        uint64_t kernels = 0;
    };
    std::map<std::string, GraphEntry> graphs;
    void drop_graphs() {
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second.exec);
        graphs.clear();
    }

    // Curve-specific device work: defined in engine_impl.cuh and instantiated
    // once per curve (inst_bn254.cu, inst_bls381.cu, inst_bls377.cu, inst_bn254g2.cu).
    // flags: ENQ_ACC_ONLY stops after the bucket sums (no window sums, no
    // result).  bucket_base (default: the engine's bucket array) receives the
    // bucket sums.
    static constexpr int ENQ_ACC_ONLY = 1;
    // Bases still being copied on another stream when the pipeline is
    // enqueued: the scalar preparation and sort (which read only scalars)
    // run first, then the engine stream waits for `ready` and, when phi_out
    // is set, writes the endomorphism image of the phi_n bases there.
    struct BasesWait {
        cudaEvent_t ready = nullptr;
        uint64_t phi_n = 0;
        uint32_t* phi_out = nullptr;
    };
    template <class C>
    void enqueue(const Plan& pl, const uint32_t* d_bases, const uint32_t* d_phi, const uint32_t* d_scalars,
                 uint32_t* d_results, int flags = 0, void* bucket_base = nullptr, const BasesWait* bw = nullptr);
    template <class C>
    void enqueue_reduce(const Plan& pl, const void* bucket_base, uint32_t* d_results,
                        std::vector<cudaEvent_t>* ev = nullptr);
    // MSD sort of the entries (k_msd_*), defined in engine_impl.cuh
    template <class C>
    void msd_sort(const Plan& pl, uint2* A, uint2* B, uint32_t* tot);
    template <class C>
    void fold_buckets(void* base, uint32_t nb, uint32_t S);
    template <class C>
    void make_phi(const uint32_t* d_bases, uint64_t n, uint32_t* d_phi);
    // Window shifts of a table of n affine points (copy 0, at d_table):
    // copies 1..copies-1, copy k = 2^(s*k) * P_i at d_table + k*n points.
    // Synchronous (returns when the table is written).
    template <class C>
    void make_shifts(uint32_t* d_table, uint64_t n, uint32_t s, uint32_t copies);
    // resident threads of k_acc_l1<C> on this device (occupancy API)
    template <class C>
    uint32_t acc_resident_threads();
    template <class C>
    void gen_bases(uint64_t seed, uint64_t index0, uint64_t n, uint32_t* d_out);
    // Histogram of the prepared half lengths of PROFILE_SAMPLES scalars of
    // d_scalars (k_scalar_profile) into h_profile; waits for the stream.
    template <class C>
    void profile_scalars(const uint32_t* d_scalars, uint64_t n, int fmt, bool glv);
    // The window override (c | nlo << 16) and the expected entry count for a
    // single n-point MSM of device scalars, chosen from a sample of them; {0,
    // 0} (layout from n alone) unless sampling is on, n >= SAMPLE_MIN_POINTS,
    // the curve splits with GLV, no window width is forced or autotuned for
    // n, and the stream is not being captured into a graph.
    struct SampledLayout {
        uint32_t window = 0;
        uint64_t entries = 0;
    };
    template <class C>
    SampledLayout sampled_layout(const uint32_t* d_scalars, uint64_t n, int fmt) {
        SampledLayout out;
        if (!scalar_sampling || n < SAMPLE_MIN_POINTS || !CurveTraits<C>::glv || tuning.glv == 0 ||
            tuning.window_bits != 0)
            return out;
        if (tuning.window_table.count({CurveTraits<C>::id * 2 + 1, nearest_log2(n)})) return out;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
            cudaGetLastError();
            return out;
        }
        profile_scalars<C>(d_scalars, n, fmt, true);
        uint64_t halves = 0;
        for (uint32_t b = 0; b < PROFILE_BINS; b++) halves += h_profile[b];
        uint64_t e = 0;
        out.window = choose_layout_sampled(h_profile, halves, n, CurveTraits<C>::half_bits, 2, &e);
        out.entries = quantize_entries(e);
        return out;
    }
    template <class C>
    void gen_scalars(uint64_t seed, uint64_t index0, uint64_t n, int dist, int fmt, uint32_t* d_out);

    // Same as run_device, through a cached CUDA graph of the whole pipeline.
    template <class C>
    void run_device_graph(const Plan& pl, const uint32_t* d_bases, const uint32_t* d_phi,
                          const uint32_t* d_scalars, uint8_t* out) {
        using P = typename C::Fp;
        ensure_workspace<C>(pl);
        std::string key;
        auto put = [&](const void* v) { key.append(reinterpret_cast<const char*>(&v), sizeof v); };
        put(&pl);
        put(d_bases);
        put(d_phi);
        put(d_scalars);
        put(stream);
        auto it = graphs.find(key);
        if (it == graphs.end()) {
            // the first call of a plan runs its launches directly: capturing
            // and instantiating costs about as much as the launches it saves
            // (~1 ms for a small MSM), which only a repeated shape pays back
            if (pl.graph_misses++ == 0) {
                run_device<C>(pl, d_bases, d_phi, d_scalars, out);
                return;
            }
            if (graphs.size() >= 64) drop_graphs();
            bool prof = profile;
            profile = false;
            uint64_t l0 = launches;
            cudaGraph_t g = nullptr;
            ZK_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            try {
                enqueue<C>(pl, d_bases, d_phi, d_scalars, w_results.as<uint32_t>());
            } catch (...) {
                cudaStreamEndCapture(stream, &g);
                if (g) cudaGraphDestroy(g);
                profile = prof;
                throw;
            }
            ZK_CUDA(cudaStreamEndCapture(stream, &g));
            profile = prof;
            GraphEntry ge;
            ge.kernels = launches - l0;
            launches = l0;
            cudaError_t ie = cudaGraphInstantiate(&ge.exec, g, 0);
            cudaGraphDestroy(g);
            ZK_CUDA(ie);
            it = graphs.emplace(key, ge).first;
        }
        ZK_CUDA(cudaGraphLaunch(it->second.exec, stream));
        launches += it->second.kernels;
        size_t bytes = pl.descs.size() * 3 * P::N * 4;
        ZK_CUDA(cudaMemcpyAsync(out, w_results.p, bytes, cudaMemcpyDeviceToHost, stream));
        ZK_CUDA(cudaStreamSynchronize(stream));
    }

    // Full MSM batch from device inputs: results copied to host `out`
    // (n_msms x 3 x fp_bytes).
    template <class C>
    void run_device(const Plan& pl, const uint32_t* d_bases, const uint32_t* d_phi, const uint32_t* d_scalars,
                    uint8_t* out) {
        using P = typename C::Fp;
        ensure_workspace<C>(pl);
        enqueue<C>(pl, d_bases, d_phi, d_scalars, w_results.as<uint32_t>());
        size_t bytes = pl.descs.size() * 3 * P::N * 4;
        ZK_CUDA(cudaMemcpyAsync(out, w_results.p, bytes, cudaMemcpyDeviceToHost, stream));
        ZK_CUDA(cudaStreamSynchronize(stream));
    }

};

// Curve-specific device code is instantiated in its own translation unit
// (inst_bn254.cu, inst_bls381.cu, inst_bls377.cu, inst_bn254g2.cu) so the curves compile in parallel.
#define ZKMSM_ENGINE_TEMPLATES(EXT, C)                                                                  \
    EXT template void Engine::enqueue<C>(const Plan&, const uint32_t*, const uint32_t*, const uint32_t*, \
                                         uint32_t*, int, void*, const BasesWait*);                      \
    EXT template void Engine::enqueue_reduce<C>(const Plan&, const void*, uint32_t*,                     \
                                                std::vector<cudaEvent_t>*);                             \
    EXT template void Engine::fold_buckets<C>(void*, uint32_t, uint32_t);                               \
    EXT template void Engine::msd_sort<C>(const Plan&, uint2*, uint2*, uint32_t*);                     \
    EXT template void Engine::make_phi<C>(const uint32_t*, uint64_t, uint32_t*);                        \
    EXT template void Engine::make_shifts<C>(uint32_t*, uint64_t, uint32_t, uint32_t);                  \
    EXT template uint32_t Engine::acc_resident_threads<C>();                                              \
    EXT template void Engine::gen_bases<C>(uint64_t, uint64_t, uint64_t, uint32_t*);                    \
    EXT template void Engine::profile_scalars<C>(const uint32_t*, uint64_t, int, bool);                 \
    EXT template void Engine::gen_scalars<C>(uint64_t, uint64_t, uint64_t, int, int, uint32_t*);

}  // namespace zkmsm
