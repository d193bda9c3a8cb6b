// Device-side halves of the Engine: kernel launch sequences.  Included only
// by the per-curve instantiation units so each curve's kernels compile once.
#pragma once
#include "engine.cuh"
#include "msm_kernels.cuh"

#include <mutex>
#include <stdexcept>
#include <utility>

namespace zkmsm {

// Exclusive scan of n u32 in place; total to d_total; optional copy.
static void scan_u32(Engine& e, uint32_t* d_in_out, uint32_t n, uint32_t* d_total, uint32_t* d_copy) {
    uint32_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (tiles <= 1) {
        k_scan_single<<<1, SCAN_THREADS, 0, e.stream>>>(d_in_out, n, d_total, d_copy);
        e.launches++;
        ZK_CUDA(cudaGetLastError());
        return;
    }
    k_scan_tiles<<<tiles, SCAN_THREADS, 0, e.stream>>>(d_in_out, n, d_in_out, e.w_tiles.as<uint32_t>());
    e.launches++;
    k_scan_sums<<<1, SCAN_THREADS, 0, e.stream>>>(e.w_tiles.as<uint32_t>(), tiles, d_total);
    e.launches++;
    k_scan_add<<<tiles, SCAN_THREADS, 0, e.stream>>>(d_in_out, n, e.w_tiles.as<uint32_t>(), d_copy);
    e.launches++;
    ZK_CUDA(cudaGetLastError());
}


// MSD sort of the entries in A by bucket id (tot[0] entries): one or two
// passes, each k_msd_count, an exclusive scan of the group totals,
// k_msd_prefix and k_msd_scatter; after two passes the result is back in A,
// after one in B.
static void msd_scatter_attr(int device) {
    // the staged tile needs more than the default 48 KB of dynamic shared
    // memory; set once per device for this unit's copy of the kernel
    static std::mutex mu;
    static bool done[64] = {};
    std::lock_guard<std::mutex> lk(mu);
    if (device < 0 || device >= 64 || done[device]) return;
    ZK_CUDA(cudaFuncSetAttribute(k_msd_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MSD_SCATTER_SMEM));
    done[device] = true;
}

template <class C>
void Engine::msd_sort(const Plan& pl, uint2* A, uint2* B, uint32_t* tot) {
    msd_scatter_attr(device);
    const uint32_t b1 = pl.msd_bits1, b2 = pl.msd_bits2, G = pl.msd_groups1, CH = pl.msd_chunks2;
    // count rows (C) and slot rows (P) of every tile, then the scan layout
    // of the groups (S)
    uint32_t* Cr = w_thist.as<uint32_t>();
    uint32_t* P = Cr + msd_rows_words(pl);
    uint32_t* S = P + msd_rows_words(pl);
    const uint32_t nseg = 1u << b1;
    uint32_t* seg_start = w_seg.as<uint32_t>();
    uint32_t* seg_tile = seg_start + nseg + 1;
    uint32_t* seg_chunk = seg_tile + nseg + 1;
    // pass 1: G groups of MSD_COUNT_PARTS count parts over the tile bound;
    // pass 2: the chunk and tile bounds (blocks past the real chunks and
    // tiles return at once)
    // pass 1 counts the digit array the digit kernel wrote at the front of
    // B (the pass-1 scatter overwrites it only after the count), pass 2 the
    // entries' keys
    auto pass = [&](const uint2* src, uint2* dst, uint32_t shift, uint32_t bits, uint32_t ng, uint32_t sub,
                    uint32_t ntiles, const uint32_t* ss, const uint32_t* st, const uint32_t* sc, uint32_t ns,
                    const uint16_t* D) {
        const uint32_t nb = 1u << bits;
        k_msd_count<<<ng * sub, MSD_THREADS, 0, stream>>>(D, src, shift, tot + 0, bits, ng, sub, ss, st, sc, ns, Cr,
                                                          S);
        launches++;
        ZK_CUDA(cudaGetLastError());
        // pass-2 totals fill a prefix of S (chunks in segment order); the
        // scan runs over the bound, and whatever lies past the prefix only
        // shifts slots past it
        scan_u32(*this, S, (uint64_t)nb * ng * sub, tot + 63, nullptr);
        k_msd_prefix<<<ng, MSD_THREADS, 0, stream>>>(tot + 0, bits, ng, sub, ss, st, sc, ns, Cr, S, P);
        k_msd_scatter<<<ntiles, MSD_THREADS, MSD_SCATTER_SMEM, stream>>>(src, tot + 0, shift, bits, ntiles, ss, st,
                                                                        ns, Cr, P, dst);
        launches += 2;
        ZK_CUDA(cudaGetLastError());
    };
    const bool two = pl.msd_passes == 2;
    pass(A, B, two ? b2 : 0, b1, G, MSD_COUNT_PARTS, pl.msd_tiles1, nullptr, nullptr, nullptr, 0,
         reinterpret_cast<const uint16_t*>(B));
    if (!two) return;
    k_msd_tiles<<<1, MSD_THREADS, 0, stream>>>(S, G * MSD_COUNT_PARTS, nseg, tot + 0, seg_start, seg_tile, seg_chunk);
    launches++;
    ZK_CUDA(cudaGetLastError());
    pass(B, A, 0, b2, CH, 1, pl.msd_tiles2, seg_start, seg_tile, seg_chunk, nseg, nullptr);
}

// ------------------------------------------------------------ pipeline
// Enqueue the whole batch; results (n_msms x 3 field elements) land in
// d_results.  No host synchronisation inside (graph capturable).
template <class C>
void Engine::enqueue(const Plan& pl, const uint32_t* d_bases, const uint32_t* d_phi, const uint32_t* d_scalars,
             uint32_t* d_results, int flags, void* bucket_base, const BasesWait* bw) {
    using P = typename C::Fp;
    const int nd = (int)pl.descs.size();
    const MsmDesc* dd = pl.d_descs.as<MsmDesc>();
    uint32_t* tot = w_totals.as<uint32_t>();
    auto ev = prof_begin();
    prof_mark(ev, 0);
    Xyzz<P>* buckets = bucket_base ? static_cast<Xyzz<P>*>(bucket_base) : w_buckets.as<Xyzz<P>>();
    ZK_CUDA(cudaMemsetAsync(buckets, 0, (size_t)pl.nbuckets * sizeof(Xyzz<P>), stream));
    // radix sort of the entries by bucket id; tot[0] = number of entries.
    // The digit pass writes to whichever buffer makes the last pass land in
    // w_ents; slot 63 of w_totals takes the (unused) totals of the scans.
    ZK_CUDA(cudaMemsetAsync(tot, 0, 4, stream));
    const uint32_t npass = pl.msd_passes ? pl.msd_passes : pl.sort_passes;
    uint2* bufA = (npass & 1) ? w_ents2.as<uint2>() : w_ents.as<uint2>();
    uint2* bufB = (npass & 1) ? w_ents.as<uint2>() : w_ents2.as<uint2>();
    // the first LSD pass's tile histogram is counted by the digit kernel
    const bool hist0 = pl.sort_passes && !pl.msd_passes;
    if (hist0) ZK_CUDA(cudaMemsetAsync(w_thist.p, 0, (size_t)(1u << pl.sort_bits) * pl.sort_tiles * 4, stream));
    if (pl.total_scalars) {
        const uint64_t g = (pl.total_scalars + pl.sort_spb - 1) / pl.sort_spb;
        // five-limb halves when every MSM splits with GLV
        bool all_glv = true;
        for (const auto& d : pl.descs) all_glv = all_glv && d.glv;
        // MSD sorts: the first pass's digit of each entry, 2 bytes, at the
        // front of the other entry buffer (free until the pass-1 scatter)
        uint16_t* D = pl.msd_passes ? reinterpret_cast<uint16_t*>(bufB) : nullptr;
        const uint32_t dshift = pl.msd_passes == 2 ? pl.msd_bits2 : 0u;
        const uint32_t dmask = pl.msd_passes ? (1u << pl.msd_bits1) - 1 : 0u;
        if (all_glv)
            k_radix_digits<C, 5><<<(unsigned)g, SORT_DTHREADS, 0, stream>>>(
                    d_scalars, dd, nd, pl.total_scalars, pl.sort_spb, bufA, tot + 0,
                    hist0 ? w_thist.as<uint32_t>() : nullptr, pl.sort_bits, pl.sort_tiles, D, dshift, dmask);
        else
            k_radix_digits<C, 9><<<(unsigned)g, SORT_DTHREADS, 0, stream>>>(
                    d_scalars, dd, nd, pl.total_scalars, pl.sort_spb, bufA, tot + 0,
                    hist0 ? w_thist.as<uint32_t>() : nullptr, pl.sort_bits, pl.sort_tiles, D, dshift, dmask);
        launches++;
        ZK_CUDA(cudaGetLastError());
    }
    if (pl.msd_passes) {
        msd_sort<C>(pl, bufA, bufB, tot);
        bufA = bufB = nullptr;
    }
    for (uint32_t ps = 0; ps < (pl.msd_passes ? 0u : pl.sort_passes); ps++) {
        const uint32_t shift = ps * pl.sort_bits, nt = pl.sort_tiles;
        if (ps > 0) {
            k_radix_hist<<<nt, SORT_ETHREADS, 0, stream>>>(bufA, tot + 0, shift, pl.sort_bits, nt,
                                                            w_thist.as<uint32_t>());
            launches++;
            ZK_CUDA(cudaGetLastError());
        }
        scan_u32(*this, w_thist.as<uint32_t>(), (1u << pl.sort_bits) * nt, tot + 63, nullptr);
        switch (pl.sort_bits) {
#define ZK_SCATTER(B)                                                                                     \
    case B:                                                                                              \
        k_radix_scatter<B><<<nt, SORT_ETHREADS, 0, stream>>>(bufA, tot + 0, shift, nt, w_thist.as<uint32_t>(), \
                                                             bufB);                                      \
        break;
            ZK_SCATTER(1) ZK_SCATTER(2) ZK_SCATTER(3) ZK_SCATTER(4)
            ZK_SCATTER(5) ZK_SCATTER(6) ZK_SCATTER(7) ZK_SCATTER(8)
#undef ZK_SCATTER
            default: throw std::runtime_error("radix digit width out of range");
        }
        launches++;
        ZK_CUDA(cudaGetLastError());
        std::swap(bufA, bufB);
    }
    if (bw) {  // nothing above reads the bases
        ZK_CUDA(cudaStreamWaitEvent(stream, bw->ready, 0));
        if (bw->phi_out) make_phi<C>(d_bases, bw->phi_n, bw->phi_out);
    }
    prof_mark(ev, 1);
    // segmented sums
    const uint32_t* keys = w_ents.as<uint32_t>();  // level 1: keys are the .x of packed entries
    uint32_t kstride = 2;
    int cur = 0;
    for (size_t l = 0; l < pl.acc_K.size(); l++) {
        uint32_t K = pl.acc_K[l], T = pl.acc_T[l];
        uint32_t* d_len = tot + l;
        uint32_t* d_next = tot + l + 1;
        k_chunk_count<<<(T + 255) / 256, 256, 0, stream>>>(keys, kstride, d_len, K, T, w_cnt.as<uint32_t>());
        launches++;
        ZK_CUDA(cudaGetLastError());
        scan_u32(*this, w_cnt.as<uint32_t>(), T, d_next, nullptr);
        uint32_t* okeys = w_pkeys[cur].as<uint32_t>();
        Xyzz<P>* ovals = w_pvals[cur].as<Xyzz<P>>();
        if (l == 0) {
            const uint32_t AT = pl.acc_threads && pl.acc_threads <= (uint32_t)AccLaunch<C>::THREADS
                                        ? pl.acc_threads
                                        : (uint32_t)AccLaunch<C>::THREADS;
            k_acc_l1<C><<<(T + AT - 1) / AT, AT, 0, stream>>>(
                    w_ents.as<uint2>(), d_len, K, d_bases,
                                                             d_phi, w_cnt.as<uint32_t>(),
                                                             buckets, okeys, ovals);
            launches++;
        } else {
            const Xyzz<P>* ivals = w_pvals[cur ^ 1].as<Xyzz<P>>();
            if (T <= RED_INLINE_MAX_NODES)  // few threads: latency-bound
                k_acc_lj<C, true><<<(T + 255) / 256, 256, 0, stream>>>(keys, ivals, d_len, K, w_cnt.as<uint32_t>(),
                                                                       buckets, okeys, ovals);
            else
                k_acc_lj<C, false><<<(T + 255) / 256, 256, 0, stream>>>(keys, ivals, d_len, K,
                                                                        w_cnt.as<uint32_t>(), buckets, okeys, ovals);
            launches++;
        }
        ZK_CUDA(cudaGetLastError());
        keys = okeys;
        kstride = 1;
        cur ^= 1;
        if (l == 0) prof_mark(ev, 2);
    }
    prof_mark(ev, 3);
    if (!(flags & ENQ_ACC_ONLY)) enqueue_reduce<C>(pl, buckets, d_results, &ev);
    prof_end(ev);
}

// Window sums from the buckets by a tree of running sums, then Horner over
// the windows and affine normalisation into d_results.
template <class C>
void Engine::enqueue_reduce(const Plan& pl, const void* bucket_base, uint32_t* d_results,
                            std::vector<cudaEvent_t>* ev) {
    using P = typename C::Fp;
    const int nd = (int)pl.descs.size();
    const MsmDesc* dd = pl.d_descs.as<MsmDesc>();
    const Xyzz<P>* inS = static_cast<const Xyzz<P>*>(bucket_base);
    const Xyzz<P>* inW = nullptr;
    int rc = 0;
    for (size_t l = 0; l < pl.red_tasks.size(); l++) {
        uint32_t nout = pl.red_nout[l];
        const RedTask* tk = pl.d_tasks.as<RedTask>() + pl.task_level_off[l];
        Xyzz<P>* oS = w_redS[rc].as<Xyzz<P>>();
        Xyzz<P>* oW = w_redW[rc].as<Xyzz<P>>();
        if (nout <= RED_INLINE_MAX_NODES)
            k_reduce_level<C, true><<<(nout + 127) / 128, 128, 0, stream>>>(inS, inW, tk, (int)pl.red_tasks[l].size(),
                                                                           nout, pl.red_L,
                                                                           (uint32_t)l * pl.red_log2L, oS, oW);
        else
            k_reduce_level<C, false><<<(nout + 127) / 128, 128, 0, stream>>>(
                    inS, inW, tk, (int)pl.red_tasks[l].size(), nout, pl.red_L, (uint32_t)l * pl.red_log2L, oS, oW);
        launches++;
        ZK_CUDA(cudaGetLastError());
        inS = oS;
        inW = oW;
        rc ^= 1;
    }
    if (ev) prof_mark(*ev, 4);
    k_combine<C><<<nd, 32 * COMBINE_WARPS, 0, stream>>>(inS, inW, dd, nd, d_results);
    launches++;
    ZK_CUDA(cudaGetLastError());
    if (ev) prof_mark(*ev, 5);
}

template <class C>
void Engine::fold_buckets(void* base, uint32_t nb, uint32_t S) {
    using P = typename C::Fp;
    if (S > 1 && nb) {
        k_bucket_fold<C><<<(nb + 127) / 128, 128, 0, stream>>>(static_cast<Xyzz<P>*>(base), nb, S);
        launches++;
        ZK_CUDA(cudaGetLastError());
    }
}

// endomorphism table for a base array
template <class C>
void Engine::make_phi(const uint32_t* d_bases, uint64_t n, uint32_t* d_phi) {
    if (!n || !CurveTraits<C>::glv) return;  // no endomorphism image without a GLV split
    k_endo<C><<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(d_bases, (uint32_t)n, d_phi);
    launches++;
    ZK_CUDA(cudaGetLastError());
}

template <class C>
void Engine::make_shifts(uint32_t* d_table, uint64_t n, uint32_t s, uint32_t copies) {
    using P = typename C::Fp;
    if (!n || copies < 2) return;
    // points per pass: the XYZZ scratch of one pass stays near 512 MB
    const uint64_t per_point = (uint64_t)(copies - 1) * sizeof(Xyzz<P>);
    const uint32_t m = (uint32_t)std::min<uint64_t>(n, std::max<uint64_t>(1024, (512ull << 20) / per_point));
    DevBuf scratch;
    scratch.ensure((size_t)m * per_point);
    Xyzz<P>* sc = scratch.as<Xyzz<P>>();
    for (uint64_t i0 = 0; i0 < n; i0 += m) {
        const uint32_t mm = (uint32_t)std::min<uint64_t>(m, n - i0);
        k_shift_chain<C><<<(mm + 127) / 128, 128, 0, stream>>>(d_table, (uint32_t)i0, mm, s, copies, sc);
        launches++;
        ZK_CUDA(cudaGetLastError());
        const uint64_t total = (uint64_t)(copies - 1) * mm;
        const uint64_t threads = (total + SHIFT_G - 1) / SHIFT_G;
        k_shift_affine<C><<<(unsigned)((threads + 127) / 128), 128, 0, stream>>>(sc, total, mm, (uint32_t)i0, n,
                                                                                 d_table);
        launches++;
        ZK_CUDA(cudaGetLastError());
    }
    ZK_CUDA(cudaStreamSynchronize(stream));
}

template <class C>
uint32_t Engine::acc_resident_threads() {
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_acc_l1<C>, AccLaunch<C>::THREADS, 0) !=
                cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return (uint32_t)(per_sm * sms * AccLaunch<C>::THREADS);
}

template <class C>
void Engine::gen_bases(uint64_t seed, uint64_t index0, uint64_t n, uint32_t* d_out) {
    using P = typename C::Fp;
    const int ci = CurveTraits<C>::id;
    static_assert(CurveTraits<C>::id < NCURVES, "per-curve arrays hold NCURVES entries");
    if (!comb_ready[ci]) {
        // one 32 x 256-entry table of affine points per curve, each slot
        // sized for the widest coordinate
        static_assert(P::N <= MAX_COORD_WORDS, "coordinate wider than the comb table slot");
        w_comb.ensure((size_t)NCURVES * 32 * 256 * 2 * MAX_COORD_WORDS * 4);
        uint32_t* tab = w_comb.as<uint32_t>() + (size_t)ci * 32 * 256 * 2 * MAX_COORD_WORDS;
        k_comb_table<C><<<(32 * 256 + 127) / 128, 128, 0, stream>>>(tab);
        launches++;
        ZK_CUDA(cudaGetLastError());
        comb_ready[ci] = true;
    }
    uint32_t* tab = w_comb.as<uint32_t>() + (size_t)ci * 32 * 256 * 2 * MAX_COORD_WORDS;
    (void)sizeof(P);
    if (n) k_gen_bases<C><<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(tab, d_out, n, seed, index0);
    launches += (n) ? 1 : 0;
    ZK_CUDA(cudaGetLastError());
    ZK_CUDA(cudaStreamSynchronize(stream));
}

template <class C>
void Engine::profile_scalars(const uint32_t* d_scalars, uint64_t n, int fmt, bool glv) {
    w_profile.ensure(PROFILE_BINS * 4);
    if (!h_profile) ZK_CUDA(cudaMallocHost(&h_profile, PROFILE_BINS * 4));
    ZK_CUDA(cudaMemsetAsync(w_profile.p, 0, PROFILE_BINS * 4, stream));
    const uint32_t m = (uint32_t)std::min<uint64_t>(n, PROFILE_SAMPLES);
    if (m) {
        k_scalar_profile<C><<<(m + 255) / 256, 256, 0, stream>>>(d_scalars, n, m, (uint32_t)fmt, glv ? 1u : 0u,
                                                                  w_profile.as<uint32_t>());
        launches++;
        ZK_CUDA(cudaGetLastError());
    }
    ZK_CUDA(cudaMemcpyAsync(h_profile, w_profile.p, PROFILE_BINS * 4, cudaMemcpyDeviceToHost, stream));
    ZK_CUDA(cudaStreamSynchronize(stream));
}

template <class C>
void Engine::gen_scalars(uint64_t seed, uint64_t index0, uint64_t n, int dist, int fmt, uint32_t* d_out) {
    if (n) k_gen_scalars<C><<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(d_out, n, seed, index0, dist, fmt);
    launches += (n) ? 1 : 0;
    ZK_CUDA(cudaGetLastError());
    ZK_CUDA(cudaStreamSynchronize(stream));
}
}  // namespace zkmsm
