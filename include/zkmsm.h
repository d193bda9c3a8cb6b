/* zkmsm.h -- C ABI of the B200 (sm_100a) multi-scalar multiplication library.
 *
 * Drop-in for the MSM part of zkMetal's C FFI.  Every entry point below that
 * exists in the reference keeps its name, argument order, byte layouts,
 * status codes and error behaviour; the citation next to each names the
 * reference declaration it replaces (paths inside the zkMetal tree).  Entry
 * points the reference does not have are marked NEW.
 *
 * Layouts (as in Sources/zkMetal-ffi/include/zkmetal.h:1-12):
 *   BN254       field element 32 B = 8 x u32 little endian, Montgomery form
 *               (R = 2^256); affine point 64 B (x, y); identity = all zero.
 *   BLS12-381   field element 48 B = 12 x u32 LE Montgomery (R = 2^384);
 *               affine point 96 B.
 *   scalars     32 B = 8 x u32 LE.  "_msm" entry points take integers
 *               (standard form, need not be reduced mod r, zkmetal.h:6);
 *               NEW "_fr" entry points take Montgomery-form Fr (s * 2^256 mod r).
 *   results     Jacobian (X, Y, Z), Montgomery form, each one field element.
 *               The library always returns Z = 1 (R mod p) for a finite point
 *               and (1, 1, 0) for the identity, so X and Y are the affine
 *               coordinates.
 *
 * Threading (zkMetal_ffi.swift:22-35, MSM/MSMEngine.swift:33-58): an engine
 * is not thread-safe; use one engine per thread.  The "_auto" functions share
 * one lazily created engine guarded by a mutex.
 */
#ifndef ZKMSM_H
#define ZKMSM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes: zkmetal.h:28-34 ------------------------------------ */
typedef int32_t ZkMetalStatus;
#define ZKMETAL_SUCCESS 0
#define ZKMETAL_ERR_NO_GPU -1
#define ZKMETAL_ERR_INVALID_INPUT -2
#define ZKMETAL_ERR_GPU_ERROR -3
#define ZKMETAL_ERR_ALLOC_FAILED -4
/* NEW: a served request was refused by admission control or cancelled */
#define ZKMETAL_ERR_BUSY -5

/* ---- engine lifecycle: zkmetal.h:40, 55-60 ------------------------------ */
typedef void* ZkMetalMSMEngine;

/* replaces zkmetal_msm_engine_create (zkmetal.h:57) */
ZkMetalStatus zkmetal_msm_engine_create(ZkMetalMSMEngine* out);
/* replaces zkmetal_msm_engine_destroy (zkmetal.h:60) */
void zkmetal_msm_engine_destroy(ZkMetalMSMEngine engine);

/* ---- BN254 G1 MSM: zkmetal.h:117-147 ------------------------------------ */

/* replaces zkmetal_bn254_msm (zkmetal.h:129-137); n_points == 0 -> INVALID_INPUT */
ZkMetalStatus zkmetal_bn254_msm(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars,
                                uint32_t n_points, uint8_t* result_x, uint8_t* result_y, uint8_t* result_z);

/* replaces zkmetal_bn254_msm_auto (zkmetal.h:140-147) */
ZkMetalStatus zkmetal_bn254_msm_auto(const uint8_t* points, const uint8_t* scalars, uint32_t n_points,
                                     uint8_t* result_x, uint8_t* result_y, uint8_t* result_z);

/* replaces zkmetal_bn254_msm_u8 / _u16 / _u32 (zkmetal.h:446-471): 1, 2 or 4
 * byte little-endian scalars, zero-extended */
ZkMetalStatus zkmetal_bn254_msm_u8(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars,
                                   uint32_t n_points, uint8_t* result_x, uint8_t* result_y, uint8_t* result_z);
ZkMetalStatus zkmetal_bn254_msm_u16(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars,
                                    uint32_t n_points, uint8_t* result_x, uint8_t* result_y, uint8_t* result_z);
ZkMetalStatus zkmetal_bn254_msm_u32(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars,
                                    uint32_t n_points, uint8_t* result_x, uint8_t* result_y, uint8_t* result_z);
/* replaces zkmetal_bn254_msm_u8_auto / _u16_auto / _u32_auto (zkmetal.h:473-484) */
ZkMetalStatus zkmetal_bn254_msm_u8_auto(const uint8_t* points, const uint8_t* scalars, uint32_t n_points,
                                        uint8_t* result_x, uint8_t* result_y, uint8_t* result_z);
ZkMetalStatus zkmetal_bn254_msm_u16_auto(const uint8_t* points, const uint8_t* scalars, uint32_t n_points,
                                         uint8_t* result_x, uint8_t* result_y, uint8_t* result_z);
ZkMetalStatus zkmetal_bn254_msm_u32_auto(const uint8_t* points, const uint8_t* scalars, uint32_t n_points,
                                         uint8_t* result_x, uint8_t* result_y, uint8_t* result_z);

/* replaces zkmetal_bn254_msm_batch (zkmetal.h:499-506): MSM i uses the next
 * counts[i] points and scalars; results[i] = 96 B (X, Y, Z); counts[i] == 0
 * writes 96 zero bytes (zkMetal_ffi.swift:1260-1264); n_msms == 0 ->
 * INVALID_INPUT.  Unlike the reference, all MSMs run in one batched launch
 * sequence instead of one after another. */
ZkMetalStatus zkmetal_bn254_msm_batch(ZkMetalMSMEngine engine, const uint8_t* all_points,
                                      const uint8_t* all_scalars, const uint32_t* counts, uint32_t n_msms,
                                      uint8_t* results);
/* replaces zkmetal_bn254_msm_batch_auto (zkmetal.h:509-515) */
ZkMetalStatus zkmetal_bn254_msm_batch_auto(const uint8_t* all_points, const uint8_t* all_scalars,
                                           const uint32_t* counts, uint32_t n_msms, uint8_t* results);

/* NEW: BN254 with Montgomery-form Fr scalars (the conversion the reference
 * does on the CPU in bn254_fr_batch_to_limbs, NeonFieldOps/bn254_msm.c:1537,
 * runs inside the GPU scalar-preparation kernel) */
ZkMetalStatus zkmetal_bn254_msm_fr(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars_mont,
                                   uint32_t n_points, uint8_t* result_x, uint8_t* result_y, uint8_t* result_z);

/* NEW: n_msms independent MSMs in one batched launch sequence, for any curve
 * and either scalar form -- the general form of zkmetal_bn254_msm_batch
 * (zkmetal.h:499), behind the Swift batch front-ends batchMSMAsync
 * (MSM/MultiMSM.swift:175), innerProductMSM (:90) and multiMSM with Fr scalar
 * sets (:63).  MSM i runs over the i-th consecutive run of counts[i] points
 * and scalars of all_points / all_scalars (host memory); results as in the
 * batch call (n_msms x 3 coordinates, counts[i] == 0 -> zero bytes). */
ZkMetalStatus zkmsm_msm_batch(ZkMetalMSMEngine engine, int curve, const uint8_t* all_points,
                              const uint8_t* all_scalars, int scalar_fmt, const uint32_t* counts, uint32_t n_msms,
                              uint8_t* results);

/* ---- BLS12-381 G1 MSM ---------------------------------------------------
 * NEW symbols: the reference FFI has none.  They replace the Swift API
 * BLS12381MSM.msm / msmFr (MSM/BLS12381MSMEngine.swift:260, 517) and the C
 * g1 Pippenger (NeonFieldOps/bls12_381_ops.c:1141).  Points 96 B, results
 * 48 B per coordinate. */
ZkMetalStatus zkmetal_bls12_381_g1_msm(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars,
                                       uint32_t n_points, uint8_t* result_x, uint8_t* result_y,
                                       uint8_t* result_z);
ZkMetalStatus zkmetal_bls12_381_g1_msm_fr(ZkMetalMSMEngine engine, const uint8_t* points,
                                          const uint8_t* scalars_mont, uint32_t n_points, uint8_t* result_x,
                                          uint8_t* result_y, uint8_t* result_z);
ZkMetalStatus zkmetal_bls12_381_g1_msm_batch(ZkMetalMSMEngine engine, const uint8_t* all_points,
                                             const uint8_t* all_scalars, const uint32_t* counts,
                                             uint32_t n_msms, uint8_t* results);

/* ---- BLS12-377 G1 MSM ---------------------------------------------------
 * NEW symbols, the same shapes as the BLS12-381 ones (96 B points, 48 B
 * coordinates).  They replace the Swift API BLS12377MSM.msm
 * (MSM/BLS12377MSMEngine.swift:266) and the C g1 Pippenger
 * (NeonFieldOps/bls12_377_ops.c:1476, GLV form :1814). */
ZkMetalStatus zkmetal_bls12_377_g1_msm(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars,
                                       uint32_t n_points, uint8_t* result_x, uint8_t* result_y,
                                       uint8_t* result_z);
ZkMetalStatus zkmetal_bls12_377_g1_msm_fr(ZkMetalMSMEngine engine, const uint8_t* points,
                                          const uint8_t* scalars_mont, uint32_t n_points, uint8_t* result_x,
                                          uint8_t* result_y, uint8_t* result_z);
ZkMetalStatus zkmetal_bls12_377_g1_msm_batch(ZkMetalMSMEngine engine, const uint8_t* all_points,
                                             const uint8_t* all_scalars, const uint32_t* counts,
                                             uint32_t n_msms, uint8_t* results);

/* ---- BN254 G2 MSM -------------------------------------------------------
 * NEW symbols.  They replace the Swift API BN254G2MSM.msm
 * (MSM/BN254G2MSMEngine.swift:51, msm at :289).  Points 128 B (x.c0, x.c1,
 * y.c0, y.c1, each 32 B Montgomery: G2AffinePoint of
 * Curve/BN254Pairing.swift:301-305); results x, y, z as 64 B Fp2 elements
 * (Z = 1 = (1, 0), or the identity (1, 1, 0) with z = 0).  Scalars as in the
 * BN254 G1 calls; the GLV split uses the twist's Frobenius endomorphism. */
ZkMetalStatus zkmetal_bn254_g2_msm(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars,
                                   uint32_t n_points, uint8_t* result_x, uint8_t* result_y, uint8_t* result_z);
ZkMetalStatus zkmetal_bn254_g2_msm_fr(ZkMetalMSMEngine engine, const uint8_t* points, const uint8_t* scalars_mont,
                                      uint32_t n_points, uint8_t* result_x, uint8_t* result_y, uint8_t* result_z);

/* ---- misc: zkmetal.h:520-530 --------------------------------------------- */
/* replaces zkmetal_set_shader_dir (zkmetal.h:524): accepted and ignored (no shaders) */
void zkmetal_set_shader_dir(const char* path);
/* replaces zkmetal_gpu_available (zkmetal.h:527): 1 if a CUDA device of compute capability 10.x is visible */
int32_t zkmetal_gpu_available(void);
/* replaces zkmetal_version (zkmetal.h:530) */
const char* zkmetal_version(void);

/* ==== NEW: device-resident data, batching, serving ======================= */

/* Curve selector for the entry points below. */
#define ZKMSM_BN254 0
#define ZKMSM_BLS12_381 1
#define ZKMSM_BLS12_377 2
#define ZKMSM_BN254_G2 3
/* Scalar encoding */
#define ZKMSM_SCALAR_INT 0
#define ZKMSM_SCALAR_MONT 1

/* Text of the last error raised on the calling thread ("" if none). */
const char* zkmsm_last_error(void);

/* MSM on device buffers (CUDA pointers): d_points n affine points, d_scalars
 * n x 32 B; result (3 field elements, Jacobian layout above) copied to HOST
 * memory `result`.  `stream` is a cudaStream_t (0 = the engine's stream). */
ZkMetalStatus zkmsm_msm_device(ZkMetalMSMEngine engine, int curve, const void* d_points, const void* d_scalars,
                               int scalar_fmt, uint32_t n_points, uint8_t* result, void* stream);

/* Enqueue-only variant for pipelined callers: all buffers are device
 * pointers; d_phi (the endomorphism image of the bases, n affine points) may
 * be NULL, in which case it is computed into engine scratch on the stream.
 * The result (3 field elements) is written to DEVICE memory d_result.  The
 * call returns without waiting; order other work on the same stream. */
ZkMetalStatus zkmsm_msm_device_async(ZkMetalMSMEngine engine, int curve, const void* d_points, const void* d_phi,
                                     const void* d_scalars, int scalar_fmt, uint32_t n_points, void* d_result,
                                     void* stream);

/* A base table kept resident in HBM (a commitment key), with its
 * endomorphism image precomputed once.  points: HOST pointer unless
 * points_on_device != 0. */
typedef void* ZkMsmTable;
ZkMetalStatus zkmsm_table_create(ZkMetalMSMEngine engine, int curve, const void* points, uint64_t n_points,
                                 int points_on_device, ZkMsmTable* out);
/* NEW: fixed-base precomputation for a resident table (replaces the
 * reference's BGMW tables, Sources/zkMetal/MSM/MSMPrecomputation.swift:17-274
 * and Sources/NeonFieldOps/bn254_msm.c:2163-2327, which store every digit
 * multiple of every window).  Extends the table in place with its window
 * shifts: copy k of every point is 2^(spacing_bits*k) * P_i, for
 * k < ceil((fr_bits + 1) / spacing_bits), so memory grows by that many
 * copies (BN254, spacing 4: 64 copies, 4 KiB per point).  MSMs over the
 * table (zkmsm_batch_commit, the commitment server) then use window widths
 * that are multiples of spacing_bits, add every window into one bucket set
 * and skip the Horner chain; results are unchanged.  spacing_bits: 2..24,
 * or 0 to drop the shifts.  Not to be called while the table is in use.
 * ZKMETAL_ERR_INVALID_INPUT if copies * n_points reaches 2^30. */
ZkMetalStatus zkmsm_table_precompute(ZkMsmTable table, int spacing_bits);
/* Spacing of the table's shifts (0: none; -1: no table). */
int zkmsm_table_shift_bits(ZkMsmTable table);
void zkmsm_table_destroy(ZkMsmTable table);
/* Device pointer of the table's affine points (for reading back / tests). */
const void* zkmsm_table_device_points(ZkMsmTable table);

/* Batched commitments over a resident table: MSM i = sum_j s_ij * T[j] for
 * j < counts[i] (a prefix of the table).  scalars: concatenated 32 B scalars
 * (HOST unless scalars_on_device), results: n_msms x 3 field elements (HOST).
 * All MSMs run as one batch; a shape that repeats is captured in a CUDA graph
 * on its second call and replayed after that.  Window width and chunking
 * come from the autotuner. */
ZkMetalStatus zkmsm_batch_commit(ZkMetalMSMEngine engine, ZkMsmTable table, const void* scalars,
                                 int scalars_on_device, int scalar_fmt, const uint32_t* counts, uint32_t n_msms,
                                 uint8_t* results);

/* Autotuner: times the MSM at equal window widths around the cost model's
 * choice, and at the model's two-width layout where it picks one (reported
 * as width 0), for every power-of-two size 2^min_log2n .. 2^max_log2n on
 * synthetic inputs and keeps the fastest per size; later plans of this
 * engine use the table (MSMs matched to the nearest power of two).  From
 * 2^14 points it then tunes the tile schedule at that layout, one knob at a
 * time: the level-1 chunk length (half or twice the cost rule's), 128
 * instead of 256 threads per accumulation block, and a bucket-reduction tree
 * of arity 4 or 16 instead of 8 (a batch plan takes the schedule of its
 * largest MSM).  A JSON summary of the timings is written to `report` (may
 * be NULL).  Replaces the reference's device tuning of window bits and
 * threadgroup sizes (Sources/zkMetal/Tuning.swift:9-127). */
ZkMetalStatus zkmsm_autotune(ZkMetalMSMEngine engine, int curve, int min_log2n, int max_log2n, char* report,
                             uint64_t report_len);
/* Persist / restore the autotuned table (text file). */
ZkMetalStatus zkmsm_tuning_save(ZkMetalMSMEngine engine, const char* path);
ZkMetalStatus zkmsm_tuning_load(ZkMetalMSMEngine engine, const char* path);

/* ---- commitment server (continuous batching) ----------------------------
 * NEW.  Requests are MSMs over a prefix of a resident table; `workers`
 * threads each own an engine (own stream and resident scratch).  A free
 * worker batches, in arrival order, the pending requests of the oldest
 * request's curve that fit `max_batch_points` (0 = 2^24) and the HBM budget
 * (`hbm_budget_bytes`, 0 = 70% of free device memory), so requests arriving
 * while others run join the next batch and batches of different workers
 * overlap on the GPU.  The caller keeps `scalars` valid until the request
 * completes.  Latency is measured from submit to completion. */
typedef void* ZkMsmServer;
ZkMetalStatus zkmsm_server_create(ZkMsmTable bn254_table, ZkMsmTable bls12_381_table, uint64_t hbm_budget_bytes,
                                  int workers, uint64_t max_batch_points, ZkMsmServer* out);
/* ZKMETAL_ERR_BUSY if the request alone exceeds the budget or the server stops */
ZkMetalStatus zkmsm_server_submit(ZkMsmServer server, int curve, const void* scalars, int scalar_fmt,
                                  uint32_t n_points, uint64_t* request_id);
/* Remove a request that has not started (ZKMETAL_ERR_BUSY if it has). */
ZkMetalStatus zkmsm_server_cancel(ZkMsmServer server, uint64_t request_id);
/* Wait up to timeout_ms (< 0: forever) for a request; returns its status
 * (ZKMETAL_ERR_BUSY on timeout or when it was cancelled), writes the result
 * (3 field elements) and the submit-to-completion latency. */
ZkMetalStatus zkmsm_server_wait(ZkMsmServer server, uint64_t request_id, int timeout_ms, uint8_t* result,
                                double* latency_ms);
/* JSON counters: completed, failed, batches, p50/p99 latency, memory in use. */
ZkMetalStatus zkmsm_server_stats(ZkMsmServer server, char* buf, uint64_t buflen);
/* Test hook: make the next `batches` batches fail on the host before any GPU work. */
ZkMetalStatus zkmsm_server_inject_failures(ZkMsmServer server, int batches);
void zkmsm_server_destroy(ZkMsmServer server);

/* NEW: request-level replicas for serving on several GPUs.  Each replica is a
 * server created (zkmsm_server_create) with its own device current and its
 * own resident tables on that device; the pool routes every submitted
 * request whole to one replica -- no collective, no data crossing GPUs.
 * Routing (zkmsm_route_pick): among replicas holding a table for the curve
 * that is long enough and a budget that can ever hold the request, one with
 * free budget for it now beats one without; then the shallowest queue
 * (points submitted and not finished, divided by relative_speed); among
 * replicas that all lack room, then the most free budget; then the first in
 * cyclic order from `first` (the pool advances it with every request, so
 * ties rotate over the replicas).  The
 * pool does not own the servers: destroy the pool first.  Ids are the
 * pool's own. */
typedef struct {
    int32_t has_table;       /* a table for the request's curve */
    uint64_t table_points;   /* its length */
    uint64_t queued_points;  /* points of requests submitted and not finished */
    uint64_t budget_bytes;   /* admission budget */
    uint64_t in_use_bytes;   /* admitted and running */
    double relative_speed;   /* 1.0 for identical GPUs */
} ZkMsmReplicaLoad;
typedef void* ZkMsmPool;
/* index of the replica for a request, or -1 when none can take it (pure host
 * logic: the rule the pool applies, callable without a GPU) */
int zkmsm_route_pick(const ZkMsmReplicaLoad* loads, uint32_t n_replicas, uint32_t request_points,
                     uint64_t request_bytes, uint32_t first);
ZkMetalStatus zkmsm_pool_create(const ZkMsmServer* servers, uint32_t n_servers, ZkMsmPool* out);
/* ZKMETAL_ERR_BUSY when no replica can take the request */
ZkMetalStatus zkmsm_pool_submit(ZkMsmPool pool, int curve, const void* scalars, int scalar_fmt, uint32_t n_points,
                                uint64_t* request_id);
ZkMetalStatus zkmsm_pool_wait(ZkMsmPool pool, uint64_t request_id, int timeout_ms, uint8_t* result,
                              double* latency_ms);
/* {"replicas": [server stats + "routed" (requests sent there) + "device"]} */
ZkMetalStatus zkmsm_pool_stats(ZkMsmPool pool, char* buf, uint64_t buflen);
void zkmsm_pool_destroy(ZkMsmPool pool);

/* Tuning overrides (0 = automatic): window bits, chunk length, GLV on/off.
 * window_bits >= 2^16 is a two-width layout c | nlo << 16: nlo windows of
 * c bits, then (c + 1)-bit windows up to the scalar width. */
ZkMetalStatus zkmsm_engine_set_tuning(ZkMetalMSMEngine engine, int window_bits, int chunk, int glv);
/* NEW: window layout from a sample of the scalars (on by default).  For a
 * single MSM of at least 2^21 points on a GLV curve, with no window width
 * forced or autotuned for its size, the engine first profiles 4096 of the
 * scalars on the device (bit lengths of their prepared halves) and picks the
 * window layout that minimises sorted entries plus bucket-reduction work for
 * that profile: skewed scalar sets (many zeros, ones or short values) get
 * fewer, narrower buckets; uniform ones keep the layout chosen from n.  The
 * result never depends on it.  The sample makes the call wait for the work
 * already queued on its stream (also in zkmsm_msm_device_async; skipped while
 * the stream is being captured).  The reference samples a window-0 bucket
 * histogram for its window choice (MSM/MSMEngine.swift:565-593, 768-783).
 * enable: 1 on, 0 off. */
ZkMetalStatus zkmsm_engine_set_sampling(ZkMetalMSMEngine engine, int enable);

/* NEW: host-buffer MSMs (zkmetal_*_msm and their _fr forms) are streamed in
 * stripes (consecutive point ranges from 2^(stripe_log2-2) points, growing
 * 1.6x per stripe up to 2^stripe_log2): each stripe's host-to-device copy
 * overlaps the previous stripe's sort and accumulation, every stripe fills
 * its own bucket array in the window layout of the largest stripe, and the
 * arrays are added and reduced once (the same point).  -1 (default):
 * automatic: largest stripe half of n's next power of two from 2^22 points,
 * and 2^20 points for BN254 G1 calls of 2^21 <= n < 2^22; none below; 0:
 * off; 2..30: fixed. */
ZkMetalStatus zkmsm_engine_set_stripe(ZkMetalMSMEngine engine, int stripe_log2);

/* Synthetic inputs on the device (seeded, counter based):
 * bases[i] = k_i * G with k_i uniform in [1, r); scalars uniform in Fr
 * (dist 0) or witness-like (dist 1: 40% 0, 20% 1, 25% < 2^32, 15% uniform). */
ZkMetalStatus zkmsm_gen_bases(ZkMetalMSMEngine engine, int curve, uint64_t seed, uint64_t index0, uint64_t n,
                              void* d_out);
ZkMetalStatus zkmsm_gen_scalars(ZkMetalMSMEngine engine, int curve, uint64_t seed, uint64_t index0,
                                uint64_t n, int dist, int scalar_fmt, void* d_out);

/* Per-phase device time: enable/disable recording CUDA events around the
 * pipeline phases of every MSM this engine enqueues; read (after waiting for
 * the recorded work) the cumulative milliseconds of phases
 * 0 scalar preparation + bucket sort, 1 first accumulation level, 2 later
 * accumulation levels, 3 bucket reduction, 4 window combine, and the number
 * of MSM batches recorded. */
ZkMetalStatus zkmsm_engine_profile(ZkMetalMSMEngine engine, int enable);
ZkMetalStatus zkmsm_engine_phase_times(ZkMetalMSMEngine engine, double* ms5, uint64_t* calls, int reset);

/* The execution plan (window widths, bucket layout, chunking of the segmented
 * sums, reduction tree) the engine would use for a batch, as JSON text in
 * buf.  Pure host computation: no device is touched. */
ZkMetalStatus zkmsm_plan_describe(int curve, const uint32_t* counts, uint32_t n_msms, int scalar_fmt,
                                  int window_bits, int chunk, int glv, int scalar_bits, char* buf, uint64_t buflen);
/* The same for MSMs over prefixes of a table of table_points points with
 * window shifts of spacing shift_bits (zkmsm_table_precompute). */
ZkMetalStatus zkmsm_plan_describe_shift(int curve, const uint32_t* counts, uint32_t n_msms, int scalar_fmt,
                                        int window_bits, int shift_bits, uint32_t table_points, char* buf,
                                        uint64_t buflen);

/* Kernels launched so far by this engine (cumulative). */
uint64_t zkmsm_engine_launch_count(ZkMetalMSMEngine engine);

/* NEW (reporting helper, no counterpart in the reference): the number of
 * sorted (bucket, point) entries of the engine's last MSM batch, i.e. the
 * mixed additions its level-1 accumulation executed.  Waits for the whole
 * device first (cudaDeviceSynchronize); 0 before the first batch. */
uint64_t zkmsm_engine_last_entries(ZkMetalMSMEngine engine);

/* Roofline denominators measured on device 0: 32x32->64-bit word products per
 * second (one low + one high multiply-add) with every SM occupied, and the
 * Montgomery multiplications per second of this library's BN254 and
 * BLS12-381 field code (either output pointer may be NULL). */
ZkMetalStatus zkmsm_measure_peaks(double* products_per_s, double* bn254_mul_per_s, double* bls381_mul_per_s);

/* Word products per second of the single-instruction 64-bit form
 * (mad.wide.u32) measured by the last zkmsm_measure_peaks call. */
double zkmsm_wide_products_per_s(void);

/* Sum `count` results (each 3 field elements in the result layout above) into
 * one; used to combine the partial MSMs of point-range shards. */
ZkMetalStatus zkmsm_sum_results(int curve, const uint8_t* results, uint32_t count, uint8_t* out);
/* Same on device buffers, enqueued on `stream` (cudaStream_t) without waiting. */
ZkMetalStatus zkmsm_sum_results_device(int curve, const void* d_results, uint32_t count, void* d_out, void* stream);

/* NEW (test helper, no counterpart in the reference): element-wise base-field
 * operation on n device operands of N little-endian u32 limbs (N = 8 BN254,
 * 12 BLS12-381), Montgomery form, each operand below 2p: op 0 r = a*b/R (the
 * product the MSM kernels use), 1 r = a^2/R (their square), 2 r = a*b/R by a
 * second implementation of the product.  Results are canonical (below p); the call
 * waits for the device. */
ZkMetalStatus zkmsm_field_op(int curve, int op, const void* d_a, const void* d_b, void* d_out, uint32_t n);

/* NEW, with no counterpart in the reference: a BN254 G1 MSM that allocates no
 * device memory, for callers that cannot call cudaMalloc -- e.g. a framework
 * that has already reserved nearly all of HBM for its own pool, or a hot loop
 * that forbids allocation after start-up because cudaMalloc/cudaFree may
 * synchronise the device.  Inputs and output are the caller's device buffers:
 * n_points affine points (64 B), n_points scalars (32 B, scalar_fmt), result
 * 3 x 32 B (Jacobian, Z = 1 or the identity).  n_points <= 8192; larger ->
 * ZKMETAL_ERR_INVALID_INPUT.  Scratch is one static device array of about
 * 7.6 MB that every GPU loading the library holds until exit and that all
 * calls share: calls whose GPU work overlaps race, so serialise them (calls
 * queued one after another on one stream are already ordered).  The first
 * call on a device looks the array's address up and caches it (make that
 * first call before any stream capture); after a cudaDeviceReset of that
 * device the cached address is stale, so do not call it again in that
 * process.  A CUDA error left pending by earlier work is reported
 * (ZKMETAL_ERR_GPU_ERROR) and left pending; nothing is enqueued then.
 * Enqueues on `stream` (cudaStream_t; 0 = legacy default stream) and returns
 * without waiting. */
ZkMetalStatus zkmsm_bn254_msm_noalloc(const void* d_points, const void* d_scalars, int scalar_fmt,
                                      uint32_t n_points, void* d_result, void* stream);

/* Device memory helpers for callers without a CUDA runtime of their own. */
void* zkmsm_device_alloc(uint64_t bytes);
void zkmsm_device_free(void* p);
ZkMetalStatus zkmsm_memcpy_h2d(void* d_dst, const void* src, uint64_t bytes);
ZkMetalStatus zkmsm_memcpy_d2h(void* dst, const void* d_src, uint64_t bytes);
ZkMetalStatus zkmsm_device_sync(void);

#ifdef __cplusplus
}
#endif

#endif /* ZKMSM_H */
