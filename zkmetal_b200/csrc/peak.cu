// Integer-multiply roofline probes and small point utilities.
//
// k_imad_peak: the denominator of the MSM roofline -- the sustained rate of
// 32x32->64-bit word products (one mad.lo + one mad.hi with carry, the unit
// the CIOS multiply is counted in) with every SM fully occupied and eight
// independent carry chains per thread.  On sm_100a a carry-chained lo/hi
// pair issues as one instruction on the heavy FMA pipe, which accepts one
// such 64-bit product every 4 cycles per scheduler (a 32-bit low product
// every 2); k_imad_wide_peak (mad.wide.u32) measures the same rate.
// k_fe_mul_peak: independent BN254 / BLS12-381 Montgomery products per
// second with per-thread operands (the field-multiply ceiling of this
// implementation).
// k_sum_results: adds a list of library results (reference Jacobian layout
// with Z = 1 or the identity) into one, for combining per-GPU partial MSMs.
#include <cuda_runtime.h>

#include "../../include/zkmsm.h"
#include "msm_kernels.cuh"

namespace zkmsm {

__global__ void __launch_bounds__(256) k_imad_peak(uint32_t iters, uint32_t seed, uint32_t* sink) {
    uint32_t a[8], b = seed ^ threadIdx.x, lo[8], hi[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        a[j] = seed * (j + 3) + threadIdx.x;
        lo[j] = j;
        hi[j] = j * 7;
    }
#pragma unroll 1
    for (uint32_t it = 0; it < iters; it++) {
#pragma unroll
        for (int r = 0; r < 8; r++) {
#pragma unroll
            for (int j = 0; j < 8; j++) {
                asm volatile("mad.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.u32 %1, %2, %3, %1;"
                             : "+r"(lo[j]), "+r"(hi[j])
                             : "r"(a[j]), "r"(b));
            }
        }
    }
    uint32_t x = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) x ^= lo[j] ^ hi[j];
    if (x == 0x12345678u) sink[0] = x;  // keep the work observable
}

// 64-bit multiply-add form of the same work: one mad.wide.u32 per product.
// The multiplier is the high word of the chain's own accumulator, so no two
// products are alike and the compiler cannot fold repeated ones into adds
// (with a loop-invariant multiplier it does, and the probe then times 64-bit
// additions instead of products).
__global__ void __launch_bounds__(256) k_imad_wide_peak(uint32_t iters, uint32_t seed, uint32_t* sink) {
    uint32_t a[8], b = seed ^ threadIdx.x;
    uint64_t acc[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        a[j] = seed * (j + 3) + threadIdx.x;
        acc[j] = ((uint64_t)(b * (j + 1)) << 32) | j;
    }
#pragma unroll 1
    for (uint32_t it = 0; it < iters; it++) {
#pragma unroll
        for (int r = 0; r < 8; r++) {
#pragma unroll
            for (int j = 0; j < 8; j++) {
                asm volatile("{\n\t.reg .u32 h;\n\tmov.b64 {_, h}, %0;\n\tmad.wide.u32 %0, %1, h, %0;\n\t}"
                             : "+l"(acc[j])
                             : "r"(a[j]));
            }
        }
    }
    uint64_t x = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) x ^= acc[j];
    if (x == 0x12345678u) sink[0] = (uint32_t)x;
}

template <class P>
__global__ void __launch_bounds__(256) k_fe_mul_peak(uint32_t iters, uint32_t* sink) {
    Fe<P> x[2], y;
#pragma unroll
    for (int i = 0; i < P::N; i++) {
        x[0].v[i] = P::ONE(i) ^ threadIdx.x;
        x[1].v[i] = P::R2(i) ^ blockIdx.x;
        y.v[i] = P::R2(i) ^ (threadIdx.x * 0x9e3779b9u) ^ blockIdx.x;  // per-thread multiplier
    }
    x[0].v[P::N - 1] &= 0x0fffffffu;
    x[1].v[P::N - 1] &= 0x0fffffffu;
    y.v[P::N - 1] &= 0x0fffffffu;
#pragma unroll 1
    for (uint32_t it = 0; it < iters; it++) {
        fe_mul(x[0], x[0], y);
        fe_mul(x[1], x[1], y);
    }
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < P::N; i++) s ^= x[0].v[i] ^ x[1].v[i];
    if (s == 0x12345678u) sink[0] = s;
}

// Element-wise field operation on n operands (limbs little endian, N words
// each): op 0 r = a*b (the library's product), 1 r = a^2 (its square),
// 2 r = a*b by the straight CIOS product (a second implementation).
template <class P>
__global__ void __launch_bounds__(128) k_field_op(int op, const uint32_t* __restrict__ a,
                                                  const uint32_t* __restrict__ b, uint32_t* __restrict__ out,
                                                  uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fe<P> x, y, z;
#pragma unroll
    for (int l = 0; l < P::N; l++) {
        x.v[l] = a[(size_t)i * P::N + l];
        y.v[l] = b[(size_t)i * P::N + l];
    }
    if (op == 0) fe_mul(z, x, y);
    else if (op == 1) fe_sqr(z, x);
    else fe_mul_body(z, x, y);
#pragma unroll
    for (int l = 0; l < P::N; l++) out[(size_t)i * P::N + l] = z.v[l];
}

template <class C>
__global__ void k_sum_results(const uint32_t* __restrict__ in, uint32_t count, uint32_t* __restrict__ out) {
    using P = typename C::Fp;
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    Xyzz<P> acc;
    xyzz_set_id(acc);
    for (uint32_t i = 0; i < count; i++) {
        const uint32_t* r = in + (size_t)i * 3 * P::N;
        bool id = true;
        for (int l = 0; l < P::N; l++) id &= r[2 * P::N + l] == 0;
        if (id) continue;
        Affine<P> a;
        for (int l = 0; l < P::N; l++) {
            a.x.v[l] = r[l];
            a.y.v[l] = r[P::N + l];
        }
        xyzz_add_affine_ni(acc, a);
    }
    Affine<P> a;
    xyzz_to_affine_ni(a, acc);
    Fe<P> one;
    fe_set_one(one);
    bool id = xyzz_is_id(acc);
    for (int l = 0; l < P::N; l++) {
        out[l] = id ? one.v[l] : a.x.v[l];
        out[P::N + l] = id ? one.v[l] : a.y.v[l];
        out[2 * P::N + l] = id ? 0u : one.v[l];
    }
}

}  // namespace zkmsm

using namespace zkmsm;

static double time_kernel(void (*launch)(cudaStream_t), cudaStream_t s) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    launch(s);  // warm-up
    cudaEventRecord(a, s);
    launch(s);
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms * 1e-3;
}

static uint32_t* g_sink = nullptr;
static double g_wide_products_per_s = 0;
static int g_blocks = 0;
constexpr uint32_t IMAD_ITERS = 2048;
constexpr uint32_t FE_ITERS = 256;

extern "C" ZkMetalStatus zkmsm_measure_peaks(double* products_per_s, double* bn254_mul_per_s,
                                             double* bls381_mul_per_s) {
    if (!products_per_s) return ZKMETAL_ERR_INVALID_INPUT;
    if (!g_sink && cudaMalloc(&g_sink, 64) != cudaSuccess) return ZKMETAL_ERR_GPU_ERROR;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, 0) != cudaSuccess) return ZKMETAL_ERR_NO_GPU;
    g_blocks = prop.multiProcessorCount * 8;  // 8 x 256 threads per SM: full occupancy
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return ZKMETAL_ERR_GPU_ERROR;
    double t = time_kernel([](cudaStream_t st) { k_imad_peak<<<g_blocks, 256, 0, st>>>(IMAD_ITERS, 7, g_sink); }, s);
    double threads = (double)g_blocks * 256;
    *products_per_s = threads * IMAD_ITERS * 64 / t;  // 64 lo+hi pairs per iteration
    double tw = time_kernel(
        [](cudaStream_t st) { k_imad_wide_peak<<<g_blocks, 256, 0, st>>>(IMAD_ITERS, 7, g_sink); }, s);
    g_wide_products_per_s = threads * IMAD_ITERS * 64 / tw;
    if (bn254_mul_per_s) {
        double t2 = time_kernel(
            [](cudaStream_t st) { k_fe_mul_peak<Bn254Fp><<<g_blocks, 256, 0, st>>>(FE_ITERS, g_sink); }, s);
        *bn254_mul_per_s = threads * FE_ITERS * 2 / t2;
    }
    if (bls381_mul_per_s) {
        double t3 = time_kernel(
            [](cudaStream_t st) { k_fe_mul_peak<Bls381Fp><<<g_blocks, 256, 0, st>>>(FE_ITERS / 2, g_sink); }, s);
        *bls381_mul_per_s = threads * (FE_ITERS / 2) * 2 / t3;
    }
    cudaError_t e = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    return e == cudaSuccess ? ZKMETAL_SUCCESS : ZKMETAL_ERR_GPU_ERROR;
}

// products/s of the single-instruction 64-bit form (mad.wide.u32), measured
// by the last zkmsm_measure_peaks call
extern "C" double zkmsm_wide_products_per_s(void) { return g_wide_products_per_s; }

extern "C" ZkMetalStatus zkmsm_sum_results_device(int curve, const void* d_results, uint32_t count, void* d_out,
                                                  void* stream) {
    if (!d_results || !d_out || count == 0) return ZKMETAL_ERR_INVALID_INPUT;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint32_t* in = static_cast<const uint32_t*>(d_results);
    uint32_t* out = static_cast<uint32_t*>(d_out);
    if (curve == ZKMSM_BN254) k_sum_results<Bn254><<<1, 32, 0, s>>>(in, count, out);
    else if (curve == ZKMSM_BLS12_381) k_sum_results<Bls381><<<1, 32, 0, s>>>(in, count, out);
    else if (curve == ZKMSM_BLS12_377) k_sum_results<Bls377><<<1, 32, 0, s>>>(in, count, out);
    else return ZKMETAL_ERR_INVALID_INPUT;
    return cudaGetLastError() == cudaSuccess ? ZKMETAL_SUCCESS : ZKMETAL_ERR_GPU_ERROR;
}

extern "C" ZkMetalStatus zkmsm_field_op(int curve, int op, const void* d_a, const void* d_b, void* d_out,
                                        uint32_t n) {
    if (!d_a || !d_b || !d_out || op < 0 || op > 2) return ZKMETAL_ERR_INVALID_INPUT;
    if (n == 0) return ZKMETAL_SUCCESS;
    const uint32_t* a = static_cast<const uint32_t*>(d_a);
    const uint32_t* b = static_cast<const uint32_t*>(d_b);
    uint32_t* o = static_cast<uint32_t*>(d_out);
    const unsigned g = (n + 127) / 128;
    if (curve == ZKMSM_BN254) k_field_op<Bn254Fp><<<g, 128>>>(op, a, b, o, n);
    else if (curve == ZKMSM_BLS12_381) k_field_op<Bls381Fp><<<g, 128>>>(op, a, b, o, n);
    else if (curve == ZKMSM_BLS12_377) k_field_op<Bls377Fp><<<g, 128>>>(op, a, b, o, n);
    else return ZKMETAL_ERR_INVALID_INPUT;
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return ZKMETAL_ERR_GPU_ERROR;
    return ZKMETAL_SUCCESS;
}

extern "C" ZkMetalStatus zkmsm_sum_results(int curve, const uint8_t* results, uint32_t count, uint8_t* out) {
    if (!results || !out || count == 0) return ZKMETAL_ERR_INVALID_INPUT;
    if (curve != ZKMSM_BN254 && curve != ZKMSM_BLS12_381 && curve != ZKMSM_BLS12_377) return ZKMETAL_ERR_INVALID_INPUT;
    size_t fb = curve == ZKMSM_BN254 ? 32 : 48;
    size_t in_bytes = (size_t)count * 3 * fb;
    uint32_t *d_in = nullptr, *d_out = nullptr;
    if (cudaMalloc(&d_in, in_bytes) != cudaSuccess || cudaMalloc(&d_out, 3 * fb) != cudaSuccess) {
        cudaFree(d_in);
        cudaGetLastError();
        return ZKMETAL_ERR_ALLOC_FAILED;
    }
    cudaMemcpy(d_in, results, in_bytes, cudaMemcpyHostToDevice);
    if (curve == ZKMSM_BN254) k_sum_results<Bn254><<<1, 32>>>(d_in, count, d_out);
    else if (curve == ZKMSM_BLS12_381) k_sum_results<Bls381><<<1, 32>>>(d_in, count, d_out);
    else k_sum_results<Bls377><<<1, 32>>>(d_in, count, d_out);
    cudaError_t e = cudaMemcpy(out, d_out, 3 * fb, cudaMemcpyDeviceToHost);
    cudaFree(d_in);
    cudaFree(d_out);
    return e == cudaSuccess ? ZKMETAL_SUCCESS : ZKMETAL_ERR_GPU_ERROR;
}
