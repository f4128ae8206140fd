// hbg_peaks.cu -- measured compute peaks of the pipes this library's kernels are bound by, for the
// rooflines of the benchmark: FP64 FMA (the FP64 residual products, the FP64 LU), FP64 warp MMA
// (mma.sync m8n8k4.f64) and TF32 tcgen05 MMA (the mixed LU's products).  Each kernel keeps its
// pipe busy from registers or shared memory only, and is timed with CUDA events.
#include <cuda_runtime.h>

namespace hbg {

// 8 independent FMA chains per thread, `iters` steps each.
__global__ void __launch_bounds__(256) k_peak_dfma(int iters, double seed, double* sink) {
    double a[8];
#pragma unroll
    for (int i = 0; i < 8; i++) a[i] = seed + threadIdx.x * 1e-9 + i;
    const double m = 0.999999999, c = 1e-12;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < 8; i++) a[i] = fma(a[i], m, c);
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; i++) s += a[i];
    if (s == 12345.678) sink[0] = s;  // never true: keeps the chains alive
}

// 4 independent m8n8k4 FP64 MMA accumulators per warp.
__global__ void __launch_bounds__(256) k_peak_dmma(int iters, double seed, double* sink) {
    double acc[4][2];
#pragma unroll
    for (int i = 0; i < 4; i++) acc[i][0] = acc[i][1] = 0.0;
    const double a = seed + (threadIdx.x & 31) * 1e-6, b = 1e-3;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int i = 0; i < 4; i++)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                         : "+d"(acc[i][0]), "+d"(acc[i][1])
                         : "d"(a), "d"(b));
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 4; i++) s += acc[i][0] + acc[i][1];
    if (s == 12345.678) sink[0] = s;
}

// One CTA per SM, one thread issuing tcgen05.mma kind::tf32 M=128 N=256 K=8 on fixed shared-memory
// operands into one TMEM accumulator, `iters` instructions, one commit at the end (bounded wait).
__global__ void __launch_bounds__(128) k_peak_tf32(int iters, int* err) {
    extern __shared__ __align__(1024) uint8_t pk_smem[];
    uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(pk_smem) + 1023) & ~uintptr_t(1023));
    float* sA = reinterpret_cast<float*>(base);          // 128 rows x 32 tf32, 128-byte swizzle
    float* sB = sA + 128 * 32;                            // 256 rows x 32
    uint64_t* done = reinterpret_cast<uint64_t*>(sB + 256 * 32);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
    for (int t = threadIdx.x; t < (128 + 256) * 32; t += blockDim.x) sA[t] = 0.f;
    if (threadIdx.x == 0) {
        tc::mbar_init(done, 1);
        tc::fence_barrier_init();
    }
    if (threadIdx.x < 32) tc::tmem_alloc(tslot, 256);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tslot;
    if (threadIdx.x == 0) {
        const uint32_t idesc = tc::idesc_tf32(128, 256);
        const uint64_t da = tc::desc_kmajor_sw128(tc::smem_u32(sA)), db = tc::desc_kmajor_sw128(tc::smem_u32(sB));
        for (int it = 0; it < iters; it++) tc::mma_tf32(tmem, da, db, idesc, it > 0);
        tc::mma_commit(done);
        if (!tc::mbar_wait(done, 0)) atomicExch(err, 1);
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    if (threadIdx.x < 32) tc::tmem_dealloc(tmem, 256);
}

// out[0] FP64 FMA TFLOP/s, out[1] FP64 MMA TFLOP/s, out[2] TF32 tcgen05 TFLOP/s (dense).
int measure_peaks(double* out, const char** msg) {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    double* sink = nullptr;
    int* err = nullptr;
    if (cudaMalloc(&sink, 64) != cudaSuccess || cudaMalloc(&err, sizeof(int)) != cudaSuccess) {
        *msg = "allocation failed";
        return HB_ERR_INTERNAL;
    }
    cudaMemset(err, 0, sizeof(int));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto timed = [&](auto launch) {
        launch();  // warm-up
        cudaEventRecord(e0);
        launch();
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return (double)ms * 1e-3;
    };
    const int blocks = nsm * 8, it64 = 1 << 14;
    double t = timed([&] { k_peak_dfma<<<blocks, 256>>>(it64, 1.0, sink); });
    out[0] = 2.0 * 8.0 * it64 * (double)blocks * 256 / t * 1e-12;
    t = timed([&] { k_peak_dmma<<<blocks, 256>>>(it64 / 4, 1.0, sink); });
    out[1] = 512.0 * 4.0 * (it64 / 4) * (double)blocks * 8 / t * 1e-12;
    const int smem = (128 + 256) * 32 * 4 + 2048;
    cudaFuncSetAttribute(k_peak_tf32, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    const int it32 = 1 << 16;
    t = timed([&] { k_peak_tf32<<<nsm, 128, smem>>>(it32, err); });
    out[2] = 2.0 * 128 * 256 * 8 * (double)it32 * nsm / t * 1e-12;
    int herr = 0;
    cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    cudaFree(err);
    if (cudaGetLastError() != cudaSuccess || herr) {
        *msg = "peak measurement failed";
        return HB_ERR_INTERNAL;
    }
    return 0;
}

}  // namespace hbg
