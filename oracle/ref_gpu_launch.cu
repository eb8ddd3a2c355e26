// ref_gpu_launch.cu — TEST INFRASTRUCTURE: drives the reference's own CUDA kernels war_count / war_canon
// (the KERNEL string of gpu/war_gpu.py, extracted unmodified into _ref/war_gpu_kernel.cu) with a
// restatement of run()'s launch loop (gpu/war_gpu.py:272-328): the same per, threads and batch_threads,
// one launch per span and a device synchronisation after each, as CuPy does.  Used only to compare the
// reference's GPU path with this repository's kernels on the same GPU (tests and oracle/ref_gpu.py).
#include <cuda_runtime.h>
#include <chrono>
#include <cstdint>
#include <cstring>
#include "_ref/war_gpu_kernel.cu"

extern "C" int ref_gpu_run(int n, int canon, int half, int rule, int hbins, int dbins, int blk, int per, int threads,
                           long long batch_threads, unsigned long long* out /* cyc, done, maxfin, shape0, shape1 */,
                           unsigned long long* hist, unsigned long long* dhist, double* ms) {
    u64 fact_h[17];
    fact_h[0] = 1;
    for (int i = 1; i <= 16; i++) fact_h[i] = fact_h[i - 1] * (u64)i;
    u64 total = canon ? fact_h[n - 1] : fact_h[n];
    if (canon) batch_threads = batch_threads / (n - 1 > 1 ? n - 1 : 1) > (1 << 12) ? batch_threads / (n - 1 > 1 ? n - 1 : 1) : (1 << 12);
    batch_threads = (batch_threads / threads) * threads;
    if (batch_threads < threads) batch_threads = threads;
    u64 *fact, *acc, *h, *shp, *dh;
    if (cudaMalloc(&fact, sizeof fact_h) || cudaMalloc(&acc, 3 * 8) || cudaMalloc(&h, 8 * (hbins > 1 ? hbins : 1)) ||
        cudaMalloc(&shp, 16) || cudaMalloc(&dh, 8 * (dbins > 1 ? dbins : 1)))
        return -1;
    cudaMemcpy(fact, fact_h, sizeof fact_h, cudaMemcpyHostToDevice);
    cudaMemset(acc, 0, 24); cudaMemset(h, 0, 8 * (hbins > 1 ? hbins : 1)); cudaMemset(shp, 0, 16);
    cudaMemset(dh, 0, 8 * (dbins > 1 ? dbins : 1));
    auto t0 = std::chrono::steady_clock::now();
    for (u64 start = 0; start < total; start += (u64)batch_threads * per) {
        u64 nthreads = (total - start + per - 1) / per;
        if (nthreads > (u64)batch_threads) nthreads = batch_threads;
        unsigned blocks = (unsigned)((nthreads + threads - 1) / threads);
        if (canon)
            war_canon<<<blocks, threads, 4 * hbins>>>(n, start, total, per, fact, blk, acc, acc + 1, acc + 2, h, hbins, shp,
                                                      rule, dh, dbins);
        else
            war_count<<<blocks, threads, 4 * hbins>>>(n, start, total, per, fact, (half ? 1 : 0) | (rule ? 2 : 0), acc,
                                                      acc + 1, acc + 2, h, hbins);
        if (cudaDeviceSynchronize() != cudaSuccess) return -2;
    }
    *ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    cudaMemcpy(out, acc, 24, cudaMemcpyDeviceToHost);
    cudaMemcpy(out + 3, shp, 16, cudaMemcpyDeviceToHost);
    if (hbins) cudaMemcpy(hist, h, 8 * hbins, cudaMemcpyDeviceToHost);
    if (dbins) cudaMemcpy(dhist, dh, 8 * dbins, cudaMemcpyDeviceToHost);
    cudaFree(fact); cudaFree(acc); cudaFree(h); cudaFree(shp); cudaFree(dh);
    return 0;
}
