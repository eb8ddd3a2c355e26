// war_peak.cu — measures the GPU's integer instruction throughput, the denominator of the roofline
// of an integer-bound kernel.  Two streams of independent 32-bit integer instructions, eight chains
// per thread so that latency is hidden:
//   alu   : LOP3 only (the ALU pipe)
//   issue : LOP3 and IMAD alternating (ALU and FMA pipes), the best case for the issue slots
// Each kernel runs a persistent grid of SMs x 2048 threads.
#include <cuda_runtime.h>
#include "war_host.h"

namespace war {

template <bool MIXED>
__global__ void __launch_bounds__(1024) int_peak_kernel(u32 iters, u32 seed, u32* out) {
    u32 a0 = seed ^ threadIdx.x, a1 = a0 * 3u, a2 = a0 * 5u, a3 = a0 * 7u, a4 = a0 * 11u, a5 = a0 * 13u,
        a6 = a0 * 17u, a7 = a0 * 19u;
    const u32 b = seed * 0x9E3779B9u + blockIdx.x, c = seed ^ 0x85EBCA6Bu;
    for (u32 i = 0; i < iters; i++) {
#define WAR_LOP(x) asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(x) : "r"(b), "r"(c))
#define WAR_MAD(x) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(x) : "r"(b), "r"(c))
        if (MIXED) {
            WAR_LOP(a0); WAR_MAD(a1); WAR_LOP(a2); WAR_MAD(a3); WAR_LOP(a4); WAR_MAD(a5); WAR_LOP(a6); WAR_MAD(a7);
            WAR_MAD(a0); WAR_LOP(a1); WAR_MAD(a2); WAR_LOP(a3); WAR_MAD(a4); WAR_LOP(a5); WAR_MAD(a6); WAR_LOP(a7);
        } else {
            WAR_LOP(a0); WAR_LOP(a1); WAR_LOP(a2); WAR_LOP(a3); WAR_LOP(a4); WAR_LOP(a5); WAR_LOP(a6); WAR_LOP(a7);
            WAR_LOP(a0); WAR_LOP(a1); WAR_LOP(a2); WAR_LOP(a3); WAR_LOP(a4); WAR_LOP(a5); WAR_LOP(a6); WAR_LOP(a7);
        }
#undef WAR_LOP
#undef WAR_MAD
    }
    u32 r = a0 ^ a1 ^ a2 ^ a3 ^ a4 ^ a5 ^ a6 ^ a7;
    if (r == 0x12345678u) out[0] = r;   // keeps the chains live
}

}  // namespace war

using namespace war;

extern "C" int war_measure_int_peak(double* issue_ops_per_s, double* alu_ops_per_s) {
    if (!issue_ops_per_s || !alu_ops_per_s) return fail(WAR_EINVAL, "NULL output");
    int st = ensure_ready();
    if (st) return st;
    std::lock_guard<std::mutex> lk(ctx().mu);
    Ctx& c = ctx();
    cudaStream_t s = cur_stream();
    const int threads = 1024, blocks = c.sm_count * 2;
    const u32 iters = 1u << 14;
    u32* out = (u32*)c.d_acc;   // scratch word, never written in practice
    double res[2];
    for (int v = 0; v < 2; v++) {
        float best = 1e30f;
        for (int rep = 0; rep < 4; rep++) {
            cudaEventRecord(c.ev0, s);
            if (v == 0) int_peak_kernel<true><<<blocks, threads, 0, s>>>(iters, 12345u + rep, out);
            else int_peak_kernel<false><<<blocks, threads, 0, s>>>(iters, 12345u + rep, out);
            note_launch();
            cudaEventRecord(c.ev1, s);
            cudaError_t e = cudaEventSynchronize(c.ev1);
            if (e != cudaSuccess) return cuda_fail(e, "int peak kernel");
            float ms = 0.f;
            cudaEventElapsedTime(&ms, c.ev0, c.ev1);
            if (rep > 0 && ms < best) best = ms;
        }
        double ops = (double)blocks * threads * iters * 16.0;
        res[v] = ops / (best * 1e-3);
    }
    *issue_ops_per_s = res[0];
    *alu_ops_per_s = res[1];
    return WAR_OK;
}
