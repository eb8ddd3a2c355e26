// war_peak.cu — measures the two ceilings of the enumeration kernels on the running GPU.
//
// Integer issue (war_measure_int_peak), the roofline of the turn loop: streams of independent 32-bit
// integer instructions, eight chains per thread so that latency is hidden, 128 of them per loop iteration
// so that the loop's own counter, compare and branch take under 3% of the issue slots:
//   alu   : LOP3 only (the ALU pipe)
//   issue : LOP3 and IMAD alternating (ALU and FMA pipes), the best case for the issue slots
// Each kernel runs a persistent grid of SMs x 2048 threads.
//
// Random gathers (war_measure_gather_peak), the roofline of the cycle memo's lookups: independent loads of
// one 8-byte word (or one 32-byte bucket) at uniformly random positions of a multi-GB table, eight in
// flight per thread, the way the memo kernel reads its table.  The result is lookups per second; the DRAM
// bytes each one costs come from a profiler capture of the same kernel.
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
#pragma unroll
        for (int k = 0; k < 8; k++) {   // 8 x 16 = 128 instructions per iteration
            if (MIXED) {
                WAR_LOP(a0); WAR_MAD(a1); WAR_LOP(a2); WAR_MAD(a3); WAR_LOP(a4); WAR_MAD(a5); WAR_LOP(a6); WAR_MAD(a7);
                WAR_MAD(a0); WAR_LOP(a1); WAR_MAD(a2); WAR_LOP(a3); WAR_MAD(a4); WAR_LOP(a5); WAR_MAD(a6); WAR_LOP(a7);
            } else {
                WAR_LOP(a0); WAR_LOP(a1); WAR_LOP(a2); WAR_LOP(a3); WAR_LOP(a4); WAR_LOP(a5); WAR_LOP(a6); WAR_LOP(a7);
                WAR_LOP(a0); WAR_LOP(a1); WAR_LOP(a2); WAR_LOP(a3); WAR_LOP(a4); WAR_LOP(a5); WAR_LOP(a6); WAR_LOP(a7);
            }
        }
#undef WAR_LOP
#undef WAR_MAD
    }
    u32 r = a0 ^ a1 ^ a2 ^ a3 ^ a4 ^ a5 ^ a6 ^ a7;
    if (r == 0x12345678u) out[0] = r;   // keeps the chains live
}

// Eight independent random loads per iteration from a table of 2^bits words.  BUCKET: a 32-byte aligned
// bucket (two 16-byte loads of one sector) instead of one word.  Positions come from a 64-bit LCG per
// thread (top bits), so consecutive loads of a thread and of neighbouring threads are unrelated.
template <bool BUCKET>
__global__ void __launch_bounds__(256) gather_peak_kernel(const u64* __restrict__ table, u32 bits, u32 iters,
                                                          u64 seed, u64* out) {
    u64 x = war_mix64(seed ^ ((u64)blockIdx.x * blockDim.x + threadIdx.x));
    u64 acc = 0;
    const u32 sh = 64u - bits;
    for (u32 i = 0; i < iters; i++) {
        u64 v[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            x = x * 6364136223846793005ull + 1442695040888963407ull;
            u64 slot = x >> sh;
            if (BUCKET) {
                const ulonglong2* p = (const ulonglong2*)(table + (slot & ~3ull));
                ulonglong2 a = __ldcg(p), b = __ldcg(p + 1);
                v[k] = a.x ^ a.y ^ b.x ^ b.y;
            } else {
                v[k] = __ldcg((const unsigned long long*)table + slot);
            }
        }
#pragma unroll
        for (int k = 0; k < 8; k++) acc ^= v[k];
    }
    if (acc == 0x9E3779B97F4A7C15ull) out[0] = acc;   // keeps the loads live
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
    const u32 iters = 1u << 11;
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
        double ops = (double)blocks * threads * iters * 128.0;
        res[v] = ops / (best * 1e-3);
    }
    *issue_ops_per_s = res[0];
    *alu_ops_per_s = res[1];
    return WAR_OK;
}

extern "C" int war_measure_gather_peak(int32_t table_bits, int32_t bucket_bytes, double* lookups_per_s) {
    if (!lookups_per_s) return fail(WAR_EINVAL, "NULL output");
    if (table_bits < 20 || table_bits > 31) return fail(WAR_EINVAL, "table_bits=%d (20..31)", table_bits);
    if (bucket_bytes != 8 && bucket_bytes != 32) return fail(WAR_EINVAL, "bucket_bytes=%d (8 or 32)", bucket_bytes);
    int st = ensure_ready();
    if (st) return st;
    std::lock_guard<std::mutex> lk(ctx().mu);
    Ctx& c = ctx();
    cudaStream_t s = cur_stream();
    cudaError_t e;
    // the memo table when it has this size (its contents do not matter), else a table of our own
    u64* table = (c.d_memo && c.memo_bits == table_bits) ? c.d_memo : nullptr;
    u64* own = nullptr;
    if (!table) {
        if ((e = cudaMalloc(&own, sizeof(u64) << table_bits)) != cudaSuccess) return cuda_fail(e, "cudaMalloc gather table");
        table = own;
    }
    const int threads = 256, blocks = c.sm_count * 8;
    const u32 iters = 256;
    u64* out = (u64*)c.d_acc;
    float best = 1e30f;
    e = cudaSuccess;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(c.ev0, s);
        if (bucket_bytes == 32) gather_peak_kernel<true><<<blocks, threads, 0, s>>>(table, (u32)table_bits, iters, 77u + rep, out);
        else gather_peak_kernel<false><<<blocks, threads, 0, s>>>(table, (u32)table_bits, iters, 77u + rep, out);
        note_launch();
        cudaEventRecord(c.ev1, s);
        if ((e = cudaEventSynchronize(c.ev1)) != cudaSuccess) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c.ev0, c.ev1);
        if (rep > 0 && ms < best) best = ms;
    }
    if (own) cudaFree(own);
    if (e != cudaSuccess) return cuda_fail(e, "gather peak kernel");
    *lookups_per_s = (double)blocks * threads * iters * 8.0 / (best * 1e-3);
    return WAR_OK;
}
