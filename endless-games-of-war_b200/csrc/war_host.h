// war_host.h — host-side state and helpers shared by the C ABI translation units.
#pragma once
#include <cuda_runtime.h>
#include <mutex>
#include <vector>
#include "war_kernels.cuh"

namespace war {

struct Ctx {
    static constexpr size_t UNIT_CAP = 1 << 16;
    std::mutex mu;                  // serialises calls that launch work
    bool ready = false;
    int device = 0, sm_count = 0;
    cudaStream_t own_stream = nullptr, user_stream = nullptr;
    DevAcc* d_acc = nullptr;        // accumulators of the running job
    DevAcc* h_acc = nullptr;        // pinned mirror
    Unit* d_units = nullptr;        // extra work units of the running job
    ulonglong2* d_sample = nullptr; // Floyd sample buffer
    size_t sample_cap = 0;
    u64* d_memo = nullptr;          // cycle memo table of the refill kernel (deals)
    int memo_bits = 0;
    int memo_n = -1, memo_rule = -1;  // job class whose cycles the memo holds
    int memo_kind = 0;                // its entry layout (prepare_memo): engine, memo form, shape values
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

struct Plan {
    int m = 0;
    u64 main_base = 0, main_count = 0;
    u64 games_per_order = 1;
    std::vector<Unit> extra;
};

struct Tune {
    int threads, blocks_per_sm, games, block_m, window, defer, variant, memo_bits, chunk;
};

Ctx& ctx();
int ensure_ready();
cudaStream_t cur_stream();
int fail(int code, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
u64 fact(int i);
u64 space_size(int n, int mode);
int check_job(const war_job* j);
void make_plan(const war_job* job, int m, Plan& p);
void merge_acc(const DevAcc& h, war_result* r, int hbins, int dbins);
void fill_fact(u64* f);
int resolve_tune(const war_job* job, const war_tune* in, Tune& t);
int floyd_sample_run(const war_job* job, war_result* out);

// Zeroes the device accumulators, runs `launch`, copies them back into c.h_acc.  Times the launch
// with events on the launching stream.
template <typename F>
inline int run_launch(F launch, double* ms) {
    Ctx& c = ctx();
    cudaStream_t st = cur_stream();
    cudaError_t e;
    if ((e = cudaMemsetAsync(c.d_acc, 0, sizeof(DevAcc), st)) != cudaSuccess) return cuda_fail(e, "memset acc");
    if ((e = cudaEventRecord(c.ev0, st)) != cudaSuccess) return cuda_fail(e, "event record");
    if ((e = launch(st)) != cudaSuccess) return cuda_fail(e, "kernel launch");
    if ((e = cudaEventRecord(c.ev1, st)) != cudaSuccess) return cuda_fail(e, "event record");
    if ((e = cudaMemcpyAsync(c.h_acc, c.d_acc, sizeof(DevAcc), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "copy acc");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "kernel execution");
    float f = 0.f;
    cudaEventElapsedTime(&f, c.ev0, c.ev1);
    if (ms) *ms += f;
    if (c.h_acc->status) return fail(WAR_ECAP, "%llu game(s) passed the turn cap", (unsigned long long)c.h_acc->status);
    return WAR_OK;
}

cudaError_t launch_sample_scan(const FloydArgs& a, int threads, u64 nthreads, ulonglong2* buf, u64 cap, DevAcc* acc,
                               cudaStream_t st);
cudaError_t launch_floyd_enum(const FloydArgs& a, int blocks, DevAcc* acc, cudaStream_t st);
int floyd_enum_blocks_per_sm(int canon, int rule);
cudaError_t launch_floyd_play(const ulonglong2* buf, u64 cap, int n, int rule, int blocks, int threads, DevAcc* acc,
                              cudaStream_t st);

}  // namespace war
