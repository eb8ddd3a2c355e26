// war_batched.cu — the persistent refill kernel (war_enumerate): a grid of SMs x resident blocks runs the
// refill loop of war_refill.cuh over one job's work units, taken from one global atomic counter.
#include "war_refill.cuh"

namespace war {

template <int RULE, int G, bool CANON, bool SHAPE, bool EXTRA, int V>
__global__ void __launch_bounds__(G == 1 ? 1024 : (G == 2 ? 512 : 256)) batched_kernel(const __grid_constant__ BatchArgs a,
                                                                     DevAcc* __restrict__ acc) {
    extern __shared__ u32 sh[];
    refill_dispatch<RULE, G, CANON, SHAPE, EXTRA, V>(a, acc, &acc->work_next, sh);
}

// ---- dispatch over the compiled variants ----------------------------------------------------------

typedef void (*BatchedFn)(const BatchArgs, DevAcc*);

// Dynamic shared memory of a block: the cycle-length and ending-length histograms (u32 bins), then one
// 8-byte chunk cursor per thread (chunk_cursor in war_refill.cuh).
static size_t batched_shmem(int hbins, int threads) {
    return sizeof(u32) * (size_t)((hbins + WAR_EBINS + 1) & ~1) + sizeof(u64) * (size_t)threads;
}

template <int RULE, int G, int V>
static BatchedFn pick_g(int canon, int shape, int extra) {
    if (!canon) return extra ? batched_kernel<RULE, G, false, false, true, V> : batched_kernel<RULE, G, false, false, false, V>;
    if constexpr ((V & 4) != 0 && (V & 16) == 0) return nullptr;   // canonical scans: the path memo only
    if (shape) return extra ? batched_kernel<RULE, G, true, true, true, V> : batched_kernel<RULE, G, true, true, false, V>;
    return extra ? batched_kernel<RULE, G, true, false, true, V> : batched_kernel<RULE, G, true, false, false, V>;
}

template <int V>
static BatchedFn pick_v(int canon, int rule, int shape, int extra, int games) {
    if (games == 4) {   // four games per lane: compiled for the product variants only (3: no memo, 31: path memo)
        if constexpr (V == 3 || V == 31) return rule ? pick_g<1, 4, V>(canon, shape, extra) : pick_g<0, 4, V>(canon, shape, extra);
        return nullptr;
    }
    if (rule) return games == 2 ? pick_g<1, 2, V>(canon, shape, extra) : pick_g<1, 1, V>(canon, shape, extra);
    return games == 2 ? pick_g<0, 2, V>(canon, shape, extra) : pick_g<0, 1, V>(canon, shape, extra);
}

// variant: bit 0 = multiply-add turn form, bit 1 = latched records, bit 2 = cycle memo (deals, latched),
// bit 3 = the memo holds every cycle state (else landmarks), bit 4 = and the paths of decided games
static BatchedFn pick(int canon, int rule, int shape, int extra, int games, int variant) {
    if ((variant & 2) == 0 || (canon && (variant & 16) == 0)) variant &= 3;
    if ((variant & 4) == 0) variant &= 7;
    if ((variant & 8) == 0) variant &= 15;
    switch (variant) {
        case 1: return pick_v<1>(canon, rule, shape, extra, games);
        case 2: return pick_v<2>(canon, rule, shape, extra, games);
        case 3: return pick_v<3>(canon, rule, shape, extra, games);
        case 6: return pick_v<6>(canon, rule, shape, extra, games);
        case 7: return pick_v<7>(canon, rule, shape, extra, games);
        case 14: return pick_v<14>(canon, rule, shape, extra, games);
        case 15: return pick_v<15>(canon, rule, shape, extra, games);
        case 30: return pick_v<30>(canon, rule, shape, extra, games);
        case 31: return pick_v<31>(canon, rule, shape, extra, games);
        default: return pick_v<0>(canon, rule, shape, extra, games);
    }
}

cudaError_t launch_batched(const BatchArgs& a, int canon, int rule, int shape, const BatchShape& bs, DevAcc* acc,
                           cudaStream_t st) {
    int extra = (a.distinct || a.sample) ? 1 : 0;
    BatchedFn fn = pick(canon, rule, canon && shape, extra, bs.games, bs.variant);
    if (!fn) return cudaErrorInvalidConfiguration;
    fn<<<bs.blocks, bs.threads, batched_shmem(a.hbins, bs.threads), st>>>(a, acc);
    note_launch();
    return cudaGetLastError();
}

int batched_max_blocks_per_sm(int canon, int rule, int shape, int distinct, int sample, int threads, int games,
                              int hbins, int variant) {
    BatchedFn fn = pick(canon, rule, canon && shape, (distinct || sample) ? 1 : 0, games, variant);
    if (!fn) return 0;   // a combination that is not compiled (four games per lane outside variants 3 and 31)
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, batched_shmem(hbins, threads)) != cudaSuccess)
        return 0;
    return nb;
}

}  // namespace war
