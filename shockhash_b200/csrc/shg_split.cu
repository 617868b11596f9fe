// RecSplit split-seed search and stable partition, one launch per tree level (one block per node);
// the node's search is split_node in shg_split.cuh.
#include "shg_split.cuh"

namespace shg {

template <int SPL, int THREADS, int ARITH>
__global__ void __launch_bounds__(THREADS) k_split(const Node *__restrict__ nodes, const uint32_t *__restrict__ ids,
                                                   uint64_t *__restrict__ keys, uint64_t *__restrict__ codes,
                                                   uint64_t max_trials, uint32_t *__restrict__ err,
                                                   unsigned long long *__restrict__ work,
                                                   unsigned long long *__restrict__ kind_work, int round_div,
                                                   const PipeK K) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    SplitSmem<SPL, THREADS> &sm = *reinterpret_cast<SplitSmem<SPL, THREADS> *>(smem_raw);
    const uint32_t id = ids[blockIdx.x];
    split_node<SPL, THREADS, ARITH>(sm, nodes[id], id, keys, codes, max_trials, err, work, kind_work, round_div, K);
}

template <int SPL, int THREADS, int ARITH>
static void launch_split_t(const Node *nodes, const uint32_t *ids, uint32_t count, uint64_t *keys, uint64_t *codes,
                           uint64_t max_trials, uint32_t *err, unsigned long long *work, unsigned long long *kind_work,
                           int round_div, cudaStream_t s) {
    const size_t smem = sizeof(SplitSmem<SPL, THREADS>);
    cudaFuncSetAttribute(k_split<SPL, THREADS, ARITH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const PipeK K{4u, 32u, 1u << 18, 2u};
    k_split<SPL, THREADS, ARITH><<<count, THREADS, smem, s>>>(nodes, ids, keys, codes, max_trials, err, work, kind_work,
                                                              round_div, K);
}

// Parameters a tuning table may set (the SIMDShockHash form is chosen by the engine, not the table).
bool split_tuning_valid(int spl, int threads, int round_div, int arith) {
    return (spl == 1 || spl == 2 || spl == 4) && (threads == 128 || threads == 256 || threads == 512) && round_div >= 1 &&
           round_div <= 64 && (arith == 0 || arith == 1);
}

void launch_split_level(const Node *nodes, const uint32_t *ids, uint32_t count, uint64_t *keys, uint64_t *codes,
                        uint64_t max_trials, uint32_t *err, unsigned long long *work, unsigned long long *kind_work,
                        const SplitTuning &t, cudaStream_t s) {
    if (!count) return;
#define SHG_SPLIT_CASE(SPL, TH, AR)                                                                              \
    if (t.spl == SPL && t.threads == TH && t.arith == AR)                                                       \
        return launch_split_t<SPL, TH, AR>(nodes, ids, count, keys, codes, max_trials, err, work, kind_work,     \
                                           t.round_div, s);
    SHG_SPLIT_CASE(1, 128, 0) SHG_SPLIT_CASE(1, 256, 0) SHG_SPLIT_CASE(1, 512, 0)
    SHG_SPLIT_CASE(2, 128, 0) SHG_SPLIT_CASE(2, 256, 0) SHG_SPLIT_CASE(2, 512, 0)
    SHG_SPLIT_CASE(4, 128, 0) SHG_SPLIT_CASE(4, 256, 0) SHG_SPLIT_CASE(4, 512, 0)
    SHG_SPLIT_CASE(1, 128, 1) SHG_SPLIT_CASE(1, 256, 1) SHG_SPLIT_CASE(1, 512, 1)
    SHG_SPLIT_CASE(2, 128, 1) SHG_SPLIT_CASE(2, 256, 1) SHG_SPLIT_CASE(2, 512, 1)
    SHG_SPLIT_CASE(4, 128, 1) SHG_SPLIT_CASE(4, 256, 1) SHG_SPLIT_CASE(4, 512, 1)
    // SIMDShockHash: its own split hash, so never the remix forms' fallback below
    SHG_SPLIT_CASE(1, 128, 2) SHG_SPLIT_CASE(1, 256, 2) SHG_SPLIT_CASE(1, 512, 2)
    SHG_SPLIT_CASE(2, 128, 2) SHG_SPLIT_CASE(2, 256, 2) SHG_SPLIT_CASE(2, 512, 2)
    SHG_SPLIT_CASE(4, 128, 2) SHG_SPLIT_CASE(4, 256, 2) SHG_SPLIT_CASE(4, 512, 2)
#undef SHG_SPLIT_CASE
    if (t.arith == kSplitArithSimd)
        return launch_split_t<2, 256, kSplitArithSimd>(nodes, ids, count, keys, codes, max_trials, err, work, kind_work,
                                                       t.round_div, s);
    launch_split_t<2, 256, 0>(nodes, ids, count, keys, codes, max_trials, err, work, kind_work, t.round_div, s);
}

} // namespace shg
