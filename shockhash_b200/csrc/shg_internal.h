// Internal declarations shared by the engine's translation units (not part of the C ABI).
#pragma once
#include <cstdint>
#include <string>
#include <memory>
#include <vector>
#include <cuda_runtime.h>
#include "shg.h"
#include "shg_common.cuh"

namespace shg {

// Node kinds of the RecSplit tree.
enum NodeKind : uint8_t { kLeaf = 0, kSplit2 = 1, kSplitK = 2 };

// One tree node as the device sees it (16 bytes). `start` is the global offset of the node's first
// key in the bucket-ordered key array; `unit` is the split point (fanout 2) or the part size.
struct __align__(16) Node {
    uint32_t start;
    uint16_t m;
    uint8_t level;  // index into start_seed of the node's search: its depth, except SIMDShockHash's
                    // aggregation nodes and leaves (kSimdSeed*)
    uint8_t kind;
    uint32_t bucket;
    uint16_t unit;
    uint8_t fanout;
    uint8_t g;  // Golomb-Rice parameter of the node's code
};
static_assert(sizeof(Node) == 16, "Node must stay 16 bytes");

// Splitting thresholds and the Golomb-Rice memo of one configuration.
// ShockHash<l>: lower = l*(l>24?4:2), upper = lower*(l>24?3:2) (ShockHash.h:63-72);
// ShockHash2<l>: lower = 4l, upper = 12l (ShockHash2.h:49-56).
// ShockHash<l, true> shares the tree, memo tables and retrieval layout of ShockHash<l, false>.
// SIMDShockHash<l, rot> shares them too; it differs in the split hash and the start seeds.
SHG_HD bool is_simd(int variant) { return variant == SHG_SIMDSHOCKHASH || variant == SHG_SIMDSHOCKHASH_ROTATION; }
SHG_HD bool is_sh1(int variant) {
    return variant == SHG_SHOCKHASH || variant == SHG_SHOCKHASH_ROTATION || is_simd(variant);
}
SHG_HD bool is_rotation(int variant) { return variant == SHG_SHOCKHASH_ROTATION || variant == SHG_SIMDSHOCKHASH_ROTATION; }
// The index into start_seed of a node's search. ShockHash and ShockHash2 start every node at its
// depth (ShockHash.h:309); SIMDShockHash starts fanout-2 nodes at their depth (SIMDShockHash.hpp:209)
// and uses fixed entries for the lower aggregation level (:582, start_seed[17]), the leaf
// aggregation level (:593, start_seed[18]) and the leaves (:411, start_seed[19]).
constexpr int kSimdSeedLower = kMaxLevels - 3, kSimdSeedLeafAggr = kMaxLevels - 2, kSimdSeedLeaf = kMaxLevels - 1;

struct ShapeCache;  // tree shapes by bucket size, built on first use (shg_plan.cpp)
struct Config {
    int variant = 0, leaf = 0;
    uint32_t lower = 0, upper = 0;
    std::vector<uint64_t> memo;  // kMaxBucket entries, fill_golomb_rice(2) layout
    std::shared_ptr<ShapeCache> shapes;  // shared by copies; kept across builds
    Config() {}
    Config(int variant, int leaf);
    int golomb(uint32_t m) const { return (int)(memo[m] >> 27); }
    uint32_t skip_bits(uint32_t m) const { return (uint32_t)(memo[m] & 0xFFFF); }
    uint32_t skip_nodes(uint32_t m) const { return (uint32_t)((memo[m] >> 16) & 0x7FF); }
};

// Tree of one bucket size, in preorder (the order the reference appends codes, ShockHash.h:303-555).
struct TNode {
    uint16_t rel;        // first key relative to the bucket start
    uint16_t m;
    uint8_t level, kind, fanout, g;
    uint8_t seed;        // index into start_seed of the node's search
    uint16_t unit;
    uint16_t fixed_off;  // bit offset of the node's fixed part within the bucket
};
struct Shape {
    std::vector<TNode> nodes;
    std::vector<uint16_t> singles;  // relative positions of size-1 children (no code, no retrieval bit)
    int depth = 0;
};
const Shape &shape_of(const Config &c, uint32_t m, std::vector<Shape> &cache, std::vector<char> &have);

// Every tree shape of one configuration for bucket sizes 0 .. rows-1, laid out for the device,
// which expands the plan of a build from it (k_plan_scan, k_plan_expand). Per size m, row m of
// `cnt` holds its node count, its size-1 children, its leaves and its split nodes per level
// (columns kColNodes, kColSingles, kColLeaves, kColLevel0 + level); its nodes sit in preorder at
// nodes[node_off[m] .. node_off[m + 1]), each with its rank in its launch list (the leaves, or the
// split nodes of its level) within the shape; its size-1 children in ascending order at
// singles[single_off[m] .. single_off[m + 1]).
enum : int { kColNodes = 0, kColSingles = 1, kColLeaves = 2, kColLevel0 = 3 };
constexpr int kMaxPlanCols = kColLevel0 + kMaxLevels;
struct __align__(16) ShapeNode {
    uint16_t rel, m;
    uint8_t level, kind, fanout, g;
    uint16_t unit, fixed_off, rank, seed;  // seed: index into start_seed of the node's search
};
static_assert(sizeof(ShapeNode) == 16, "ShapeNode must stay 16 bytes");
struct ShapeTables {
    uint32_t rows = 0;
    int ncol = kColLevel0;
    std::vector<uint32_t> cnt;  // [rows][ncol]
    std::vector<ShapeNode> nodes;
    std::vector<uint32_t> node_off;  // [rows + 1]
    std::vector<uint16_t> singles;
    std::vector<uint32_t> single_off;  // [rows + 1]
};
void make_shape_tables(const Config &c, uint32_t rows, ShapeTables &t);

// Start of each launch list in the id array of a build: split levels in order, then the leaves.
struct ListOffsets {
    uint32_t level[kMaxLevels];
    uint32_t leaf;
};

// ShockHash2Flat<k> constants (ShockHash2Flat.h:16-46).
struct FlatConsts {
    uint32_t k = 0, threshold_bits = 0, threshold_range = 0, seed_bits = 0;
    std::vector<uint32_t> mapping;  // THRESHOLD_MAPPING
};
FlatConsts flat_consts(uint32_t k);
void flat_launch_murmur(const uint8_t *bytes, const uint64_t *offsets, uint64_t n, uint64_t *out, cudaStream_t s);
void flat_launch_count(uint64_t *mhc, uint64_t n, uint32_t nb, bool rehash, uint32_t *counts, cudaStream_t s);
void flat_launch_scatter(const uint64_t *mhc, uint64_t n, uint32_t nb, uint32_t *cursor, uint64_t *out, cudaStream_t s);
void flat_launch_sort_flush(uint64_t *keys, const uint64_t *acc, uint32_t nb, uint32_t k, const uint32_t *mapping,
                            uint32_t range, uint64_t layer_base, uint8_t *thr, uint64_t *free_cnt, uint64_t *bump_cnt,
                            uint32_t *bump_first, uint32_t *err, cudaStream_t s);
void flat_launch_emit(const uint64_t *keys, const uint64_t *acc, uint32_t nb, uint64_t layer_base, const uint64_t *free_cnt,
                      const uint64_t *free_off, const uint64_t *bump_cnt, const uint64_t *bump_off, const uint32_t *bump_first,
                      uint64_t *free_out, uint64_t *bump_out, cudaStream_t s);
void flat_launch_assign(const uint64_t *mhc0, uint64_t n, uint32_t layers, const uint64_t *layer_bases, const uint8_t *thr,
                        const uint32_t *mapping, uint64_t *bucket, uint64_t *last_mhc, cudaStream_t s);
void flat_launch_fallback_list(const uint64_t *bucket, uint64_t n, unsigned long long *count, uint64_t *list, cudaStream_t s);
void flat_launch_gather(const uint64_t *idx, const uint64_t *src, uint64_t cnt, uint64_t *out, cudaStream_t s);
void flat_launch_set_buckets(const uint64_t *idx, const uint64_t *val, uint64_t cnt, uint64_t *bucket, cudaStream_t s);
void flat_launch_group(const uint64_t *bucket, uint64_t n, uint64_t nbuckets, uint32_t k, uint32_t *cursor,
                       uint32_t *slot_idx, const uint64_t *mhc0, uint64_t *leaf_keys, uint32_t *err, cudaStream_t s);

// Records the message returned by shg_last_error() on this thread and passes the status through.
shg_status shg_set_error(shg_status st, const std::string &msg);

// Device error flag bits.
enum : uint32_t { kErrTrialLimit = 1, kErrScratch = 2, kErrBucket = 4, kErrInternal = 8, kErrArg = 16 };

// ----------------------------------------------------------------- kernels (shg_kernels.cu)
void launch_spooky_u64(const uint64_t *keys, uint64_t n, uint64_t *first, uint64_t *second, cudaStream_t s);
void launch_spooky_strings(const uint8_t *bytes, const uint64_t *offsets, uint64_t n, uint64_t *first,
                           uint64_t *second, cudaStream_t s);
void launch_bucket_count(const uint64_t *first, uint64_t n, uint64_t nb, uint64_t nb_map, uint64_t b0, uint32_t *counts,
                         uint32_t *err, cudaStream_t s);
void launch_scan_counts(const uint32_t *counts, uint64_t nb, uint64_t *acc, uint32_t *cursor, uint32_t *maxsz,
                        cudaStream_t s);
void launch_bucket_scatter(const uint64_t *first, uint64_t n, uint64_t nb, uint64_t nb_map, uint64_t b0, uint32_t *cursor,
                           uint64_t *sfirst, uint32_t *sidx, uint64_t idx_base, cudaStream_t s);
void launch_bucket_sort(const uint64_t *acc, uint64_t nb, const uint64_t *sfirst, const uint32_t *sidx,
                        const uint64_t *second, uint64_t *keys, cudaStream_t s);
// Speed-only launch parameters of the search kernels for one configuration (variant, leaf size):
// every choice gives identical results. The defaults are the untuned values; a tuning table
// (shg_engine_load_tuning) replaces them per configuration.
struct SplitTuning {
    int spl = 2;         // seeds per lane: 1, 2 or 4
    int threads = 256;   // threads per split block (one node per block): 128, 256 or 512
    int round_div = 8;   // warp groups make a round about 1/round_div of a node's expected trials (1..64)
    int arith = 0;       // 0: remix as the compiler schedules it; 1: split between integer and multiply pipes;
                         // kSplitArithSimd: SIMDShockHash's split hash (set by the engine, not by the table)
};
constexpr int kSplitArithSimd = 2;
struct Tuning {
    SplitTuning split;
    int leaf_bps = 0;    // leaf grid in blocks per SM (0: as many as shared memory allows, at most 8)
    int leaf_minb = 6;   // bipartite leaves of up to 64 keys: launch bound of 4, 6 or 8 blocks per SM
    int sh1_spl = 2;     // original leaves: seeds per lane, 1 or 2
    int queue_lag = 8;   // work-queue item order: lag between a bucket's levels in rounds of the grid
                         // (0: none, the levels one after another and the leaves last; 1..64)
};
bool split_tuning_valid(int spl, int threads, int round_div, int arith);
constexpr int kTuningFlat = 4;  // tuning-table variant key of ShockHash2Flat<k> (leaf size = k)
// work[0] += useful evaluations; kind_work[k] += the same per inner loop (k = compared thresholds
// - 1, or 3 for quarter-split moments)
void launch_split_level(const Node *nodes, const uint32_t *ids, uint32_t count, uint64_t *keys,
                        uint64_t *codes, uint64_t max_trials, uint32_t *err, unsigned long long *work,
                        unsigned long long *kind_work, const SplitTuning &t, cudaStream_t s);
int leaves_sh1_warps_per_block();
// Inner-loop peaks of the bipartite leaf search (kind 0 scan, 1 pair filter, 2 pseudoforest edges),
// 256-thread blocks; operations per thread and iteration from sh2_op_peak_per_iter.
void launch_sh2_op_peak(int kind, int blocks, uint64_t iters, unsigned long long *sink);
int sh2_op_peak_per_iter(int kind);
// The work-queue schedule of a ShockHash2 build with leaves of up to 64 keys (shg_leaves_sh2.cu):
// the split nodes and leaves of the launch lists `ids` ([0, nsplit) the split levels in order, then
// the leaves) in one persistent launch of `grid` blocks, taken in the order of `seq` (*nitems items,
// both from launch_queue_order); offs/stride/nlevels are the plan's per-bucket list offsets,
// done[nbuckets] zeroed counters, ctr[2] zeroed item counters.
// Where the queue kernel writes request r's retrieval input (out[r]; buckets from b_first on, keys
// from key_off, size-1 positions from single_off in the batch's arrays): compacted keys and bits,
// host-mapped pinned memory.
struct QueueOut {
    uint64_t b_first, key_off, single_off;
    uint64_t *keys;
    uint8_t *bits;
};
int tree_queue_warps_per_block();
int tree_queue_smem_per_block(int spl);
// Time slots T of the staggered item order (nb + nlevels * lag); launch_queue_order writes the items
// into seq[0 .. nsplit + buckets with leaves), with scratch cnt[T] and pos[T + 1] (pos[T]: the
// item count). Without groups the sequence holds the split nodes only, and the queue kernel is
// given nleaf_tail = the leaf count: its warps take the leaves one by one after the last item.
uint64_t queue_order_slots(uint64_t nb, uint32_t nlevels, uint32_t lag);
void launch_queue_order(const uint32_t *offs, uint64_t stride, uint64_t nb, uint32_t nlevels, uint32_t lag, bool groups,
                        const ListOffsets &lists, uint32_t nsplit, uint32_t *cnt, uint32_t *pos, uint32_t *seq,
                        cudaStream_t s);
void launch_tree_queue(const Node *nodes, const uint32_t *ids, const uint32_t *seq, const uint32_t *nitems, uint32_t nsplit,
                       const uint32_t *offs, uint64_t stride, uint32_t nlevels, uint32_t *done, uint64_t *keys,
                       uint64_t *codes, uint8_t *rib_bits, uint8_t *scratch, uint64_t per_warp, uint32_t smax, uint32_t cmax,
                       uint64_t max_trials, uint32_t *err, unsigned long long *work, unsigned long long *kind_work,
                       unsigned int *ctr, uint32_t nleaf_tail, const uint64_t *acc, const uint64_t *singles,
                       const QueueOut *out, uint32_t nreq, const SplitTuning &t, int grid, cudaStream_t s);
void launch_gr_bucket_bits(const Node *nodes, const uint32_t *bnb, uint64_t nb, const uint64_t *acc,
                           const uint64_t *codes, const uint32_t *memo_skip_bits, uint64_t *bucket_bits,
                           cudaStream_t s);
void launch_scan_u64(const uint64_t *in, uint64_t n, uint64_t *out_excl_plus_total, cudaStream_t s);
void launch_gr_write(const Node *nodes, const uint16_t *fixed_off, const uint32_t *bnb, uint64_t nb,
                     const uint64_t *acc, const uint64_t *pos_acc, const uint64_t *codes,
                     const uint32_t *memo_skip_bits, unsigned long long *words, cudaStream_t s);
void launch_set_bit(unsigned long long *words, uint64_t bit, cudaStream_t s);
void launch_compact_ribbon(const uint64_t *keys, const uint8_t *bits, uint64_t n, const uint64_t *singles,
                           uint64_t nsingles, uint64_t single_base, uint64_t *out_keys, uint8_t *out_bits,
                           cudaStream_t s);
void launch_plan_scan(const uint64_t *acc, uint64_t nb, const uint32_t *cnt, uint32_t rows, int ncol, uint32_t *offs,
                      cudaStream_t s);
void launch_plan_expand(const uint64_t *acc, uint64_t nb, uint32_t rows, const uint32_t *offs, const ShapeNode *shape_nodes,
                        const uint32_t *node_off, const uint16_t *shape_singles, const uint32_t *single_off,
                        const ListOffsets &lists, Node *nodes, uint16_t *fixed_off, uint32_t *ids, uint64_t *singles,
                        cudaStream_t s);

} // namespace shg
