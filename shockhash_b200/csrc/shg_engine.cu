// Engine: device buffers, the build pipeline and the C ABI (include/shg.h).
//
// Pipeline of one build (all on the engine's stream):
//   hash (optional) -> bucket count/scan -> scatter + per-bucket sort  [partition, Sorter.hpp:15-36]
//   -> plan of the RecSplit trees: per-size shapes stamped out per bucket [ShockHash.h:303-555]
//   -> split-seed search per tree level                                 [ShockHash.h:451-547]
//   -> leaf searches                                                    [ShockHash.h:404-434 / ShockHash2.h:267-285]
//   -> Golomb-Rice encode                                               [RiceBitVector.h:67-127]
//   -> copy-out of descriptors, accumulators and retrieval input.
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include <dlfcn.h>
#include <cuda_runtime.h>
#include "shg.h"
#include "shg_common.cuh"
#include "shg_internal.h"

namespace shg {
uint64_t sh2_scratch_bytes(uint32_t smax, uint32_t cmax, int max_leaf);
void launch_leaves_sh1_ctr(const Node *nodes, const uint32_t *ids, uint32_t count, const uint64_t *keys, uint64_t *codes,
                           uint64_t *rib_keys, uint8_t *rib_bits, uint64_t max_trials, uint32_t *err,
                           unsigned long long *work, unsigned int *ctr, int grid, cudaStream_t s, uint32_t rot_leaf = 0,
                           int spl = 2);
void launch_leaves_sh2_ctr(const Node *nodes, const uint32_t *ids, uint32_t count, const uint64_t *keys, uint64_t *codes,
                           uint8_t *rib_bits, uint8_t *scratch, uint64_t scratch_per_warp, uint32_t smax, uint32_t cmax,
                           uint32_t *err, unsigned long long *work, unsigned int *ctr, int grid, cudaStream_t s,
                           int max_leaf, uint32_t quad_min = kQuadMinRecSplit, int minb = 6);
int sh2_smem_per_warp(int max_leaf);
int leaves_sh1_warps_per_block();
} // namespace shg

using namespace shg;

static thread_local std::string g_last_error;

static shg_status fail(shg_status st, const std::string &msg) {
    g_last_error = msg;
    return st;
}

namespace shg {
shg_status shg_set_error(shg_status st, const std::string &msg) { return fail(st, msg); }
} // namespace shg

#define CU(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return fail(SHG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = std::max<size_t>(bytes, 256);
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    template <class T> T *as() const { return (T *)p; }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

} // namespace

// Pinned host block that a result's arrays live in; reused across builds once released. One
// process-wide mutex guards every engine's pool, so a result can be released from any thread and
// after its engine is gone: the engine's destructor frees the idle blocks and orphans the ones
// still held by results (eng = nullptr), which are freed when those results are released.
struct PinnedBlock {
    void *p = nullptr;
    size_t cap = 0;
    bool in_use = false;
    bool host = false;  // plain malloc (merged shards), freed on release
    int refs = 0;       // results that point into the block (a batch's results share one)
    shg_engine *eng = nullptr;
};
static std::mutex g_pool_mu;

static void release_pinned(PinnedBlock *b) {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (--b->refs > 0) return;
    if (b->eng) {
        b->in_use = false;
        return;
    }
    if (b->host)
        free(b->p);
    else if (b->p)
        cudaFreeHost(b->p);
    delete b;
}

struct shg_engine {
    std::vector<PinnedBlock *> pool;
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    DevBuf in_keys, in_bytes, in_offsets, first, second, sfirst, sidx, counts, cursor, acc, keys, nodes, ids, codes,
        fixed_off, bucket_bits, pos_acc, words, rib_keys, rib_bits, scratch, misc, singles, ckeys, cbits;
    // ShockHash2Flat state kept across its nested fallback build
    DevBuf f_bytes, f_offs, f_mhc0, f_cur, f_sorted, f_next, f_thr, f_counts, f_cursor, f_acc, f_free_cnt, f_bump_cnt,
        f_first, f_free_off, f_bump_off, f_free_out, f_bucket, f_last, f_list, f_slot, f_leaf_keys, f_nodes, f_ids, f_codes,
        f_bits, f_mapping, f_lb, f_tmp, f_tmp2;
    // device shape tables of the configurations this engine has built, grown to the largest bucket
    struct Shapes {
        int variant = 0, leaf = 0;
        ShapeTables host;
        DevBuf cnt, nodes, node_off, singles, single_off, skip_bits;
    };
    std::vector<Shapes *> shapes;
    DevBuf plan_offs, ret_scratch, qdone, qorder;
    cudaEvent_t ev[8] = {};
    cudaStream_t stream2 = nullptr;  // leaves of the pipelined mode
    static constexpr int kMaxChunks = 64;
    cudaEvent_t chunk_ev[kMaxChunks] = {};
    cudaEvent_t join_ev = nullptr;
    int pipe_chunks = 8;
    // pinned staging of large copies from pageable host memory (h2d_from_host), made on first use
    void *stage[2] = {nullptr, nullptr};
    cudaEvent_t stage_ev[2] = {};
    unsigned long long split_kind[4] = {};  // of the last build (shg_engine_last_work)
    uint64_t split_launches = 0, leaf_scan = 0;
    unsigned long long flat_work[5] = {};  // leaf work of the last ShockHash2Flat build (shg_engine_last_work)
    // launch parameters per configuration (variant, leaf size); absent = the Tuning defaults
    std::map<std::pair<int, int>, Tuning> tuning;
    std::mutex tuning_mu;
    std::string tuning_source;  // the table file loaded at creation, or ""
    Tuning tuning_of(int variant, int leaf) {
        std::lock_guard<std::mutex> lock(tuning_mu);
        if (variant == SHG_SHOCKHASH_ROTATION) variant = SHG_SHOCKHASH;  // same searches
        if (variant == SHG_SIMDSHOCKHASH_ROTATION) variant = SHG_SIMDSHOCKHASH;
        auto it = tuning.find({variant, leaf});
        Tuning t = it == tuning.end() ? Tuning() : it->second;
        if (is_simd(variant)) t.split.arith = kSplitArithSimd;  // the format's own split hash
        return t;
    }
    ~shg_engine() {
        DevBuf *all[] = {&in_keys, &in_bytes, &in_offsets, &first, &second, &sfirst, &sidx, &counts, &cursor,
                         &acc, &keys, &nodes, &ids, &codes, &fixed_off, &bucket_bits, &pos_acc, &words,
                         &rib_keys, &rib_bits, &scratch, &misc, &singles, &ckeys, &cbits, &f_bytes, &f_offs,
                         &f_mhc0, &f_cur, &f_sorted, &f_next, &f_thr, &f_counts, &f_cursor, &f_acc, &f_free_cnt,
                         &f_bump_cnt, &f_first, &f_free_off, &f_bump_off, &f_free_out, &f_bucket, &f_last, &f_list,
                         &f_slot, &f_leaf_keys, &f_nodes, &f_ids, &f_codes, &f_bits, &f_mapping, &f_lb, &f_tmp, &f_tmp2};
        for (DevBuf *b : all) b->release();
        plan_offs.release();
        ret_scratch.release();
        qdone.release();
        qorder.release();
        for (Shapes *sh : shapes) {
            DevBuf *sb[] = {&sh->cnt, &sh->nodes, &sh->node_off, &sh->singles, &sh->single_off, &sh->skip_bits};
            for (DevBuf *b : sb) b->release();
            delete sh;
        }
        {
            std::lock_guard<std::mutex> lock(g_pool_mu);
            for (PinnedBlock *b : pool) {
                if (b->in_use) {
                    b->eng = nullptr;  // freed by release_pinned when its result is released
                    continue;
                }
                if (b->p) cudaFreeHost(b->p);
                delete b;
            }
            pool.clear();
        }
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
        for (auto &e : chunk_ev)
            if (e) cudaEventDestroy(e);
        if (join_ev) cudaEventDestroy(join_ev);
        for (int i = 0; i < 2; i++) {
            if (stage_ev[i]) {
                cudaEventSynchronize(stage_ev[i]);
                cudaEventDestroy(stage_ev[i]);
            }
            if (stage[i]) cudaFreeHost(stage[i]);
        }
        if (stream2) cudaStreamDestroy(stream2);
        if (stream) cudaStreamDestroy(stream);
    }
};

shg_status hash_strings_into(shg_engine *e, const char *bytes, const uint64_t *offsets, uint64_t n, float &ms);

namespace {

// Host-to-device copy of `bytes` from host memory that may be pageable. A pageable source of at
// least two staging buffers goes through the engine's two pinned buffers of kStageBytes: host
// threads fill one while the copy engine drains the other (a copy straight from pageable memory ran
// at about 11 GB/s). The source may be reused when this returns; the device copy is ordered on s.
constexpr size_t kStageBytes = 64ull << 20;

// fn(0) .. fn(nt - 1) on nt host threads (this one included); the parts a thread could not be
// started for run on this thread, so no exception leaves through the C ABI.
template <class F> void run_parts(unsigned nt, F &fn) {
    std::vector<std::thread> pool;
    unsigned started = 1;
    try {
        for (unsigned t = 1; t < nt; t++, started++) pool.emplace_back(fn, t);
    } catch (...) {
    }
    fn(0u);
    for (unsigned t = started; t < nt; t++) fn(t);
    for (auto &th : pool) th.join();
}

shg_status h2d_from_host(shg_engine *e, void *dst, const void *src, size_t bytes, cudaStream_t s) {
    if (!bytes) return SHG_OK;
    cudaPointerAttributes attr{};
    const bool pinned = cudaPointerGetAttributes(&attr, src) == cudaSuccess && attr.type == cudaMemoryTypeHost;
    cudaGetLastError();  // a pageable pointer may leave an error behind on some drivers
    if (pinned || bytes < 2 * kStageBytes) {
        CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
        return SHG_OK;
    }
    for (int i = 0; i < 2; i++) {
        if (!e->stage[i] && cudaHostAlloc(&e->stage[i], kStageBytes, cudaHostAllocDefault) != cudaSuccess) {
            e->stage[i] = nullptr;  // no pinned memory to spare: copy directly
            cudaGetLastError();
            CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
            return SHG_OK;
        }
        if (!e->stage_ev[i]) CU(cudaEventCreateWithFlags(&e->stage_ev[i], cudaEventDisableTiming));
    }
    const unsigned nt = std::min(8u, std::max(1u, std::thread::hardware_concurrency()));
    for (size_t off = 0, c = 0; off < bytes; off += kStageBytes, c++) {
        const size_t len = std::min(kStageBytes, bytes - off);
        const int b = (int)(c & 1);
        CU(cudaEventSynchronize(e->stage_ev[b]));  // the copy that last read this buffer is done
        char *d = (char *)e->stage[b];
        const char *from = (const char *)src + off;
        auto part = [&](unsigned t) {
            const size_t a = len * t / nt, z = len * (t + 1) / nt;
            memcpy(d + a, from + a, z - a);
        };
        run_parts(nt, part);
        CU(cudaMemcpyAsync((char *)dst + off, d, len, cudaMemcpyHostToDevice, s));
        CU(cudaEventRecord(e->stage_ev[b], s));
    }
    return SHG_OK;
}

PinnedBlock *acquire_pinned(shg_engine *e, size_t bytes, int refs = 1) {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    PinnedBlock *best = nullptr;
    for (PinnedBlock *b : e->pool)
        if (!b->in_use && b->cap >= bytes && (!best || b->cap < best->cap)) best = b;
    if (!best) {
        best = new PinnedBlock();
        best->eng = e;
        best->cap = bytes + bytes / 8 + 4096;
        if (cudaMallocHost(&best->p, best->cap) != cudaSuccess) {
            delete best;
            return nullptr;
        }
        e->pool.push_back(best);
    }
    best->in_use = true;
    best->refs = refs;
    return best;
}

struct Misc {  // small device-side counters, one allocation
    uint32_t err;
    uint32_t maxsz;
    unsigned int leaf_ctr;
    unsigned int pad;
    unsigned long long work[8];
    unsigned long long split_kind[4];  // useful split evaluations by inner loop (see launch_split_level)
    unsigned int qctr[2];              // work-queue schedule: split and leaf items taken
};

// Memo tables are cached per configuration (they cost ~3000 transcendental evaluations).
const Config &config_of(int variant, int leaf) {
    static std::mutex mu;
    static std::vector<Config *> cache;
    std::lock_guard<std::mutex> lock(mu);
    for (Config *c : cache)
        if (c->variant == variant && c->leaf == leaf) return *c;
    cache.push_back(new Config(variant, leaf));
    return *cache.back();
}

// The device shape tables of a configuration covering bucket sizes below `rows` (grown in steps of
// a quarter, then uploaded once; later builds of the configuration reuse them).
shg_status ensure_shapes(shg_engine *e, const Config &cfg, uint32_t rows, shg_engine::Shapes *&out) {
    shg_engine::Shapes *sh = nullptr;
    for (shg_engine::Shapes *x : e->shapes)
        if (x->variant == cfg.variant && x->leaf == cfg.leaf) sh = x;
    if (!sh) {
        sh = new shg_engine::Shapes();
        sh->variant = cfg.variant;
        sh->leaf = cfg.leaf;
        e->shapes.push_back(sh);
    }
    out = sh;
    if (rows <= sh->host.rows) return SHG_OK;
    rows = std::min<uint32_t>(kMaxBucket, ((rows + rows / 4 + 255) / 256) * 256);
    try {
        make_shape_tables(cfg, rows, sh->host);
    } catch (const std::exception &ex) {
        sh->host = ShapeTables();
        return fail(SHG_ERR_ARG, ex.what());
    }
    const ShapeTables &t = sh->host;
    std::vector<uint32_t> skip(rows);
    for (uint32_t m = 0; m < rows; m++) skip[m] = cfg.skip_bits(m);
    auto up = [&](DevBuf &b, const void *src, size_t bytes) -> cudaError_t {
        cudaError_t err = b.ensure(std::max<size_t>(bytes, 16));
        if (err == cudaSuccess && bytes) err = cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, e->stream);
        return err;
    };
    cudaError_t err = up(sh->cnt, t.cnt.data(), t.cnt.size() * 4);
    if (err == cudaSuccess) err = up(sh->nodes, t.nodes.data(), t.nodes.size() * sizeof(ShapeNode));
    if (err == cudaSuccess) err = up(sh->node_off, t.node_off.data(), t.node_off.size() * 4);
    if (err == cudaSuccess) err = up(sh->singles, t.singles.data(), t.singles.size() * 2);
    if (err == cudaSuccess) err = up(sh->single_off, t.single_off.data(), t.single_off.size() * 4);
    if (err == cudaSuccess) err = up(sh->skip_bits, skip.data(), skip.size() * 4);
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);  // the host vectors may change later
    if (err != cudaSuccess) {
        sh->host = ShapeTables();
        return fail(SHG_ERR_CUDA, std::string("shape tables: ") + cudaGetErrorString(err));
    }
    return SHG_OK;
}

shg_status check_params(const shg_params *p, uint64_t n) {
    if (!p) return fail(SHG_ERR_ARG, "null params");
    if (!is_sh1(p->variant) && p->variant != SHG_SHOCKHASH2) return fail(SHG_ERR_ARG, "unknown variant");
    const int maxleaf = is_sh1(p->variant) ? kMaxLeaf1 : kMaxLeaf2;
    if (p->leaf_size < 2 || p->leaf_size > maxleaf) return fail(SHG_ERR_ARG, "leaf size out of range");
    if (p->bucket_size < 1) return fail(SHG_ERR_ARG, "bucket size must be >= 1");
    if (n >= (1ull << 32)) return fail(SHG_ERR_ARG, "at most 2^32 - 1 keys per build");
    if (p->mode < SHG_MODE_DEFAULT || p->mode > SHG_MODE_QUEUE) return fail(SHG_ERR_ARG, "unknown mode");
    return SHG_OK;
}

// The core build from 128-bit fingerprints already in device memory (e->first / e->second).
// The build of a batch of R independent key sets (requests) whose 128-bit fingerprints lie back to
// back in d_first / d_second (request r holds nr[r] keys). Every request gets its own bucket range
// and its own products (as if built alone); the partition, the split levels and the leaf search of
// all requests share the same launches.
// A request that is one shard of a larger structure: it owns buckets [b0, b1) of nb_global
// (nb_global 0: the request is a whole structure). `shards` holds one entry per request, or is null.
struct ShardSpec {
    uint64_t nb_global, b0, b1;
};

shg_status build_batch(shg_engine *e, const shg_params *p, const uint64_t *d_first, const uint64_t *d_second,
                       const std::vector<uint64_t> &nr, shg_result *outs, float hash_ms,
                       const ShardSpec *shards = nullptr) {
    const Config &cfg = config_of(p->variant, p->leaf_size);
    cudaStream_t s = e->stream;
    const size_t R = nr.size();

    std::vector<uint64_t> off(R + 1, 0), nbr(R), boff(R + 1, 0), nb_map(R), b0(R, 0);
    for (size_t r = 0; r < R; r++) {
        off[r + 1] = off[r] + nr[r];
        nbr[r] = std::max<uint64_t>(1, (nr[r] + p->bucket_size - 1) / p->bucket_size);  // ShockHash.h:616
        nb_map[r] = nbr[r];
        if (shards && shards[r].nb_global) {  // request r holds buckets [b0, b1) of a larger structure
            nbr[r] = shards[r].b1 - shards[r].b0;
            nb_map[r] = shards[r].nb_global;
            b0[r] = shards[r].b0;
        }
        boff[r + 1] = boff[r] + nbr[r];
        memset(&outs[r], 0, sizeof(shg_result));
        outs[r].n = nr[r];
        outs[r].nbuckets = nbr[r];
    }
    const uint64_t n = off[R], nb = boff[R];
    if (n >= (1ull << 32)) return fail(SHG_ERR_ARG, "at most 2^32 - 1 keys per batch");

    CU(e->misc.ensure(sizeof(Misc)));
    Misc *misc = e->misc.as<Misc>();
    CU(cudaMemsetAsync(misc, 0, sizeof(Misc), s));
    CU(e->counts.ensure(nb * 4));
    CU(e->cursor.ensure(nb * 4));
    CU(e->acc.ensure((nb + 1) * 8));
    CU(e->sfirst.ensure(std::max<uint64_t>(n, 1) * 8));
    CU(e->sidx.ensure(std::max<uint64_t>(n, 1) * 4));
    CU(e->keys.ensure(std::max<uint64_t>(n, 1) * 8));

    // ---- partition: each request's keys into its own bucket range, then one sort pass; the
    // plan's per-bucket offsets are scanned from the bucket sizes before the host looks at them
    shg_engine::Shapes *shp = nullptr;
    {
        const shg_status st = ensure_shapes(e, cfg, std::min<uint64_t>(kMaxBucket, 2 * p->bucket_size + 64), shp);
        if (st != SHG_OK) return st;
    }
    const uint64_t offs_stride = nb + 1;
    uint64_t plan_launches = 0;
    auto plan_scan = [&]() -> cudaError_t {
        plan_launches++;
        cudaError_t err = e->plan_offs.ensure(((uint64_t)shp->host.ncol * offs_stride + kMaxPlanCols) * 4);
        if (err == cudaSuccess)
            launch_plan_scan(e->acc.as<uint64_t>(), nb, shp->cnt.as<uint32_t>(), shp->host.rows, shp->host.ncol,
                             e->plan_offs.as<uint32_t>(), s);
        return err;
    };
    CU(cudaEventRecord(e->ev[0], s));
    for (size_t r = 0; r < R; r++)
        launch_bucket_count(d_first + off[r], nr[r], nbr[r], nb_map[r], b0[r], e->counts.as<uint32_t>() + boff[r], &misc->err,
                            s);
    launch_scan_counts(e->counts.as<uint32_t>(), nb, e->acc.as<uint64_t>(), e->cursor.as<uint32_t>(), &misc->maxsz, s);
    CU(plan_scan());
    std::vector<uint64_t> acc(nb + 1);
    uint32_t totals[kMaxPlanCols] = {};
    uint32_t maxsz = 0;
    CU(cudaMemcpyAsync(acc.data(), e->acc.p, (nb + 1) * 8, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(&maxsz, &misc->maxsz, 4, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(totals, e->plan_offs.as<uint32_t>() + shp->host.ncol * offs_stride, shp->host.ncol * 4,
                       cudaMemcpyDeviceToHost, s));
    uint32_t perr = 0;
    CU(cudaMemcpyAsync(&perr, &misc->err, 4, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (perr & kErrArg) return fail(SHG_ERR_ARG, "a key lies outside the shard's bucket range");
    if (maxsz >= (uint32_t)kMaxBucket)
        return fail(SHG_ERR_BUCKET, "a bucket holds " + std::to_string(maxsz) + " keys (MAX_BUCKET_SIZE is 3000)");
    if (maxsz >= shp->host.rows) {  // a bucket larger than the shape tables cover: grow them, scan again
        const shg_status st = ensure_shapes(e, cfg, maxsz + 1, shp);
        if (st != SHG_OK) return st;
        CU(plan_scan());
        CU(cudaMemcpyAsync(totals, e->plan_offs.as<uint32_t>() + shp->host.ncol * offs_stride, shp->host.ncol * 4,
                           cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
    }
    const ShapeTables &tab = shp->host;
    for (size_t r = 0; r < R; r++)
        launch_bucket_scatter(d_first + off[r], nr[r], nbr[r], nb_map[r], b0[r], e->cursor.as<uint32_t>() + boff[r],
                              e->sfirst.as<uint64_t>(),
                              e->sidx.as<uint32_t>(), off[r], s);
    launch_bucket_sort(e->acc.as<uint64_t>(), nb, e->sfirst.as<uint64_t>(), e->sidx.as<uint32_t>(), d_second,
                       e->keys.as<uint64_t>(), s);
    CU(cudaEventRecord(e->ev[1], s));

    // ---- plan: launch lists are the split levels in order, then the leaves
    const uint64_t nn = totals[kColNodes];
    const uint64_t nsingles = totals[kColSingles];
    const uint32_t nleaves = totals[kColLeaves];
    const int nlevels = tab.ncol - kColLevel0;
    ListOffsets lists{};
    std::vector<uint64_t> level_count(nlevels), level_off(nlevels);
    uint64_t nids = 0;
    for (int lv = 0; lv < nlevels; lv++) {
        level_off[lv] = lists.level[lv] = (uint32_t)nids;
        level_count[lv] = totals[kColLevel0 + lv];
        nids += level_count[lv];
    }
    const uint64_t leaf_off = lists.leaf = (uint32_t)nids;
    nids += nleaves;
    CU(e->nodes.ensure(std::max<uint64_t>(nn, 1) * sizeof(Node)));
    CU(e->fixed_off.ensure(std::max<uint64_t>(nn, 1) * 2));
    CU(e->codes.ensure(std::max<uint64_t>(nn, 1) * 8));
    CU(e->ids.ensure(std::max<uint64_t>(nids, 1) * 4));
    CU(e->bucket_bits.ensure(nb * 8));
    CU(e->pos_acc.ensure((nb + 1) * 8));
    CU(e->rib_bits.ensure(std::max<uint64_t>(n, 1)));
    if (is_sh1(p->variant)) CU(e->rib_keys.ensure(std::max<uint64_t>(n, 1) * 8));
    CU(e->singles.ensure(std::max<uint64_t>(nsingles, 1) * 8));
    plan_launches += nb ? 1 : 0;
    launch_plan_expand(e->acc.as<uint64_t>(), nb, tab.rows, e->plan_offs.as<uint32_t>(), shp->nodes.as<ShapeNode>(),
                       shp->node_off.as<uint32_t>(), shp->singles.as<uint16_t>(), shp->single_off.as<uint32_t>(), lists,
                       e->nodes.as<Node>(), e->fixed_off.as<uint16_t>(), e->ids.as<uint32_t>(), e->singles.as<uint64_t>(), s);
    const uint32_t *d_bnb = e->plan_offs.as<uint32_t>() + kColNodes * offs_stride;  // first node of each bucket
    const uint32_t *d_skip = shp->skip_bits.as<uint32_t>();
    if (p->variant == SHG_SHOCKHASH2) {
        // bipartite leaf scratch for the widest leaf grid any schedule uses (grown once, then reused)
        const uint32_t sm_ = p->leaf_size > 64 ? 16384 : 4096, cm_ = p->leaf_size > 64 ? 16384 : 2048;
        const uint64_t pw = (sh2_scratch_bytes(sm_, cm_, p->leaf_size) + 255) & ~255ull;
        const int bps = std::max(1, std::min(8, (228 * 1024) / (4 * sh2_smem_per_warp(p->leaf_size) + 1024)));
        CU(e->scratch.ensure(pw * (uint64_t)e->sms * bps * 4));
    }
    // per request: its nodes, its size-1 positions (no retrieval bit) and its fixed code bits,
    // from the host copy of the shape table
    std::vector<uint64_t> soff(R + 1, 0), rnv(R), rnodes(R, 0), rfixed(R, 0);
    for (size_t r = 0; r < R; r++) {
        uint64_t singles_r = 0;
        for (uint64_t b = boff[r]; b < boff[r + 1]; b++) {
            const uint32_t m = (uint32_t)(acc[b + 1] - acc[b]);
            const uint32_t *row = &tab.cnt[(size_t)m * tab.ncol];
            rnodes[r] += row[kColNodes];
            singles_r += row[kColSingles];
            rfixed[r] += cfg.skip_bits(m);
        }
        soff[r + 1] = soff[r] + singles_r;
        rnv[r] = nr[r] - singles_r;
    }
    CU(e->ckeys.ensure(std::max<uint64_t>(n, 1) * 8));
    CU(e->cbits.ensure(std::max<uint64_t>(n, 1)));
    // Bipartite retrieval keys are final once the splits are done (the leaves only add the bits),
    // so in the level schedule they go to the host on the second stream while the leaf kernel
    // runs. The pinned block is then taken before the splits, with room for descriptor words
    // bounded by the fixed bits plus 8 unary bits per node; a longer stream (not seen in
    // practice) takes a new block after encoding.
    // the work-queue schedule: bipartite leaves of up to 64 keys (other builds take the level schedule)
    // (the default schedule for these builds: measured faster than the level schedule on B200)
    const bool queue = (p->mode == SHG_MODE_QUEUE || p->mode == SHG_MODE_DEFAULT) && p->variant == SHG_SHOCKHASH2 &&
                       p->leaf_size <= 64;
    const Tuning tun = e->tuning_of(p->variant, p->leaf_size);
    // with per-bucket leaf groups, the queue kernel writes each bucket's retrieval keys and bits
    // straight into the pinned result block as the bucket's leaves finish
    const bool stream_out = queue && tun.queue_lag > 0;
    const bool early_keys = p->variant == SHG_SHOCKHASH2 && p->mode != SHG_MODE_PIPELINED && !queue;
    std::vector<uint64_t> wcap(R, 0);
    std::vector<size_t> roff(R + 1, 0);
    auto layout = [&]() {
        for (size_t r = 0; r < R; r++) {
            const size_t acc_bytes = (nbr[r] + 1) * 8;
            roff[r + 1] = roff[r] + ((2 * acc_bytes + rnv[r] * 9 + wcap[r] * 8 + 64 + 63) & ~(size_t)63);
        }
    };
    PinnedBlock *blk = nullptr;
    if (early_keys || stream_out) {
        for (size_t r = 0; r < R; r++) {
            const uint64_t bits = rfixed[r] + 8 * rnodes[r] + 1;
            wcap[r] = ((bits + 7) / 8 + 14) / 8;
        }
        layout();
        blk = acquire_pinned(e, roff[R], (int)R);
        if (!blk) return fail(SHG_ERR_OOM, "pinned host allocation failed");
    }
    auto keys_host = [&](PinnedBlock *b, size_t r) { return (uint64_t *)((uint8_t *)b->p + roff[r] + 2 * (nbr[r] + 1) * 8); };
    auto release_all = [&](PinnedBlock *b) {  // drop every reference a failed build still holds
        for (size_t r = 0; r < R; r++) release_pinned(b);
    };
    CU(cudaEventRecord(e->ev[2], s));

    // ---- splits and leaves
    uint64_t launches = 0;
    const uint32_t *d_ids = e->ids.as<uint32_t>();
    const bool sh2 = p->variant == SHG_SHOCKHASH2;
    const bool pipelined = p->mode == SHG_MODE_PIPELINED;
    // leaf kernel launch shape and scratch
    const int maxm = p->leaf_size;
    const uint32_t smax = maxm > 64 ? 16384 : 4096, cmax = maxm > 64 ? 16384 : 2048;
    const uint64_t per_warp = (sh2_scratch_bytes(smax, cmax, maxm) + 255) & ~255ull;
    int leaf_grid;
    if (sh2) {
        const int per_block_smem = 4 * sh2_smem_per_warp(maxm);
        int blocks_per_sm = std::max(1, std::min(8, (228 * 1024) / (per_block_smem + 1024)));
        if (tun.leaf_bps > 0) blocks_per_sm = std::min(blocks_per_sm, tun.leaf_bps);
        // next to running split launches, leaves take part of each SM (the splits are ALU bound,
        // the leaves latency bound, so the two interleave)
        const int bps = pipelined ? std::max(1, blocks_per_sm / 2) : blocks_per_sm;
        leaf_grid = p->mode == SHG_MODE_PER_LEAF ? 1 : std::max(1, std::min<int>(e->sms * bps, (int)((nleaves + 3) / 4)));
    } else {
        const int wpb = leaves_sh1_warps_per_block();
        const int bps = tun.leaf_bps > 0 ? tun.leaf_bps : 8;
        leaf_grid = std::max(1, std::min<int>(e->sms * (pipelined ? std::max(1, bps / 2) : bps), (int)((nleaves + wpb - 1) / wpb)));
    }
    auto split_range = [&](size_t lv, uint64_t a, uint64_t b, cudaStream_t st) {
        if (b <= a) return;
        launch_split_level(e->nodes.as<Node>(), d_ids + level_off[lv] + a, (uint32_t)(b - a), e->keys.as<uint64_t>(),
                           e->codes.as<uint64_t>(), p->max_trials, &misc->err, &misc->work[0], misc->split_kind, tun.split,
                           st);
        launches++;
    };
    auto leaf_range = [&](uint64_t a, uint64_t b, cudaStream_t st, int grid) {
        if (b <= a) return;
        if (sh2)
            launch_leaves_sh2_ctr(e->nodes.as<Node>(), d_ids + leaf_off + a, (uint32_t)(b - a), e->keys.as<uint64_t>(),
                                  e->codes.as<uint64_t>(), e->rib_bits.as<uint8_t>(), e->scratch.as<uint8_t>(), per_warp, smax,
                                  cmax, &misc->err, misc->work, &misc->leaf_ctr, grid, st, maxm, kQuadMinRecSplit,
                                  tun.leaf_minb);
        else
            launch_leaves_sh1_ctr(e->nodes.as<Node>(), d_ids + leaf_off + a, (uint32_t)(b - a), e->keys.as<uint64_t>(),
                                  e->codes.as<uint64_t>(), e->rib_keys.as<uint64_t>(), e->rib_bits.as<uint8_t>(), p->max_trials,
                                  &misc->err, misc->work, &misc->leaf_ctr, grid, st,
                                  is_rotation(p->variant) ? (uint32_t)p->leaf_size : 0, tun.sh1_spl);
        launches++;
    };
    if (queue) {
        // one persistent launch over the staggered item order: split nodes and per-bucket leaf groups
        const int qsmem = tree_queue_smem_per_block(tun.split.spl);
        int qbps = std::max(1, std::min(3, (228 * 1024) / (qsmem + 1024)));
        if (tun.leaf_bps > 0) qbps = std::min(qbps, tun.leaf_bps);
        const int qgrid = std::max(1, std::min<int>(e->sms * qbps, (int)std::max<uint64_t>(leaf_off + nb, 1)));
        // lag between a bucket's levels: queue_lag rounds of the grid's blocks, in buckets of
        // (split nodes + one leaf group) each, so that a node's parent has finished when it is
        // taken; none (0): lag nb, the levels one after another, then the leaf groups
        const uint64_t per_bucket = std::max<uint64_t>(1, (leaf_off + nb) / std::max<uint64_t>(nb, 1));
        const uint64_t lag_b = tun.queue_lag > 0 ? ((uint64_t)tun.queue_lag * qgrid + per_bucket - 1) / per_bucket : nb;
        const uint32_t lag = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(nb, 1), std::max<uint64_t>(1, lag_b));
        const uint64_t T = queue_order_slots(nb, (uint32_t)nlevels, lag);
        const uint64_t seq_words = leaf_off + nb;
        const uint64_t order_words = (2 * T + 1 + seq_words + 1) & ~1ull;  // the request table after it, 8-byte aligned
        CU(e->qorder.ensure(order_words * 4 + (stream_out ? R * sizeof(QueueOut) : 0) + 256));
        uint32_t *q_cnt = e->qorder.as<uint32_t>(), *q_pos = q_cnt + T, *q_seq = q_pos + T + 1;
        QueueOut *q_out = nullptr;
        if (stream_out) {
            // where each request's compacted retrieval keys and bits go in the pinned block
            std::vector<QueueOut> qo(R);
            for (size_t r = 0; r < R; r++)
                qo[r] = QueueOut{boff[r], off[r], soff[r], keys_host(blk, r), (uint8_t *)keys_host(blk, r) + rnv[r] * 8};
            q_out = (QueueOut *)(e->qorder.as<uint32_t>() + order_words);
            CU(cudaMemcpyAsync(q_out, qo.data(), R * sizeof(QueueOut), cudaMemcpyHostToDevice, s));
            CU(cudaStreamSynchronize(s));  // qo is pageable and leaves scope
        }
        CU(e->scratch.ensure(per_warp * (uint64_t)qgrid * tree_queue_warps_per_block()));
        CU(e->qdone.ensure(std::max<uint64_t>(nb, 1) * 4));
        CU(cudaMemsetAsync(e->qdone.p, 0, nb * 4, s));
        CU(cudaMemsetAsync(misc->qctr, 0, sizeof(misc->qctr), s));
        const bool groups = tun.queue_lag > 0;
        launch_queue_order(e->plan_offs.as<uint32_t>(), offs_stride, nb, (uint32_t)nlevels, lag, groups, lists,
                           (uint32_t)leaf_off, q_cnt, q_pos, q_seq, s);
        launches += T ? 3 : 0;
        if (T == 0) CU(cudaMemsetAsync(q_pos, 0, 4, s));  // no buckets: no items
        launch_tree_queue(e->nodes.as<Node>(), d_ids, q_seq, q_pos + T, (uint32_t)leaf_off, e->plan_offs.as<uint32_t>(),
                          offs_stride, (uint32_t)nlevels, e->qdone.as<uint32_t>(), e->keys.as<uint64_t>(),
                          e->codes.as<uint64_t>(), e->rib_bits.as<uint8_t>(), e->scratch.as<uint8_t>(), per_warp, smax, cmax,
                          p->max_trials, &misc->err, misc->work, misc->split_kind, misc->qctr, groups ? 0u : nleaves,
                          e->acc.as<uint64_t>(), e->singles.as<uint64_t>(), q_out, (uint32_t)R, tun.split, qgrid, s);
        launches++;
        CU(cudaEventRecord(e->ev[3], s));  // the split stage's time covers the whole queue launch
    } else if (pipelined) {
        // Buckets in chunks: chunk c's split levels run on the engine stream, its leaves on the
        // second stream as soon as those splits are done, overlapping the next chunk's splits.
        // Node and leaf lists are in bucket order, so a chunk is a contiguous range of each list.
        const int C = (int)std::max<uint64_t>(1, std::min<uint64_t>(nb, (uint64_t)e->pipe_chunks));
        // bounds of each launch list at the chunk borders: the per-bucket list offsets of the plan
        std::vector<uint32_t> offs_h((uint64_t)tab.ncol * offs_stride);
        CU(cudaMemcpyAsync(offs_h.data(), e->plan_offs.p, offs_h.size() * 4, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        auto chunk_bounds = [&](int col, std::vector<uint64_t> &bounds) {
            bounds.assign(C + 1, 0);
            for (int c = 0; c <= C; c++) bounds[c] = offs_h[(uint64_t)col * offs_stride + nb * (uint64_t)c / C];
        };
        std::vector<std::vector<uint64_t>> lvb(nlevels);
        for (int lv = 0; lv < nlevels; lv++) chunk_bounds(kColLevel0 + lv, lvb[lv]);
        std::vector<uint64_t> lb;
        chunk_bounds(kColLeaves, lb);
        for (int c = 0; c < C; c++) {
            for (int lv = 0; lv < nlevels; lv++) split_range(lv, lvb[lv][c], lvb[lv][c + 1], s);
            CU(cudaEventRecord(e->chunk_ev[c], s));
            CU(cudaStreamWaitEvent(e->stream2, e->chunk_ev[c], 0));
            leaf_range(lb[c], lb[c + 1], e->stream2, leaf_grid);
        }
        CU(cudaEventRecord(e->ev[3], s));  // last split launch done
        CU(cudaEventRecord(e->join_ev, e->stream2));
        CU(cudaStreamWaitEvent(s, e->join_ev, 0));
    } else {
        for (int lv = 0; lv < nlevels; lv++) split_range(lv, 0, level_count[lv], s);
        CU(cudaEventRecord(e->ev[3], s));
        if (early_keys) {
            // compaction on the engine stream before the leaf kernel takes every SM; only the
            // copies run on the second stream, next to the leaves
            for (size_t r = 0; r < R; r++)
                if (rnv[r])
                    launch_compact_ribbon(e->keys.as<uint64_t>() + off[r], nullptr, nr[r], e->singles.as<uint64_t>() + soff[r],
                                          soff[r + 1] - soff[r], off[r], e->ckeys.as<uint64_t>() + off[r], nullptr, s);
            CU(cudaEventRecord(e->chunk_ev[0], s));
            CU(cudaStreamWaitEvent(e->stream2, e->chunk_ev[0], 0));
            for (size_t r = 0; r < R; r++)
                if (rnv[r])
                    CU(cudaMemcpyAsync(keys_host(blk, r), e->ckeys.as<uint64_t>() + off[r], rnv[r] * 8, cudaMemcpyDeviceToHost,
                                       e->stream2));
            CU(cudaEventRecord(e->join_ev, e->stream2));
        }
        if (p->mode == SHG_MODE_PER_LEAF)
            for (uint32_t l = 0; l < nleaves; l++) leaf_range(l, l + 1, s, 1);
        else
            leaf_range(0, nleaves, s, leaf_grid);
    }
    CU(cudaGetLastError());
    CU(cudaEventRecord(e->ev[4], s));

    // ---- Golomb-Rice encode, one stream per request
    CU(e->pos_acc.ensure((nb + R) * 8));
    for (size_t r = 0; r < R; r++) {
        launch_gr_bucket_bits(e->nodes.as<Node>(), d_bnb + boff[r], nbr[r], e->acc.as<uint64_t>() + boff[r],
                              e->codes.as<uint64_t>(), d_skip, e->bucket_bits.as<uint64_t>() + boff[r], s);
        launch_scan_u64(e->bucket_bits.as<uint64_t>() + boff[r], nbr[r], e->pos_acc.as<uint64_t>() + boff[r] + r, s);
    }
    std::vector<uint64_t> pos(nb + R);
    CU(cudaMemcpyAsync(pos.data(), e->pos_acc.p, (nb + R) * 8, cudaMemcpyDeviceToHost, s));
    uint32_t err = 0;
    CU(cudaMemcpyAsync(&err, &misc->err, 4, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (err && blk) {
        cudaStreamSynchronize(e->stream2);
        release_all(blk);
    }
    if (err & kErrTrialLimit) return fail(SHG_ERR_TRIAL_LIMIT, "a seed search exceeded its trial cap (duplicate keys?)");
    if (err & kErrScratch) return fail(SHG_ERR_TRIAL_LIMIT, "a bipartite leaf exceeded its candidate capacity (duplicate keys?)");
    if (err) return fail(SHG_ERR_CUDA, "internal device error flag " + std::to_string(err));
    std::vector<uint64_t> total(R), words(R), wbase(R + 1, 0);
    for (size_t r = 0; r < R; r++) {
        total[r] = pos[boff[r] + r + nbr[r]];
        const uint64_t bits = total[r] + 1;          // + sentinel (ShockHash.h:652)
        words[r] = ((bits + 7) / 8 + 7 + 7) / 8;     // the builder's final size (RiceBitVector.h:71)
        wbase[r + 1] = wbase[r] + words[r];
    }
    CU(e->words.ensure(wbase[R] * 8));
    CU(cudaMemsetAsync(e->words.p, 0, wbase[R] * 8, s));
    for (size_t r = 0; r < R; r++) {
        unsigned long long *w = e->words.as<unsigned long long>() + wbase[r];
        launch_gr_write(e->nodes.as<Node>(), e->fixed_off.as<uint16_t>(), d_bnb + boff[r], nbr[r],
                        e->acc.as<uint64_t>() + boff[r], e->pos_acc.as<uint64_t>() + boff[r] + r, e->codes.as<uint64_t>(),
                        d_skip, w, s);
        launch_set_bit(w, total[r], s);
        launches += 4;
    }
    CU(cudaGetLastError());
    CU(cudaEventRecord(e->ev[5], s));

    // ---- copy-out: the products of each request into the pinned block (one block per batch,
    // each result holding a reference); the retrieval input is compacted on the device first.
    bool keys_done = early_keys || stream_out, bits_done = stream_out;
    if (early_keys || stream_out) {
        bool fits = true;
        for (size_t r = 0; r < R; r++) fits = fits && words[r] <= wcap[r];
        if (!fits) {  // descriptor stream longer than the bound: a new block, keys (and bits) copied again
            CU(cudaStreamSynchronize(e->stream2));
            release_all(blk);
            blk = nullptr;
            keys_done = bits_done = false;
        }
    }
    if (!blk) {
        for (size_t r = 0; r < R; r++) wcap[r] = words[r];
        layout();
        blk = acquire_pinned(e, roff[R], (int)R);
        if (!blk) return fail(SHG_ERR_OOM, "pinned host allocation failed");
    }
    const uint64_t *src_keys = is_sh1(p->variant) ? e->rib_keys.as<uint64_t>() : e->keys.as<uint64_t>();
    for (size_t r = 0; r < R; r++) {
        shg_result *out = &outs[r];
        const uint64_t ns = soff[r + 1] - soff[r], rn = rnv[r];
        if (!bits_done)
            launch_compact_ribbon(src_keys + off[r], e->rib_bits.as<uint8_t>() + off[r], nr[r], e->singles.as<uint64_t>() + soff[r],
                                  ns, off[r], keys_done ? nullptr : e->ckeys.as<uint64_t>() + off[r],
                                  e->cbits.as<uint8_t>() + off[r], s);
        const size_t acc_bytes = (nbr[r] + 1) * 8;
        uint8_t *hp = (uint8_t *)blk->p + roff[r];
        out->owner = blk;
        out->bucket_size_acc = (uint64_t *)hp;
        out->bucket_pos_acc = (uint64_t *)(hp + acc_bytes);
        out->ribbon_keys = (uint64_t *)(hp + 2 * acc_bytes);
        out->ribbon_bits = hp + 2 * acc_bytes + rn * 8;
        out->descriptors = (uint64_t *)(hp + ((2 * acc_bytes + rn * 9 + 7) & ~(size_t)7));
        for (uint64_t b = 0; b <= nbr[r]; b++) out->bucket_size_acc[b] = acc[boff[r] + b] - acc[boff[r]];
        CU(cudaMemcpyAsync(out->bucket_pos_acc, e->pos_acc.as<uint64_t>() + boff[r] + r, acc_bytes, cudaMemcpyDeviceToHost, s));
        CU(cudaMemcpyAsync(out->descriptors, e->words.as<uint64_t>() + wbase[r], words[r] * 8, cudaMemcpyDeviceToHost, s));
        if (rn) {
            if (!keys_done)
                CU(cudaMemcpyAsync(out->ribbon_keys, e->ckeys.as<uint64_t>() + off[r], rn * 8, cudaMemcpyDeviceToHost, s));
            if (!bits_done)
                CU(cudaMemcpyAsync(out->ribbon_bits, e->cbits.as<uint8_t>() + off[r], rn, cudaMemcpyDeviceToHost, s));
        }
        out->desc_words = words[r];
        out->desc_bits = total[r] + 1;
        out->ribbon_n = rn;
    }
    if (keys_done && early_keys) CU(cudaStreamWaitEvent(s, e->join_ev, 0));  // the keys copied during the leaves
    unsigned long long work[8];
    CU(cudaMemcpyAsync(work, misc->work, sizeof(work), cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(e->split_kind, misc->split_kind, sizeof(e->split_kind), cudaMemcpyDeviceToHost, s));
    CU(cudaEventRecord(e->ev[6], s));
    CU(cudaStreamSynchronize(s));
    e->split_launches = 0;
    for (int lv = 0; lv < nlevels; lv++) e->split_launches += level_count[lv] ? 1 : 0;
    e->leaf_scan = work[5];  // the leaf kernel's candidate-scan count (the slot is reported as leaves below)
    float ms[6] = {};
    cudaEventElapsedTime(&ms[0], e->ev[0], e->ev[1]);
    cudaEventElapsedTime(&ms[1], e->ev[1], e->ev[2]);
    cudaEventElapsedTime(&ms[2], e->ev[2], e->ev[3]);
    cudaEventElapsedTime(&ms[3], e->ev[3], e->ev[4]);
    cudaEventElapsedTime(&ms[4], e->ev[4], e->ev[5]);
    cudaEventElapsedTime(&ms[5], e->ev[5], e->ev[6]);
    for (size_t r = 0; r < R; r++) {
        shg_result *out = &outs[r];
        out->stage_ms[0] = hash_ms;
        for (int i = 0; i < 6; i++) out->stage_ms[1 + i] = ms[i];
        out->stage_ms[7] = hash_ms + ms[0] + ms[1] + ms[2] + ms[3] + ms[4] + ms[5];
        for (int i = 0; i < 7; i++) out->work[i] = work[i];
        out->work[5] = nleaves;
        out->work[6] = nn - nleaves;
        // kernels of this build: hashing (when the keys were hashed on the device), partition
        // (count and scatter per request, one scan, one sort), plan (offset scan and expansion),
        // split levels and leaves, Golomb-Rice encoding (4 per request, counted above), retrieval
        // compaction (keys and bits together, or keys before the leaves and bits after them)
        out->work[7] = (hash_ms > 0.f ? 1 : 0) + 2 * R + 2 + plan_launches + launches +
                      R * ((early_keys ? 1 : 0) + (bits_done ? 0 : 1));
    }
    return SHG_OK;
}

shg_status build_core(shg_engine *e, const shg_params *p, const uint64_t *d_first, const uint64_t *d_second, uint64_t n,
                      shg_result *out, float hash_ms) {
    return build_batch(e, p, d_first, d_second, std::vector<uint64_t>{n}, out, hash_ms);
}


// ------------------------------------------------------------------ ShockHash2Flat<k>
double ms_since(std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

shg_status build_flat(shg_engine *e, uint64_t k, const char *bytes, const uint64_t *offsets, uint64_t n,
                      shg_flat_result *out) {
    using clk = std::chrono::steady_clock;
    const auto t_start = clk::now();
    cudaStream_t s = e->stream;
    const FlatConsts fc = flat_consts((uint32_t)k);
    memset(out, 0, sizeof(*out));
    out->n = n;
    out->k = k;
    out->threshold_bits = fc.threshold_bits;
    out->seed_bits = fc.seed_bits;
    const uint64_t nbuckets = n / k;                   // ShockHash2Flat.h:68
    const uint64_t keys_in_end_bucket = n - nbuckets * k;
    out->nbuckets = nbuckets;
    CU(e->misc.ensure(sizeof(Misc)));
    Misc *misc = e->misc.as<Misc>();
    CU(cudaMemsetAsync(misc, 0, sizeof(Misc), s));

    // ---- MurmurHash64 of every key
    const uint64_t nbytes = n ? offsets[n] : 0;
    const uint64_t nn = std::max<uint64_t>(n, 1);
    CU(e->f_bytes.ensure(std::max<uint64_t>(nbytes, 1)));
    CU(e->f_offs.ensure((n + 1) * 8));
    CU(e->f_mhc0.ensure(nn * 8));
    CU(e->f_cur.ensure(nn * 8));
    CU(e->f_sorted.ensure(nn * 8));
    CU(e->f_next.ensure(nn * 8));
    CU(e->f_thr.ensure(std::max<uint64_t>(nbuckets, 1)));
    CU(e->f_mapping.ensure(fc.threshold_range * 4 + 4));
    CU(e->f_lb.ensure(4 * 8));
    if (shg_status cs = h2d_from_host(e, e->f_bytes.p, bytes, nbytes, s)) return cs;
    if (shg_status cs = h2d_from_host(e, e->f_offs.p, offsets, (n + 1) * 8, s)) return cs;
    CU(cudaMemcpyAsync(e->f_mapping.p, fc.mapping.data(), fc.threshold_range * 4, cudaMemcpyHostToDevice, s));
    CU(cudaMemsetAsync(e->f_thr.p, 0, std::max<uint64_t>(nbuckets, 1), s));  // thresholdsAndSeeds starts zeroed
    flat_launch_murmur(e->f_bytes.as<uint8_t>(), e->f_offs.as<uint64_t>(), n, e->f_mhc0.as<uint64_t>(), s);
    if (n) CU(cudaMemcpyAsync(e->f_cur.p, e->f_mhc0.p, n * 8, cudaMemcpyDeviceToDevice, s));
    CU(cudaStreamSynchronize(s));
    out->stage_ms[0] = ms_since(t_start);
    auto t = clk::now();

    // ---- threshold layers (ShockHash2Flat.h:86-122)
    std::vector<uint64_t> layer_bases{0};
    std::vector<uint64_t> free_positions;
    uint64_t layers = 2, cur_n = n;
    uint64_t buckets_this_layer = (uint64_t)std::ceil(0.9 * (double)nbuckets);  // :70
    if (buckets_this_layer == 0) layers = 0;
    for (uint64_t layer = 0; layer < layers; layer++) {
        const uint64_t base = layer_bases.back();
        if (layer != 0) {
            buckets_this_layer = (uint64_t)(0.9 * (double)(cur_n / k));  // :89-90
            buckets_this_layer = std::min(buckets_this_layer, nbuckets - base);
            if (buckets_this_layer == 0) {
                layers = 1;
                break;
            }
        }
        const uint32_t B = (uint32_t)buckets_this_layer;
        layer_bases.push_back(base + B);
        CU(e->f_counts.ensure(B * 4ull));
        CU(e->f_cursor.ensure(B * 4ull));
        CU(e->f_acc.ensure((B + 1ull) * 8));
        CU(e->f_free_cnt.ensure(B * 8ull));
        CU(e->f_bump_cnt.ensure(B * 8ull));
        CU(e->f_first.ensure(B * 4ull));
        CU(e->f_free_off.ensure((B + 1ull) * 8));
        CU(e->f_bump_off.ensure((B + 1ull) * 8));
        flat_launch_count(e->f_cur.as<uint64_t>(), cur_n, B, layer != 0, e->f_counts.as<uint32_t>(), s);
        launch_scan_counts(e->f_counts.as<uint32_t>(), B, e->f_acc.as<uint64_t>(), e->f_cursor.as<uint32_t>(), &misc->maxsz, s);
        flat_launch_scatter(e->f_cur.as<uint64_t>(), cur_n, B, e->f_cursor.as<uint32_t>(), e->f_sorted.as<uint64_t>(), s);
        flat_launch_sort_flush(e->f_sorted.as<uint64_t>(), e->f_acc.as<uint64_t>(), B, (uint32_t)k, e->f_mapping.as<uint32_t>(),
                               fc.threshold_range, base, e->f_thr.as<uint8_t>(), e->f_free_cnt.as<uint64_t>(),
                               e->f_bump_cnt.as<uint64_t>(), e->f_first.as<uint32_t>(), &misc->err, s);
        launch_scan_u64(e->f_free_cnt.as<uint64_t>(), B, e->f_free_off.as<uint64_t>(), s);
        launch_scan_u64(e->f_bump_cnt.as<uint64_t>(), B, e->f_bump_off.as<uint64_t>(), s);
        uint64_t tot[2];
        CU(cudaMemcpyAsync(&tot[0], e->f_free_off.as<uint64_t>() + B, 8, cudaMemcpyDeviceToHost, s));
        CU(cudaMemcpyAsync(&tot[1], e->f_bump_off.as<uint64_t>() + B, 8, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        CU(e->f_free_out.ensure(std::max<uint64_t>(tot[0], 1) * 8));
        flat_launch_emit(e->f_sorted.as<uint64_t>(), e->f_acc.as<uint64_t>(), B, base, e->f_free_cnt.as<uint64_t>(),
                         e->f_free_off.as<uint64_t>(), e->f_bump_cnt.as<uint64_t>(), e->f_bump_off.as<uint64_t>(),
                         e->f_first.as<uint32_t>(), e->f_free_out.as<uint64_t>(), e->f_next.as<uint64_t>(), s);
        const size_t old = free_positions.size();
        free_positions.resize(old + tot[0]);
        if (tot[0]) CU(cudaMemcpyAsync(free_positions.data() + old, e->f_free_out.p, tot[0] * 8, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        std::swap(e->f_cur, e->f_next);
        cur_n = tot[1];
    }
    uint32_t err0 = 0;
    CU(cudaMemcpy(&err0, &misc->err, 4, cudaMemcpyDeviceToHost));
    if (err0) return fail(SHG_ERR_BUCKET, "a threshold-layer bucket holds more than 1024 keys");
    out->layers = layers;
    for (size_t i = 0; i < layer_bases.size() && i < 3; i++) out->layer_bases[i] = layer_bases[i];
    out->stage_ms[1] = ms_since(t);
    t = clk::now();

    // ---- fallback PHF over the keys bumped from the last layer (:124-128)
    std::vector<uint64_t> bumped(cur_n);
    if (cur_n) CU(cudaMemcpy(bumped.data(), e->f_cur.p, cur_n * 8, cudaMemcpyDeviceToHost));
    std::string fb_bytes;
    std::vector<uint64_t> fb_offs{0};
    for (uint64_t h : bumped) {
        fb_bytes += std::to_string(h);
        fb_offs.push_back(fb_bytes.size());
    }
    out->nfallback_keys = cur_n;
    shg_params fp{SHG_SHOCKHASH2, (int)k, 2000, SHG_MODE_DEFAULT, 0};
    {
        float hms = 0;
        shg_status st = hash_strings_into(e, fb_bytes.data(), fb_offs.data(), cur_n, hms);
        if (st) return st;
        st = build_core(e, &fp, e->first.as<uint64_t>(), e->second.as<uint64_t>(), cur_n, &out->fallback, hms);
        if (st) return st;
    }
    shg_mphf *fbq = nullptr;
    {
        shg_status st = shg_mphf_create(&fp, &out->fallback, &fbq);
        if (st) return fail(st, "fallback query object");
    }
    // free positions of the fallback keys (:129-139)
    const uint64_t additional = cur_n - free_positions.size();
    const uint64_t handled = layer_bases.back();
    {
        uint64_t i = 0;
        for (; i < additional - keys_in_end_bucket; i++) free_positions.push_back(handled + i / k);
        for (; i < additional; i++) free_positions.push_back(nbuckets + i);
    }
    out->stage_ms[2] = ms_since(t);
    t = clk::now();

    // ---- every key's bucket (evaluateKPerfect), fallback keys through the fallback PHF
    CU(e->f_bucket.ensure(nn * 8));
    CU(e->f_last.ensure(nn * 8));
    CU(e->f_list.ensure(nn * 8));
    CU(cudaMemcpyAsync(e->f_lb.p, layer_bases.data(), layer_bases.size() * 8, cudaMemcpyHostToDevice, s));
    flat_launch_assign(e->f_mhc0.as<uint64_t>(), n, (uint32_t)layers, e->f_lb.as<uint64_t>(), e->f_thr.as<uint8_t>(),
                       e->f_mapping.as<uint32_t>(), e->f_bucket.as<uint64_t>(), e->f_last.as<uint64_t>(), s);
    unsigned long long *cnt = &misc->work[7];
    flat_launch_fallback_list(e->f_bucket.as<uint64_t>(), n, cnt, e->f_list.as<uint64_t>(), s);
    unsigned long long nfb = 0;
    CU(cudaMemcpyAsync(&nfb, cnt, 8, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (nfb) {
        std::vector<uint64_t> idx(nfb), last(nfb), vals(nfb);
        CU(cudaMemcpy(idx.data(), e->f_list.p, nfb * 8, cudaMemcpyDeviceToHost));
        {  // input order: the device listed them in any order; key indices are below 2^32, so two
           // 16-bit counting passes sort them
            std::vector<uint64_t> tmp(nfb);
            std::vector<uint64_t> cnt(1 << 16);
            for (int pass = 0; pass < 2; pass++) {
                const int sh = 16 * pass;
                std::fill(cnt.begin(), cnt.end(), 0);
                for (uint64_t v : idx) cnt[(v >> sh) & 0xFFFF]++;
                uint64_t sum = 0;
                for (uint64_t &c : cnt) {
                    const uint64_t x = c;
                    c = sum;
                    sum += x;
                }
                for (uint64_t v : idx) tmp[cnt[(v >> sh) & 0xFFFF]++] = v;
                idx.swap(tmp);
            }
        }
        // re-mixed hashes of the fallback keys, gathered on the device
        CU(e->f_tmp.ensure(nfb * 8));
        CU(e->f_tmp2.ensure(nfb * 8));
        CU(cudaMemcpyAsync(e->f_tmp.p, idx.data(), nfb * 8, cudaMemcpyHostToDevice, s));
        flat_launch_gather(e->f_tmp.as<uint64_t>(), e->f_last.as<uint64_t>(), nfb, e->f_tmp2.as<uint64_t>(), s);
        CU(cudaMemcpyAsync(last.data(), e->f_tmp2.p, nfb * 8, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        // each fallback key is the decimal string of its re-mixed hash, queried through the fallback
        // PHF (a read-only host object) on the host's threads, a contiguous range each
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const uint64_t nt = std::max<uint64_t>(1, std::min<uint64_t>(hw, nfb / 16384));
        std::vector<shg_status> tst(nt, SHG_OK);
        auto query_range = [&](uint64_t t) {
            const uint64_t j0 = nfb * t / nt, j1 = nfb * (t + 1) / nt;
            std::string qb;
            std::vector<uint64_t> qo{0};
            for (uint64_t j = j0; j < j1; j++) {
                qb += std::to_string(last[j]);
                qo.push_back(qb.size());
            }
            std::vector<uint64_t> phf(j1 - j0);
            tst[t] = shg_mphf_query_strings(fbq, qb.data(), qo.data(), j1 - j0, phf.data());
            for (uint64_t j = j0; j < j1 && tst[t] == SHG_OK; j++) {
                const uint64_t q = phf[j - j0];
                if (q >= free_positions.size()) {
                    tst[t] = SHG_ERR_CUDA;
                    break;
                }
                const uint64_t b = free_positions[q];  // select1(phf + 1) - phf (:295)
                vals[j] = b < nbuckets ? b : ~1ull;    // keys past the last full bucket are not searched
            }
        };
        auto query_part = [&](unsigned t) { query_range(t); };
        run_parts((unsigned)nt, query_part);
        for (shg_status qs : tst)
            if (qs) return fail(qs, qs == SHG_ERR_CUDA ? "fallback value outside the free positions" : "fallback query");
        CU(cudaMemcpyAsync(e->f_tmp2.p, vals.data(), nfb * 8, cudaMemcpyHostToDevice, s));
        flat_launch_set_buckets(e->f_tmp.as<uint64_t>(), e->f_tmp2.as<uint64_t>(), nfb, e->f_bucket.as<uint64_t>(), s);
    }
    shg_mphf_destroy(fbq);
    // keys grouped k per bucket, input order inside a bucket (:149-158)
    const uint64_t leaf_n = nbuckets * k;
    CU(e->f_slot.ensure(std::max<uint64_t>(leaf_n, 1) * 4));
    CU(e->f_leaf_keys.ensure(std::max<uint64_t>(leaf_n, 1) * 8));
    CU(e->f_cursor.ensure(std::max<uint64_t>(nbuckets, 1) * 4));
    flat_launch_group(e->f_bucket.as<uint64_t>(), n, nbuckets, (uint32_t)k, e->f_cursor.as<uint32_t>(), e->f_slot.as<uint32_t>(),
                      e->f_mhc0.as<uint64_t>(), e->f_leaf_keys.as<uint64_t>(), &misc->err, s);
    out->stage_ms[3] = ms_since(t);
    t = clk::now();

    // ---- one bipartite leaf search per bucket (:160-168)
    std::vector<Node> nodes(nbuckets);
    std::vector<uint32_t> ids(nbuckets);
    const Config &c2 = config_of(SHG_SHOCKHASH2, kMaxLeaf2);
    for (uint64_t b = 0; b < nbuckets; b++) {
        Node &nd = nodes[b];
        memset(&nd, 0, sizeof nd);
        nd.start = (uint32_t)(b * k);
        nd.m = (uint16_t)k;
        nd.kind = kLeaf;
        nd.g = (uint8_t)c2.golomb((uint32_t)k);
        ids[b] = (uint32_t)b;
    }
    CU(e->f_nodes.ensure(std::max<uint64_t>(nbuckets, 1) * sizeof(Node)));
    CU(e->f_ids.ensure(std::max<uint64_t>(nbuckets, 1) * 4));
    CU(e->f_codes.ensure(std::max<uint64_t>(nbuckets, 1) * 8));
    CU(e->f_bits.ensure(std::max<uint64_t>(leaf_n, 1)));
    if (nbuckets) {
        CU(cudaMemcpyAsync(e->f_nodes.p, nodes.data(), nbuckets * sizeof(Node), cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(e->f_ids.p, ids.data(), nbuckets * 4, cudaMemcpyHostToDevice, s));
        const uint32_t smax = k > 64 ? 16384 : 4096, cmax = k > 64 ? 16384 : 2048;
        const uint64_t per_warp = (sh2_scratch_bytes(smax, cmax, (int)k) + 255) & ~255ull;
        const Tuning ftun = e->tuning_of(kTuningFlat, (int)k);
        int bps = std::max(1, std::min(8, (228 * 1024) / (4 * sh2_smem_per_warp((int)k) + 1024)));
        if (ftun.leaf_bps > 0) bps = std::min(bps, ftun.leaf_bps);
        const int grid = std::max(1, std::min<int>(e->sms * bps, (int)((nbuckets + 3) / 4)));
        CU(e->scratch.ensure(per_warp * (uint64_t)grid * 4));
        CU(cudaMemsetAsync(&misc->work[1], 0, 5 * sizeof(unsigned long long), s));  // the fallback build's counts
        launch_leaves_sh2_ctr(e->f_nodes.as<Node>(), e->f_ids.as<uint32_t>(), (uint32_t)nbuckets, e->f_leaf_keys.as<uint64_t>(),
                              e->f_codes.as<uint64_t>(), e->f_bits.as<uint8_t>(), e->scratch.as<uint8_t>(), per_warp, smax, cmax,
                              &misc->err, misc->work, &misc->leaf_ctr, grid, s, (int)k, kQuadMinFlat, ftun.leaf_minb);
        CU(cudaGetLastError());
        CU(cudaMemcpyAsync(e->flat_work, &misc->work[1], sizeof(e->flat_work), cudaMemcpyDeviceToHost, s));
    } else {
        for (auto &w : e->flat_work) w = 0;
    }
    uint32_t err = 0;
    CU(cudaMemcpyAsync(&err, &misc->err, 4, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (err & kErrInternal) return fail(SHG_ERR_CUDA, "a bucket did not receive exactly k keys");
    if (err) return fail(SHG_ERR_TRIAL_LIMIT, "a bucket's leaf search exceeded its capacity (duplicate keys?)");
    out->stage_ms[4] = ms_since(t);
    t = clk::now();

    // ---- products: packed thresholds and seeds, seed fallback map, free positions, retrieval input
    std::vector<uint64_t> seeds(nbuckets);
    std::vector<uint8_t> thr(nbuckets);
    if (nbuckets) {
        CU(cudaMemcpyAsync(seeds.data(), e->f_codes.p, nbuckets * 8, cudaMemcpyDeviceToHost, s));
        CU(cudaMemcpyAsync(thr.data(), e->f_thr.p, nbuckets, cudaMemcpyDeviceToHost, s));
    }
    CU(cudaStreamSynchronize(s));
    std::vector<uint64_t> fbb, fbs;
    const uint64_t max_seed = fc.seed_bits >= 64 ? ~0ull : (1ull << fc.seed_bits);
    const size_t block_bytes = nbuckets * 8 + 2 * nbuckets * 8 + free_positions.size() * 8 + leaf_n * 9 + 256;
    PinnedBlock *blk = acquire_pinned(e, block_bytes);
    if (!blk) return fail(SHG_ERR_OOM, "pinned host allocation failed");
    uint8_t *hp = (uint8_t *)blk->p;
    out->owner = blk;
    out->thresholds_and_seeds = (uint64_t *)hp;
    hp += nbuckets * 8;
    for (uint64_t b = 0; b < nbuckets; b++) {
        uint64_t sd = seeds[b];
        if (sd >= max_seed || sd == 0) {  // :163-166
            fbb.push_back(b);
            fbs.push_back(sd);
            sd = 0;
        }
        out->thresholds_and_seeds[b] = sd << fc.threshold_bits | thr[b];
    }
    out->nfallback_seeds = fbb.size();
    out->fallback_seed_buckets = (uint64_t *)hp;
    memcpy(hp, fbb.data(), fbb.size() * 8);
    hp += nbuckets * 8;
    out->fallback_seeds = (uint64_t *)hp;
    memcpy(hp, fbs.data(), fbs.size() * 8);
    hp += nbuckets * 8;
    out->nfree = free_positions.size();
    out->free_positions = (uint64_t *)hp;
    memcpy(hp, free_positions.data(), free_positions.size() * 8);
    hp += free_positions.size() * 8;
    out->ribbon_n = leaf_n;
    out->ribbon_keys = (uint64_t *)hp;
    hp += leaf_n * 8;
    out->ribbon_bits = hp;
    if (leaf_n) {
        CU(cudaMemcpyAsync(out->ribbon_keys, e->f_leaf_keys.p, leaf_n * 8, cudaMemcpyDeviceToHost, s));
        CU(cudaMemcpyAsync(out->ribbon_bits, e->f_bits.p, leaf_n, cudaMemcpyDeviceToHost, s));
    }
    CU(cudaStreamSynchronize(s));
    out->stage_ms[5] = ms_since(t);
    out->stage_ms[7] = ms_since(t_start);
    return SHG_OK;
}

} // namespace

namespace shg {
// The engine's stream and device, for the other translation units' entry points.
cudaStream_t engine_stream(shg_engine *e, int *device) {
    *device = e->device;
    return e->stream;
}
// Reusable device buffers of the engine for the retrieval build: slot 0 its scratch region, 1 and 2
// the staging of host keys and bits (the input buffers of the other builds).
void *engine_scratch(shg_engine *e, int slot, size_t bytes, cudaError_t &err) {
    DevBuf &b = slot == 0 ? e->ret_scratch : slot == 1 ? e->in_keys : e->in_bytes;
    err = b.ensure(bytes);
    return err == cudaSuccess ? b.p : nullptr;
}
} // namespace shg

extern "C" {

// ------------------------------------------------------------------ tuning table
// One parameter per line: "<variant> <leaf size> <name> <value>" (variant as shg_variant, or 4 for
// ShockHash2Flat<k>); '#' starts a comment. Unknown names or out-of-range values reject the file.
static shg_status set_tuning(shg_engine *e, int variant, int leaf, const std::string &name, int64_t v) {
    if (variant < 1 || variant > SHG_SIMDSHOCKHASH_ROTATION || leaf < 1 || leaf > kMaxLeaf2)
        return fail(SHG_ERR_ARG, "tuning: no configuration variant " + std::to_string(variant) + " leaf " + std::to_string(leaf));
    if (variant == SHG_SHOCKHASH_ROTATION) variant = SHG_SHOCKHASH;
    if (variant == SHG_SIMDSHOCKHASH_ROTATION) variant = SHG_SIMDSHOCKHASH;
    std::lock_guard<std::mutex> lock(e->tuning_mu);
    Tuning t = e->tuning.count({variant, leaf}) ? e->tuning[{variant, leaf}] : Tuning();
    if (name == "split_seeds_per_lane") t.split.spl = (int)v;
    else if (name == "split_threads") t.split.threads = (int)v;
    else if (name == "split_round_div") t.split.round_div = (int)v;
    else if (name == "split_arith") t.split.arith = (int)v;
    else if (name == "leaf_blocks_per_sm" && v >= 0 && v <= 16) t.leaf_bps = (int)v;
    else if (name == "leaf_min_blocks" && (v == 4 || v == 6 || v == 8)) t.leaf_minb = (int)v;
    else if (name == "sh1_seeds_per_lane" && (v == 1 || v == 2)) t.sh1_spl = (int)v;
    else if (name == "queue_lag_rounds" && v >= 0 && v <= 64) t.queue_lag = (int)v;
    else return fail(SHG_ERR_ARG, "tuning: bad parameter " + name + " = " + std::to_string(v));
    if (!split_tuning_valid(t.split.spl, t.split.threads, t.split.round_div, t.split.arith))
        return fail(SHG_ERR_ARG, "tuning: bad parameter " + name + " = " + std::to_string(v));
    e->tuning[{variant, leaf}] = t;
    return SHG_OK;
}

static shg_status load_tuning(shg_engine *e, const char *path) {
    FILE *f = fopen(path, "r");
    if (!f) return fail(SHG_ERR_ARG, std::string("tuning: cannot open ") + path);
    char line[512];
    shg_status st = SHG_OK;
    while (st == SHG_OK && fgets(line, sizeof line, f)) {
        if (char *hash = strchr(line, '#')) *hash = 0;
        int variant = 0, leaf = 0;
        char name[128];
        long long v = 0;
        const int got = sscanf(line, "%d %d %127s %lld", &variant, &leaf, name, &v);
        if (got <= 0) continue;  // blank or comment
        st = got == 4 ? set_tuning(e, variant, leaf, name, v) : fail(SHG_ERR_ARG, std::string("tuning: malformed line in ") + path);
    }
    fclose(f);
    if (st == SHG_OK) e->tuning_source = path;
    return st;
}

// The table next to the package (shockhash_b200/tuning.tsv beside _lib/libshg.so), or the file
// named by SHG_TUNING_TABLE (empty: none).
static std::string default_tuning_path() {
    if (const char *env = getenv("SHG_TUNING_TABLE")) return env;
    Dl_info info;
    if (!dladdr((void *)&default_tuning_path, &info) || !info.dli_fname) return "";
    std::string so = info.dli_fname;
    const size_t slash = so.rfind('/');
    const std::string dir = slash == std::string::npos ? "." : so.substr(0, slash);
    return dir + "/../tuning.tsv";
}

shg_status shg_engine_set_tuning(shg_engine *e, int variant, int leaf_size, const char *name, int64_t value) {
    if (!e || !name) return fail(SHG_ERR_ARG, "null argument");
    return set_tuning(e, variant, leaf_size, name, value);
}

shg_status shg_engine_get_tuning(shg_engine *e, int variant, int leaf_size, const char *name, int64_t *value) {
    if (!e || !name || !value) return fail(SHG_ERR_ARG, "null argument");
    const Tuning t = e->tuning_of(variant, leaf_size);
    const std::string n = name;
    if (n == "split_seeds_per_lane") *value = t.split.spl;
    else if (n == "split_threads") *value = t.split.threads;
    else if (n == "split_round_div") *value = t.split.round_div;
    else if (n == "split_arith") *value = t.split.arith;
    else if (n == "leaf_blocks_per_sm") *value = t.leaf_bps;
    else if (n == "leaf_min_blocks") *value = t.leaf_minb;
    else if (n == "sh1_seeds_per_lane") *value = t.sh1_spl;
    else if (n == "queue_lag_rounds") *value = t.queue_lag;
    else return fail(SHG_ERR_ARG, "tuning: unknown parameter " + n);
    return SHG_OK;
}

shg_status shg_engine_load_tuning(shg_engine *e, const char *path) {
    if (!e || !path) return fail(SHG_ERR_ARG, "null argument");
    return load_tuning(e, path);
}

const char *shg_engine_tuning_source(const shg_engine *e) { return e ? e->tuning_source.c_str() : ""; }

shg_status shg_engine_create(int device, shg_engine **out) {
    if (!out) return fail(SHG_ERR_ARG, "null output");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return fail(SHG_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= count) return fail(SHG_ERR_ARG, "device index out of range");
    CU(cudaSetDevice(device));
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return fail(SHG_ERR_NO_DEVICE, "libshg is built for sm_100a (B200); found sm_" + std::to_string(prop.major) + std::to_string(prop.minor));
    auto *e = new shg_engine();
    e->device = device;
    e->sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete e;
        return fail(SHG_ERR_CUDA, "stream creation failed");
    }
    for (auto &ev : e->ev) cudaEventCreate(&ev);
    for (auto &ev : e->chunk_ev) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&e->join_ev, cudaEventDisableTiming);
    if (cudaStreamCreateWithFlags(&e->stream2, cudaStreamNonBlocking) != cudaSuccess) {
        delete e;
        return fail(SHG_ERR_CUDA, "stream creation failed");
    }
    if (const char *c = getenv("SHG_PIPE_CHUNKS")) e->pipe_chunks = std::max(1, std::min(shg_engine::kMaxChunks, atoi(c)));
    const std::string tpath = default_tuning_path();
    if (!tpath.empty()) {
        if (FILE *f = fopen(tpath.c_str(), "r")) {  // a table that exists must be valid
            fclose(f);
            const shg_status st = load_tuning(e, tpath.c_str());
            if (st != SHG_OK) {
                delete e;
                return st;
            }
        }
    }
    *out = e;
    return SHG_OK;
}

void shg_engine_destroy(shg_engine *e) {
    if (!e) return;
    cudaSetDevice(e->device);
    delete e;
}

static shg_status timed_hash_u64(shg_engine *e, const uint64_t *d_keys, uint64_t n, float &ms) {
    CU(e->first.ensure(std::max<uint64_t>(n, 1) * 8));
    CU(e->second.ensure(std::max<uint64_t>(n, 1) * 8));
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, e->stream);
    launch_spooky_u64(d_keys, n, e->first.as<uint64_t>(), e->second.as<uint64_t>(), e->stream);
    cudaEventRecord(b, e->stream);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CU(cudaGetLastError());
    return SHG_OK;
}

shg_status shg_build_hash128_device(shg_engine *e, const shg_params *p, const uint64_t *d_first, const uint64_t *d_second,
                                    uint64_t n, shg_result *out) {
    if (!e || !out) return fail(SHG_ERR_ARG, "null engine or result");
    shg_status st = check_params(p, n);
    if (st) return st;
    CU(cudaSetDevice(e->device));
    return build_core(e, p, d_first, d_second, n, out, 0.f);
}

shg_status shg_build_hash128(shg_engine *e, const shg_params *p, const uint64_t *first, const uint64_t *second, uint64_t n,
                             shg_result *out) {
    if (!e || !out || (n && (!first || !second))) return fail(SHG_ERR_ARG, "null argument");
    shg_status st = check_params(p, n);
    if (st) return st;
    CU(cudaSetDevice(e->device));
    CU(e->first.ensure(std::max<uint64_t>(n, 1) * 8));
    CU(e->second.ensure(std::max<uint64_t>(n, 1) * 8));
    if (n) {
        if (shg_status cs = h2d_from_host(e, e->first.p, first, n * 8, e->stream)) return cs;
        if (shg_status cs = h2d_from_host(e, e->second.p, second, n * 8, e->stream)) return cs;
    }
    return build_core(e, p, e->first.as<uint64_t>(), e->second.as<uint64_t>(), n, out, 0.f);
}

shg_status shg_build_shard_hash128(shg_engine *e, const shg_params *p, const uint64_t *first, const uint64_t *second,
                                   uint64_t n, uint64_t nb_global, uint64_t b0, uint64_t b1, shg_result *out) {
    if (!e || !out || (n && (!first || !second))) return fail(SHG_ERR_ARG, "null argument");
    if (b0 >= b1 || b1 > nb_global) return fail(SHG_ERR_ARG, "bucket range must satisfy b0 < b1 <= nb_global");
    shg_status st = check_params(p, n);
    if (st) return st;
    CU(cudaSetDevice(e->device));
    CU(e->first.ensure(std::max<uint64_t>(n, 1) * 8));
    CU(e->second.ensure(std::max<uint64_t>(n, 1) * 8));
    if (n) {
        if (shg_status cs = h2d_from_host(e, e->first.p, first, n * 8, e->stream)) return cs;
        if (shg_status cs = h2d_from_host(e, e->second.p, second, n * 8, e->stream)) return cs;
    }
    const ShardSpec shard{nb_global, b0, b1};
    return build_batch(e, p, e->first.as<uint64_t>(), e->second.as<uint64_t>(), std::vector<uint64_t>{n}, out, 0.f, &shard);
}

shg_status shg_hash_u64_device(shg_engine *e, const uint64_t *d_keys, uint64_t n, uint64_t *d_first, uint64_t *d_second) {
    if (!e || (n && (!d_keys || !d_first || !d_second))) return fail(SHG_ERR_ARG, "null argument");
    if (!n) return SHG_OK;
    CU(cudaSetDevice(e->device));
    launch_spooky_u64(d_keys, n, d_first, d_second, e->stream);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(e->stream));
    return SHG_OK;
}

shg_status shg_build_batch_items(shg_engine *e, const shg_params *p, const shg_batch_item *items, uint64_t nitems,
                                 shg_result *outs) {
    if (!e || !outs || !items || nitems == 0) return fail(SHG_ERR_ARG, "null argument or empty batch");
    uint64_t total = 0, nkeys = 0;
    std::vector<uint64_t> nr(nitems);
    std::vector<ShardSpec> specs(nitems, ShardSpec{0, 0, 0});
    for (uint64_t r = 0; r < nitems; r++) {
        const shg_batch_item &it = items[r];
        if (it.n && !it.keys && (!it.first || !it.second)) return fail(SHG_ERR_ARG, "item without keys or fingerprints");
        if (it.b1 > it.b0) {
            if (it.b1 > it.nb_global) return fail(SHG_ERR_ARG, "bucket range must satisfy b0 < b1 <= nb_global");
            specs[r] = ShardSpec{it.nb_global, it.b0, it.b1};
        }
        nr[r] = it.n;
        total += it.n;
        if (it.keys) nkeys += it.n;
    }
    shg_status st = check_params(p, total);
    if (st) return st;
    CU(cudaSetDevice(e->device));
    cudaStream_t s = e->stream;
    CU(e->first.ensure(std::max<uint64_t>(total, 1) * 8));
    CU(e->second.ensure(std::max<uint64_t>(total, 1) * 8));
    CU(e->in_keys.ensure(std::max<uint64_t>(nkeys, 1) * 8));
    CU(cudaEventRecord(e->ev[7], s));
    uint64_t off = 0, koff = 0;
    for (uint64_t r = 0; r < nitems; r++) {
        const shg_batch_item &it = items[r];
        if (!it.n) continue;
        if (it.keys) {  // uint64 keys, hashed on the device as 8-byte strings
            CU(cudaMemcpyAsync(e->in_keys.as<uint64_t>() + koff, it.keys, it.n * 8, cudaMemcpyHostToDevice, s));
            launch_spooky_u64(e->in_keys.as<uint64_t>() + koff, it.n, e->first.as<uint64_t>() + off,
                              e->second.as<uint64_t>() + off, s);
            koff += it.n;
        } else {
            CU(cudaMemcpyAsync(e->first.as<uint64_t>() + off, it.first, it.n * 8, cudaMemcpyHostToDevice, s));
            CU(cudaMemcpyAsync(e->second.as<uint64_t>() + off, it.second, it.n * 8, cudaMemcpyHostToDevice, s));
        }
        off += it.n;
    }
    CU(cudaGetLastError());
    CU(cudaEventRecord(e->ev[0], s));
    CU(cudaEventSynchronize(e->ev[0]));
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev[7], e->ev[0]);
    return build_batch(e, p, e->first.as<uint64_t>(), e->second.as<uint64_t>(), nr, outs, ms, specs.data());
}

shg_status shg_build_shard_hash128_device(shg_engine *e, const shg_params *p, const uint64_t *d_first,
                                          const uint64_t *d_second, uint64_t n, uint64_t nb_global, uint64_t b0,
                                          uint64_t b1, shg_result *out) {
    if (!e || !out || (n && (!d_first || !d_second))) return fail(SHG_ERR_ARG, "null argument");
    if (b0 >= b1 || b1 > nb_global) return fail(SHG_ERR_ARG, "bucket range must satisfy b0 < b1 <= nb_global");
    shg_status st = check_params(p, n);
    if (st) return st;
    CU(cudaSetDevice(e->device));
    const ShardSpec shard{nb_global, b0, b1};
    return build_batch(e, p, d_first, d_second, std::vector<uint64_t>{n}, out, 0.f, &shard);
}

// On-disk form of a build result (no counterpart in the reference classes, which persist only the
// RiceBitVector, RiceBitVector.h:133-141). Little-endian: "SHGMPHF1", variant u32, leaf size u32,
// bucket size u64, n, nbuckets, desc_bits, ribbon_n (u64 each), bucket_size_acc and bucket_pos_acc
// ([nbuckets + 1] u64 each), the descriptors in RiceBitVector's stream layout (u64 word count, then
// the words, as sux::util::Vector writes them), ribbon_keys ([ribbon_n] u64), ribbon_bits
// ([ribbon_n] u8).
static const char kSaveMagic[8] = {'S', 'H', 'G', 'M', 'P', 'H', 'F', '1'};

shg_status shg_result_save(const shg_params *p, const shg_result *r, const char *path) {
    if (!p || !r || !path) return fail(SHG_ERR_ARG, "null argument");
    if (r->nbuckets == 0 || !r->bucket_size_acc || !r->bucket_pos_acc || (r->desc_words && !r->descriptors) ||
        (r->ribbon_n && (!r->ribbon_keys || !r->ribbon_bits)))
        return fail(SHG_ERR_ARG, "not a build result");
    FILE *f = fopen(path, "wb");
    if (!f) return fail(SHG_ERR_ARG, std::string("cannot open ") + path + " for writing");
    const uint32_t vl[2] = {(uint32_t)p->variant, (uint32_t)p->leaf_size};
    const uint64_t head[5] = {p->bucket_size, r->n, r->nbuckets, r->desc_bits, r->ribbon_n};
    const size_t acc = r->nbuckets + 1;
    bool ok = fwrite(kSaveMagic, 1, 8, f) == 8 && fwrite(vl, 4, 2, f) == 2 && fwrite(head, 8, 5, f) == 5 &&
              fwrite(r->bucket_size_acc, 8, acc, f) == acc && fwrite(r->bucket_pos_acc, 8, acc, f) == acc &&
              fwrite(&r->desc_words, 8, 1, f) == 1 &&
              fwrite(r->descriptors, 8, r->desc_words, f) == r->desc_words &&
              fwrite(r->ribbon_keys, 8, r->ribbon_n, f) == r->ribbon_n &&
              fwrite(r->ribbon_bits, 1, r->ribbon_n, f) == r->ribbon_n;
    ok = (fclose(f) == 0) && ok;
    return ok ? SHG_OK : fail(SHG_ERR_ARG, std::string("write to ") + path + " failed");
}

shg_status shg_result_load(const char *path, shg_params *p, shg_result *out) {
    if (!path || !p || !out) return fail(SHG_ERR_ARG, "null argument");
    memset(out, 0, sizeof(shg_result));
    FILE *f = fopen(path, "rb");
    if (!f) return fail(SHG_ERR_ARG, std::string("cannot open ") + path);
    auto bad = [&](const char *why) {
        fclose(f);
        return fail(SHG_ERR_ARG, std::string(path) + ": " + why);
    };
    char magic[8];
    uint32_t vl[2];
    uint64_t head[5], words = 0;
    if (fread(magic, 1, 8, f) != 8 || memcmp(magic, kSaveMagic, 8) != 0) return bad("not a saved build result");
    if (fread(vl, 4, 2, f) != 2 || fread(head, 8, 5, f) != 5) return bad("truncated header");
    const uint64_t n = head[1], nb = head[2], bits = head[3], rn = head[4];
    if (fseek(f, 0, SEEK_END) != 0) return bad("seek failed");
    const uint64_t fsize = (uint64_t)ftell(f);
    const uint64_t fixed = 8 + 8 + 40;
    {  // the configuration must be one this library builds
        shg_params cp{(int)vl[0], (int)vl[1], head[0], SHG_MODE_DEFAULT, 0};
        if (vl[0] > 16 || vl[1] > 4096 || check_params(&cp, 0) != SHG_OK) return bad("unknown configuration");
    }
    // every count is bounded by the file size before any product is formed
    if (nb == 0 || nb > fsize / 16 || rn > n || rn > fsize / 9 || bits < 1 || bits > 8 * fsize)
        return bad("inconsistent sizes");
    if (fseek(f, (long)(fixed + 16 * (nb + 1)), SEEK_SET) != 0 || fread(&words, 8, 1, f) != 1) return bad("truncated");
    if (words > fsize / 8 || words != ((bits + 7) / 8 + 14) / 8) return bad("descriptor word count does not match its bit count");
    if (fsize != fixed + 16 * (nb + 1) + 8 + 8 * words + 9 * rn) return bad("file size does not match its header");
    const size_t acc_bytes = (nb + 1) * 8;
    const size_t bytes = 2 * acc_bytes + words * 8 + rn * 9 + 64;
    auto *blk = new PinnedBlock();
    blk->host = true;
    blk->in_use = true;
    blk->refs = 1;
    blk->p = calloc(1, bytes);
    blk->cap = bytes;
    if (!blk->p) {
        delete blk;
        return bad("host allocation failed");
    }
    uint8_t *hp = (uint8_t *)blk->p;
    out->owner = blk;
    out->n = n;
    out->nbuckets = nb;
    out->bucket_size_acc = (uint64_t *)hp;
    out->bucket_pos_acc = (uint64_t *)(hp + acc_bytes);
    out->descriptors = (uint64_t *)(hp + 2 * acc_bytes);
    out->ribbon_keys = (uint64_t *)(hp + 2 * acc_bytes + words * 8);
    out->ribbon_bits = hp + 2 * acc_bytes + words * 8 + rn * 8;
    out->desc_words = words;
    out->desc_bits = bits;
    out->ribbon_n = rn;
    fseek(f, (long)fixed, SEEK_SET);
    const bool ok = fread(out->bucket_size_acc, 8, nb + 1, f) == nb + 1 && fread(out->bucket_pos_acc, 8, nb + 1, f) == nb + 1 &&
                    fseek(f, 8, SEEK_CUR) == 0 && fread(out->descriptors, 8, words, f) == words &&
                    fread(out->ribbon_keys, 8, rn, f) == rn && fread(out->ribbon_bits, 1, rn, f) == rn;
    fclose(f);
    // the accumulators start at zero, never decrease, end at n keys and within the code bits
    bool mono = ok && out->bucket_size_acc[0] == 0 && out->bucket_pos_acc[0] == 0;
    for (uint64_t b = 0; mono && b < nb; b++)
        mono = out->bucket_size_acc[b] <= out->bucket_size_acc[b + 1] && out->bucket_pos_acc[b] <= out->bucket_pos_acc[b + 1];
    if (!mono || out->bucket_size_acc[nb] != n || out->bucket_pos_acc[nb] >= bits) {
        release_pinned(blk);
        memset(out, 0, sizeof(shg_result));
        return fail(SHG_ERR_ARG, std::string(path) + ": truncated or inconsistent arrays");
    }
    p->variant = (int)vl[0];
    p->leaf_size = (int)vl[1];
    p->bucket_size = head[0];
    p->mode = SHG_MODE_DEFAULT;
    p->max_trials = 0;
    return SHG_OK;
}

shg_status shg_merge_shards(const shg_params *p, const shg_result *shards, uint64_t nshards, shg_result *out) {
    if (!p || !shards || !out || nshards == 0) return fail(SHG_ERR_ARG, "null argument or no shards");
    memset(out, 0, sizeof(shg_result));
    uint64_t n = 0, nb = 0, code_bits = 0, rn = 0;
    for (uint64_t g = 0; g < nshards; g++) {
        const shg_result &r = shards[g];
        if (r.nbuckets == 0 || !r.bucket_size_acc || !r.bucket_pos_acc || r.desc_bits < 1 ||
            (r.desc_words && !r.descriptors) || (r.ribbon_n && (!r.ribbon_keys || !r.ribbon_bits)))
            return fail(SHG_ERR_ARG, "shard " + std::to_string(g) + " is not a build result");
        if (r.bucket_size_acc[r.nbuckets] != r.n) return fail(SHG_ERR_ARG, "shard key count mismatch");
        n += r.n;
        nb += r.nbuckets;
        code_bits += r.desc_bits - 1;  // without the shard's sentinel
        rn += r.ribbon_n;
    }
    if (nb != std::max<uint64_t>(1, (n + p->bucket_size - 1) / p->bucket_size))
        return fail(SHG_ERR_ARG, "shards do not cover the buckets of one structure of " + std::to_string(n) + " keys");
    // RiceBitVector::Builder: the sentinel appendFixed(1, 1), then the word count of its final resize
    const uint64_t bits = code_bits + 1;
    const uint64_t words = ((bits + 7) / 8 + 14) / 8;
    const size_t acc_bytes = (nb + 1) * 8;
    const size_t bytes = 2 * acc_bytes + words * 8 + rn * 8 + rn + 64;
    auto *blk = new PinnedBlock();
    blk->host = true;
    blk->in_use = true;
    blk->refs = 1;
    blk->p = calloc(1, bytes);
    blk->cap = bytes;
    if (!blk->p) {
        delete blk;
        return fail(SHG_ERR_OOM, "host allocation failed");
    }
    uint8_t *hp = (uint8_t *)blk->p;
    out->owner = blk;
    out->n = n;
    out->nbuckets = nb;
    out->bucket_size_acc = (uint64_t *)hp;
    out->bucket_pos_acc = (uint64_t *)(hp + acc_bytes);
    out->descriptors = (uint64_t *)(hp + 2 * acc_bytes);
    out->ribbon_keys = (uint64_t *)(hp + 2 * acc_bytes + words * 8);
    out->ribbon_bits = hp + 2 * acc_bytes + words * 8 + rn * 8;
    out->desc_words = words;
    out->desc_bits = bits;
    out->ribbon_n = rn;
    uint64_t kb = 0, bb = 0, bitpos = 0, ro = 0;
    for (uint64_t g = 0; g < nshards; g++) {
        const shg_result &r = shards[g];
        for (uint64_t b = 0; b < r.nbuckets; b++) {
            out->bucket_size_acc[bb + b] = kb + r.bucket_size_acc[b];
            out->bucket_pos_acc[bb + b] = bitpos + r.bucket_pos_acc[b];
        }
        // appendRiceBitVector (RiceBitVector.h:102-120): the shard's code bits at the current bit position
        const uint64_t nbits = r.desc_bits - 1;
        for (uint64_t w = 0; w * 64 < nbits; w++) {
            uint64_t v = r.descriptors[w];
            const uint64_t left = nbits - w * 64;
            if (left < 64) v &= (1ull << left) - 1;
            const uint64_t at = bitpos + w * 64;
            out->descriptors[at / 64] |= v << (at % 64);
            if (at % 64) out->descriptors[at / 64 + 1] |= v >> (64 - at % 64);
        }
        if (r.ribbon_n) {
            memcpy(out->ribbon_keys + ro, r.ribbon_keys, r.ribbon_n * 8);
            memcpy(out->ribbon_bits + ro, r.ribbon_bits, r.ribbon_n);
        }
        kb += r.n;
        bb += r.nbuckets;
        bitpos += nbits;
        ro += r.ribbon_n;
    }
    out->bucket_size_acc[nb] = kb;
    out->bucket_pos_acc[nb] = bitpos;
    out->descriptors[bitpos / 64] |= 1ull << (bitpos % 64);  // sentinel
    return SHG_OK;
}

shg_status shg_build_u64_device(shg_engine *e, const shg_params *p, const uint64_t *d_keys, uint64_t n, shg_result *out) {
    if (!e || !out) return fail(SHG_ERR_ARG, "null engine or result");
    shg_status st = check_params(p, n);
    if (st) return st;
    CU(cudaSetDevice(e->device));
    float ms = 0;
    st = timed_hash_u64(e, d_keys, n, ms);
    if (st) return st;
    return build_core(e, p, e->first.as<uint64_t>(), e->second.as<uint64_t>(), n, out, ms);
}

shg_status shg_build_u64(shg_engine *e, const shg_params *p, const uint64_t *keys, uint64_t n, shg_result *out) {
    if (!e || !out || (n && !keys)) return fail(SHG_ERR_ARG, "null argument");
    shg_status st = check_params(p, n);
    if (st) return st;
    CU(cudaSetDevice(e->device));
    CU(e->in_keys.ensure(std::max<uint64_t>(n, 1) * 8));
    if (shg_status cs = h2d_from_host(e, e->in_keys.p, keys, n * 8, e->stream)) return cs;
    float ms = 0;
    st = timed_hash_u64(e, e->in_keys.as<uint64_t>(), n, ms);
    if (st) return st;
    return build_core(e, p, e->first.as<uint64_t>(), e->second.as<uint64_t>(), n, out, ms);
}

shg_status shg_build_batch_u64(shg_engine *e, const shg_params *p, const uint64_t *const *keys, const uint64_t *n,
                               uint64_t nreq, shg_result *outs) {
    if (!e || !outs || !keys || !n || nreq == 0) return fail(SHG_ERR_ARG, "null argument or empty batch");
    uint64_t total = 0;
    for (uint64_t r = 0; r < nreq; r++) {
        if (n[r] && !keys[r]) return fail(SHG_ERR_ARG, "null key array");
        total += n[r];
    }
    shg_status st = check_params(p, total);
    if (st) return st;
    CU(cudaSetDevice(e->device));
    CU(e->in_keys.ensure(std::max<uint64_t>(total, 1) * 8));
    uint64_t off = 0;
    for (uint64_t r = 0; r < nreq; r++) {
        if (n[r]) CU(cudaMemcpyAsync(e->in_keys.as<uint64_t>() + off, keys[r], n[r] * 8, cudaMemcpyHostToDevice, e->stream));
        off += n[r];
    }
    float ms = 0;
    st = timed_hash_u64(e, e->in_keys.as<uint64_t>(), total, ms);
    if (st) return st;
    return build_batch(e, p, e->first.as<uint64_t>(), e->second.as<uint64_t>(), std::vector<uint64_t>(n, n + nreq), outs, ms);
}

static shg_status hash_strings_dev(shg_engine *e, const char *bytes, const uint64_t *offsets, uint64_t n, float &ms) {
    return hash_strings_into(e, bytes, offsets, n, ms);
}
}  // extern "C"
shg_status hash_strings_into(shg_engine *e, const char *bytes, const uint64_t *offsets, uint64_t n, float &ms) {
    const uint64_t nbytes = n ? offsets[n] : 0;
    CU(e->in_bytes.ensure(std::max<uint64_t>(nbytes, 1)));
    CU(e->in_offsets.ensure((n + 1) * 8));
    CU(e->first.ensure(std::max<uint64_t>(n, 1) * 8));
    CU(e->second.ensure(std::max<uint64_t>(n, 1) * 8));
    if (shg_status cs = h2d_from_host(e, e->in_bytes.p, bytes, nbytes, e->stream)) return cs;
    if (shg_status cs = h2d_from_host(e, e->in_offsets.p, offsets, (n + 1) * 8, e->stream)) return cs;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, e->stream);
    launch_spooky_strings(e->in_bytes.as<uint8_t>(), e->in_offsets.as<uint64_t>(), n, e->first.as<uint64_t>(),
                          e->second.as<uint64_t>(), e->stream);
    cudaEventRecord(b, e->stream);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CU(cudaGetLastError());
    return SHG_OK;
}

extern "C" {
shg_status shg_build_strings(shg_engine *e, const shg_params *p, const char *bytes, const uint64_t *offsets, uint64_t n,
                             shg_result *out) {
    if (!e || !out || !offsets || (n && !bytes)) return fail(SHG_ERR_ARG, "null argument");
    shg_status st = check_params(p, n);
    if (st) return st;
    CU(cudaSetDevice(e->device));
    float ms = 0;
    st = hash_strings_dev(e, bytes, offsets, n, ms);
    if (st) return st;
    return build_core(e, p, e->first.as<uint64_t>(), e->second.as<uint64_t>(), n, out, ms);
}

shg_status shg_hash_strings(shg_engine *e, const char *bytes, const uint64_t *offsets, uint64_t n, uint64_t *first,
                            uint64_t *second) {
    if (!e || !offsets || !first || !second || (n && !bytes)) return fail(SHG_ERR_ARG, "null argument");
    CU(cudaSetDevice(e->device));
    float ms = 0;
    shg_status st = hash_strings_dev(e, bytes, offsets, n, ms);
    if (st) return st;
    if (n) {
        CU(cudaMemcpyAsync(first, e->first.p, n * 8, cudaMemcpyDeviceToHost, e->stream));
        CU(cudaMemcpyAsync(second, e->second.p, n * 8, cudaMemcpyDeviceToHost, e->stream));
    }
    CU(cudaStreamSynchronize(e->stream));
    return SHG_OK;
}

void shg_result_free(shg_result *r) {
    if (!r) return;
    if (r->owner) release_pinned((PinnedBlock *)r->owner);
    r->owner = nullptr;
    r->bucket_size_acc = r->bucket_pos_acc = r->descriptors = r->ribbon_keys = nullptr;
    r->ribbon_bits = nullptr;
}

static shg_status leaves_common(shg_engine *e, const uint64_t *keys, const uint64_t *leaf_offsets, uint64_t nleaves,
                                int max_leaf, int level, std::vector<Node> &nodes) {
    if (!e || !keys || !leaf_offsets) return fail(SHG_ERR_ARG, "null argument");
    nodes.resize(nleaves);
    for (uint64_t j = 0; j < nleaves; j++) {
        const uint64_t m = leaf_offsets[j + 1] - leaf_offsets[j];
        if (m < 2 || m > (uint64_t)max_leaf) return fail(SHG_ERR_ARG, "leaf size out of range");
        if (leaf_offsets[j + 1] >= (1ull << 32)) return fail(SHG_ERR_ARG, "too many keys");
        Node &n = nodes[j];
        memset(&n, 0, sizeof n);
        n.start = (uint32_t)leaf_offsets[j];
        n.m = (uint16_t)m;
        n.level = (uint8_t)level;
        n.kind = kLeaf;
        const Config &c = config_of(max_leaf == kMaxLeaf1 ? SHG_SHOCKHASH : SHG_SHOCKHASH2, max_leaf);
        n.g = (uint8_t)c.golomb((uint32_t)m);
    }
    return SHG_OK;
}

shg_status shg_sh2_construct_leaves(shg_engine *e, const uint64_t *keys, const uint64_t *leaf_offsets, uint64_t nleaves,
                                    uint64_t *seeds, uint8_t *bits) {
    std::vector<Node> nodes;
    shg_status st = leaves_common(e, keys, leaf_offsets, nleaves, kMaxLeaf2, 0, nodes);
    if (st) return st;
    if (!seeds || !bits) return fail(SHG_ERR_ARG, "null output");
    if (!nleaves) return SHG_OK;
    CU(cudaSetDevice(e->device));
    cudaStream_t s = e->stream;
    const uint64_t n = leaf_offsets[nleaves];
    std::vector<uint32_t> ids(nleaves);
    for (uint64_t j = 0; j < nleaves; j++) ids[j] = (uint32_t)j;
    CU(e->keys.ensure(n * 8));
    CU(e->nodes.ensure(nleaves * sizeof(Node)));
    CU(e->ids.ensure(nleaves * 4));
    CU(e->codes.ensure(nleaves * 8));
    CU(e->rib_bits.ensure(n));
    CU(e->misc.ensure(sizeof(Misc)));
    Misc *misc = e->misc.as<Misc>();
    CU(cudaMemsetAsync(misc, 0, sizeof(Misc), s));
    CU(cudaMemcpyAsync(e->keys.p, keys, n * 8, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(e->nodes.p, nodes.data(), nleaves * sizeof(Node), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(e->ids.p, ids.data(), nleaves * 4, cudaMemcpyHostToDevice, s));
    uint64_t maxm = 0;
    for (auto &nd : nodes) maxm = std::max<uint64_t>(maxm, nd.m);
    const uint32_t smax = maxm > 64 ? 16384 : 4096, cmax = maxm > 64 ? 16384 : 2048;
    const uint64_t per_warp = (sh2_scratch_bytes(smax, cmax, (int)maxm) + 255) & ~255ull;
    const int per_block_smem = 4 * sh2_smem_per_warp((int)maxm);
    const int blocks_per_sm = std::max(1, std::min(8, (228 * 1024) / (per_block_smem + 1024)));
    const int grid = std::max(1, std::min<int>(e->sms * blocks_per_sm, (int)((nleaves + 3) / 4)));
    CU(e->scratch.ensure(per_warp * (uint64_t)grid * 4));
    launch_leaves_sh2_ctr(e->nodes.as<Node>(), e->ids.as<uint32_t>(), (uint32_t)nleaves, e->keys.as<uint64_t>(),
                          e->codes.as<uint64_t>(), e->rib_bits.as<uint8_t>(), e->scratch.as<uint8_t>(), per_warp, smax, cmax,
                          &misc->err, misc->work, &misc->leaf_ctr, grid, s, (int)maxm);
    CU(cudaGetLastError());
    uint32_t err = 0;
    CU(cudaMemcpyAsync(seeds, e->codes.p, nleaves * 8, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(bits, e->rib_bits.p, n, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(&err, &misc->err, 4, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (err) return fail(SHG_ERR_TRIAL_LIMIT, "leaf search failed (error flags " + std::to_string(err) + ")");
    return SHG_OK;
}

shg_status shg_sh1_construct_leaves(shg_engine *e, const uint64_t *keys, const uint64_t *leaf_offsets, uint64_t nleaves,
                                    int level, uint64_t *codes, uint64_t *keys_by_cell, uint8_t *bits) {
    if (level < 0 || level >= kMaxLevels) return fail(SHG_ERR_ARG, "level out of range");
    std::vector<Node> nodes;
    shg_status st = leaves_common(e, keys, leaf_offsets, nleaves, kMaxLeaf1, level, nodes);
    if (st) return st;
    if (!codes || !keys_by_cell || !bits) return fail(SHG_ERR_ARG, "null output");
    if (!nleaves) return SHG_OK;
    CU(cudaSetDevice(e->device));
    cudaStream_t s = e->stream;
    const uint64_t n = leaf_offsets[nleaves];
    std::vector<uint32_t> ids(nleaves);
    for (uint64_t j = 0; j < nleaves; j++) ids[j] = (uint32_t)j;
    CU(e->keys.ensure(n * 8));
    CU(e->nodes.ensure(nleaves * sizeof(Node)));
    CU(e->ids.ensure(nleaves * 4));
    CU(e->codes.ensure(nleaves * 8));
    CU(e->rib_bits.ensure(n));
    CU(e->rib_keys.ensure(n * 8));
    CU(e->misc.ensure(sizeof(Misc)));
    Misc *misc = e->misc.as<Misc>();
    CU(cudaMemsetAsync(misc, 0, sizeof(Misc), s));
    CU(cudaMemcpyAsync(e->keys.p, keys, n * 8, cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(e->nodes.p, nodes.data(), nleaves * sizeof(Node), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(e->ids.p, ids.data(), nleaves * 4, cudaMemcpyHostToDevice, s));
    const int wpb = leaves_sh1_warps_per_block();
    const int grid = std::max(1, std::min<int>(e->sms * 8, (int)((nleaves + wpb - 1) / wpb)));
    launch_leaves_sh1_ctr(e->nodes.as<Node>(), e->ids.as<uint32_t>(), (uint32_t)nleaves, e->keys.as<uint64_t>(),
                          e->codes.as<uint64_t>(), e->rib_keys.as<uint64_t>(), e->rib_bits.as<uint8_t>(), 0, &misc->err,
                          misc->work, &misc->leaf_ctr, grid, s);
    CU(cudaGetLastError());
    uint32_t err = 0;
    CU(cudaMemcpyAsync(codes, e->codes.p, nleaves * 8, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(keys_by_cell, e->rib_keys.p, n * 8, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(bits, e->rib_bits.p, n, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(&err, &misc->err, 4, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (err) return fail(SHG_ERR_TRIAL_LIMIT, "leaf search failed (error flags " + std::to_string(err) + ")");
    return SHG_OK;
}

shg_status shg_build_flat_strings(shg_engine *e, uint64_t k, const char *bytes, const uint64_t *offsets, uint64_t n,
                                  shg_flat_result *out) {
    if (!e || !out || !offsets || (n && !bytes)) return fail(SHG_ERR_ARG, "null argument");
    if (k < 4 || k > (uint64_t)kMaxLeaf2) return fail(SHG_ERR_ARG, "ShockHash2Flat needs 4 <= k <= 128");
    if (n >= (1ull << 32)) return fail(SHG_ERR_ARG, "at most 2^32 - 1 keys per build");
    CU(cudaSetDevice(e->device));
    shg_status st = build_flat(e, k, bytes, offsets, n, out);
    if (st) shg_flat_result_free(out);
    return st;
}

void shg_flat_result_free(shg_flat_result *r) {
    if (!r) return;
    shg_result_free(&r->fallback);
    if (r->owner) release_pinned((PinnedBlock *)r->owner);
    r->owner = nullptr;
    r->thresholds_and_seeds = r->fallback_seed_buckets = r->fallback_seeds = r->free_positions = r->ribbon_keys = nullptr;
    r->ribbon_bits = nullptr;
}

uint64_t shg_sh2_query(uint64_t leaf_size, uint64_t seed, uint64_t key, uint64_t retrieved) {
    return sh2_leaf_query((uint32_t)leaf_size, seed, key, retrieved);
}

shg_status shg_memo_table(int variant, int leaf_size, uint64_t *out) {
    if (!out) return fail(SHG_ERR_ARG, "null output");
    if (!is_sh1(variant) && variant != SHG_SHOCKHASH2) return fail(SHG_ERR_ARG, "unknown variant");
    const int maxleaf = is_sh1(variant) ? kMaxLeaf1 : kMaxLeaf2;
    if (leaf_size < 2 || leaf_size > maxleaf) return fail(SHG_ERR_ARG, "leaf size out of range");
    const Config &c = config_of(variant, leaf_size);
    memcpy(out, c.memo.data(), kMaxBucket * 8);
    return SHG_OK;
}

shg_status shg_engine_last_work(const shg_engine *e, uint64_t *out, int n) {
    if (!e || !out || n < 0) return fail(SHG_ERR_ARG, "null argument");
    const uint64_t v[13] = {e->split_kind[0], e->split_kind[1], e->split_kind[2], e->split_kind[3], e->split_launches,
                            e->leaf_scan, 0, 0, e->flat_work[0], e->flat_work[1], e->flat_work[2], e->flat_work[3],
                            e->flat_work[4]};
    for (int k = 0; k < n && k < 13; k++) out[k] = v[k];
    return SHG_OK;
}

shg_status shg_device_memory(int device, uint64_t *free_bytes, uint64_t *total_bytes) {
    if (!free_bytes || !total_bytes) return fail(SHG_ERR_ARG, "null output");
    CU(cudaSetDevice(device));
    size_t f = 0, t = 0;
    CU(cudaMemGetInfo(&f, &t));
    *free_bytes = f;
    *total_bytes = t;
    return SHG_OK;
}

const char *shg_last_error(void) { return g_last_error.c_str(); }

} // extern "C"
