/*
 * shg.h — C ABI of the B200 ShockHash construction engine (libshg.so).
 *
 * Plain C types only. Every build entry point reproduces, bit for bit, what the reference's
 * constructors compute (paths relative to the ShockHash reference project):
 *   - the Golomb-Rice descriptor words   (RiceBitVector::Builder, include/shockhash/RiceBitVector.h:67-127)
 *   - bucket_size_acc / bucket_pos_acc   (hash_gen, include/ShockHash.h:616-654; ShockHash2.h:455-494)
 *   - the retrieval input (key, bit)      (ShockHash.h:425-428; ShockHash2-internal.h:548-572),
 *     in the reference's push order.
 * The Elias-Fano structure built from those arrays stays on the host; the retrieval input can go
 * to the reference's SimpleRibbon or to the compact retrieval structure built on the device
 * (shg_retrieval_*).
 *
 * Errors: every entry point returns an shg_status; no C++ exception crosses this boundary. The
 * message of the last failure on the calling thread is available from shg_last_error().
 * Threading: an engine owns one CUDA stream and its device buffers and is not thread-safe; use one
 * engine per host thread. Result arrays live in pinned host memory owned by the engine that built
 * them; they stay valid until shg_result_free() or shg_engine_destroy(), whichever comes first.
 */
#ifndef SHG_H
#define SHG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum shg_status {
    SHG_OK = 0,
    SHG_ERR_ARG = 1,          /* invalid argument (leaf size, bucket size, null pointer, n >= 2^32) */
    SHG_ERR_OOM = 2,          /* device or host allocation failed */
    SHG_ERR_TRIAL_LIMIT = 3,  /* a seed search exceeded its trial cap (duplicate keys loop forever in the reference) */
    SHG_ERR_CUDA = 4,         /* a CUDA call failed; see shg_last_error() */
    SHG_ERR_BUCKET = 5,       /* a bucket holds >= 3000 keys (MAX_BUCKET_SIZE, ShockHash.h:33) */
    SHG_ERR_NO_DEVICE = 6     /* no CUDA device or the kernels are not loadable on it */
} shg_status;

/* Which reference class the build reproduces. */
typedef enum shg_variant {
    SHG_SHOCKHASH = 1,   /* shockhash::ShockHash<leaf_size, false>            (include/ShockHash.h:134) */
    SHG_SHOCKHASH2 = 2,  /* shockhash::ShockHash2<leaf_size>                  (include/ShockHash2.h:117) */
    SHG_SHOCKHASH_ROTATION = 3, /* shockhash::ShockHash<leaf_size, true>: leaves of exactly leaf_size keys
                                   use rotation fitting (ShockHash.h:316-399); leaf_size 2..60 */
    SHG_SIMDSHOCKHASH = 5,      /* shockhash::SIMDShockHash<leaf_size, false> (include/SIMDShockHash.hpp:105), the
                                   class the reference's SIMD benchmark builds as ShockHash<l>: the same tree and
                                   leaves as ShockHash<l, false>, with its own split hash (remixAndRemap,
                                   SIMDShockHash.hpp:762-766) and start seeds (:209, :582, :593, :411); leaf_size 2..60 */
    SHG_SIMDSHOCKHASH_ROTATION = 6 /* shockhash::SIMDShockHash<leaf_size, true>: rotation fitting for leaves of
                                   exactly leaf_size keys (SIMDShockHash.hpp:419-512) */
} shg_variant;

/* How the search stages are scheduled on the device. All modes give identical results. */
typedef enum shg_mode {
    SHG_MODE_DEFAULT = 0,     /* the fastest measured schedule: SHG_MODE_QUEUE for ShockHash2 with leaves of up
                                 to 64 keys, SHG_MODE_LEVELS otherwise */
    SHG_MODE_LEVELS = 1,      /* one launch per RecSplit level (a block per split node), then one persistent
                                 leaf launch whose warps drain all leaves from a device counter */
    SHG_MODE_PER_LEAF = 2,    /* comparison form: per-level split launches and one launch per leaf */
    SHG_MODE_PIPELINED = 3,   /* buckets in chunks; a chunk's leaf launch (second stream) overlaps the next
                                 chunk's split launches (measured slower on B200: both compete for issue slots) */
    SHG_MODE_QUEUE = 4        /* ShockHash2 with leaves of up to 64 keys: every split node and leaf in ONE
                                 persistent launch that takes them from a device work list, a node as soon as
                                 its bucket's levels above it are done, leaves once their bucket's splits are;
                                 other variants run the level schedule */
} shg_mode;

typedef struct shg_params {
    int variant;              /* shg_variant */
    int leaf_size;            /* ShockHash, SIMDShockHash: 2..60; ShockHash2: 2..128 */
    uint64_t bucket_size;     /* expected keys per bucket (the reference's bucket_size argument) */
    int mode;                 /* shg_mode */
    uint64_t max_trials;      /* seeds tried at most per split node / original leaf; 0 = library default,
                                 2^(g+12) per split and 2^(g+10) per leaf (g = the node's Rice parameter),
                                 about a thousand times the expected count */
} shg_params;

typedef struct shg_result {
    uint64_t n;                  /* number of keys */
    uint64_t nbuckets;           /* max(1, ceil(n / bucket_size)) (ShockHash.h:616) */
    uint64_t *bucket_size_acc;   /* [nbuckets + 1] cumulative bucket sizes */
    uint64_t *bucket_pos_acc;    /* [nbuckets + 1] bit offset of each bucket's codes */
    uint64_t *descriptors;       /* [desc_words] Golomb-Rice stream incl. the (1,1) sentinel */
    uint64_t desc_words;         /* ((bits + 7) / 8 + 14) / 8 words, the builder's final size */
    uint64_t desc_bits;          /* bits written, sentinel included */
    uint64_t *ribbon_keys;       /* [ribbon_n] retrieval input keys (hash.second), reference push order */
    uint8_t *ribbon_bits;        /* [ribbon_n] retrieval input values */
    uint64_t ribbon_n;           /* keys in leaves of size >= 2 */
    double stage_ms[8];          /* device time per stage: hash, partition, tree, splits, leaves, encode, copy-out, total */
    uint64_t work[8];            /* split evaluations, leaf evaluations, candidate pairs, filtered pairs,
                                    pseudoforest edge operations, leaves, split nodes, kernel launches */
    void *owner;                 /* library-internal: the pinned host block the arrays live in */
} shg_result;

typedef struct shg_engine shg_engine;

/* Create an engine on CUDA device `device` (its own non-blocking stream). */
shg_status shg_engine_create(int device, shg_engine **out);
void shg_engine_destroy(shg_engine *e);

/* Build from 128-bit key fingerprints in HOST memory: first[i], second[i] are the halves of the
 * reference's hash128_t (ShockHash.h:187, ShockHash2.h:167). The arrays are not modified (the
 * reference sorts its argument vector in place; this entry point leaves the caller's data alone). */
shg_status shg_build_hash128(shg_engine *e, const shg_params *p, const uint64_t *first,
                             const uint64_t *second, uint64_t n, shg_result *out);

/* Build from string keys in HOST memory: bytes + offsets[n+1]; keys are hashed on the device with
 * SpookyHash V2 seed 0, as the reference's string constructors do (ShockHash.h:159-185). */
shg_status shg_build_strings(shg_engine *e, const shg_params *p, const char *bytes,
                             const uint64_t *offsets, uint64_t n, shg_result *out);

/* Build from uint64 keys in HOST memory, each hashed as its 8-byte little-endian string. */
shg_status shg_build_u64(shg_engine *e, const shg_params *p, const uint64_t *keys, uint64_t n,
                         shg_result *out);

/* Same as shg_build_hash128 / shg_build_u64 with inputs already in DEVICE memory (device pointers
 * on the engine's device); outputs are still returned in host memory. */
shg_status shg_build_hash128_device(shg_engine *e, const shg_params *p, const uint64_t *d_first,
                                    const uint64_t *d_second, uint64_t n, shg_result *out);
shg_status shg_build_u64_device(shg_engine *e, const shg_params *p, const uint64_t *d_keys,
                                uint64_t n, shg_result *out);

/* Batched construction of nreq independent key sets (uint64 keys in HOST memory, hashed as 8-byte
 * strings): request r's keys[r][0..n[r]) give outs[r], exactly what shg_build_u64 gives for that
 * request alone. All requests' split nodes and leaves go through the same kernel launches (one
 * persistent leaf launch for the whole batch); encoding and copy-out are per request. This is the
 * unit of the continuous-batching build loop (shockhash_b200/serve.py). */
shg_status shg_build_batch_u64(shg_engine *e, const shg_params *p, const uint64_t *const *keys, const uint64_t *n,
                               uint64_t nreq, shg_result *outs);

/* One item of a mixed batch (shg_build_batch_items): n uint64 keys (`keys`, hashed on the device as
 * 8-byte strings) or n 128-bit fingerprints (`first`/`second` when `keys` is NULL), in HOST memory;
 * with b1 > b0 the item is one piece of a larger structure of nb_global buckets and holds exactly
 * the keys of its buckets [b0, b1) (as shg_build_shard_hash128), else a whole structure. */
typedef struct shg_batch_item {
    const uint64_t *keys;
    const uint64_t *first, *second;
    uint64_t n;
    uint64_t nb_global, b0, b1;
} shg_batch_item;

/* Batched construction of mixed items (no counterpart in the reference): whole key sets and pieces
 * of larger ones share the kernel launches; outs[i] is what building item i alone gives (for a
 * piece, what shg_build_shard_hash128 gives, to be joined by shg_merge_shards). The build service
 * uses it to interleave the bucket-range pieces of large requests with smaller requests. */
shg_status shg_build_batch_items(shg_engine *e, const shg_params *p, const shg_batch_item *items, uint64_t nitems,
                                 shg_result *outs);

void shg_result_free(shg_result *r);

/* A build result on disk and back (no counterpart in the reference classes, which persist only
 * the RiceBitVector, RiceBitVector.h:133-141; the descriptors section of the file is in that
 * stream layout: u64 word count, then the words). A loaded result is freed with shg_result_free
 * and feeds shg_mphf_create / shg_dmphf_create like a fresh one; `p` receives the configuration. */
shg_status shg_result_save(const shg_params *p, const shg_result *r, const char *path);
shg_status shg_result_load(const char *path, shg_params *p, shg_result *out);

/* Shards of one structure (no counterpart in the reference, whose compute_thread splits the same
 * bucket ranges over threads, ShockHash.h:566-570). Bucket b = remap128(first, nb_global) is
 * monotone in `first`, so a key set can be split by bucket range over GPUs or processes:
 * shg_build_shard_hash128 builds the buckets [b0, b1) of a structure with nb_global buckets from
 * exactly the keys that fall in them (any other key is SHG_ERR_ARG); its result holds those
 * buckets only (accumulators from 0, no other shard's bits). shg_merge_shards joins the shard
 * results, given in bucket order, into the result a single build of all keys produces, bit for
 * bit: accumulators offset, Golomb-Rice codes concatenated at bit granularity
 * (appendRiceBitVector, RiceBitVector.h:102-120), one sentinel, retrieval input concatenated.
 * nb_global must be max(1, ceil(N / bucket_size)) for the total key count N. The merged result
 * lives in plain host memory and is released with shg_result_free like any other. */
shg_status shg_build_shard_hash128(shg_engine *e, const shg_params *p, const uint64_t *first,
                                   const uint64_t *second, uint64_t n, uint64_t nb_global, uint64_t b0,
                                   uint64_t b1, shg_result *out);
/* Same with the fingerprints in DEVICE memory on the engine's device (the keys a rank received
 * from the exchange stay on its GPU). */
shg_status shg_build_shard_hash128_device(shg_engine *e, const shg_params *p, const uint64_t *d_first,
                                          const uint64_t *d_second, uint64_t n, uint64_t nb_global, uint64_t b0,
                                          uint64_t b1, shg_result *out);
/* The 128-bit fingerprints of uint64 keys (each hashed as its 8-byte string, SpookyV2 seed 0) from
 * and into DEVICE memory on the engine's device; synchronous. What a rank exchanges before a
 * sharded build. */
shg_status shg_hash_u64_device(shg_engine *e, const uint64_t *d_keys, uint64_t n, uint64_t *d_first, uint64_t *d_second);
/* The send side of the exchange before a sharded build: every key's (first, second) pair written to
 * pairs[2 i], pairs[2 i + 1] in owner-rank order, stable (input order inside a rank), with the key
 * count per rank in counts[world]. Rank g of `world` owns buckets [floor(nb g / world),
 * floor(nb (g + 1) / world)) of remap128(first, nb). shg_shard_partition runs on the host (host
 * pointers); shg_shard_partition_device on the engine's device (device pointers; counts in host
 * memory; synchronous). Both give the same order. 1 <= world <= 64, 1 <= nb < 2^32. */
shg_status shg_shard_partition(const uint64_t *first, const uint64_t *second, uint64_t n, uint64_t nb, int world,
                               uint64_t *pairs, uint64_t *counts);
/* The same fingerprints as shg_hash_u64_device, on the host with up to `threads` threads. */
shg_status shg_hash_u64_host(const uint64_t *keys, uint64_t n, uint64_t *first, uint64_t *second, int threads);
/* Host uint64 keys in, host (first, second) pairs out in bucket-range order: the keys are copied to
 * the engine's device, hashed (shg_hash_u64_device) and partitioned into `parts` bucket ranges of
 * nb buckets (shg_shard_partition_device), and the pairs and per-range counts copied back. The
 * build service splits large requests this way into pieces for shg_build_batch_items. */
shg_status shg_partition_u64(shg_engine *e, const uint64_t *keys, uint64_t n, uint64_t nb, int parts, uint64_t *pairs,
                             uint64_t *counts);
shg_status shg_shard_partition_device(shg_engine *e, const uint64_t *d_first, const uint64_t *d_second, uint64_t n,
                                      uint64_t nb, int world, uint64_t *d_pairs, uint64_t *counts);
shg_status shg_merge_shards(const shg_params *p, const shg_result *shards, uint64_t nshards, shg_result *out);

/* Hash n string keys (bytes + offsets[n+1], host memory) to 128-bit fingerprints on the device:
 * sux spooky(key, len, 0) as used by ShockHash.h:129. */
shg_status shg_hash_strings(shg_engine *e, const char *bytes, const uint64_t *offsets, uint64_t n,
                            uint64_t *first, uint64_t *second);

/* Batched bipartite leaf search: the device counterpart of the reference's plugin seam
 * shockhash2construct (include/shockhash/ShockHash2-precompiled.h:9-10,
 * src/ShockHash2-precompiled.cpp:24-47), for many leaves in one call. Leaf j holds keys
 * [leaf_offsets[j], leaf_offsets[j+1]) (2..128 keys each, host memory). Writes seeds[j] and, for
 * every key in order, the retrieval bit bits[k] that constructRetrieval would push. */
shg_status shg_sh2_construct_leaves(shg_engine *e, const uint64_t *keys, const uint64_t *leaf_offsets,
                                    uint64_t nleaves, uint64_t *seeds, uint8_t *bits);

/* No counterpart in the reference. The bipartite leaf search of shg_sh2_construct_leaves for callers
 * that cannot allocate device memory (a framework-owned memory pool that forbids cudaMalloc, a
 * real-time host path, code that must not grow its footprint): it calls no cudaMalloc, cudaFree or
 * allocating library routine, and no engine is needed. Inputs and outputs are DEVICE pointers on
 * the current device: keys, leaf_offsets[nleaves+1] (leaves of 2..64 keys, at most 2^32 - 1 keys),
 * seeds[nleaves], bits[total keys]; `stream` is a cudaStream_t (NULL = default stream). The call
 * synchronizes that stream to report errors. Scratch is a fixed 16 MiB array in the library's own
 * device image, held by every GPU that loads the library until the process exits; a leaf needing
 * more than 512 raw seeds or 512 candidates fails with SHG_ERR_TRIAL_LIMIT, a leaf outside 2..64
 * keys with SHG_ERR_ARG. The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress, once per device); make that first call before any stream capture begins.
 * All calls share the array, so calls that overlap on the GPU (other streams, other host threads)
 * race. */
shg_status shg_sh2_construct_leaves_noalloc(const uint64_t *d_keys, const uint64_t *d_leaf_offsets, uint64_t nleaves,
                                            uint64_t *d_seeds, uint8_t *d_bits, void *stream);

/* Batched original-ShockHash leaf search at tree depth `level` (include/ShockHash.h:404-434):
 * codes[j] = x - start_seed[level]; keys_by_cell/bits are written per leaf in cell order, as the
 * reference pushes its retrieval input. Leaves of 2..60 keys. */
shg_status shg_sh1_construct_leaves(shg_engine *e, const uint64_t *keys, const uint64_t *leaf_offsets,
                                    uint64_t nleaves, int level, uint64_t *codes, uint64_t *keys_by_cell,
                                    uint8_t *bits);

/* Leaf query of the bipartite variant: shockhash2query (ShockHash2-precompiled.h:8). */
uint64_t shg_sh2_query(uint64_t leaf_size, uint64_t seed, uint64_t key, uint64_t retrieved);

/* Host query object over a build result: the reference's operator() (ShockHash.h:199-270,
 * ShockHash2.h:178-230) and getBits() (ShockHash.h:283-286, ShockHash2.h:243-246). The result's
 * arrays are copied; the caller still frees the result. */
typedef struct shg_mphf shg_mphf;
shg_status shg_mphf_create(const shg_params *p, shg_result *r, shg_mphf **out);
void shg_mphf_destroy(shg_mphf *f);
/* operator()(const hash128_t&) for n fingerprints (host memory). */
shg_status shg_mphf_query_hash(const shg_mphf *f, const uint64_t *first, const uint64_t *second, uint64_t n,
                               uint64_t *out);
/* operator()(const string&) for n string keys (bytes + offsets[n+1]). */
shg_status shg_mphf_query_strings(const shg_mphf *f, const char *bytes, const uint64_t *offsets, uint64_t n,
                                  uint64_t *out);
/* getBits(): size estimate in bits, with the same component formulas as the reference classes. */
uint64_t shg_mphf_bits(const shg_mphf *f);
/* size(): number of keys. */
uint64_t shg_mphf_size(const shg_mphf *f);

/* Device query object: the same operator() evaluated on the GPU for many keys per call, one thread
 * per key (bucket lookup, Golomb-Rice walk RiceBitVector.h:149-213, leaf hash, retrieval bit from
 * a device hash table built from the result's retrieval input). No counterpart in the reference,
 * which queries one key per call on the host; the outputs equal shg_mphf_query_* key for key.
 * Calls are synchronous on the object's own stream; one object is not thread-safe. */
typedef struct shg_dmphf shg_dmphf;
shg_status shg_dmphf_create(int device, const shg_params *p, const shg_result *r, shg_dmphf **out);
void shg_dmphf_destroy(shg_dmphf *f);
/* Fingerprints (first, second) or results in host memory. */
shg_status shg_dmphf_query_hash128(shg_dmphf *f, const uint64_t *first, const uint64_t *second, uint64_t n,
                                   uint64_t *out);
/* uint64 keys, each hashed as its 8-byte little-endian string (SpookyV2-128 fused in the kernel). */
shg_status shg_dmphf_query_u64(shg_dmphf *f, const uint64_t *keys, uint64_t n, uint64_t *out);
/* String keys (bytes + offsets[n+1]), hashed in the kernel. */
shg_status shg_dmphf_query_strings(shg_dmphf *f, const char *bytes, const uint64_t *offsets, uint64_t n,
                                   uint64_t *out);
/* Device-memory forms of the two above (all pointers on the object's device). */
shg_status shg_dmphf_query_hash128_device(shg_dmphf *f, const uint64_t *d_first, const uint64_t *d_second,
                                          uint64_t n, uint64_t *d_out);
shg_status shg_dmphf_query_u64_device(shg_dmphf *f, const uint64_t *d_keys, uint64_t n, uint64_t *d_out);
uint64_t shg_dmphf_bits(const shg_dmphf *f);
uint64_t shg_dmphf_size(const shg_dmphf *f);
/* Device time of the last query kernel, in milliseconds (CUDA events on the object's stream). */
float shg_dmphf_last_kernel_ms(const shg_dmphf *f);
/* The same object with the compact retrieval structure (shg_retrieval_*, below) built on the device
 * in place of the exact table: outputs equal shg_mphf_query_* for every key of the build (other
 * keys may differ, as they may between any two retrieval structures). Size in bits of the
 * object's retrieval part, compact structure or table. */
shg_status shg_dmphf_create_compact(int device, const shg_params *p, const shg_result *r, shg_dmphf **out);
uint64_t shg_dmphf_retrieval_bits(const shg_dmphf *f);

/* ------------------------------------------------------------------ retrieval structure
 * Compact 1-bit retrieval built on the GPU from a retrieval input (key, bit): the role of
 * SimpleRibbon<1, w> in the reference (built at ShockHash.h:657 and ShockHash2.h:497 from
 * ribbonInput, read by retrieve() at ShockHash.h:267-270 and ShockHash2.h:226-229). SimpleRibbon's
 * source is absent from the reference tree, so the format is this library's own: levels of buckets
 * of ~240 keys, each bucket a 256-bit GF(2) solution and an 8-bit priority threshold (keys at or
 * above it go to the next level), about 1.1 bits per key. query(key) returns the stored bit of
 * every input key (any bit for other keys). Duplicate keys with different bits fail with
 * SHG_ERR_ARG. */
typedef struct shg_retrieval shg_retrieval;
/* Build from host arrays (copied to the engine's device) or from device arrays; synchronous. */
shg_status shg_retrieval_build(shg_engine *e, const uint64_t *keys, const uint8_t *bits, uint64_t n,
                               shg_retrieval **out);
shg_status shg_retrieval_build_device(shg_engine *e, const uint64_t *d_keys, const uint8_t *d_bits, uint64_t n,
                                      shg_retrieval **out);
/* A structure from its arrays (as read back with the accessors below): host queries only. */
shg_status shg_retrieval_load(const uint64_t *level_buckets, uint32_t levels, const uint64_t *solutions,
                              const uint8_t *thresholds, uint64_t n, shg_retrieval **out);
void shg_retrieval_destroy(shg_retrieval *r);
/* Host query, and device query over device arrays (synchronous, on the building engine's device). */
shg_status shg_retrieval_query(const shg_retrieval *r, const uint64_t *keys, uint64_t n, uint8_t *out);
shg_status shg_retrieval_query_device(shg_retrieval *r, const uint64_t *d_keys, uint64_t n, uint8_t *d_out);
/* Format accessors: levels, buckets of a level, 4 solution words per bucket and one threshold per
 * bucket (levels back to back), size in bits, device times of the build and of the last query. */
uint32_t shg_retrieval_levels(const shg_retrieval *r);
uint64_t shg_retrieval_buckets(const shg_retrieval *r, uint32_t level);
const uint64_t *shg_retrieval_solutions(const shg_retrieval *r);
const uint8_t *shg_retrieval_thresholds(const shg_retrieval *r);
uint64_t shg_retrieval_bits(const shg_retrieval *r);
float shg_retrieval_build_ms(const shg_retrieval *r);
float shg_retrieval_query_ms(const shg_retrieval *r);

/* ------------------------------------------------------------------ ShockHash2Flat<k>
 * k-perfect "flat" variant (include/ShockHash2Flat.h:37-302): MurmurHash64 keys, two threshold
 * layers of k-key buckets, a fallback ShockHash2<k> for bumped keys, one bipartite leaf search per
 * bucket. k in 4..128. */
typedef struct shg_flat_result {
    uint64_t n, k, nbuckets, layers;
    uint64_t layer_bases[3];           /* layerBases (ShockHash2Flat.h:49) */
    uint32_t threshold_bits, seed_bits;
    uint64_t *thresholds_and_seeds;    /* [nbuckets] seed << threshold_bits | compact threshold (:173-192) */
    uint64_t nfallback_seeds;          /* seedsFallback (:48): buckets whose seed is 0 or >= 2^seed_bits */
    uint64_t *fallback_seed_buckets;   /* ascending */
    uint64_t *fallback_seeds;
    uint64_t nfree;
    uint64_t *free_positions;          /* freePositions (:71, 129-146) */
    uint64_t nfallback_keys;           /* keys of the fallback PHF */
    shg_result fallback;               /* ShockHash2<k>(to_string(mhc) of the bumped keys, 2000) (:124-128) */
    uint64_t *ribbon_keys;             /* [ribbon_n] retrieval input (mhc, bit), bucket order (:159-170) */
    uint8_t *ribbon_bits;
    uint64_t ribbon_n;
    double stage_ms[8];                /* hash, layers, fallback build, assign, leaves, copy-out, -, total */
    void *owner;
} shg_flat_result;
shg_status shg_build_flat_strings(shg_engine *e, uint64_t k, const char *bytes, const uint64_t *offsets, uint64_t n,
                                  shg_flat_result *out);
void shg_flat_result_free(shg_flat_result *r);
/* Query object: operator()(const string&) / operator()(uint64_t) and getBits() (ShockHash2Flat.h:236-277). */
typedef struct shg_flat shg_flat;
shg_status shg_flat_create(const shg_flat_result *r, shg_flat **out);
void shg_flat_destroy(shg_flat *f);
shg_status shg_flat_query_strings(const shg_flat *f, const char *bytes, const uint64_t *offsets, uint64_t n, uint64_t *out);
shg_status shg_flat_query_hash(const shg_flat *f, const uint64_t *mhc, uint64_t n, uint64_t *out);
uint64_t shg_flat_bits(const shg_flat *f);
/* Device query object for ShockHash2Flat<k>: operator()(const string&) / operator()(uint64_t)
 * (ShockHash2Flat.h:258-301) for many keys per call, one GPU thread per key (MurmurHash64, the
 * threshold layers, the fallback ShockHash2<k> over the decimal string of the hash, seed fallback,
 * retrieval bit). No counterpart in the reference, which queries one key per call on the host;
 * outputs equal shg_flat_query_* key for key. Synchronous; one object is not thread-safe. */
typedef struct shg_dflat shg_dflat;
shg_status shg_dflat_create(int device, const shg_flat_result *r, shg_dflat **out);
void shg_dflat_destroy(shg_dflat *f);
shg_status shg_dflat_query_strings(shg_dflat *f, const char *bytes, const uint64_t *offsets, uint64_t n,
                                   uint64_t *out);
shg_status shg_dflat_query_hash(shg_dflat *f, const uint64_t *mhc, uint64_t n, uint64_t *out);
float shg_dflat_last_kernel_ms(const shg_dflat *f);

/* Golomb-Rice memo table of a configuration (ShockHash.h:121-127 / ShockHash2.h:106-115):
 * out[m] for m < 3000 packs golomb parameter << 27 | subtree nodes << 16 | subtree fixed bits. */
shg_status shg_memo_table(int variant, int leaf_size, uint64_t *out);

/* Benchmark utilities (no counterpart in the reference interface). n keys drawn from
 * std::mt19937_64(seed) with duplicates redrawn, as the benchmark configurations specify. */
void shg_keys_mt19937_64(uint64_t seed, uint64_t n, uint64_t *out);
/* n distinct uint64 keys out[j] = remix(seed ^ (j * 0x9E3779B97F4A7C15)) (Stafford Mix13, a bijection),
 * filled by up to `threads` host threads: the per-request key sets of the serving stream. */
void shg_keys_mix(uint64_t seed, uint64_t n, uint64_t *out, int threads);
/* Integer-pipe peak of the split-search arithmetic (remix + 16-bit part thresholds, operands in
 * registers) on `device`, in evaluations per second: the roofline denominator of the searches. */
int shg_int_peak(int device, uint64_t iters, double *evals_per_s, double *ms);
/* Same for the inner loop of one search: 0 = split quarter-split moments (as shg_int_peak),
 * 1 = original leaf coverage (remix, two fastrange32 cells, half masks), 2 = bipartite raw seeds
 * (remix, fastrange64, mask), 3 / 4 / 5 = split compare-and-count against 1 / 2 / 3 part
 * thresholds (fanout-2 and uneven split nodes), 6 = bipartite candidate-scan mask pairs,
 * 7 = bipartite isolated-key pair filter, 8 = bipartite pseudoforest edges (union-find),
 * 9 / 10 / 11 / 12 = kinds 0 / 3 / 4 / 5 with the split kernel's pipe-split arithmetic
 * (tuning parameter split_arith 1), 13 / 14 / 15 = kinds 6 / 7 / 8 for bipartite leaves of more
 * than 64 keys (64-bit masks, 100-edge tests), 16 / 17 / 18 / 19 = kinds 0 / 3 / 4 / 5 under
 * SIMDShockHash's split hash (SIMDShockHash.hpp:762-766), 20 = kind 13 with the other form of the
 * mask test ((a | t) == full instead of (~t & ~a) == 0; the faster of 13 and 20 bounds the scan). */
int shg_int_peak_kind(int device, int kind, uint64_t iters, double *evals_per_s, double *ms);

/* Work counts of the engine's last RecSplit build beyond shg_result.work (measurement utility, no
 * counterpart in the reference; the weights of the search stages' roofline denominators). Writes
 * min(n, 13) values: [0..2] useful split evaluations of nodes comparing 1, 2 or 3 part thresholds
 * (fanout-2 and uneven nodes), [3] of quarter splits (moment sums), [4] split level launches,
 * [5] bipartite leaves' candidate-scan mask-pair tests (for each raw seed, the earlier raw seeds
 * it is paired with), [6..7] zero; [8..12] the last ShockHash2Flat build's leaf search: hash
 * evaluations, candidate pairs, pairs left by the isolated-key filter, union-find edges,
 * candidate-scan mask-pair tests. */
shg_status shg_engine_last_work(const shg_engine *e, uint64_t *out, int n);

/* Launch parameters of the search kernels per configuration (no counterpart in the reference; they
 * change speed only, never a result). variant is an shg_variant (SHG_SHOCKHASH_ROTATION shares
 * SHG_SHOCKHASH's entry) or 4 for ShockHash2Flat<k> with leaf_size = k. Names and ranges:
 *   split_seeds_per_lane 1, 2, 4; split_threads 128, 256, 512; split_round_div 1..64 (a round of
 *   seeds aims at 1/round_div of a split node's expected trials); split_arith 0, 1 (1: remix's
 *   shifts partly as multiply-highs, moving work from the integer to the multiply pipe);
 *   leaf_blocks_per_sm 0..16 (0 =
 *   as many as shared memory allows); leaf_min_blocks 4, 6, 8 (bipartite leaves up to 64 keys:
 *   register bound); sh1_seeds_per_lane 1, 2 (original leaves); queue_lag_rounds 0..64 (work-queue
 *   schedule: lag between a bucket's tree levels in the item order, in rounds of the grid; default
 *   8; 0 = the levels one after another, then the leaves).
 * At creation an engine loads the table shockhash_b200/tuning.tsv beside the library (or the file
 * named by the SHG_TUNING_TABLE environment variable; empty = none), written by the autotuner
 * (python -m shockhash_b200.tune); lines "<variant> <leaf> <name> <value>", '#' comments. */
shg_status shg_engine_set_tuning(shg_engine *e, int variant, int leaf_size, const char *name, int64_t value);
shg_status shg_engine_get_tuning(shg_engine *e, int variant, int leaf_size, const char *name, int64_t *value);
shg_status shg_engine_load_tuning(shg_engine *e, const char *path);
/* Path of the table the engine loaded ("" if none). */
const char *shg_engine_tuning_source(const shg_engine *e);

/* Free and total device memory (cudaMemGetInfo), for admission control. */
shg_status shg_device_memory(int device, uint64_t *free_bytes, uint64_t *total_bytes);

/* Message of the last failure on this thread ("" if none). */
const char *shg_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* SHG_H */
