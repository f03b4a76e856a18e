/*
 * gmpt.h -- handle-based C ABI of the B200 MPT library (libgmpt_b200.so).
 *
 * One call per method of the reference's GpuMPT::Compress::MPT surface
 * (mpt-with-compress/include/mpt/gpu_mpt.cuh:18-192) that the batched update
 * path uses, plus the additive status / buffer calls the reference lacks.
 * Plain pointers and sizes only; every call is synchronous on the trie's own
 * CUDA stream and returns a gmpt_status (0 = ok).
 *
 * Batch layout (as in the reference): keys_hexs holds hex-nibble keys (one
 * byte per nibble, 16 = terminator, util/utils.cuh:340-349); keys_indexs and
 * values_indexs hold inclusive [start, end] pairs (int / int64_t); values_hps
 * (may be NULL) are the caller's host pointers that lookups echo back.
 * Semantics: keys of one batch are applied as if inserted in index order
 * (the last occurrence of a key wins) and an existing key's value is
 * replaced, for both insert strategies.
 */
#ifndef GMPT_H
#define GMPT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gmpt_trie gmpt_trie;

enum gmpt_status {
  GMPT_OK = 0,
  GMPT_E_CUDA = 1,        /* CUDA runtime error (message in gmpt_last_error_message) */
  GMPT_E_BAD_KEY = 2,     /* nibble > 16, terminator not last, prefix key, too long */
  GMPT_E_CAPACITY = 3,    /* more than 2^30 nodes of one kind, or out of memory */
  GMPT_E_RETRY_LIMIT = 4, /* a LockNU insert exceeded its CAS retry budget */
  GMPT_E_ARG = 5,         /* invalid argument */
  GMPT_E_INTERNAL = 6
};

/* Encoding of children shorter than 32 bytes and of the root. */
enum gmpt_encode_mode {
  GMPT_MODE_REF = 0,  /* the reference: RLP string of the raw child, raw small root */
  GMPT_MODE_GETH = 1  /* go-ethereum: embedded child, root always hashed */
};

typedef struct gmpt_stats {
  uint64_t n_full, n_short, n_value, n_records;
  uint64_t key_bytes, value_bytes;
  uint64_t last_unique, last_new, last_pseudo, last_dirty, last_levels, last_hash_levels;
  uint64_t device_bytes;
  uint32_t sort_passes, build_levels;
  float t_stage_ms, t_sort_ms, t_walk_ms, t_build_ms, t_hash_ms;
  uint64_t last_hashed, last_enc_bytes, last_keccak_blocks; /* last PhaseHC pass (timing mode only, else 0) */
  float t_hash_kernels_ms; /* encode+Keccak kernels of the last pass (timing mode) */
  uint32_t hash_launches, pad;
} gmpt_stats;

int gmpt_version(void);

/* MPT::MPT() (gpu_mpt.cuh:162-173): an empty trie on `device`. */
gmpt_trie *gmpt_create(int device, int encode_mode);
void gmpt_destroy(gmpt_trie *t);

/* A forest: max_tries independent tries (ids 0 .. max_tries-1) that share
 * one set of node pools and arenas, so a batch touching many tries (a block's
 * state trie and its accounts' storage tries) is one insert and one PhaseHC
 * pass.  No counterpart in the reference, which holds one trie per MPT
 * object (gpu_mpt.cuh:162-173); trie 0 of a forest is what every
 * single-trie call below addresses. */
gmpt_trie *gmpt_create_forest(int device, int encode_mode, int max_tries);
/* gmpt_create_forest with flags.  GMPT_CREATE_UNIFIED_MEMORY: the node
 * pools, key / value arenas and dirty list live in unified memory
 * (cudaMallocManaged, preferred location and accessed-by the device), so a
 * trie may grow past the device's memory with pages migrating on demand --
 * the reference's out-of-core UMMPT (mpt/um_mpt.cuh:13-52).  Results are
 * the same; speed drops once pages migrate. */
enum { GMPT_CREATE_UNIFIED_MEMORY = 1 };
gmpt_trie *gmpt_create_ex(int device, int encode_mode, int max_tries, unsigned flags);
int gmpt_max_tries(gmpt_trie *t);
/* drop every node (capacity is kept) */
int gmpt_reset(gmpt_trie *t);

/* puts_2phase_with_valuehp (gpu_mpt.cuh:95-97, 1262-1399): PhaseNU batch
 * insert from HOST arrays.  Marks the touched nodes dirty; call
 * gmpt_hash_onepass() to rehash. */
int gmpt_puts_2phase(gmpt_trie *t, const uint8_t *keys_hexs, const int *keys_indexs,
                     const uint8_t *values_bytes, const int64_t *values_indexs,
                     const uint8_t *const *values_hps, int n);

/* puts_latching_with_valuehp_v2 (gpu_mpt.cuh:69-71, 554-615): LockNU batch
 * insert from HOST arrays. */
int gmpt_puts_latching(gmpt_trie *t, const uint8_t *keys_hexs, const int *keys_indexs,
                       const uint8_t *values_bytes, const int64_t *values_indexs,
                       const uint8_t *const *values_hps, int n);

/* Same two inserts with DEVICE-resident inputs (d_values_hps: n uint64 host
 * addresses in device memory, or NULL); keys_bytes / values_bytes are the
 * lengths of the key and value streams. */
int gmpt_puts_2phase_device(gmpt_trie *t, const uint8_t *d_keys_hexs, const int *d_keys_indexs,
                            const uint8_t *d_values_bytes, const int64_t *d_values_indexs,
                            const uint64_t *d_values_hps, int n, int64_t keys_bytes,
                            int64_t values_bytes);
int gmpt_puts_latching_device(gmpt_trie *t, const uint8_t *d_keys_hexs, const int *d_keys_indexs,
                              const uint8_t *d_values_bytes, const int64_t *d_values_indexs,
                              const uint64_t *d_values_hps, int n, int64_t keys_bytes,
                              int64_t values_bytes);

/* Forest inserts from HOST arrays: key i goes into trie trie_ids[i].  Same
 * semantics per trie as the single-trie calls above; the tries' roots come
 * from gmpt_get_roots after gmpt_hash_onepass. */
int gmpt_puts_2phase_forest(gmpt_trie *t, const uint8_t *keys_hexs, const int *keys_indexs,
                            const uint8_t *values_bytes, const int64_t *values_indexs,
                            const uint8_t *const *values_hps, const int *trie_ids, int n);
int gmpt_puts_latching_forest(gmpt_trie *t, const uint8_t *keys_hexs, const int *keys_indexs,
                              const uint8_t *values_bytes, const int64_t *values_indexs,
                              const uint8_t *const *values_hps, const int *trie_ids, int n);

/* One block of a forest in ONE persistent launch (no counterpart in the
 * reference, whose per-trie puts_latching_with_valuehp_v2 + hash_onepass_v2
 * pairs this replaces for a whole set of tries, gpu_mpt.cuh:554-615 and
 * 1162-1191):
 *   stage 0 = keys [0, n0): LockNU insert into tries trie_ids[i], PhaseHC;
 *   stage 1 = keys [n0, n): key i with patch_trie[i] >= 0 first gets the 32
 *     root bytes of trie patch_trie[i] (after stage 0; zero-padded when the
 *     root is shorter or the trie empty) written into its value at byte
 *     offset patch_off[i]; then LockNU insert and PhaseHC.
 * This is the Ethereum block shape: storage tries in stage 0, the state trie
 * in stage 1 with storageRoot patched into each account's RLP.  Key and
 * value index pairs must tile their streams (keys back to back).  patch_trie
 * and patch_off may both be NULL.  On return out32[32 j..] / out_sizes[j]
 * hold the root of trie out_ids[j] (host array) after the block.  The
 * staging copy and the persistent kernel are replayed from one captured CUDA
 * graph, rebuilt only when a buffer or node pool grows.  Stage semantics per
 * trie equal gmpt_puts_latching_forest + gmpt_hash_onepass. */
int gmpt_block_update(gmpt_trie *t, const uint8_t *keys_hexs, const int *keys_indexs, const uint8_t *values_bytes,
                      const int64_t *values_indexs, const int *trie_ids, const int *patch_trie, const int *patch_off,
                      int n, int n0, const int *out_ids, int n_out, uint8_t *out32, int *out_sizes);
/* Same with device-resident key/value/trie/patch arrays (out_ids stays a
 * host array). */
int gmpt_block_update_device(gmpt_trie *t, const uint8_t *d_keys_hexs, const int *d_keys_indexs,
                             const uint8_t *d_values_bytes, const int64_t *d_values_indexs, const int *d_trie_ids,
                             const int *d_patch_trie, const int *d_patch_off, int n, int n0, int64_t keys_bytes,
                             int64_t values_bytes, const int *out_ids, int n_out, uint8_t *out32, int *out_sizes);
/* The last block: hash levels of stage 0 / 1, dirty nodes of stage 0 / 1,
 * CTAs of the persistent kernel, graph captures so far, block launches so
 * far, 0. */
int gmpt_block_info(gmpt_trie *t, uint32_t out[8]);
/* With gmpt_set_timing on: the last block's input copies, graph replay and
 * whole call, in ms (CUDA events on the trie's stream). */
int gmpt_block_times(gmpt_trie *t, float out[3]);
/* Device timeline of the last block (globaltimer ns, up to cap entries):
 * staging start, persistent kernel start, each grid barrier, end.  *n =
 * entries recorded. */
int gmpt_block_timeline(gmpt_trie *t, uint64_t *out_ns, int cap, int *n);
/* Grow the node pools and arenas now for n_keys more keys carrying
 * key_bytes / value_bytes stream bytes, so later inserts (and block graphs)
 * do not stall on growth.  No counterpart in the reference, whose arenas are
 * fixed at construction (util/allocator.cuh:152-157). */
int gmpt_reserve(gmpt_trie *t, int64_t n_keys, int64_t key_bytes, int64_t value_bytes);
/* gmpt_reserve with explicit headroom: free slots for `full` branch nodes,
 * `shorts` short nodes, `values` value nodes and `records` value records,
 * and key_bytes / value_bytes more arena bytes, beyond what is in use. */
int gmpt_reserve_nodes(gmpt_trie *t, int64_t full, int64_t shorts, int64_t values, int64_t records, int64_t key_bytes,
                       int64_t value_bytes);
/* Size the gmpt_block_update buffers for blocks of up to max_keys keys,
 * max_key_bytes / max_value_bytes stream bytes and max_out reported roots,
 * and capture the block graph now, so that no block of that size pays for
 * buffer growth or a capture.  Also reserves the node pools for one such
 * block. */
int gmpt_reserve_block(gmpt_trie *t, int64_t max_keys, int64_t max_key_bytes, int64_t max_value_bytes,
                       int64_t max_out);

/* Forest inserts from DEVICE arrays (two_phase: PhaseNU, else LockNU);
 * d_trie_ids may be NULL (trie 0). */
int gmpt_puts_forest_device(gmpt_trie *t, int two_phase, const uint8_t *d_keys_hexs, const int *d_keys_indexs,
                            const uint8_t *d_values_bytes, const int64_t *d_values_indexs, const uint64_t *d_values_hps,
                            const int *d_trie_ids, int n, int64_t keys_bytes, int64_t values_bytes);
/* gets_parallel with DEVICE keys (and trie ids, or NULL for trie 0); the
 * results land in the host arrays as for gmpt_gets_parallel. */
int gmpt_gets_forest_device(gmpt_trie *t, const uint8_t *d_keys_hexs, const int *d_keys_indexs, const int *d_trie_ids,
                            int n, int64_t keys_bytes, const uint8_t **values_hps, int *values_sizes);
/* The same with DEVICE result arrays: d_values_hps[i] (the host pointer
 * given with the value, as a uint64) and d_values_sizes[i] are written by the
 * lookup kernel; nothing crosses to the host.  Synchronous on the trie's
 * stream. */
int gmpt_gets_device(gmpt_trie *t, const uint8_t *d_keys_hexs, const int *d_keys_indexs, const int *d_trie_ids, int n,
                     int64_t keys_bytes, uint64_t *d_values_hps, int *d_values_sizes);

/* ---- synthetic request batches in device memory (bench and tests) ----
 * gmpt_gen_ids: n ids; each is fresh (next_new, next_new + 1, ... in batch
 * order) with probability p_new, else zipf(theta) over [0, n_existing)
 * (Gray et al.'s generator, ranks scrambled by FNV-1a-64); *n_new = fresh
 * ids used.  gmpt_gen_keys: key_bytes bytes per id from a splitmix64 stream
 * of (seed, id), as hex nibbles + terminator back to back with int32 index
 * pairs.  gmpt_gen_values: value_bytes random bytes per batch position.
 * Synchronous on `stream` (a cudaStream_t or NULL). */
int gmpt_gen_ids(uint64_t seed, int64_t n, int64_t n_existing, int64_t next_new, double p_new, double theta,
                 int64_t *d_ids, int64_t *n_new, void *stream);
int gmpt_gen_keys(uint64_t seed, const int64_t *d_ids, int64_t n, int key_bytes, uint8_t *d_keys_hexs,
                  int *d_keys_indexs, void *stream);
int gmpt_gen_values(uint64_t seed, int64_t n, int value_bytes, uint8_t *d_values, int64_t *d_values_indexs,
                    void *stream);

/* Schedule-selector features of a device-resident key batch, from 64 evenly
 * spaced keys: out[0] mean key length (nibbles), out[1] its standard
 * deviation, out[2] share of sampled keys repeating an earlier sample,
 * out[3] mean longest common prefix of a sample with any other sample over
 * the mean length.  Reads only bytes [0, keys_bytes) of the key stream.
 * One kernel, no allocation; synchronous on `stream`. */
int gmpt_batch_features_device(const uint8_t *d_keys_hexs, const int *d_keys_indexs, int n, int64_t keys_bytes,
                               float out[4], void *stream);

/* A sequence of HOST batches, each inserted (two_phase[i] != 0: PhaseNU,
 * else LockNU), hashed and its root read (roots32[32 i..], root_sizes[i]),
 * with the host -> device copy of batch i+1 running on a second stream while
 * batch i is inserted and hashed (the reference's two-stream pipelines,
 * puts_2phase_pipeline gpu_mpt.cuh:1715-1823 and puts_latching_pipeline_v2
 * gpu_mpt.cuh:926-982).  Per-batch arrays as for gmpt_puts_2phase;
 * values_hps may be NULL (or hold NULL entries).  Copies overlap only from
 * page-locked host memory. */
int gmpt_puts_pipeline(gmpt_trie *t, int count, const uint8_t *const *keys_hexs, const int *const *keys_indexs,
                       const uint8_t *const *values_bytes, const int64_t *const *values_indexs,
                       const uint8_t *const *const *values_hps, const int *counts, const int *two_phase,
                       uint8_t *roots32, int *root_sizes);

/* ---- deletes ----
 * Remove keys (hex-nibble keys with terminator, index pairs as for the puts;
 * trie_ids may be NULL: trie 0); absent keys are ignored.  After
 * gmpt_hash_onepass the trie is the canonical trie of the remaining keys:
 * a branch left with one child becomes a short node merged with the
 * extension above it, an emptied branch disappears.  No counterpart in the
 * reference, which has no delete path (go-ethereum deletes empty accounts
 * and zeroed storage slots on commit).
 * Space is not reclaimed: unlinked branches, dead short nodes, the deleted
 * keys' value records and the old key bytes stay in the pools and arenas,
 * and every collapsed branch appends one short node plus its merged key
 * (extension key + 1 + the child's key, in nibbles) to them.  A workload
 * that deletes and re-inserts keys block after block grows the pools until
 * gmpt_reset, or until the live keys are re-loaded into a fresh trie. */
int gmpt_deletes(gmpt_trie *t, const uint8_t *keys_hexs, const int *keys_indexs, const int *trie_ids, int n);
/* The same with DEVICE key / index / trie-id arrays; keys_bytes = key stream length. */
int gmpt_deletes_device(gmpt_trie *t, const uint8_t *d_keys_hexs, const int *d_keys_indexs, const int *d_trie_ids,
                        int n, int64_t keys_bytes);

/* ---- mixed read/write batches ----
 * puts_latching_with_valuehp_v2_with_read (gpu_mpt.cuh:684-765) and
 * puts_2phase_with_valuehp_with_read (gpu_mpt.cuh:1609-1713): rw_flags[i] = 0
 * (READ_FLAG, util/utils.cuh:26) looks key i up, 1 (WRITE_FLAG) puts it; any
 * other flag is GMPT_E_ARG.  Every key has a value pair (ignored for reads;
 * empty pairs allowed).  Deterministic where the reference is not: the batch
 * acts as if applied in index order -- a read returns the last earlier write
 * of its key in the batch, else the value before the batch -- and read i's
 * result is at its rank among the reads (the reference fills read slots in
 * atomicAdd order, its reads race with the batch's writes).  Results: the
 * host pointer given with the value (NULL if absent or none was given) and
 * the size (0 if absent); *read_num = number of reads.  Writes then behave as
 * gmpt_puts_2phase / gmpt_puts_latching (last write of a key wins) and need
 * gmpt_hash_onepass like them. */
int gmpt_puts_latching_with_read(gmpt_trie *t, const uint8_t *keys_hexs, const int *keys_indexs, int *read_num,
                                 const uint8_t *rw_flags, const uint8_t *values_bytes, const int64_t *values_indexs,
                                 const uint8_t *const *values_hps, int n, const uint8_t **read_values_hps,
                                 int *read_values_sizes);
int gmpt_puts_2phase_with_read(gmpt_trie *t, const uint8_t *keys_hexs, const int *keys_indexs, int *read_num,
                               const uint8_t *rw_flags, const uint8_t *values_bytes, const int64_t *values_indexs,
                               const uint8_t *const *values_hps, int n, const uint8_t **read_values_hps,
                               int *read_values_sizes);
/* The same over a forest (trie_ids may be NULL: trie 0); two_phase picks
 * PhaseNU (1) or LockNU (0). */
int gmpt_puts_with_read_forest(gmpt_trie *t, int two_phase, const uint8_t *keys_hexs, const int *keys_indexs,
                               const uint8_t *rw_flags, const uint8_t *values_bytes, const int64_t *values_indexs,
                               const uint8_t *const *values_hps, const int *trie_ids, int n,
                               const uint8_t **read_values_hps, int *read_values_sizes, int *read_num);
/* DEVICE inputs and DEVICE result arrays (n entries each; the first
 * *read_num are written); *read_num is a host int. */
int gmpt_puts_with_read_device(gmpt_trie *t, int two_phase, const uint8_t *d_keys_hexs, const int *d_keys_indexs,
                               const uint8_t *d_rw_flags, const uint8_t *d_values_bytes,
                               const int64_t *d_values_indexs, const uint64_t *d_values_hps, const int *d_trie_ids,
                               int n, int64_t keys_bytes, int64_t values_bytes, uint64_t *d_read_values_hps,
                               int *d_read_values_sizes, int *read_num);

/* ---- raw-key batches ----
 * The reference's callers convert every key to hex nibbles on the host
 * (test/experiments.cu:50-73 keys_bytes_to_hexs over util/utils.cuh:340-349
 * key_bytes_to_hex) and pass the nibble stream to the puts above.  These take the
 * raw key bytes instead: keys_indexs[2 i], [2 i + 1] is the inclusive byte
 * range of key i (end = start - 1 for the empty key), and the device writes
 * nibbles (high, low per byte) plus terminator 16 straight into the trie's
 * key arena.  Results are identical to the hex puts on key_bytes_to_hex of
 * the same keys; the key stream crosses PCIe at half the size.  two_phase
 * picks PhaseNU (1) or LockNU (0); trie_ids may be NULL (trie 0).  No
 * counterpart in the reference. */
int gmpt_puts_raw(gmpt_trie *t, int two_phase, const uint8_t *keys, const int *keys_indexs,
                  const uint8_t *values_bytes, const int64_t *values_indexs, const uint8_t *const *values_hps,
                  const int *trie_ids, int n);
/* gmpt_puts_raw with DEVICE arrays (read in place; keys_bytes = raw key bytes). */
int gmpt_puts_raw_device(gmpt_trie *t, int two_phase, const uint8_t *d_keys, const int *d_keys_indexs,
                         const uint8_t *d_values_bytes, const int64_t *d_values_indexs, const uint64_t *d_values_hps,
                         const int *d_trie_ids, int n, int64_t keys_bytes, int64_t values_bytes);
/* gmpt_puts_pipeline with raw-key host batches. */
int gmpt_puts_pipeline_raw(gmpt_trie *t, int count, const uint8_t *const *keys, const int *const *keys_indexs,
                           const uint8_t *const *values_bytes, const int64_t *const *values_indexs,
                           const uint8_t *const *const *values_hps, const int *counts, const int *two_phase,
                           uint8_t *roots32, int *root_sizes);

/* hash_onepass_v2 (gpu_mpt.cuh:131, 1162-1191): PhaseHC over every node made
 * dirty since the last call. */
int gmpt_hash_onepass(gmpt_trie *t);

/* The device array of dirty node references pending for gmpt_hash_onepass
 * (the reference returns it from the puts as std::tuple<Node**, int>). */
int gmpt_pending_targets(gmpt_trie *t, const uint32_t **d_targets, int *n);

/* get_root_hash (gpu_mpt.cuh:151-152, 1217-1247): *size = 0 for an empty
 * trie, < 32 for a raw root in GMPT_MODE_REF, else 32. */
int gmpt_get_root_hash(gmpt_trie *t, uint8_t out[32], int *size);

/* Roots of tries trie_ids[0..n) (NULL: tries 0..n-1), as get_root_hash:
 * out32[32 i ..] zero-padded, sizes[i] = 0 / < 32 / 32. */
int gmpt_get_roots(gmpt_trie *t, const int *trie_ids, int n, uint8_t *out32, int *sizes);

/* gets_parallel (gpu_mpt.cuh:139-140, 984-1036): values_hps[i] receives the
 * host pointer given with the stored value (NULL when the key is absent or
 * none was given) and values_sizes[i] its length (0 when absent). */
int gmpt_gets_parallel(gmpt_trie *t, const uint8_t *keys_hexs, const int *keys_indexs, int n,
                       const uint8_t **values_hps, int *values_sizes);

/* gets_parallel on a forest: key i is looked up in trie trie_ids[i]. */
int gmpt_gets_forest(gmpt_trie *t, const uint8_t *keys_hexs, const int *keys_indexs, const int *trie_ids, int n,
                     const uint8_t **values_hps, int *values_sizes);

/* Value bytes stored for each key, concatenated into out (capacity out_cap);
 * out_indexs[2i], out_indexs[2i+1] = inclusive range, or -1, -1 if absent.
 * *out_len = bytes written (or needed, when out_cap is too small). */
int gmpt_get_values(gmpt_trie *t, const uint8_t *keys_hexs, const int *keys_indexs, int n,
                    uint8_t *out, int64_t out_cap, int64_t *out_indexs, int64_t *out_len);

int gmpt_get_stats(gmpt_trie *t, gmpt_stats *out);

/* The commit nodeset: (hash, RLP encoding) of every node hashed since the
 * previous gmpt_flush_dirty (or since tracking began) that is still in a
 * trie and is referenced by hash -- encoding of 32 bytes or more, or a root
 * -- in its current state, each once, ordered by node reference.  hashs =
 * 32 bytes per node (a root shorter than 32 bytes: its raw encoding,
 * zero-padded), encs + inclusive [start, end] pairs encs_indexs[2 * num];
 * the three arrays are malloc'd, release them with gmpt_free_buffer.  Needs
 * the "track_dirty" option set to 1 before the puts whose nodes are to be
 * exported (hash passes then keep a record of their nodes, 4 bytes per node,
 * until the flush; persistent block updates are not recorded).  The
 * reference exports every node on a set of key paths instead
 * (MPT::flush_dirty_nodes, gpu_mpt.cuh:1039-1122, behind get_all_nodes,
 * lib/libgmpt.cu:216-238); go-ethereum commits only the changed nodes. */
int gmpt_flush_dirty(gmpt_trie *t, const uint8_t **hashs, const uint8_t **encs,
                     const unsigned long long **encs_indexs, unsigned long long *num);
/* Tuning knobs of the batch pipeline (results never depend on them):
 *   "local_build" 1/0: finish build segments of <= 2048 keys inside one CTA
 *                      each (default 1) or keep every level device-wide;
 *   "local_sort"  1/0: same for the still-tied runs of the batch sort;
 *   "local_build_cap", "local_sort_cap" N (<= 2048; 0 = 2048): the largest
 *                      segment / run finished inside one CTA;
 *   "latch_ways"  1/2/4: keys each LockNU thread walks together (default 4:
 *                      more loads in flight; 1: more threads for small batches);
 *   "latch_dedup" 0/1/2: LockNU drops repeated keys of a batch before the
 *                      walk: never / batches of >= 64K keys (default) / always;
 *   "sort_dedup"  0/1/2: PhaseNU drops repeated keys of a batch (keeping the
 *                      last) before sorting: never / batches of >= 64K keys
 *                      whose 64K-key sample holds more than 1 % repeats
 *                      (default) / always;
 *   "warp_full_max" N: PhaseHC hashes a level's branches one warp each when
 *                      the level has at most N branches (default 4096);
 *   "block_grid"  N:   CTAs of the persistent block kernel (0 = one per SM,
 *                      capped at what can be co-resident);
 *   "block_graph" 1/0: replay block launches from a captured CUDA graph
 *                      (default 1) or issue them one by one;
 *   "track_dirty" 1/0: record the nodes each hash pass rehashes for
 *                      gmpt_flush_dirty (default 0).
 * Failure bounds (the reference instead spins without bound, util/lock.cuh:
 * 17-21, and asserts on arena overflow, util/allocator.cuh:115-118):
 *   "retry_limit" N:   failed CASes one LockNU key may take before the batch
 *                      reports GMPT_E_RETRY_LIMIT (default 2^20).  Keys that
 *                      hit it are left out and every other key is in; putting
 *                      the batch again completes it;
 *   "block_barrier_ns" N: longest grid-barrier wait of the persistent block
 *                      kernel (default 2e9); a wait that runs out ends the
 *                      launch with GMPT_E_INTERNAL ("grid barrier wait gave
 *                      up") with the block partly applied: gmpt_reset and
 *                      reload the trie;
 *   "max_branch_nodes" N: the branch pool stops growing at N nodes (0 = no
 *                      cap); a batch that needs more fails with
 *                      GMPT_E_CAPACITY from the kernel that ran out, partly
 *                      applied: gmpt_reset and reload the trie. */
int gmpt_set_option(gmpt_trie *t, const char *name, int64_t value);

/* ---- schedules and the schedule selector ----
 * A put batch can run under several schedules -- PhaseNU or LockNU with
 * their knobs, or the persistent launch (LockNU insert + PhaseHC in one
 * graph-replayed kernel) -- and every one gives the same trie, so choosing
 * only changes time.  No counterpart in the reference, which fixes LockNU
 * (lib/libgmpt.cu:107-111) and fits its cost model offline
 * (test/experiments.cu:3250-3348).
 * gmpt_schedule_info(k, out): out = {PhaseNU, persistent, local_build,
 * local_sort, latch_ways, latch_dedup, block_grid, warp_full_max}. */
int gmpt_schedule_count(void);
const char *gmpt_schedule_name(int k);
int gmpt_schedule_info(int k, int out[8]);
/* Insert a batch under schedule k (host arrays; trie_ids may be NULL).  A
 * persistent schedule also hashes the trie; a batch it cannot take (caller
 * host pointers, index pairs that do not tile the key stream) runs as LockNU. */
int gmpt_puts_schedule(gmpt_trie *t, int k, const uint8_t *keys_hexs, const int *keys_indexs,
                       const uint8_t *values_bytes, const int64_t *values_indexs, const uint8_t *const *values_hps,
                       const int *trie_ids, int n);
/* The same with device arrays (d_trie_ids may be NULL). */
int gmpt_puts_schedule_device(gmpt_trie *t, int k, const uint8_t *d_keys_hexs, const int *d_keys_indexs,
                              const uint8_t *d_values_bytes, const int64_t *d_values_indexs, const int *d_trie_ids,
                              int n, int64_t keys_bytes, int64_t values_bytes);
/* The selector's features of a put batch into t:
 *   out[0] log2(n + 1)          out[4] log2(value nodes in t + 1)
 *   out[1] mean key nibbles/64  out[5] log2(mean value bytes + 1)
 *   out[2] key-length spread/64 out[6] mean longest common prefix of a
 *   out[3] repeated-key share          sampled key with the others / mean length
 *                               out[7] log2(tries the batch touches)
 * out[2], out[3], out[6] come from 64 evenly spaced keys (host arrays: on the
 * host; device arrays: the kernel of gmpt_batch_features_device). */
int gmpt_batch_features(gmpt_trie *t, const uint8_t *keys_hexs, const int *keys_indexs,
                        const int64_t *values_indexs, const int *trie_ids, int n, float out[8]);
/* Device key arrays, stream totals given.  tries_touched > 0 fills out[7]
 * and trie_keys >= 0 (keys of the tries the batch touches) out[4]; otherwise
 * they come from the whole trie object. */
int gmpt_batch_features_trie_device(gmpt_trie *t, const uint8_t *d_keys_hexs, const int *d_keys_indexs, int n,
                                    int64_t keys_bytes, int64_t values_bytes, int tries_touched, int64_t trie_keys,
                                    float out[8]);
/* A schedule selector: an autotuned rule table (coarse buckets of batch
 * size, trie size and repeated-key share -> the schedule measured fastest
 * there) and optionally the MLP of gmpt_mlp_* predicting every schedule's
 * log time (inference on the device), with the rule as fallback outside the
 * network's training range.  path = a file written by the Python trainer
 * (gmpt.tuner.Selector.save); NULL = the built-in rule (empty trie: PhaseNU;
 * up to 64K keys: persistent launch; else LockNU, 4 keys per thread). */
typedef struct gmpt_selector gmpt_selector;
gmpt_selector *gmpt_selector_create(int device, const char *path);
void gmpt_selector_destroy(gmpt_selector *s);
int gmpt_selector_choose(gmpt_selector *s, const float features[8], int *schedule, int *used_net);
/* out[0] = choices so far, out[1] = of which the rule made (fallbacks) */
int gmpt_selector_counts(gmpt_selector *s, uint64_t out[2]);
/* Insert a batch under the schedule the selector picks for it (sel NULL: the
 * library's selector of the trie's device -- the file named by the
 * GMPT_SELECTOR environment variable, else the built-in rule).  *chosen
 * (may be NULL) = the schedule run.  Setting GMPT_SCHEDULE=auto makes the
 * reference ABI's build_mpt_* / insert_mpt_* calls (libgmpt.h) go this way. */
int gmpt_puts_auto(gmpt_trie *t, gmpt_selector *sel, const uint8_t *keys_hexs, const int *keys_indexs,
                   const uint8_t *values_bytes, const int64_t *values_indexs, const uint8_t *const *values_hps,
                   const int *trie_ids, int n, int *chosen);
/* Device arrays; tries_touched / trie_keys as for gmpt_batch_features_trie_device. */
int gmpt_puts_auto_device(gmpt_trie *t, gmpt_selector *sel, const uint8_t *d_keys_hexs, const int *d_keys_indexs,
                          const uint8_t *d_values_bytes, const int64_t *d_values_indexs, const int *d_trie_ids, int n,
                          int64_t keys_bytes, int64_t values_bytes, int tries_touched, int64_t trie_keys,
                          int *chosen);
/* per-phase CUDA-event timing into gmpt_stats (adds synchronisation) */
int gmpt_set_timing(gmpt_trie *t, int on);

/* The trie's CUDA stream (a cudaStream_t), for callers that order their own
 * work or events against it. */
void *gmpt_stream(gmpt_trie *t);

/* Keccak-256 (Ethereum padding) of n messages: data + inclusive int64
 * [start, end] pairs -> out32[32 * n].  Host arrays; the reference's
 * standalone batch kernel is keccak_kernel_batch
 * (hash/batch_mode_hash.cuh:89-115). */
int gmpt_keccak256_batch(const uint8_t *data, const int64_t *indexs, int n, uint8_t *out32);
/* Same with device arrays, on `stream` (a cudaStream_t, or NULL). */
int gmpt_keccak256_batch_device(const uint8_t *d_data, const int64_t *d_indexs, int n, uint8_t *d_out32,
                                void *stream);
/* gmpt_keccak256_batch without any device allocation.  No counterpart in the
 * reference.  For callers that cannot allocate device memory at the point of
 * the call: a process whose device memory is already owned by another
 * allocator (a framework's caching allocator that reserved the GPU), or code
 * that must not call cudaMalloc/cudaFree there.  Same inputs, outputs and
 * results as gmpt_keccak256_batch (host arrays), but every device-side copy
 * goes through one fixed 3.5 MiB array inside the library that each GPU
 * loading the library keeps until the process exits.
 * Limits: at most 32768 messages and 2 MiB of message bytes per call (every
 * end index below 2^21); larger calls fail with GMPT_E_ARG and a message
 * naming the limit, before any device work.
 * Memory: the array lives in the library's device module.  CUDA loads that
 * module, and allocates its memory (the array included), on the first call
 * on a device that uses any of the library's kernels -- this function's
 * first call, or any earlier library call.  Callers whose device memory is
 * later handed to another allocator should make one call before that.  The
 * first call on a device also looks up the array's device address (set-up,
 * once per device, on the current device); make that first call before any
 * stream capture.
 * Ordering: the copies and the kernel run on the calling thread's per-thread
 * default stream (cudaStreamPerThread), and the call returns when they have
 * finished; they do not wait for other non-blocking streams.  All calls share
 * the one array, so calls from this process are serialised; work that
 * overlaps a call on the same GPU through other means races with it. */
int gmpt_keccak256_batch_noalloc(const uint8_t *data, const int64_t *indexs, int n, uint8_t *out32);
/* Measurement aid: Keccak-f[1600] permutations per second of a
 * register-only loop on `device` (the integer-pipe ceiling of the hash
 * stage's permutation code). */
int gmpt_keccak_peak(int device, double *perm_per_s);
/* Number of kernels this library has launched in this process. */
uint64_t gmpt_launch_count(void);

/* ---- schedule selector network --------------------------------------
 * A two-hidden-layer ReLU MLP (n_in <= 16, n_hidden <= 64, n_out <= 16, fp32)
 * with hand-written CUDA inference, gradient and Adam training kernels; the
 * library's schedule selector predicts per-configuration batch times with it.
 * No counterpart in the reference, whose insert strategy is fixed
 * (libgmpt.cu:107-111) and whose model fitting happens offline
 * (experiments.cu:3250-3348).  Parameters, flat: W1[H][I] b1[H] W2[H][H]
 * b2[H] W3[O][H] b3[O]; He-uniform weights from `seed`, zero biases.
 * Loss: sum of mask * (y - target)^2 over all outputs / sum of mask. */
typedef struct gmpt_mlp gmpt_mlp;
gmpt_mlp *gmpt_mlp_create(int device, int n_in, int n_hidden, int n_out, uint64_t seed);
void gmpt_mlp_destroy(gmpt_mlp *m);
int gmpt_mlp_num_params(gmpt_mlp *m);
int gmpt_mlp_get_params(gmpt_mlp *m, float *out);
/* also clears the Adam moments and step count */
int gmpt_mlp_set_params(gmpt_mlp *m, const float *in);
/* y[n][n_out] for x[n][n_in] (host arrays) */
int gmpt_mlp_forward(gmpt_mlp *m, const float *x, int n, float *y);
/* loss and gradient (n_params floats) over all n samples */
int gmpt_mlp_loss_grad(gmpt_mlp *m, const float *x, const float *t, const float *mask, int n, float *loss,
                       float *grad);
/* Adam (0.9, 0.999, 1e-8) over `epochs` passes in mini-batches of `batch`
 * (1..64) samples, one launch; epoch e visits positions j of [0, P), P the
 * next power of two >= n, as sample (a_e j + b_e) mod P, skipping images >= n,
 * with a_e odd and b_e from splitmix64 of seed and e.  *loss = mean
 * mini-batch loss of the last epoch. */
int gmpt_mlp_train(gmpt_mlp *m, const float *x, const float *t, const float *mask, int n, int epochs, int batch,
                   float lr, uint64_t seed, float *loss);

/* Status of the last failed call on this thread, and its message. */
int gmpt_last_error(void);
const char *gmpt_last_error_message(void);
/* Free memory returned by the libgmpt.h calls (roots, nodesets). */
void gmpt_free_buffer(void *p);

#ifdef __cplusplus
}
#endif
#endif
