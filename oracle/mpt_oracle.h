/*
 * mpt_oracle.h -- CPU restatement of the reference Merkle Patricia Trie
 * (TEST INFRASTRUCTURE ONLY: the checker for the GPU path, never shipped).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load this library.  It restates, in plain C, the algorithm of the
 * reference's CPU MPT:
 *   insert   mpt-with-compress/include/mpt/cpu_mpt.cuh:232-378 (dfs_put_baseline,
 *            puts_baseline): sequential, last write wins, split into
 *            branch + optional extension, nil -> new leaf.
 *   hash     cpu_mpt.cuh:380-505 (dfs_hashs_dirty_flag): encode, Keccak-256
 *            when the encoding is >= 32 bytes, else keep the raw encoding;
 *            a value node's "hash" is its raw value bytes.
 *   encode   node.cuh:46-112 (full), node.cuh:226-270 (short),
 *            util/rlp.cuh:9-155, util/utils.cuh:361-396 (hex_to_compact).
 *   keccak   hash/cpu_hash.h:35-127 (Keccak-f[1600], rate 136, pad 0x01).
 *   get      cpu_mpt.cuh:507-579, root cpu_mpt.cuh:915-934.
 *
 * Two encode modes:
 *   OMT_MODE_REF  (0): byte-for-byte the reference: a child whose encoding is
 *                      shorter than 32 bytes is written as an RLP *string* of
 *                      its raw encoding (node.cuh:75,442) and a root shorter
 *                      than 32 bytes is returned unhashed (cpu_mpt.cuh:413-418).
 *   OMT_MODE_GETH (1): go-ethereum's rule: such a child is embedded as-is and
 *                      the root is always hashed.
 */
#ifndef MPT_ORACLE_H
#define MPT_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OMT_MODE_REF = 0, OMT_MODE_GETH = 1 };

enum {
  OMT_OK = 0,
  OMT_ERR_BAD_KEY = 1,   /* nibble > 16, or a key that is a prefix of another */
  OMT_ERR_NOMEM = 2,
};

typedef struct omt_trie omt_trie;

/* Accounting of the last omt_hash() pass: the dirty set and its encodings. */
typedef struct omt_stats {
  uint64_t hashed_nodes;     /* full + short nodes re-encoded */
  uint64_t hashed_full;      /* of which full (branch) nodes */
  uint64_t hashed_short;     /* of which short (extension / leaf) nodes */
  uint64_t enc_bytes;        /* sum of encoding lengths of re-encoded nodes */
  uint64_t keccak_blocks;    /* sum of ceil((enc+1)/136) over hashed (>=32 B) */
  uint64_t keccak_calls;     /* nodes whose encoding was >= 32 bytes */
  uint64_t nodes_full;       /* live node counts of the whole trie */
  uint64_t nodes_short;
  uint64_t nodes_value;
  uint64_t max_depth_nibbles;
} omt_stats;

/* --- Keccak (hash/cpu_hash.h:35-127) ------------------------------------ */
void omt_keccak_f1600(uint64_t st[25]);
/* Keccak-256 (pad 0x01), what the trie uses. */
void omt_keccak256(const uint8_t *in, size_t len, uint8_t out[32]);
/* FIPS-202 SHA3-256 (pad 0x06): same permutation; used to pin it. */
void omt_sha3_256(const uint8_t *in, size_t len, uint8_t out[32]);
/* Keccak-256 of each of `rows` messages of `width` bytes laid out back to
 * back -> out[32 * rows]. */
void omt_keccak256_rows(const uint8_t *in, size_t rows, size_t width, uint8_t *out);

/* --- helpers (util/utils.cuh) ------------------------------------------- */
int omt_key_bytes_to_hex(const uint8_t *key, int len, uint8_t *hex);
int omt_hex_to_compact(const uint8_t *hex, int hex_len, uint8_t *out);

/* --- trie ---------------------------------------------------------------- */
omt_trie *omt_new(int mode);
void omt_free(omt_trie *t);
/* Sequential puts in index order; key/value bytes are copied into the trie.
 * keys_indexs / values_indexs are inclusive [start, end] pairs. */
int omt_puts(omt_trie *t, const uint8_t *keys_hexs, const int *keys_indexs,
             const uint8_t *values, const int64_t *values_indexs, int n);
/* Re-hash dirty nodes; fills the stats of this pass. */
void omt_hash(omt_trie *t);
/* Root reference: returns its length (0 = empty trie, <32 = raw encoding in
 * OMT_MODE_REF, 32 = Keccak-256). */
int omt_root(const omt_trie *t, uint8_t out[32]);
/* Lookups: out_ptr[i] = address of the stored value bytes (0 if absent),
 * out_len[i] = its length.  The addresses stay valid until omt_free. */
void omt_gets(const omt_trie *t, const uint8_t *keys_hexs,
              const int *keys_indexs, int n, uint64_t *out_ptr,
              int *out_len);
void omt_get_stats(const omt_trie *t, omt_stats *out);
/* Commit nodeset (call after omt_hash): (hash, encoding) of every node
 * reachable from the root that a put visited or created since the last
 * omt_flush and that is referenced by hash (hash length 32) or is the root;
 * hashs[32 * num] (zero-padded), encs + inclusive pairs encs_indexs[2 * num],
 * children before parents.  Clears the marks.  Free the arrays with
 * omt_free_buffer. */
int omt_flush(omt_trie *t, uint8_t **hashs, uint8_t **encs, uint64_t **encs_indexs,
              uint64_t *num);
void omt_free_buffer(void *p);
uint64_t omt_count_stats(omt_trie *t); /* refresh live node counts; returns total */

#ifdef __cplusplus
}
#endif
#endif
