/*
 * libgmpt.h -- drop-in C ABI of the reference's libgmpt, served by the B200
 * MPT library (libgmpt_b200.so).
 *
 * Same symbols, enum and struct as mpt-with-compress/lib/libgmpt.h:1-55, with
 * the behaviour fixes documented per function.  Every entry point is
 * extern "C", takes plain pointers and sizes, and never exits the process:
 * failures return NULL / a zero nodeset and set gmpt_last_error()
 * (declared in gmpt.h).
 *
 * Conventions kept from the reference: keys are hex-nibble bytes with the
 * terminator 16 (util/utils.cuh:340-349); index arrays are inclusive
 * [start, end] pairs, int for keys and int64_t for values
 * (util/utils.cuh:254-301); values_hps are caller host pointers echoed back by
 * lookups (NULL allowed).
 */
#ifndef LIBGMPT_H
#define LIBGMPT_H

#ifdef __cplusplus
extern "C" {
#endif

#include "stdint.h"

/* lib/libgmpt.h:7-11 */
enum TrieType {
  STATE_TRIE = 0,
  TRANSACTION_TRIE = 1,
  RECEIPT_TRIE = 2,
};

/* lib/libgmpt.h:13-18: hashs[32 * num], encs[...], encs_indexs[2 * num]
 * inclusive pairs into encs.  Release each array with gmpt_free_buffer(). */
struct nodeset {
  const uint8_t *hashs;
  const uint8_t *encs;
  const unsigned long long *encs_indexs;
  unsigned long long num;
};

/* lib/libgmpt.cu:45-129 (reference: runs LockNU despite the name).  Here:
 * PhaseNU batch insert into the global trie of `trie_type`, PhaseHC, and the
 * root.  Returns a malloc'd 32-byte root (a root encoding shorter than 32
 * bytes is zero-padded) or NULL for an empty trie / on error. */
const uint8_t *build_mpt_2phase(enum TrieType trie_type,
                                const uint8_t *keys_hexs, int *keys_hexs_indexs,
                                const uint8_t *values_bytes,
                                int64_t *values_bytes_indexs,
                                const uint8_t **values_hps, int insert_num);

/* lib/libgmpt.cu:131-214: LockNU batch insert + PhaseHC + root. */
const uint8_t *build_mpt_olc(enum TrieType trie_type, const uint8_t *keys_hexs,
                             int *keys_hexs_indexs, const uint8_t *values_bytes,
                             int64_t *values_bytes_indexs,
                             const uint8_t **values_hps, int insert_num);

/* lib/libgmpt.cu:25-43: (re)creates the three global tries.  The device is
 * GMPT_DEVICE (default 0) instead of a hard-coded device 1, and it does not
 * reset the device.  Returns 1 on success, 0 on failure. */
int preprocess();

/* lib/libgmpt.cu:216-238: (hash, RLP encoding) of every node on the paths of
 * the given keys in the STATE trie (any trie_type is accepted here; the
 * reference asserts STATE and deletes the other two tries, this does not). */
struct nodeset get_all_nodes(enum TrieType trie_type, const uint8_t *keys_hexs,
                             int *keys_hexs_indexs, int num);

/* ------------------------------------------------------------------------ */
/* lib/libgmpt.cu:323-327: a new empty trie on the current device. */
void *init_mpt();

/* lib/libgmpt.cu:240-246 is an empty stub in the reference; here PhaseNU +
 * PhaseHC + root on the given trie. */
const uint8_t *insert_mpt_2phase(void *mpt, const uint8_t *keys_hexs,
                                 int *keys_hexs_indexs,
                                 const uint8_t *values_bytes,
                                 int64_t *values_bytes_indexs,
                                 const uint8_t **values_hps, int insert_num);
/* lib/libgmpt.cu:248-321: LockNU + PhaseHC + root on the given trie. */
const uint8_t *insert_mpt_olc(void *mpt, const uint8_t *keys_hexs,
                              int *keys_hexs_indexs,
                              const uint8_t *values_bytes,
                              int64_t *values_bytes_indexs,
                              const uint8_t **values_hps, int insert_num);

/* lib/libgmpt.cu:329-332 resets the whole device; here it frees only `mpt`. */
void free_mpt(void *mpt);
/* ------------------------------------------------------------------------ */

#ifdef __cplusplus
}
#endif
#endif
