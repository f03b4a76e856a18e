/*
 * mpt_oracle.c -- CPU restatement of the reference MPT (TEST INFRASTRUCTURE).
 * See mpt_oracle.h for the reference lines each part follows.
 */
#include "mpt_oracle.h"

#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Keccak-f[1600] (FIPS 202; reference loop form hash/cpu_hash.h:35-76)     */
/* ------------------------------------------------------------------------ */

static const uint64_t kRoundConst[24] = {
    0x0000000000000001ULL, 0x0000000000008082ULL, 0x800000000000808aULL,
    0x8000000080008000ULL, 0x000000000000808bULL, 0x0000000080000001ULL,
    0x8000000080008081ULL, 0x8000000000008009ULL, 0x000000000000008aULL,
    0x0000000000000088ULL, 0x0000000080008009ULL, 0x000000008000000aULL,
    0x000000008000808bULL, 0x800000000000008bULL, 0x8000000000008089ULL,
    0x8000000000008003ULL, 0x8000000000008002ULL, 0x8000000000000080ULL,
    0x000000000000800aULL, 0x800000008000000aULL, 0x8000000080008081ULL,
    0x8000000000008080ULL, 0x0000000080000001ULL, 0x8000000080008008ULL};

/* rho offsets r[x + 5y] */
static const int kRho[25] = {0,  1,  62, 28, 27, 36, 44, 6,  55, 20, 3,  10, 43,
                             25, 39, 41, 45, 15, 21, 8,  18, 2,  61, 56, 14};

static inline uint64_t rotl64(uint64_t v, int n) {
  return n == 0 ? v : (v << n) | (v >> (64 - n));
}

void omt_keccak_f1600(uint64_t a[25]) {
  for (int round = 0; round < 24; ++round) {
    uint64_t c[5], d[5], b[25];
    for (int x = 0; x < 5; ++x)
      c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
    for (int x = 0; x < 5; ++x) d[x] = c[(x + 4) % 5] ^ rotl64(c[(x + 1) % 5], 1);
    for (int i = 0; i < 25; ++i) a[i] ^= d[i % 5];
    /* rho + pi: B[y, 2x+3y] = rot(A[x, y], r[x, y]) */
    for (int x = 0; x < 5; ++x)
      for (int y = 0; y < 5; ++y)
        b[y + 5 * ((2 * x + 3 * y) % 5)] = rotl64(a[x + 5 * y], kRho[x + 5 * y]);
    /* chi */
    for (int y = 0; y < 5; ++y)
      for (int x = 0; x < 5; ++x)
        a[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
    /* iota */
    a[0] ^= kRoundConst[round];
  }
}

static void sponge256(const uint8_t *in, size_t len, uint8_t pad, uint8_t out[32]) {
  enum { RATE = 136 };
  uint64_t st[25];
  uint8_t blk[RATE];
  memset(st, 0, sizeof(st));
  while (len >= RATE) {
    for (int i = 0; i < RATE / 8; ++i) {
      uint64_t w;
      memcpy(&w, in + 8 * i, 8); /* little-endian lanes */
      st[i] ^= w;
    }
    omt_keccak_f1600(st);
    in += RATE;
    len -= RATE;
  }
  memset(blk, 0, sizeof(blk));
  memcpy(blk, in, len);
  blk[len] ^= pad;
  blk[RATE - 1] ^= 0x80;
  for (int i = 0; i < RATE / 8; ++i) {
    uint64_t w;
    memcpy(&w, blk + 8 * i, 8);
    st[i] ^= w;
  }
  omt_keccak_f1600(st);
  memcpy(out, st, 32);
}

void omt_keccak256(const uint8_t *in, size_t len, uint8_t out[32]) {
  sponge256(in, len, 0x01, out);
}

void omt_sha3_256(const uint8_t *in, size_t len, uint8_t out[32]) {
  sponge256(in, len, 0x06, out);
}

void omt_keccak256_rows(const uint8_t *in, size_t rows, size_t width, uint8_t *out) {
  for (size_t r = 0; r < rows; ++r) sponge256(in + r * width, width, 0x01, out + 32 * r);
}

/* ------------------------------------------------------------------------ */
/* RLP (util/rlp.cuh:9-155) and compact keys (util/utils.cuh:340-396)        */
/* ------------------------------------------------------------------------ */

static int putint_size(uint64_t i) {
  int size = 1;
  while ((i >>= 8) != 0) ++size;
  return size;
}

static int putint(uint8_t *b, uint64_t i) {
  int n = putint_size(i);
  for (int k = 0; k < n; ++k) b[k] = (uint8_t)(i >> (8 * (n - 1 - k)));
  return n;
}

/* size of an RLP string holding `bytes` */
static int rlp_str_size(const uint8_t *bytes, int len) {
  if (len == 1 && bytes[0] <= 0x7f) return 1;
  if (len < 56) return 1 + len;
  return 1 + putint_size((uint64_t)len) + len;
}

static int rlp_str(uint8_t *out, const uint8_t *bytes, int len) {
  if (len == 1 && bytes[0] <= 0x7f) {
    out[0] = bytes[0];
    return 1;
  }
  int h;
  if (len < 56) {
    out[0] = (uint8_t)(0x80 + len);
    h = 1;
  } else {
    int s = putint(out + 1, (uint64_t)len);
    out[0] = (uint8_t)(0xb7 + s);
    h = 1 + s;
  }
  memcpy(out + h, bytes, (size_t)len);
  return h + len;
}

static int rlp_list_head_size(uint64_t payload) {
  return payload < 56 ? 1 : 1 + putint_size(payload);
}

static int rlp_list_head(uint8_t *out, uint64_t payload) {
  if (payload < 56) {
    out[0] = (uint8_t)(0xc0 + payload);
    return 1;
  }
  int s = putint(out + 1, payload);
  out[0] = (uint8_t)(0xf7 + s);
  return 1 + s;
}

int omt_key_bytes_to_hex(const uint8_t *key, int len, uint8_t *hex) {
  for (int i = 0; i < len; ++i) {
    hex[2 * i] = key[i] >> 4;
    hex[2 * i + 1] = key[i] & 15;
  }
  hex[2 * len] = 16;
  return 2 * len + 1;
}

static int compact_size(const uint8_t *hex, int len) {
  if (len > 0 && hex[len - 1] == 16) --len;
  return len / 2 + 1;
}

int omt_hex_to_compact(const uint8_t *hex, int len, uint8_t *out) {
  uint8_t term = 0;
  if (len > 0 && hex[len - 1] == 16) {
    term = 1;
    --len;
  }
  int n = len / 2 + 1;
  out[0] = (uint8_t)(term << 5);
  if (len & 1) {
    out[0] |= (uint8_t)(0x10 | hex[0]);
    ++hex;
    --len;
  }
  for (int bi = 1, ni = 0; ni < len; ++bi, ni += 2)
    out[bi] = (uint8_t)((hex[ni] << 4) | hex[ni + 1]);
  return n;
}

/* ------------------------------------------------------------------------ */
/* Trie nodes and owned storage                                              */
/* ------------------------------------------------------------------------ */

enum { T_FULL = 1, T_SHORT = 2, T_VALUE = 3 };

typedef struct onode {
  uint8_t type;
  uint8_t dirty;
  uint8_t touched;    /* on a put path since the last omt_flush */
  uint8_t hlen;       /* length of hash[] (full/short nodes) */
  uint8_t hash[32];   /* Keccak-256, or the raw encoding if it is < 32 B */
  /* full */
  struct onode *child[17];
  /* short */
  const uint8_t *key;
  int klen;
  struct onode *val;
  /* value */
  const uint8_t *v;
  int vlen;
} onode;

typedef struct chunk {
  struct chunk *next;
  size_t used, cap;
  unsigned char data[];
} chunk;

struct omt_trie {
  int mode;
  onode *root;
  chunk *mem;
  omt_stats stats;
  uint8_t *enc;      /* scratch encoding buffer */
  size_t enc_cap;
};

static void *arena_alloc(omt_trie *t, size_t n) {
  n = (n + 15) & ~(size_t)15;
  if (!t->mem || t->mem->used + n > t->mem->cap) {
    size_t cap = n > (1u << 22) ? n : (1u << 22);
    chunk *c = (chunk *)malloc(sizeof(chunk) + cap);
    if (!c) return NULL;
    c->next = t->mem;
    c->used = 0;
    c->cap = cap;
    t->mem = c;
  }
  void *p = t->mem->data + t->mem->used;
  t->mem->used += n;
  return p;
}

static onode *new_node(omt_trie *t, int type) {
  onode *n = (onode *)arena_alloc(t, sizeof(onode));
  if (!n) return NULL;
  memset(n, 0, sizeof(*n));
  n->type = (uint8_t)type;
  n->dirty = 1;
  return n;
}

omt_trie *omt_new(int mode) {
  omt_trie *t = (omt_trie *)calloc(1, sizeof(omt_trie));
  if (!t) return NULL;
  t->mode = mode;
  return t;
}

void omt_free(omt_trie *t) {
  if (!t) return;
  chunk *c = t->mem;
  while (c) {
    chunk *nx = c->next;
    free(c);
    c = nx;
  }
  free(t->enc);
  free(t);
}

/* ------------------------------------------------------------------------ */
/* Insert: cpu_mpt.cuh:232-346 (dfs_put_baseline)                            */
/* ------------------------------------------------------------------------ */

static int prefix_len(const uint8_t *a, int alen, const uint8_t *b, int blen) {
  int m = 0;
  while (m < alen && m < blen && a[m] == b[m]) ++m;
  return m;
}

/* returns the new subtree root; *dirty tells whether anything changed;
 * *err is set on malformed (prefix) keys. */
static onode *put_rec(omt_trie *t, onode *node, const uint8_t *key, int klen,
                      onode *value, int *dirty, int *err) {
  if (node && node->type != T_VALUE) node->touched = 1;
  if (klen == 0) {
    if (node && node->type == T_VALUE) {
      *dirty = !(node->vlen == value->vlen &&
                 memcmp(node->v, value->v, (size_t)value->vlen) == 0);
      return value;
    }
    if (node) *err = OMT_ERR_BAD_KEY; /* key ends inside an inner node */
    *dirty = 1;
    return value;
  }
  if (!node) {
    onode *s = new_node(t, T_SHORT);
    if (!s) {
      *err = OMT_ERR_NOMEM;
      return NULL;
    }
    s->key = key;
    s->klen = klen;
    s->val = value;
    s->touched = 1;
    *dirty = 1;
    return s;
  }
  if (node->type == T_SHORT) {
    int m = prefix_len(node->key, node->klen, key, klen);
    if (m == node->klen) {
      int d = 0;
      node->val = put_rec(t, node->val, key + m, klen - m, value, &d, err);
      if (d) node->dirty = 1;
      *dirty = d;
      return node;
    }
    if (m == klen) { /* new key is a proper prefix of a stored one */
      *err = OMT_ERR_BAD_KEY;
      *dirty = 0;
      return node;
    }
    onode *br = new_node(t, T_FULL);
    if (!br) {
      *err = OMT_ERR_NOMEM;
      return node;
    }
    br->touched = 1;
    int d1 = 0, d2 = 0;
    br->child[node->key[m]] = put_rec(t, NULL, node->key + m + 1,
                                      node->klen - m - 1, node->val, &d1, err);
    br->child[key[m]] = put_rec(t, NULL, key + m + 1, klen - m - 1, value, &d2, err);
    *dirty = 1;
    if (m == 0) return br;
    node->klen = m; /* the old short node becomes the extension */
    node->val = br;
    node->dirty = 1;
    return node;
  }
  if (node->type == T_FULL) {
    int d = 0;
    onode *c = put_rec(t, node->child[key[0]], key + 1, klen - 1, value, &d, err);
    if (d) {
      node->child[key[0]] = c;
      node->dirty = 1;
    }
    *dirty = d;
    return node;
  }
  /* a value node reached with key left over: stored key is a prefix */
  *err = OMT_ERR_BAD_KEY;
  *dirty = 0;
  return node;
}

int omt_puts(omt_trie *t, const uint8_t *keys_hexs, const int *keys_indexs,
             const uint8_t *values, const int64_t *values_indexs, int n) {
  int err = OMT_OK;
  for (int i = 0; i < n; ++i) {
    int ks = keys_indexs[2 * i], klen = keys_indexs[2 * i + 1] - ks + 1;
    int64_t vs = values_indexs[2 * i];
    int vlen = (int)(values_indexs[2 * i + 1] - vs + 1);
    for (int j = 0; j < klen; ++j) {
      uint8_t nb = keys_hexs[ks + j];
      if (nb > 16 || (nb == 16 && j != klen - 1)) return OMT_ERR_BAD_KEY;
    }
    uint8_t *kc = (uint8_t *)arena_alloc(t, (size_t)klen + 1);
    uint8_t *vc = (uint8_t *)arena_alloc(t, (size_t)vlen + 1);
    onode *v = new_node(t, T_VALUE);
    if (!kc || !vc || !v) return OMT_ERR_NOMEM;
    memcpy(kc, keys_hexs + ks, (size_t)klen);
    memcpy(vc, values + vs, (size_t)vlen);
    v->v = vc;
    v->vlen = vlen;
    int dirty = 0;
    t->root = put_rec(t, t->root, kc, klen, v, &dirty, &err);
    if (err) return err;
  }
  return OMT_OK;
}

/* ------------------------------------------------------------------------ */
/* Hash: cpu_mpt.cuh:380-505 (dfs_hashs_dirty_flag) + node.cuh encoders      */
/* ------------------------------------------------------------------------ */

/* the bytes a parent writes for child c */
static void child_ref(const onode *c, const uint8_t **p, int *len) {
  if (c->type == T_VALUE) {
    *p = c->v;
    *len = c->vlen;
  } else {
    *p = c->hash;
    *len = c->hlen;
  }
}

/* size of the item a parent writes for child c */
static int child_item_size(const omt_trie *t, const onode *c) {
  const uint8_t *p;
  int len;
  child_ref(c, &p, &len);
  if (t->mode == OMT_MODE_GETH && c->type != T_VALUE && len < 32) return len;
  return rlp_str_size(p, len);
}

static int child_item(const omt_trie *t, uint8_t *out, const onode *c) {
  const uint8_t *p;
  int len;
  child_ref(c, &p, &len);
  if (t->mode == OMT_MODE_GETH && c->type != T_VALUE && len < 32) {
    memcpy(out, p, (size_t)len); /* embedded node (go-ethereum) */
    return len;
  }
  return rlp_str(out, p, len);
}

static uint8_t *enc_buf(omt_trie *t, size_t n) {
  if (n > t->enc_cap) {
    free(t->enc);
    t->enc_cap = n * 2;
    t->enc = (uint8_t *)malloc(t->enc_cap);
  }
  return t->enc;
}

static void finish_hash(omt_trie *t, onode *node, const uint8_t *enc, int len,
                        int force) {
  t->stats.hashed_nodes++;
  t->stats.enc_bytes += (uint64_t)len;
  if (len < 32 && !force) {
    memcpy(node->hash, enc, (size_t)len);
    node->hlen = (uint8_t)len;
  } else {
    omt_keccak256(enc, (size_t)len, node->hash);
    node->hlen = 32;
    t->stats.keccak_calls++;
    t->stats.keccak_blocks += (uint64_t)(len + 1 + 135) / 136;
  }
}

/* RLP encoding of a full or short node from its children's current
 * references (node.cuh:46-112, 226-270) into the scratch buffer; returns
 * its length. */
static int encode_node(omt_trie *t, const onode *node, uint8_t **out) {
  if (node->type == T_SHORT) {
    uint8_t kcbuf[256];
    uint8_t *kc = node->klen / 2 + 1 <= (int)sizeof(kcbuf)
                      ? kcbuf
                      : (uint8_t *)arena_alloc(t, (size_t)node->klen / 2 + 1);
    int kn = omt_hex_to_compact(node->key, node->klen, kc);
    uint64_t payload = (uint64_t)rlp_str_size(kc, kn) + (uint64_t)child_item_size(t, node->val);
    int len = rlp_list_head_size(payload) + (int)payload;
    uint8_t *e = enc_buf(t, (size_t)len);
    int o = rlp_list_head(e, payload);
    o += rlp_str(e + o, kc, kn);
    o += child_item(t, e + o, node->val);
    (void)o;
    *out = e;
    return len;
  }
  uint64_t payload = 0;
  for (int i = 0; i < 17; ++i)
    payload += node->child[i] ? (uint64_t)child_item_size(t, node->child[i]) : 1;
  int len = rlp_list_head_size(payload) + (int)payload;
  uint8_t *e = enc_buf(t, (size_t)len);
  int o = rlp_list_head(e, payload);
  for (int i = 0; i < 17; ++i) {
    if (node->child[i])
      o += child_item(t, e + o, node->child[i]);
    else
      e[o++] = 0x80;
  }
  *out = e;
  return len;
}

static void hash_rec(omt_trie *t, onode *node, int is_root) {
  if (!node) return;
  if (node->type == T_VALUE) return; /* hash := raw value bytes */
  if (!node->dirty) return;
  int force = is_root && t->mode == OMT_MODE_GETH;
  if (node->type == T_SHORT)
    hash_rec(t, node->val, 0);
  else
    for (int i = 0; i < 17; ++i) hash_rec(t, node->child[i], 0);
  uint8_t *e;
  int len = encode_node(t, node, &e);
  if (node->type == T_SHORT)
    t->stats.hashed_short++;
  else
    t->stats.hashed_full++;
  finish_hash(t, node, e, len, force);
  node->dirty = 0;
}

/* ------------------------------------------------------------------------ */
/* Commit nodeset: reachable nodes on put paths since the last flush          */
/* ------------------------------------------------------------------------ */

typedef struct flushbuf {
  uint8_t *hashs, *encs;
  uint64_t *idx;
  uint64_t num, cap, ebytes, ecap;
} flushbuf;

static int flush_rec(omt_trie *t, onode *node, int is_root, flushbuf *f) {
  if (!node || node->type == T_VALUE) return 0;
  if (node->type == T_SHORT) {
    if (flush_rec(t, node->val, 0, f)) return 1;
  } else {
    for (int i = 0; i < 17; ++i)
      if (flush_rec(t, node->child[i], 0, f)) return 1;
  }
  if (!node->touched) return 0;
  node->touched = 0;
  if (node->hlen != 32 && !is_root) return 0; /* embedded in its parent */
  uint8_t *e;
  int len = encode_node(t, node, &e);
  if (f->num == f->cap) {
    f->cap = f->cap ? 2 * f->cap : 1024;
    f->hashs = (uint8_t *)realloc(f->hashs, 32 * f->cap);
    f->idx = (uint64_t *)realloc(f->idx, 16 * f->cap);
    if (!f->hashs || !f->idx) return 1;
  }
  if (f->ebytes + (uint64_t)len > f->ecap) {
    f->ecap = 2 * (f->ebytes + (uint64_t)len) + 4096;
    f->encs = (uint8_t *)realloc(f->encs, f->ecap);
    if (!f->encs) return 1;
  }
  memset(f->hashs + 32 * f->num, 0, 32);
  memcpy(f->hashs + 32 * f->num, node->hash, node->hlen);
  memcpy(f->encs + f->ebytes, e, (size_t)len);
  f->idx[2 * f->num] = f->ebytes;
  f->idx[2 * f->num + 1] = f->ebytes + (uint64_t)len - 1;
  f->ebytes += (uint64_t)len;
  f->num++;
  return 0;
}

int omt_flush(omt_trie *t, uint8_t **hashs, uint8_t **encs, uint64_t **encs_indexs,
              uint64_t *num) {
  flushbuf f;
  memset(&f, 0, sizeof(f));
  int rc = flush_rec(t, t->root, 1, &f);
  *hashs = f.hashs;
  *encs = f.encs;
  *encs_indexs = f.idx;
  *num = f.num;
  return rc ? OMT_ERR_NOMEM : OMT_OK;
}

void omt_free_buffer(void *p) { free(p); }

void omt_hash(omt_trie *t) {
  omt_stats keep = t->stats;
  memset(&t->stats, 0, sizeof(t->stats));
  t->stats.nodes_full = keep.nodes_full;
  t->stats.nodes_short = keep.nodes_short;
  t->stats.nodes_value = keep.nodes_value;
  t->stats.max_depth_nibbles = keep.max_depth_nibbles;
  hash_rec(t, t->root, 1);
}

int omt_root(const omt_trie *t, uint8_t out[32]) {
  const onode *r = t->root;
  if (!r) return 0;
  if (r->type == T_VALUE) { /* degenerate trie of one empty key */
    int n = r->vlen < 32 ? r->vlen : 32;
    memcpy(out, r->v, (size_t)n);
    return n;
  }
  memcpy(out, r->hash, r->hlen);
  return r->hlen;
}

/* ------------------------------------------------------------------------ */
/* Get: cpu_mpt.cuh:507-579                                                  */
/* ------------------------------------------------------------------------ */

void omt_gets(const omt_trie *t, const uint8_t *keys_hexs,
              const int *keys_indexs, int n, uint64_t *out_ptr, int *out_len) {
  for (int i = 0; i < n; ++i) {
    const uint8_t *key = keys_hexs + keys_indexs[2 * i];
    int klen = keys_indexs[2 * i + 1] - keys_indexs[2 * i] + 1;
    const onode *node = t->root;
    int pos = 0;
    out_ptr[i] = 0;
    out_len[i] = 0;
    while (node) {
      if (node->type == T_VALUE) {
        if (pos == klen) {
          out_ptr[i] = (uint64_t)(uintptr_t)node->v;
          out_len[i] = node->vlen;
        }
        break;
      }
      if (node->type == T_SHORT) {
        if (klen - pos < node->klen ||
            memcmp(node->key, key + pos, (size_t)node->klen) != 0)
          break;
        pos += node->klen;
        node = node->val;
      } else {
        if (pos >= klen || key[pos] > 16) break;
        node = node->child[key[pos]];
        pos += 1;
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Stats                                                                     */
/* ------------------------------------------------------------------------ */

static void count_rec(omt_stats *s, const onode *n, uint64_t depth) {
  if (!n) return;
  if (n->type == T_VALUE) {
    s->nodes_value++;
    if (depth > s->max_depth_nibbles) s->max_depth_nibbles = depth;
  } else if (n->type == T_SHORT) {
    s->nodes_short++;
    count_rec(s, n->val, depth + (uint64_t)n->klen);
  } else {
    s->nodes_full++;
    for (int i = 0; i < 17; ++i) count_rec(s, n->child[i], depth + 1);
  }
}

uint64_t omt_count_stats(omt_trie *t) {
  t->stats.nodes_full = t->stats.nodes_short = t->stats.nodes_value = 0;
  t->stats.max_depth_nibbles = 0;
  count_rec(&t->stats, t->root, 0);
  return t->stats.nodes_full + t->stats.nodes_short + t->stats.nodes_value;
}

void omt_get_stats(const omt_trie *t, omt_stats *out) { *out = t->stats; }
