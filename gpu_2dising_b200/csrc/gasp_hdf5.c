/*
 * gasp_hdf5.c -- the PyGASP side files gridstates.hdf5 / pBgrids.hdf5
 * (create_ising_grids_hdf5 / write_ising_grids_hdf5, src/io.c:132-301),
 * written without libhdf5.
 *
 * The files follow the HDF5 file format specification with the structures
 * libhdf5 writes under its default (earliest-format) settings: a version 0
 * superblock (8-byte offsets and lengths, group leaf K 4, group internal K
 * 16), version 1 object headers, and symbol-table groups (a version 1 B-tree
 * of group nodes over symbol-table nodes, link names in a local heap).
 * Content, as the reference writes it:
 *   /L, /ngrids, /tot_nsweeps     scalar int32
 *   /h, /beta                     scalar IEEE double
 *   /total_saved_grids            scalar int32: grids written so far
 *   /sweep_<isweep>/grid_<g>      int32 [L][L], contiguous, with the
 *                                 variable-length ASCII string attributes
 *                                 magnetisation and lclus_size ("%g" of the
 *                                 value, or "null"), committor and
 *                                 committor_error ("null")
 * Each write appends to the end of the file: the grids' data, global heap
 * collections holding the attribute strings, the datasets' object headers,
 * the new group's local heap, symbol-table nodes, B-tree and object header,
 * then a rebuilt index of the root group.  Last, the root object header's
 * symbol-table message, the superblock (root index, end of file) and
 * total_saved_grids are updated in place.  The superseded root index stays in
 * the file, unreferenced (under 1 KB per write for a few hundred groups).
 * Appending reads back only the superblock, the root group and
 * total_saved_grids, so it works on files this writer created.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/types.h>

#include "gasp.h"

#define H5_UNDEF 0xFFFFFFFFFFFFFFFFull
#define H5_FREE_NULL 1u /* "no free block" in a local heap (libhdf5's encoding) */

enum {
  kLeafK = 4,                                   /* symbol-table node: 2K entries */
  kNodeK = 16,                                  /* group B-tree node: 2K children */
  kEntry = 40,                                  /* symbol-table entry, 8-byte offsets */
  kSnodSize = 8 + 2 * kLeafK * kEntry,          /* 328 */
  kTreeSize = 24 + (2 * kNodeK + 1) * 8 + 2 * kNodeK * 8, /* 544 */
  kSuperSize = 96,
  kRootOhdrAt = kSuperSize,                     /* root object header, fixed */
  kGcolMaxObjs = 2048                           /* strings per global heap collection */
};

enum {
  kMsgDataspace = 0x0001,
  kMsgDatatype = 0x0003,
  kMsgFill = 0x0005,
  kMsgLayout = 0x0008,
  kMsgAttribute = 0x000C,
  kMsgSymtab = 0x0011
};

/* ------------------------------------------------------------ byte buffer */
typedef struct {
  uint8_t *p;
  size_t n, cap;
  int oom;
} buf_t;

static void b_need(buf_t *b, size_t extra) {
  if (b->oom || b->n + extra <= b->cap) return;
  size_t cap = b->cap ? b->cap : 4096;
  while (cap < b->n + extra) cap *= 2;
  uint8_t *q = (uint8_t *)realloc(b->p, cap);
  if (!q) {
    b->oom = 1;
    return;
  }
  b->p = q;
  b->cap = cap;
}
static void b_put(buf_t *b, const void *src, size_t n) {
  b_need(b, n);
  if (b->oom) return;
  memcpy(b->p + b->n, src, n);
  b->n += n;
}
static void b_zero(buf_t *b, size_t n) {
  b_need(b, n);
  if (b->oom) return;
  memset(b->p + b->n, 0, n);
  b->n += n;
}
static void b_le(buf_t *b, uint64_t v, int nbytes) {
  uint8_t t[8];
  for (int i = 0; i < nbytes; ++i) t[i] = (uint8_t)(v >> (8 * i));
  b_put(b, t, (size_t)nbytes);
}
#define b_u8(b, v) b_le((b), (v), 1)
#define b_u16(b, v) b_le((b), (v), 2)
#define b_u32(b, v) b_le((b), (v), 4)
#define b_u64(b, v) b_le((b), (v), 8)
static void b_pad8(buf_t *b) { b_zero(b, (8 - (b->n & 7)) & 7); }
static void set_le(uint8_t *p, uint64_t v, int nbytes) {
  for (int i = 0; i < nbytes; ++i) p[i] = (uint8_t)(v >> (8 * i));
}
static uint64_t get_le(const uint8_t *p, int nbytes) {
  uint64_t v = 0;
  for (int i = nbytes - 1; i >= 0; --i) v = (v << 8) | p[i];
  return v;
}
static size_t pad8(size_t n) { return (n + 7) & ~(size_t)7; }

/* ------------------------------------------------------------ file access */
static int f_read_at(FILE *f, uint64_t off, void *dst, size_t n) {
  if (fseeko(f, (off_t)off, SEEK_SET) != 0) return -1;
  return fread(dst, 1, n, f) == n ? 0 : -1;
}
static int f_write_at(FILE *f, uint64_t off, const void *src, size_t n) {
  if (fseeko(f, (off_t)off, SEEK_SET) != 0) return -1;
  return fwrite(src, 1, n, f) == n ? 0 : -1;
}

/* ------------------------------------------------------- object headers */
/* Version 1 object header: 16-byte prefix (version, reserved, message count,
 * reference count, chunk size, 4 bytes of alignment), then messages of an
 * 8-byte header (type, size, flags, 3 reserved) and data padded to 8 bytes. */
typedef struct {
  size_t start;
  int nmsgs;
} ohdr_t;

static ohdr_t oh_begin(buf_t *b) {
  ohdr_t o = {b->n, 0};
  b_u8(b, 1);
  b_u8(b, 0);
  b_u16(b, 0); /* message count, set by oh_end */
  b_u32(b, 1); /* reference count */
  b_u32(b, 0); /* chunk size, set by oh_end */
  b_u32(b, 0);
  return o;
}
/* Starts a message; returns the offset of its data within b. */
static size_t oh_msg(buf_t *b, ohdr_t *o, unsigned type, size_t size, unsigned flags) {
  b_u16(b, type);
  b_u16(b, pad8(size));
  b_u8(b, flags);
  b_zero(b, 3);
  o->nmsgs++;
  return b->n;
}
static void oh_end(buf_t *b, ohdr_t *o) {
  if (b->oom) return;
  set_le(b->p + o->start + 2, (uint64_t)o->nmsgs, 2);
  set_le(b->p + o->start + 8, (uint64_t)(b->n - o->start - 16), 4);
}

/* Dataspace message, version 1 (rank 0: scalar). */
static void msg_dataspace(buf_t *b, ohdr_t *o, int rank, const uint64_t *dims) {
  oh_msg(b, o, kMsgDataspace, 8 + 8 * (size_t)rank, 0);
  b_u8(b, 1);
  b_u8(b, (unsigned)rank);
  b_u8(b, 0); /* no maximum dimensions, no permutation */
  b_zero(b, 5);
  for (int i = 0; i < rank; ++i) b_u64(b, dims[i]);
}
/* Datatype descriptions (version 1). */
static void dt_int(buf_t *b, unsigned size, int is_signed) {
  b_u8(b, 0x10); /* version 1, class 0: fixed point */
  b_u8(b, is_signed ? 0x08 : 0x00); /* little-endian, zero padding */
  b_zero(b, 2);
  b_u32(b, size);
  b_u16(b, 0);        /* bit offset */
  b_u16(b, 8 * size); /* bit precision */
}
static void dt_double(buf_t *b) {
  b_u8(b, 0x11); /* version 1, class 1: floating point */
  b_u8(b, 0x20); /* little-endian, implied leading mantissa bit */
  b_u8(b, 63);   /* sign bit position */
  b_u8(b, 0);
  b_u32(b, 8);
  b_u16(b, 0);
  b_u16(b, 64);
  b_u8(b, 52); /* exponent location */
  b_u8(b, 11); /* exponent size */
  b_u8(b, 0);  /* mantissa location */
  b_u8(b, 52); /* mantissa size */
  b_u32(b, 1023);
}
enum { kDtIntSize = 12, kDtDoubleSize = 20, kDtVlenStrSize = 20 };
/* Variable-length string: null-terminated ASCII over unsigned 8-bit chars;
 * an element is a 4-byte length and a global heap ID (collection address,
 * object index). */
static void dt_vlen_str(buf_t *b) {
  b_u8(b, 0x19); /* version 1, class 9: variable length */
  b_u8(b, 0x01); /* string, null-terminated padding */
  b_u8(b, 0x00); /* ASCII */
  b_u8(b, 0);
  b_u32(b, 4 + 8 + 4);
  dt_int(b, 1, 0); /* base type */
}
static void msg_fill(buf_t *b, ohdr_t *o) {
  oh_msg(b, o, kMsgFill, 4, 1);
  b_u8(b, 2); /* version 2 */
  b_u8(b, 2); /* space allocated late */
  b_u8(b, 2); /* fill written only if one is set */
  b_u8(b, 0); /* no fill value defined */
  b_zero(b, 4);
}
static void msg_layout(buf_t *b, ohdr_t *o, uint64_t addr, uint64_t size) {
  oh_msg(b, o, kMsgLayout, 18, 0);
  b_u8(b, 3); /* version 3 */
  b_u8(b, 1); /* contiguous */
  b_u64(b, addr);
  b_u64(b, size);
  b_zero(b, 6);
}
static size_t msg_symtab(buf_t *b, ohdr_t *o, uint64_t btree, uint64_t heap) {
  const size_t at = oh_msg(b, o, kMsgSymtab, 16, 0);
  b_u64(b, btree);
  b_u64(b, heap);
  return at;
}
/* Scalar variable-length string attribute, version 1. */
static void msg_attr_str(buf_t *b, ohdr_t *o, const char *name, uint64_t gcol, uint32_t idx,
                         uint32_t len) {
  const size_t nlen = strlen(name) + 1;
  oh_msg(b, o, kMsgAttribute, 8 + pad8(nlen) + pad8(kDtVlenStrSize) + 8 + 16, 0);
  b_u8(b, 1);
  b_u8(b, 0);
  b_u16(b, nlen);
  b_u16(b, kDtVlenStrSize);
  b_u16(b, 8);
  b_put(b, name, nlen);
  b_pad8(b);
  dt_vlen_str(b);
  b_pad8(b);
  b_u8(b, 1); /* scalar dataspace, version 1 */
  b_zero(b, 7);
  b_u32(b, len);
  b_u64(b, gcol);
  b_u32(b, idx);
}

/* Object header of a contiguous dataset (scalar when rank == 0). */
static void dataset_ohdr(buf_t *b, int rank, const uint64_t *dims, int is_double, uint64_t addr,
                         uint64_t size, ohdr_t *o_out) {
  ohdr_t o = oh_begin(b);
  msg_dataspace(b, &o, rank, dims);
  oh_msg(b, &o, kMsgDatatype, is_double ? kDtDoubleSize : kDtIntSize, 1);
  if (is_double)
    dt_double(b);
  else
    dt_int(b, 4, 1);
  b_pad8(b);
  msg_fill(b, &o);
  msg_layout(b, &o, addr, size);
  *o_out = o;
}

/* --------------------------------------------------------------- groups */
typedef struct {
  char *name;
  uint64_t ohdr;
  uint32_t cache; /* 1: a group, scratch-pad holds its B-tree and heap */
  uint64_t btree, heap;
} link_t;

static int link_cmp(const void *a, const void *b) {
  return strcmp(((const link_t *)a)->name, ((const link_t *)b)->name);
}

static void sym_entry(buf_t *b, uint64_t name_off, const link_t *l) {
  b_u64(b, name_off);
  b_u64(b, l->ohdr);
  b_u32(b, l->cache);
  b_u32(b, 0);
  if (l->cache == 1) {
    b_u64(b, l->btree);
    b_u64(b, l->heap);
  } else {
    b_zero(b, 16);
  }
}

/* Appends a group's index for the links (sorted by name) to b, whose first
 * byte sits at file offset base: the local heap (names), symbol-table nodes of
 * up to 2*kLeafK entries and a B-tree of nodes of up to 2*kNodeK children.
 * A key of a group node is the heap offset of a name: child i of a node holds
 * the names above key i up to key i+1, key 0 of the leftmost node is the empty
 * name at heap offset 0, and key i+1 is the last name under child i. */
static int group_index(buf_t *b, uint64_t base, const link_t *links, int n, uint64_t *btree_out,
                       uint64_t *heap_out) {
  uint64_t *name_off = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(n ? n : 1));
  if (!name_off) return GASP_ERR_ALLOC;
  size_t seg = 8; /* offset 0: the empty name */
  for (int i = 0; i < n; ++i) {
    name_off[i] = seg;
    seg += pad8(strlen(links[i].name) + 1);
  }
  const uint64_t heap = base + b->n;
  b_put(b, "HEAP", 4);
  b_u8(b, 0);
  b_zero(b, 3);
  b_u64(b, seg);
  b_u64(b, H5_FREE_NULL);
  b_u64(b, heap + 32);
  b_zero(b, 8);
  for (int i = 0; i < n; ++i) {
    const size_t len = strlen(links[i].name) + 1;
    b_put(b, links[i].name, len);
    b_zero(b, pad8(len) - len);
  }
  /* symbol-table nodes */
  const int per_snod = 2 * kLeafK;
  int nchild = (n + per_snod - 1) / per_snod;
  uint64_t *child = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(nchild ? nchild : 1));
  uint64_t *ckey = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(nchild ? nchild : 1));
  if (!child || !ckey) {
    free(name_off);
    free(child);
    free(ckey);
    return GASP_ERR_ALLOC;
  }
  for (int s = 0; s < nchild; ++s) {
    const int lo = s * per_snod, hi = lo + per_snod < n ? lo + per_snod : n;
    child[s] = base + b->n;
    ckey[s] = name_off[hi - 1];
    b_put(b, "SNOD", 4);
    b_u8(b, 1);
    b_u8(b, 0);
    b_u16(b, (uint64_t)(hi - lo));
    for (int i = lo; i < hi; ++i) sym_entry(b, name_off[i], &links[i]);
    b_zero(b, (size_t)(per_snod - (hi - lo)) * kEntry);
  }
  free(name_off);
  /* B-tree levels, bottom up, until one node remains */
  int level = 0;
  const int per_node = 2 * kNodeK;
  for (;;) {
    const int nnodes = nchild ? (nchild + per_node - 1) / per_node : 1;
    const uint64_t first = base + b->n;
    for (int j = 0; j < nnodes; ++j) {
      const int lo = j * per_node, hi = lo + per_node < nchild ? lo + per_node : nchild;
      b_put(b, "TREE", 4);
      b_u8(b, 0); /* group node */
      b_u8(b, (unsigned)level);
      b_u16(b, (uint64_t)(hi - lo));
      b_u64(b, j > 0 ? first + (uint64_t)(j - 1) * kTreeSize : H5_UNDEF);
      b_u64(b, j + 1 < nnodes ? first + (uint64_t)(j + 1) * kTreeSize : H5_UNDEF);
      b_u64(b, lo > 0 ? ckey[lo - 1] : 0);
      for (int i = lo; i < hi; ++i) {
        b_u64(b, child[i]);
        b_u64(b, ckey[i]);
      }
      b_zero(b, (size_t)(per_node - (hi - lo)) * 16);
    }
    /* the nodes of this level become the children of the next */
    for (int j = 0; j < nnodes; ++j) {
      const int hi = (j + 1) * per_node < nchild ? (j + 1) * per_node : nchild;
      child[j] = first + (uint64_t)j * kTreeSize;
      ckey[j] = nchild ? ckey[hi - 1] : 0;
    }
    if (nnodes == 1) {
      *btree_out = first;
      break;
    }
    nchild = nnodes;
    ++level;
  }
  free(child);
  free(ckey);
  *heap_out = heap;
  return b->oom ? GASP_ERR_ALLOC : GASP_OK;
}

/* ----------------------------------------------------- reading a file back */
typedef struct {
  FILE *f;
  uint64_t eof;
  uint64_t root_ohdr, root_btree, root_heap;
  uint64_t root_symtab_at; /* file offset of the root symbol-table message data */
  uint8_t *heap_seg;
  uint64_t heap_len;
  link_t *links;
  int nlinks, cap;
} h5file_t;

static void h5_release(h5file_t *h) {
  for (int i = 0; i < h->nlinks; ++i) free(h->links[i].name);
  free(h->links);
  free(h->heap_seg);
  h->links = NULL;
  h->heap_seg = NULL;
  h->nlinks = h->cap = 0;
}

static int add_link(h5file_t *h, const char *name, uint64_t ohdr, uint32_t cache, uint64_t bt,
                    uint64_t hp) {
  if (h->nlinks == h->cap) {
    const int cap = h->cap ? 2 * h->cap : 16;
    link_t *q = (link_t *)realloc(h->links, sizeof(link_t) * (size_t)cap);
    if (!q) return GASP_ERR_ALLOC;
    h->links = q;
    h->cap = cap;
  }
  char *s = strdup(name);
  if (!s) return GASP_ERR_ALLOC;
  link_t l = {s, ohdr, cache, bt, hp};
  h->links[h->nlinks++] = l;
  return GASP_OK;
}

/* Walks the root group's B-tree (depth-first, children in order). */
static int read_tree(h5file_t *h, uint64_t addr, int depth) {
  if (depth > 16 || addr >= h->eof) return GASP_ERR_FORMAT;
  uint8_t node[kTreeSize];
  if (f_read_at(h->f, addr, node, sizeof node)) return GASP_ERR_FORMAT;
  if (memcmp(node, "TREE", 4) || node[4] != 0) return GASP_ERR_FORMAT;
  const int level = node[5], used = (int)get_le(node + 6, 2);
  if (used > 2 * kNodeK) return GASP_ERR_FORMAT;
  for (int i = 0; i < used; ++i) {
    const uint64_t c = get_le(node + 24 + 8 + 16 * (size_t)i, 8);
    int rc;
    if (level > 0) {
      rc = read_tree(h, c, depth + 1);
    } else {
      uint8_t sn[kSnodSize];
      if (c >= h->eof || f_read_at(h->f, c, sn, sizeof sn)) return GASP_ERR_FORMAT;
      if (memcmp(sn, "SNOD", 4) || sn[4] != 1) return GASP_ERR_FORMAT;
      const int ns = (int)get_le(sn + 6, 2);
      if (ns > 2 * kLeafK) return GASP_ERR_FORMAT;
      rc = GASP_OK;
      for (int e = 0; e < ns && rc == GASP_OK; ++e) {
        const uint8_t *en = sn + 8 + (size_t)e * kEntry;
        const uint64_t off = get_le(en, 8);
        if (off >= h->heap_len || !memchr(h->heap_seg + off, 0, h->heap_len - off))
          return GASP_ERR_FORMAT;
        rc = add_link(h, (const char *)h->heap_seg + off, get_le(en + 8, 8),
                      (uint32_t)get_le(en + 16, 4), get_le(en + 24, 8), get_le(en + 32, 8));
      }
    }
    if (rc) return rc;
  }
  return GASP_OK;
}

/* Finds the data of a message of `type` in the object header at addr; its
 * file offset and size. */
static int find_msg(h5file_t *h, uint64_t addr, unsigned type, uint64_t *at, size_t *size) {
  uint8_t pre[16];
  if (addr >= h->eof || f_read_at(h->f, addr, pre, sizeof pre) || pre[0] != 1)
    return GASP_ERR_FORMAT;
  const int nm = (int)get_le(pre + 2, 2);
  const uint64_t chunk = get_le(pre + 8, 4);
  uint64_t p = addr + 16;
  const uint64_t end = p + chunk;
  for (int i = 0; i < nm && p + 8 <= end; ++i) {
    uint8_t mh[8];
    if (f_read_at(h->f, p, mh, sizeof mh)) return GASP_ERR_FORMAT;
    const unsigned t = (unsigned)get_le(mh, 2);
    const size_t sz = (size_t)get_le(mh + 2, 2);
    if (t == type) {
      *at = p + 8;
      *size = sz;
      return GASP_OK;
    }
    p += 8 + sz;
  }
  return GASP_ERR_FORMAT;
}

/* Opens a file this writer made and lists its root group. */
static int h5_open(h5file_t *h, const char *filename) {
  memset(h, 0, sizeof *h);
  h->f = fopen(filename, "r+b");
  if (!h->f) return GASP_ERR_IO;
  uint8_t sb[kSuperSize];
  if (f_read_at(h->f, 0, sb, sizeof sb)) return GASP_ERR_FORMAT;
  static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  if (memcmp(sb, sig, 8) || sb[8] != 0 || sb[13] != 8 || sb[14] != 8 ||
      get_le(sb + 16, 2) != kLeafK || get_le(sb + 18, 2) != kNodeK || get_le(sb + 24, 8) != 0)
    return GASP_ERR_FORMAT;
  h->eof = get_le(sb + 40, 8);
  if (fseeko(h->f, 0, SEEK_END) != 0 || (uint64_t)ftello(h->f) < h->eof || (h->eof & 7))
    return GASP_ERR_FORMAT;
  h->root_ohdr = get_le(sb + 56 + 8, 8);
  size_t sz = 0;
  int rc = find_msg(h, h->root_ohdr, kMsgSymtab, &h->root_symtab_at, &sz);
  if (rc || sz < 16) return GASP_ERR_FORMAT;
  uint8_t st[16];
  if (f_read_at(h->f, h->root_symtab_at, st, sizeof st)) return GASP_ERR_FORMAT;
  h->root_btree = get_le(st, 8);
  h->root_heap = get_le(st + 8, 8);
  uint8_t hp[32];
  if (h->root_heap >= h->eof || f_read_at(h->f, h->root_heap, hp, sizeof hp) ||
      memcmp(hp, "HEAP", 4) || hp[4] != 0)
    return GASP_ERR_FORMAT;
  h->heap_len = get_le(hp + 8, 8);
  const uint64_t seg = get_le(hp + 24, 8);
  if (h->heap_len == 0 || seg + h->heap_len > h->eof) return GASP_ERR_FORMAT;
  h->heap_seg = (uint8_t *)malloc(h->heap_len);
  if (!h->heap_seg) return GASP_ERR_ALLOC;
  if (f_read_at(h->f, seg, h->heap_seg, h->heap_len)) return GASP_ERR_FORMAT;
  return read_tree(h, h->root_btree, 0);
}

/* Writes a rebuilt root index at the end of the file and points the root
 * object header and the superblock at it (end of file updated last). */
static int h5_commit_root(h5file_t *h) {
  qsort(h->links, (size_t)h->nlinks, sizeof(link_t), link_cmp);
  buf_t b = {0};
  uint64_t bt = 0, hp = 0;
  int rc = group_index(&b, h->eof, h->links, h->nlinks, &bt, &hp);
  if (!rc && f_write_at(h->f, h->eof, b.p, b.n)) rc = GASP_ERR_IO;
  if (!rc) {
    h->eof += b.n;
    uint8_t st[16], eo[8];
    set_le(st, bt, 8);
    set_le(st + 8, hp, 8);
    set_le(eo, h->eof, 8);
    if (f_write_at(h->f, h->root_symtab_at, st, 16) || f_write_at(h->f, 56 + 24, st, 16) ||
        f_write_at(h->f, 40, eo, 8))
      rc = GASP_ERR_IO;
    h->root_btree = bt;
    h->root_heap = hp;
  }
  free(b.p);
  return rc;
}

/* ------------------------------------------------------------ entry points */
int gasp_create_ising_grids_hdf5(int L, int ngrids, int tot_nsweeps, double h, double beta,
                                 int itask, const char *filename) {
  (void)itask; /* accepted and unused, as in the reference */
  if (!filename) return GASP_ERR_INVALID;
  FILE *f = fopen(filename, "w+b");
  if (!f) {
    fprintf(stderr, "Error: failed to create HDF5 file '%s'\n", filename);
    return GASP_ERR_IO;
  }
  h5file_t hf;
  memset(&hf, 0, sizeof hf);
  hf.f = f;
  buf_t b = {0};
  /* superblock (end of file and root index patched by h5_commit_root) */
  static const uint8_t sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  b_put(&b, sig, 8);
  b_u8(&b, 0); /* superblock version */
  b_u8(&b, 0); /* free-space storage version */
  b_u8(&b, 0); /* root group symbol-table entry version */
  b_u8(&b, 0);
  b_u8(&b, 0); /* shared header message format version */
  b_u8(&b, 8); /* size of offsets */
  b_u8(&b, 8); /* size of lengths */
  b_u8(&b, 0);
  b_u16(&b, kLeafK);
  b_u16(&b, kNodeK);
  b_u32(&b, 0);        /* consistency flags */
  b_u64(&b, 0);        /* base address */
  b_u64(&b, H5_UNDEF); /* free-space info */
  b_u64(&b, 0);        /* end of file */
  b_u64(&b, H5_UNDEF); /* driver information */
  b_u64(&b, 0);        /* root entry: link name offset */
  b_u64(&b, kRootOhdrAt);
  b_u32(&b, 1); /* cache type 1: scratch-pad holds the B-tree and heap */
  b_u32(&b, 0);
  b_zero(&b, 16);
  /* root group object header: one symbol-table message */
  ohdr_t ro = oh_begin(&b);
  hf.root_symtab_at = msg_symtab(&b, &ro, H5_UNDEF, H5_UNDEF);
  oh_end(&b, &ro);
  /* the six scalars: value, then object header */
  const int32_t ivals[4] = {L, ngrids, tot_nsweeps, 0};
  const char *inames[4] = {"L", "ngrids", "tot_nsweeps", "total_saved_grids"};
  const double dvals[2] = {h, beta};
  const char *dnames[2] = {"h", "beta"};
  int rc = GASP_OK;
  for (int i = 0; i < 6 && !rc; ++i) {
    const int dbl = i >= 4;
    const uint64_t at = b.n;
    if (dbl)
      b_put(&b, &dvals[i - 4], 8);
    else
      b_put(&b, &ivals[i], 4);
    b_pad8(&b);
    const uint64_t oh = b.n;
    ohdr_t o;
    dataset_ohdr(&b, 0, NULL, dbl, at, dbl ? 8 : 4, &o);
    oh_end(&b, &o);
    rc = add_link(&hf, dbl ? dnames[i - 4] : inames[i], oh, 0, 0, 0);
  }
  if (!rc && b.oom) rc = GASP_ERR_ALLOC;
  if (!rc && f_write_at(f, 0, b.p, b.n)) rc = GASP_ERR_IO;
  hf.eof = b.n;
  free(b.p);
  if (!rc) rc = h5_commit_root(&hf);
  h5_release(&hf);
  if (fclose(f) != 0 && !rc) rc = GASP_ERR_IO;
  if (rc) fprintf(stderr, "Error: failed to write HDF5 file '%s'\n", filename);
  return rc;
}

static const char *attr_value(const float *v, int g, char *tmp, size_t n) {
  if (!v) return "null";
  snprintf(tmp, n, "%g", (double)v[g]);
  return tmp;
}

int gasp_write_ising_grids_hdf5(int L, int ngrids, const int *ising_grids, int isweep,
                                const float *magnetisation, const float *lclus_size,
                                const char *cv, double dn_thr, double up_thr,
                                const char *filename) {
  (void)cv; /* accepted and unused, as in the reference */
  (void)dn_thr;
  (void)up_thr;
  if (!filename || L <= 0 || ngrids < 0 || (ngrids > 0 && !ising_grids)) return GASP_ERR_INVALID;
  h5file_t hf;
  int rc = h5_open(&hf, filename);
  if (rc) {
    fprintf(stderr, "Error: failed to open HDF5 file '%s' for writing\n", filename);
    if (hf.f) fclose(hf.f);
    h5_release(&hf);
    return rc;
  }
  char gname[64];
  snprintf(gname, sizeof gname, "sweep_%d", isweep);
  uint64_t tot_addr = 0;
  int has_total = 0;
  for (int i = 0; i < hf.nlinks; ++i) {
    if (!strcmp(hf.links[i].name, gname)) {
      fprintf(stderr, "Error: failed to create group '/%s' in HDF5 file\n", gname);
      fclose(hf.f);
      h5_release(&hf);
      return GASP_ERR_IO;
    }
    if (!strcmp(hf.links[i].name, "total_saved_grids")) {
      uint64_t at = 0;
      size_t sz = 0;
      uint8_t lay[18];
      if (!find_msg(&hf, hf.links[i].ohdr, kMsgLayout, &at, &sz) && sz >= 18 &&
          !f_read_at(hf.f, at, lay, sizeof lay) && lay[0] == 3 && lay[1] == 1) {
        tot_addr = get_le(lay + 2, 8);
        has_total = tot_addr + 4 <= hf.eof;
      }
    }
  }
  /* The reference deletes the group again when no grid was written. */
  if (ngrids == 0) {
    fclose(hf.f);
    h5_release(&hf);
    return GASP_OK;
  }
  const uint64_t N = (uint64_t)L * L, gbytes = 4 * N;
  const uint64_t data0 = hf.eof;
  const uint64_t data_len = pad8((size_t)(gbytes * (uint64_t)ngrids));
  /* 1. the grids' values, as given (int32, little-endian host) */
  if (f_write_at(hf.f, data0, ising_grids, (size_t)(gbytes * (uint64_t)ngrids)) ||
      fwrite("\0\0\0\0\0\0\0", 1, data_len - gbytes * (uint64_t)ngrids, hf.f) !=
          data_len - gbytes * (uint64_t)ngrids)
    rc = GASP_ERR_IO;
  const uint64_t meta0 = data0 + data_len;
  buf_t b = {0};
  static const char *anames[4] = {"magnetisation", "lclus_size", "committor", "committor_error"};
  /* 2. global heap collections: the four strings of each grid, in order */
  const int nstr = 4 * ngrids;
  uint64_t *s_col = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)nstr);
  uint32_t *s_len = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)nstr);
  link_t *gl = (link_t *)calloc((size_t)ngrids, sizeof(link_t));
  if (!s_col || !s_len || !gl) rc = rc ? rc : GASP_ERR_ALLOC;
  for (int s0 = 0; s0 < nstr && !rc; s0 += kGcolMaxObjs) {
    const int s1 = s0 + kGcolMaxObjs < nstr ? s0 + kGcolMaxObjs : nstr;
    const size_t start = b.n;
    const uint64_t col = meta0 + start;
    b_put(&b, "GCOL", 4);
    b_u8(&b, 1);
    b_zero(&b, 3);
    b_u64(&b, 0); /* collection size, set below */
    for (int s = s0; s < s1; ++s) {
      char tmp[64];
      const int g = s / 4, k = s % 4;
      const char *v = k == 0   ? attr_value(magnetisation, g, tmp, sizeof tmp)
                      : k == 1 ? attr_value(lclus_size, g, tmp, sizeof tmp)
                               : "null";
      const size_t len = strlen(v);
      b_u16(&b, (uint64_t)(s - s0 + 1)); /* object index */
      b_u16(&b, 0);                      /* reference count */
      b_u32(&b, 0);
      b_u64(&b, len);
      b_put(&b, v, len); /* stored without the terminating null */
      b_pad8(&b);
      s_col[s] = col;
      s_len[s] = (uint32_t)len;
    }
    /* free space (object 0) to the minimum collection size of 4096 bytes */
    size_t used = b.n - start;
    size_t total = used + 16 < 4096 ? 4096 : used + 16;
    b_u16(&b, 0);
    b_u16(&b, 0);
    b_u32(&b, 0);
    b_u64(&b, total - used);
    b_zero(&b, total - used - 16);
    if (!b.oom) set_le(b.p + start + 8, total, 8);
  }
  /* 3. the datasets' object headers */
  const uint64_t dims[2] = {(uint64_t)L, (uint64_t)L};
  char dname[32];
  for (int g = 0; g < ngrids && !rc; ++g) {
    const uint64_t oh = meta0 + b.n;
    ohdr_t o;
    dataset_ohdr(&b, 2, dims, 0, data0 + (uint64_t)g * gbytes, gbytes, &o);
    for (int k = 0; k < 4; ++k)
      msg_attr_str(&b, &o, anames[k], s_col[4 * g + k], (uint32_t)((4 * g + k) % kGcolMaxObjs + 1),
                   s_len[4 * g + k]);
    oh_end(&b, &o);
    snprintf(dname, sizeof dname, "grid_%d", g);
    gl[g].name = strdup(dname);
    gl[g].ohdr = oh;
    if (!gl[g].name) rc = GASP_ERR_ALLOC;
  }
  /* 4. the group: its index (names sorted), then its object header */
  uint64_t gbt = 0, ghp = 0, goh = 0;
  if (!rc) {
    qsort(gl, (size_t)ngrids, sizeof(link_t), link_cmp);
    rc = group_index(&b, meta0, gl, ngrids, &gbt, &ghp);
  }
  if (!rc) {
    goh = meta0 + b.n;
    ohdr_t o = oh_begin(&b);
    msg_symtab(&b, &o, gbt, ghp);
    oh_end(&b, &o);
    if (b.oom) rc = GASP_ERR_ALLOC;
  }
  if (!rc && f_write_at(hf.f, meta0, b.p, b.n)) rc = GASP_ERR_IO;
  if (!rc) {
    hf.eof = meta0 + b.n;
    rc = add_link(&hf, gname, goh, 1, gbt, ghp);
  }
  /* 5. root index, superblock; 6. total_saved_grids */
  if (!rc) rc = h5_commit_root(&hf);
  if (!rc && has_total) {
    uint8_t t[4];
    if (f_read_at(hf.f, tot_addr, t, 4)) {
      rc = GASP_ERR_IO;
    } else {
      set_le(t, (uint64_t)(uint32_t)((int32_t)get_le(t, 4) + ngrids), 4);
      if (f_write_at(hf.f, tot_addr, t, 4)) rc = GASP_ERR_IO;
    }
  }
  if (gl)
    for (int g = 0; g < ngrids; ++g) free(gl[g].name);
  free(gl);
  free(s_col);
  free(s_len);
  free(b.p);
  h5_release(&hf);
  if (fclose(hf.f) != 0 && !rc) rc = GASP_ERR_IO;
  if (rc) fprintf(stderr, "Error: failed to write HDF5 file '%s'\n", filename);
  return rc;
}
