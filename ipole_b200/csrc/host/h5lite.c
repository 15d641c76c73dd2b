/* HDF5 subset reader/writer; see h5lite.h for the scope.  Structure names and
 * field orders follow the HDF5 File Format Specification (version 3); section
 * numbers below refer to it. */
#define _POSIX_C_SOURCE 200809L
#include "h5lite.h"

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

#define UNDEF 0xffffffffffffffffULL

static char g_err[256];
const char *h5l_error(void) { return g_err; }

static int fail(int code, const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

static const unsigned char SIG[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

/* the signature sits at offset 0, 512, 1024, 2048, ... (after a user block) */
int h5l_is_hdf5(const char *fname)
{
  FILE *fp = fopen(fname, "rb");
  if (!fp) return 0;
  unsigned char b[8];
  int ok = 0;
  for (long o = 0; o <= (1L << 30) && !ok; o = o ? 2 * o : 512) {
    if (fseek(fp, o, SEEK_SET) != 0 || fread(b, 1, 8, fp) != 8) break;
    ok = memcmp(b, SIG, 8) == 0;
  }
  fclose(fp);
  return ok;
}

/* ===================================================================== */
/* reader                                                                 */
/* ===================================================================== */
typedef struct {
  const uint8_t *b;
  uint64_t n;
  int so, sl; /* size of offsets, size of lengths */
} H5F;

static uint64_t rdn(const uint8_t *p, int nb)
{
  uint64_t v = 0;
  for (int i = nb - 1; i >= 0; i--) v = (v << 8) | p[i];
  return v;
}

static int inside(const H5F *F, uint64_t off, uint64_t len) { return off <= F->n && len <= F->n - off; }

typedef struct {
  int type, flags;
  uint64_t size;
  const uint8_t *data;
} Msg;

typedef struct {
  Msg *m;
  int n, cap;
} MsgList;

static void msg_add(MsgList *L, int type, int flags, uint64_t size, const uint8_t *data)
{
  if (L->n == L->cap) {
    L->cap = L->cap ? 2 * L->cap : 16;
    L->m = (Msg *)realloc(L->m, L->cap * sizeof(Msg));
  }
  Msg *m = &L->m[L->n++];
  m->type = type;
  m->flags = flags;
  m->size = size;
  m->data = data;
}

/* object headers, sections IV.A.1.a (version 1) and IV.A.1.b (version 2),
 * with continuation messages (IV.A.2.q) */
static int read_ohdr(const H5F *F, uint64_t addr, MsgList *L)
{
  memset(L, 0, sizeof(*L));
  if (!inside(F, addr, 16)) return fail(-1, "object header address out of range");
  const uint8_t *p = F->b + addr;
  uint64_t blocks[64][2];
  int nblk = 0;
  if (memcmp(p, "OHDR", 4) == 0) {
    int flags = p[5];
    uint64_t off = addr + 6;
    if (flags & 0x20) off += 16;
    if (flags & 0x10) off += 4;
    int csz = 1 << (flags & 3);
    if (!inside(F, off, csz)) return fail(-1, "truncated object header");
    uint64_t size0 = rdn(F->b + off, csz);
    off += csz;
    blocks[nblk][0] = off;
    blocks[nblk][1] = size0;
    nblk++;
    for (int k = 0; k < nblk; k++) {
      uint64_t o = blocks[k][0], end = blocks[k][0] + blocks[k][1];
      if (k > 0) {
        if (!inside(F, o, 4) || memcmp(F->b + o, "OCHK", 4) != 0) return fail(-1, "bad continuation block");
        o += 4;
        end -= 4; /* checksum */
      }
      if (!inside(F, o, end - o)) return fail(-1, "truncated object header");
      while (o + 4 <= end) {
        int type = F->b[o];
        uint64_t size = rdn(F->b + o + 1, 2);
        int mflags = F->b[o + 3];
        o += 4;
        if (flags & 0x04) o += 2;
        if (o + size > end) break;
        if (type == 0x10) {
          if (nblk == 64) return fail(-2, "too many object header continuation blocks");
          blocks[nblk][0] = rdn(F->b + o, F->so);
          blocks[nblk][1] = rdn(F->b + o + F->so, F->sl);
          nblk++;
        } else if (type != 0) {
          msg_add(L, type, mflags, size, F->b + o);
        }
        o += size;
      }
    }
    return 0;
  }
  if (p[0] != 1) return fail(-2, "object header version %d", p[0]);
  uint64_t hsize = rdn(p + 8, 4);
  blocks[nblk][0] = addr + 16;
  blocks[nblk][1] = hsize;
  nblk++;
  for (int k = 0; k < nblk; k++) {
    uint64_t o = blocks[k][0], end = blocks[k][0] + blocks[k][1];
    if (!inside(F, o, end - o)) return fail(-1, "truncated object header");
    while (o + 8 <= end) {
      int type = (int)rdn(F->b + o, 2);
      uint64_t size = rdn(F->b + o + 2, 2);
      int mflags = F->b[o + 4];
      o += 8;
      if (o + size > end) break;
      if (type == 0x10) {
        if (nblk == 64) return fail(-2, "too many object header continuation blocks");
        blocks[nblk][0] = rdn(F->b + o, F->so);
        blocks[nblk][1] = rdn(F->b + o + F->so, F->sl);
        nblk++;
      } else if (type != 0) {
        msg_add(L, type, mflags, size, F->b + o);
      }
      o += size;
    }
  }
  return 0;
}

static const Msg *find_msg(const MsgList *L, int type)
{
  for (int i = 0; i < L->n; i++)
    if (L->m[i].type == type) return &L->m[i];
  return NULL;
}

/* dataspace, IV.A.2.b */
typedef struct {
  int rank;
  uint64_t dims[IPGC_MAXRANK];
} Dspace;

static int parse_dspace(const H5F *F, const uint8_t *d, uint64_t size, Dspace *s)
{
  int ver = d[0];
  s->rank = d[1];
  if (s->rank > IPGC_MAXRANK) return fail(-2, "dataspace rank %d", s->rank);
  const uint8_t *q;
  if (ver == 1) {
    q = d + 8;
  } else if (ver == 2) {
    if (d[3] == 2) return fail(-2, "null dataspace");
    q = d + 4;
  } else {
    return fail(-2, "dataspace version %d", ver);
  }
  if ((uint64_t)(q - d) + (uint64_t)s->rank * F->sl > size) return fail(-1, "truncated dataspace");
  for (int i = 0; i < s->rank; i++) s->dims[i] = rdn(q + (size_t)i * F->sl, F->sl);
  return 0;
}

/* datatype, IV.A.2.d */
typedef struct {
  int cls, size, be, is_signed, vlen_str;
} Dtype;

static int parse_dtype(const uint8_t *d, uint64_t size, Dtype *t)
{
  if (size < 8) return fail(-1, "truncated datatype");
  memset(t, 0, sizeof(*t));
  t->cls = d[0] & 0x0f;
  unsigned bf = d[1] | (d[2] << 8) | (d[3] << 16);
  t->size = (int)rdn(d + 4, 4);
  switch (t->cls) {
    case 0: /* fixed point */
      t->be = bf & 1;
      t->is_signed = (bf >> 3) & 1;
      if (t->size != 1 && t->size != 2 && t->size != 4 && t->size != 8) return fail(-2, "integer size %d", t->size);
      return 0;
    case 1: /* floating point */
      t->be = bf & 1;
      if (t->size != 4 && t->size != 8) return fail(-2, "float size %d", t->size);
      return 0;
    case 3: /* fixed-length string */
      return 0;
    case 8: { /* enumeration: read as its integer base type */
      int rc = parse_dtype(d + 8, size - 8, t);
      if (rc) return rc;
      if (t->cls != 0) return fail(-2, "enumeration over datatype class %d", t->cls);
      return 0;
    }
    case 9: /* variable length */
      if ((bf & 0xf) != 1) return fail(-2, "variable-length sequence");
      t->vlen_str = 1;
      return 0;
  }
  return fail(-2, "datatype class %d", t->cls);
}

/* global heap object (for variable-length strings), III.E */
static int gheap_obj(const H5F *F, uint64_t addr, uint32_t index, const uint8_t **data, uint64_t *len)
{
  if (!inside(F, addr, 16) || memcmp(F->b + addr, "GCOL", 4) != 0) return fail(-1, "bad global heap");
  uint64_t csize = rdn(F->b + addr + 8, F->sl);
  uint64_t o = addr + 8 + F->sl, end = addr + csize;
  if (!inside(F, addr, csize)) return fail(-1, "truncated global heap");
  while (o + 8 + F->sl <= end) {
    uint32_t idx = (uint32_t)rdn(F->b + o, 2);
    uint64_t osz = rdn(F->b + o + 8, F->sl);
    const uint8_t *od = F->b + o + 8 + F->sl;
    if (idx == index) {
      *data = od;
      *len = osz;
      return 0;
    }
    if (idx == 0) break;
    o += 8 + F->sl + ((osz + 7) & ~7ULL);
  }
  return fail(-1, "global heap object %u not found", index);
}

/* raw data in file order -> ipgc entry (floats to doubles, integers to
 * 32-bit ints when they fit, else doubles; strings as bytes) */
static int put_data(const H5F *F, ipgc_file *f, const char *path, const Dspace *s, const Dtype *t,
                    const uint8_t *raw, uint64_t rawlen)
{
  uint64_t n = 1;
  for (int i = 0; i < s->rank; i++) n *= s->dims[i];
  if (t->vlen_str) {
    if (n != 1) return fail(-2, "%s: arrays of variable-length strings", path);
    if (rawlen < 4 + (uint64_t)F->so + 4) return fail(-1, "%s: truncated string", path);
    const uint8_t *sd = NULL;
    uint64_t slen = 0;
    uint64_t gaddr = rdn(raw + 4, F->so);
    uint32_t gidx = (uint32_t)rdn(raw + 4 + F->so, 4);
    int rc = gheap_obj(F, gaddr, gidx, &sd, &slen);
    if (rc) return rc;
    ipgc_put(f, path, IPGC_STR, 0, NULL, sd, slen);
    return 0;
  }
  if (rawlen < n * (uint64_t)t->size) return fail(-1, "%s: %llu bytes of data for %llu elements", path,
                                                 (unsigned long long)rawlen, (unsigned long long)n);
  if (t->cls == 3) {
    ipgc_put(f, path, IPGC_STR, s->rank, s->dims, raw, n * (uint64_t)t->size);
    return 0;
  }
  unsigned char el[8];
  if (t->cls == 1) {
    double *v = (double *)malloc((n ? n : 1) * sizeof(double));
    for (uint64_t k = 0; k < n; k++) {
      const uint8_t *e = raw + k * t->size;
      for (int b = 0; b < t->size; b++) el[b] = t->be ? e[t->size - 1 - b] : e[b];
      if (t->size == 8) {
        memcpy(&v[k], el, 8);
      } else {
        float x;
        memcpy(&x, el, 4);
        v[k] = x;
      }
    }
    ipgc_put(f, path, IPGC_F64, s->rank, s->dims, v, n * sizeof(double));
    free(v);
    return 0;
  }
  /* integers */
  int64_t *iv = (int64_t *)malloc((n ? n : 1) * sizeof(int64_t));
  int fits = 1;
  for (uint64_t k = 0; k < n; k++) {
    const uint8_t *e = raw + k * t->size;
    for (int b = 0; b < t->size; b++) el[b] = t->be ? e[t->size - 1 - b] : e[b];
    uint64_t u = rdn(el, t->size);
    int64_t x;
    if (t->is_signed && t->size < 8 && (u >> (8 * t->size - 1)) & 1) u |= ~0ULL << (8 * t->size);
    x = (int64_t)u;
    if (!t->is_signed && t->size == 8 && (u >> 63)) fits = 0;
    iv[k] = x;
    if (x < INT32_MIN || x > INT32_MAX) fits = 0;
  }
  if (fits) {
    int32_t *v = (int32_t *)malloc((n ? n : 1) * sizeof(int32_t));
    for (uint64_t k = 0; k < n; k++) v[k] = (int32_t)iv[k];
    ipgc_put(f, path, IPGC_I32, s->rank, s->dims, v, n * sizeof(int32_t));
    free(v);
  } else {
    double *v = (double *)malloc((n ? n : 1) * sizeof(double));
    for (uint64_t k = 0; k < n; k++) v[k] = (double)iv[k];
    ipgc_put(f, path, IPGC_F64, s->rank, s->dims, v, n * sizeof(double));
    free(v);
  }
  free(iv);
  return 0;
}

/* filter pipeline, IV.A.2.l: deflate (1) and shuffle (2) */
typedef struct {
  int n;
  int id[8];
} Filters;

static int parse_filters(const uint8_t *d, uint64_t size, Filters *fl)
{
  fl->n = 0;
  int ver = d[0], nf = d[1];
  uint64_t o = (ver == 1) ? 8 : 2;
  for (int i = 0; i < nf; i++) {
    if (o + 2 > size) return fail(-1, "truncated filter pipeline");
    int id = (int)rdn(d + o, 2);
    int namelen = 0;
    if (ver == 1 || id >= 256) {
      namelen = (int)rdn(d + o + 2, 2);
      o += 2;
    }
    int nv = (int)rdn(d + o + 4, 2);
    o += 6;
    if (ver == 1) {
      o += (namelen + 7) & ~7;
      o += 4 * (uint64_t)nv + ((ver == 1 && (nv & 1)) ? 4 : 0);
    } else {
      o += namelen + 4 * (uint64_t)nv;
    }
    if (id != 1 && id != 2) return fail(-2, "filter %d (only deflate and shuffle are read)", id);
    if (fl->n == 8) return fail(-2, "too many filters");
    fl->id[fl->n++] = id;
  }
  return 0;
}

/* undo the pipeline on one chunk; returns a malloc'd buffer of `want` bytes */
static int unfilter(const Filters *fl, const uint8_t *in, uint64_t inlen, uint32_t mask, int esize, uint64_t want,
                    uint8_t **out)
{
  uint8_t *cur = (uint8_t *)malloc(inlen ? inlen : 1);
  memcpy(cur, in, inlen);
  uint64_t curlen = inlen;
  for (int i = fl->n - 1; i >= 0; i--) {
    if (mask & (1u << i)) continue;
    if (fl->id[i] == 1) {
      uLongf dl = (uLongf)want;
      uint8_t *dst = (uint8_t *)malloc(want ? want : 1);
      if (uncompress(dst, &dl, cur, (uLong)curlen) != Z_OK) {
        free(dst);
        free(cur);
        return fail(-1, "deflate stream error");
      }
      free(cur);
      cur = dst;
      curlen = dl;
    } else { /* shuffle */
      uint8_t *dst = (uint8_t *)malloc(curlen ? curlen : 1);
      uint64_t ne = curlen / esize;
      for (uint64_t k = 0; k < ne; k++)
        for (int b = 0; b < esize; b++) dst[k * esize + b] = cur[b * ne + k];
      memcpy(dst + ne * esize, cur + ne * esize, curlen - ne * esize);
      free(cur);
      cur = dst;
    }
  }
  if (curlen < want) {
    free(cur);
    return fail(-1, "chunk shorter than its extent");
  }
  *out = cur;
  return 0;
}

typedef struct {
  const H5F *F;
  const Filters *fl;
  int rank;
  const uint64_t *dims;
  const uint64_t *cdims;
  int esize;
  uint8_t *dst;
} ChunkCtx;

/* chunk index, v1 B-tree of node type 1 (III.A.1) */
static int walk_chunks(const ChunkCtx *C, uint64_t addr, int depth)
{
  const H5F *F = C->F;
  if (depth > 64) return fail(-1, "chunk B-tree too deep");
  if (!inside(F, addr, 8 + 2 * (uint64_t)F->so) || memcmp(F->b + addr, "TREE", 4) != 0 || F->b[addr + 4] != 1)
    return fail(-1, "bad chunk B-tree node");
  int level = F->b[addr + 5], used = (int)rdn(F->b + addr + 6, 2);
  uint64_t keysz = 8 + 8 * (uint64_t)(C->rank + 1);
  uint64_t o = addr + 8 + 2 * (uint64_t)F->so;
  uint64_t csz = C->esize;
  for (int i = 0; i < C->rank; i++) csz *= C->cdims[i];
  for (int e = 0; e < used; e++) {
    const uint8_t *key = F->b + o;
    if (!inside(F, o, keysz + F->so)) return fail(-1, "truncated chunk B-tree");
    uint64_t child = rdn(F->b + o + keysz, F->so);
    if (level > 0) {
      int rc = walk_chunks(C, child, depth + 1);
      if (rc) return rc;
    } else {
      uint32_t nbytes = (uint32_t)rdn(key, 4), mask = (uint32_t)rdn(key + 4, 4);
      uint64_t off[IPGC_MAXRANK];
      for (int i = 0; i < C->rank; i++) off[i] = rdn(key + 8 + 8 * i, 8);
      if (!inside(F, child, nbytes)) return fail(-1, "chunk out of range");
      uint8_t *buf = NULL;
      int rc = unfilter(C->fl, F->b + child, nbytes, mask, C->esize, csz, &buf);
      if (rc) return rc;
      /* copy the part of the chunk inside the dataset */
      uint64_t idx[IPGC_MAXRANK] = {0};
      uint64_t nel = csz / C->esize;
      for (uint64_t k = 0; k < nel; k++) {
        int ok = 1;
        uint64_t lin = 0;
        for (int i = 0; i < C->rank; i++) {
          uint64_t g = off[i] + idx[i];
          if (g >= C->dims[i]) ok = 0;
          lin = lin * C->dims[i] + g;
        }
        if (ok) memcpy(C->dst + lin * C->esize, buf + k * C->esize, C->esize);
        for (int i = C->rank - 1; i >= 0; i--) {
          if (++idx[i] < C->cdims[i]) break;
          idx[i] = 0;
        }
      }
      free(buf);
    }
    o += keysz + F->so;
  }
  return 0;
}

/* the raw bytes of a dataset or attribute payload: contiguous, compact or chunked (IV.A.2.i) */
static int dataset_raw(const H5F *F, const MsgList *L, const Dspace *s, const Dtype *t, uint8_t **raw, uint64_t *len)
{
  const Msg *lm = find_msg(L, 0x08);
  if (!lm) return fail(-1, "dataset without layout");
  const uint8_t *d = lm->data;
  uint64_t n = 1;
  for (int i = 0; i < s->rank; i++) n *= s->dims[i];
  int esize = t->vlen_str ? 4 + F->so + 4 : t->size;
  uint64_t want = n * (uint64_t)esize;
  int ver = d[0];
  int cls;
  uint64_t addr = UNDEF, size = 0;
  const uint8_t *compact = NULL;
  uint64_t btree = UNDEF;
  uint64_t cdims[IPGC_MAXRANK];
  if (ver == 1 || ver == 2) {
    int r = d[1];
    cls = d[2];
    const uint8_t *q = d + 8;
    if (cls != 0) {
      addr = rdn(q, F->so);
      q += F->so;
    }
    if (cls == 2) {
      btree = addr;
      for (int i = 0; i < r - 1 && i < IPGC_MAXRANK; i++) cdims[i] = rdn(q + 4 * i, 4);
    } else if (cls == 1) {
      size = want;
    } else {
      q += 4 * r;
      size = rdn(q, 4);
      compact = q + 4;
    }
  } else if (ver == 3 || ver == 4) {
    cls = d[1];
    if (cls == 0) {
      size = rdn(d + 2, 2);
      compact = d + 4;
    } else if (cls == 1) {
      addr = rdn(d + 2, F->so);
      size = rdn(d + 2 + F->so, F->sl);
    } else if (cls == 2 && ver == 3) {
      int r = d[2];
      btree = rdn(d + 3, F->so);
      for (int i = 0; i < r - 1 && i < IPGC_MAXRANK; i++) cdims[i] = rdn(d + 3 + F->so + 4 * i, 4);
    } else {
      return fail(-2, "layout version %d class %d", ver, cls);
    }
  } else {
    return fail(-2, "layout version %d", ver);
  }
  *raw = (uint8_t *)calloc(want ? want : 1, 1);
  *len = want;
  if (compact) {
    memcpy(*raw, compact, size < want ? size : want);
    return 0;
  }
  if (cls == 1) {
    if (addr == UNDEF) return 0; /* never written: fill value (zero) */
    if (!inside(F, addr, want)) return fail(-1, "contiguous data out of range");
    memcpy(*raw, F->b + addr, want);
    return 0;
  }
  Filters fl = {0, {0}};
  const Msg *fm = find_msg(L, 0x0B);
  if (fm) {
    int rc = parse_filters(fm->data, fm->size, &fl);
    if (rc) return rc;
  }
  if (btree == UNDEF) return 0;
  ChunkCtx C = {F, &fl, s->rank, s->dims, cdims, esize, *raw};
  return walk_chunks(&C, btree, 0);
}

/* attribute message, IV.A.2.m */
static int read_attr(const H5F *F, ipgc_file *f, const char *objpath, const Msg *m)
{
  const uint8_t *d = m->data;
  int ver = d[0];
  uint64_t nsz = rdn(d + 2, 2), tsz = rdn(d + 4, 2), ssz = rdn(d + 6, 2);
  uint64_t o = (ver == 3) ? 9 : 8;
  const uint8_t *name = d + o;
  o += (ver == 1) ? ((nsz + 7) & ~7ULL) : nsz;
  const uint8_t *td = d + o;
  o += (ver == 1) ? ((tsz + 7) & ~7ULL) : tsz;
  const uint8_t *sd = d + o;
  o += (ver == 1) ? ((ssz + 7) & ~7ULL) : ssz;
  if (o > m->size) return fail(-1, "truncated attribute");
  Dtype t;
  Dspace s;
  int rc = parse_dtype(td, tsz, &t);
  if (!rc) rc = parse_dspace(F, sd, ssz, &s);
  if (rc == -2) return 0; /* a type or shape outside the subset: the attribute is skipped */
  if (rc) return rc;
  char path[1100];
  snprintf(path, sizeof(path), "%s@%.*s", objpath[0] ? objpath : "/", (int)strnlen((const char *)name, nsz),
           (const char *)name);
  return put_data(F, f, path, &s, &t, d + o, m->size - o);
}

static int visit(const H5F *F, ipgc_file *f, const char *path, uint64_t addr, int depth, uint64_t *seen, int *nseen);

static int visit_child(const H5F *F, ipgc_file *f, const char *path, const char *name, uint64_t addr, int depth,
                       uint64_t *seen, int *nseen)
{
  char cp[1024];
  snprintf(cp, sizeof(cp), "%s/%s", path, name);
  return visit(F, f, cp, addr, depth + 1, seen, nseen);
}

/* symbol-table group: v1 B-tree of node type 0 over symbol-table nodes (III.A.1, III.C, III.D) */
static int walk_group_btree(const H5F *F, ipgc_file *f, const char *path, uint64_t addr, const uint8_t *heap,
                            uint64_t heapsz, int depth, uint64_t *seen, int *nseen)
{
  if (depth > 64) return fail(-1, "group B-tree too deep");
  if (!inside(F, addr, 8 + 2 * (uint64_t)F->so) || memcmp(F->b + addr, "TREE", 4) != 0 || F->b[addr + 4] != 0)
    return fail(-1, "bad group B-tree node");
  int level = F->b[addr + 5], used = (int)rdn(F->b + addr + 6, 2);
  uint64_t o = addr + 8 + 2 * (uint64_t)F->so;
  for (int e = 0; e < used; e++) {
    uint64_t child = rdn(F->b + o + F->sl, F->so);
    o += F->sl + F->so;
    if (level > 0) {
      int rc = walk_group_btree(F, f, path, child, heap, heapsz, depth + 1, seen, nseen);
      if (rc) return rc;
      continue;
    }
    if (!inside(F, child, 8) || memcmp(F->b + child, "SNOD", 4) != 0) return fail(-1, "bad symbol-table node");
    int nsym = (int)rdn(F->b + child + 6, 2);
    uint64_t ent = child + 8, esz = 2 * (uint64_t)F->so + 8 + 16;
    for (int k = 0; k < nsym; k++, ent += esz) {
      if (!inside(F, ent, esz)) return fail(-1, "truncated symbol-table node");
      uint64_t noff = rdn(F->b + ent, F->so), oh = rdn(F->b + ent + F->so, F->so);
      if (noff >= heapsz) return fail(-1, "name offset outside the local heap");
      char name[512];
      snprintf(name, sizeof(name), "%.*s", (int)strnlen((const char *)heap + noff, heapsz - noff),
               (const char *)heap + noff);
      int rc = visit_child(F, f, path, name, oh, depth, seen, nseen);
      if (rc) return rc;
    }
  }
  return 0;
}

static int visit(const H5F *F, ipgc_file *f, const char *path, uint64_t addr, int depth, uint64_t *seen, int *nseen)
{
  if (depth > 64) return fail(-1, "object nesting too deep");
  for (int i = 0; i < *nseen; i++)
    if (seen[i] == addr) return 0; /* a second hard link to an object already read */
  if (*nseen < 4096) seen[(*nseen)++] = addr;
  MsgList L;
  int rc = read_ohdr(F, addr, &L);
  if (rc) return rc;
  const Msg *stab = find_msg(&L, 0x11), *lay = find_msg(&L, 0x08);
  int is_group = stab || find_msg(&L, 0x06) || find_msg(&L, 0x02);
  if (is_group) {
    if (path[0]) ipgc_put_group(f, path);
  } else if (lay) {
    const Msg *sm = find_msg(&L, 0x01), *tm = find_msg(&L, 0x03);
    if (!sm || !tm) {
      free(L.m);
      return fail(-1, "%s: dataset without dataspace or datatype", path);
    }
    Dspace s;
    Dtype t;
    rc = parse_dspace(F, sm->data, sm->size, &s);
    if (!rc) rc = parse_dtype(tm->data, tm->size, &t);
    if (!rc) {
      uint8_t *raw = NULL;
      uint64_t len = 0;
      rc = dataset_raw(F, &L, &s, &t, &raw, &len);
      if (!rc) rc = put_data(F, f, path, &s, &t, raw, len);
      free(raw);
    }
    /* a dataset whose type or shape is outside the subset is skipped; a
     * reader that needs it finds it missing */
    if (rc == -1) {
      free(L.m);
      return rc;
    }
    rc = 0;
  }
  for (int i = 0; i < L.n && !rc; i++)
    if (L.m[i].type == 0x0C) rc = read_attr(F, f, path, &L.m[i]);
  if (rc) {
    free(L.m);
    return rc;
  }
  if (stab) {
    uint64_t bt = rdn(stab->data, F->so), hp = rdn(stab->data + F->so, F->so);
    if (!inside(F, hp, 8 + 2 * (uint64_t)F->sl + F->so) || memcmp(F->b + hp, "HEAP", 4) != 0) {
      free(L.m);
      return fail(-1, "bad local heap");
    }
    uint64_t hsz = rdn(F->b + hp + 8, F->sl), hda = rdn(F->b + hp + 8 + 2 * F->sl, F->so);
    if (!inside(F, hda, hsz)) {
      free(L.m);
      return fail(-1, "local heap data out of range");
    }
    rc = walk_group_btree(F, f, path, bt, F->b + hda, hsz, depth, seen, nseen);
  } else {
    const Msg *li = find_msg(&L, 0x02);
    if (li) {
      int flags = li->data[1];
      uint64_t fheap = rdn(li->data + 2 + ((flags & 1) ? 8 : 0), F->so);
      if (fheap != UNDEF) {
        free(L.m);
        return fail(-2, "%s: dense group storage (fractal heap)", path[0] ? path : "/");
      }
    }
    for (int i = 0; i < L.n && !rc; i++) {
      if (L.m[i].type != 0x06) continue;
      /* link message, IV.A.2.g */
      const uint8_t *d = L.m[i].data;
      int flags = d[1];
      uint64_t o = 2;
      int ltype = 0;
      if (flags & 0x08) ltype = d[o++];
      if (flags & 0x04) o += 8;
      if (flags & 0x10) o++;
      int lsz = 1 << (flags & 3);
      uint64_t nlen = rdn(d + o, lsz);
      o += lsz;
      char name[512];
      snprintf(name, sizeof(name), "%.*s", (int)nlen, (const char *)d + o);
      o += nlen;
      if (ltype != 0) continue; /* soft and external links are not followed */
      rc = visit_child(F, f, path, name, rdn(d + o, F->so), depth, seen, nseen);
    }
  }
  free(L.m);
  return rc;
}

int h5l_read(const char *fname, ipgc_file *f)
{
  memset(f, 0, sizeof(*f));
  g_err[0] = 0;
  FILE *fp = fopen(fname, "rb");
  if (!fp) return fail(-1, "cannot open %s", fname);
  fseek(fp, 0, SEEK_END);
  long sz = ftell(fp);
  fseek(fp, 0, SEEK_SET);
  if (sz < 64) {
    fclose(fp);
    return fail(-1, "%s: too short for HDF5", fname);
  }
  uint8_t *buf = (uint8_t *)malloc((size_t)sz);
  if (fread(buf, 1, (size_t)sz, fp) != (size_t)sz) {
    fclose(fp);
    free(buf);
    return fail(-1, "%s: read error", fname);
  }
  fclose(fp);
  /* superblock (II.A): searched at 0, 512, 1024, ... */
  uint64_t sb = UNDEF;
  for (uint64_t o = 0; o + 8 <= (uint64_t)sz; o = o ? 2 * o : 512)
    if (memcmp(buf + o, SIG, 8) == 0) {
      sb = o;
      break;
    }
  if (sb == UNDEF) {
    free(buf);
    return fail(-1, "%s: no HDF5 signature", fname);
  }
  H5F F = {buf, (uint64_t)sz, 8, 8};
  const uint8_t *p = buf + sb;
  int ver = p[8];
  uint64_t root, base;
  if (ver == 0 || ver == 1) {
    F.so = p[13];
    F.sl = p[14];
    uint64_t o = sb + 24 + (ver == 1 ? 4 : 0);
    if (F.so != 4 && F.so != 8) goto badsizes;
    base = rdn(buf + o, F.so);
    o += 4 * (uint64_t)F.so; /* base, free space, end of file, driver info */
    if (o + 2 * (uint64_t)F.so > (uint64_t)sz) goto truncated;
    root = rdn(buf + o + F.so, F.so); /* root symbol-table entry: name offset, object header */
  } else if (ver == 2 || ver == 3) {
    F.so = p[9];
    F.sl = p[10];
    if (F.so != 4 && F.so != 8) goto badsizes;
    if (sb + 12 + 4 * (uint64_t)F.so > (uint64_t)sz) goto truncated;
    base = rdn(p + 12, F.so);
    root = rdn(p + 12 + 3 * (uint64_t)F.so, F.so);
  } else {
    free(buf);
    return fail(-2, "superblock version %d", ver);
  }
  if (F.sl != 4 && F.sl != 8) goto badsizes;
  /* addresses are relative to the base address (the superblock's offset
   * when the file has a user block) */
  if (base > (uint64_t)sz) goto truncated;
  F.b = buf + base;
  F.n = (uint64_t)sz - base;
  uint64_t *seen = (uint64_t *)malloc(4096 * sizeof(uint64_t));
  int nseen = 0;
  int rc = visit(&F, f, "", root, 0, seen, &nseen);
  free(seen);
  free(buf);
  if (rc) ipgc_free(f);
  return rc;
badsizes:
  free(buf);
  return fail(-2, "offset/length sizes %d/%d", F.so, F.sl);
truncated:
  free(buf);
  return fail(-1, "%s: truncated superblock", fname);
}

/* ===================================================================== */
/* writer                                                                 */
/* ===================================================================== */
typedef struct {
  uint8_t *b;
  uint64_t n, cap;
} Buf;

static uint64_t bpos(Buf *B) { return B->n; }
static void bgrow(Buf *B, uint64_t need)
{
  if (B->n + need <= B->cap) return;
  while (B->n + need > B->cap) B->cap = B->cap ? 2 * B->cap : 1 << 16;
  B->b = (uint8_t *)realloc(B->b, B->cap);
}
static void wbytes(Buf *B, const void *p, uint64_t n)
{
  bgrow(B, n);
  if (p)
    memcpy(B->b + B->n, p, n);
  else
    memset(B->b + B->n, 0, n);
  B->n += n;
}
/* v as nb little-endian bytes (zeros past the eighth) */
static void wn(Buf *B, uint64_t v, uint64_t nb)
{
  uint8_t t[8];
  uint64_t k = nb < 8 ? nb : 8;
  for (uint64_t i = 0; i < k; i++) t[i] = (uint8_t)(v >> (8 * i));
  wbytes(B, t, k);
  if (nb > 8) wbytes(B, NULL, nb - 8);
}
static void patch(Buf *B, uint64_t at, uint64_t v, int nb)
{
  for (int i = 0; i < nb; i++) B->b[at + i] = (uint8_t)(v >> (8 * i));
}
static void align8(Buf *B)
{
  while (B->n & 7) wn(B, 0, 1);
}

/* a node of the group tree being written */
typedef struct WNode {
  const char *name;      /* last path component */
  const ipgc_entry *ds;  /* dataset entry, or NULL for a group */
  const ipgc_entry **at; /* attributes */
  int nat;
  struct WNode **kid;
  int nkid;
  uint64_t oh, btree, heap; /* addresses once written */
} WNode;

static WNode *wnode_new(const char *name)
{
  WNode *w = (WNode *)calloc(1, sizeof(WNode));
  w->name = name;
  return w;
}

static WNode *wnode_child(WNode *g, const char *name, size_t len, int create)
{
  for (int i = 0; i < g->nkid; i++)
    if (strlen(g->kid[i]->name) == len && strncmp(g->kid[i]->name, name, len) == 0) return g->kid[i];
  if (!create) return NULL;
  char *nm = (char *)malloc(len + 1);
  memcpy(nm, name, len);
  nm[len] = 0;
  WNode *c = wnode_new(nm);
  g->kid = (WNode **)realloc(g->kid, (g->nkid + 1) * sizeof(WNode *));
  g->kid[g->nkid++] = c;
  return c;
}

static WNode *wnode_path(WNode *root, const char *path)
{
  WNode *g = root;
  const char *p = path;
  while (*p == '/') p++;
  while (*p) {
    const char *e = strchr(p, '/');
    size_t len = e ? (size_t)(e - p) : strlen(p);
    if (len) g = wnode_child(g, p, len, 1);
    if (!e) break;
    p = e + 1;
  }
  return g;
}

static void wnode_free(WNode *w, int top)
{
  for (int i = 0; i < w->nkid; i++) wnode_free(w->kid[i], 0);
  free(w->kid);
  free(w->at);
  if (!top) free((char *)w->name);
  free(w);
}

static int cmp_kid(const void *a, const void *b)
{
  return strcmp((*(const WNode *const *)a)->name, (*(const WNode *const *)b)->name);
}

/* datatype message bodies (IV.A.2.d) */
static uint64_t dtype_size(const ipgc_entry *e) { return e->kind == IPGC_F64 ? 20 : (e->kind == IPGC_I32 ? 12 : 8); }
static void w_dtype(Buf *B, const ipgc_entry *e)
{
  if (e->kind == IPGC_F64) {
    uint8_t h[8] = {0x11, 0x20, 0x3f, 0x00, 8, 0, 0, 0};
    wbytes(B, h, 8);
    wn(B, 0, 2);   /* bit offset */
    wn(B, 64, 2);  /* precision */
    wn(B, 52, 1);  /* exponent location */
    wn(B, 11, 1);  /* exponent size */
    wn(B, 0, 1);   /* mantissa location */
    wn(B, 52, 1);  /* mantissa size */
    wn(B, 1023, 4);
  } else if (e->kind == IPGC_I32) {
    uint8_t h[8] = {0x10, 0x08, 0x00, 0x00, 4, 0, 0, 0};
    wbytes(B, h, 8);
    wn(B, 0, 2);
    wn(B, 32, 2);
  } else { /* fixed-length, null-terminated ASCII string */
    uint64_t n = 1;
    for (int i = 0; i < e->rank; i++) n *= e->dims[i];
    uint64_t len = n ? e->nbytes / n : e->nbytes;
    if (len == 0) len = 1;
    uint8_t h[4] = {0x13, 0x00, 0x00, 0x00};
    wbytes(B, h, 4);
    wn(B, len, 4);
  }
}
/* dataspace version 1 (IV.A.2.b) */
static void w_dspace(Buf *B, const ipgc_entry *e)
{
  wn(B, 1, 1);
  wn(B, e->rank, 1);
  wn(B, 0, 1);
  wn(B, 0, 5);
  for (int i = 0; i < e->rank; i++) wn(B, e->dims[i], 8);
}
static void w_msg_head(Buf *B, int type, uint64_t size, int flags)
{
  wn(B, type, 2);
  wn(B, size, 2);
  wn(B, flags, 1);
  wn(B, 0, 3);
}
static uint64_t pad8(uint64_t n) { return (n + 7) & ~7ULL; }

/* string payload padded to the stored length (null-terminated type) */
static const void *payload(const ipgc_entry *e, uint64_t *n)
{
  *n = e->nbytes;
  return e->data;
}

/* attribute message version 1 (IV.A.2.m) */
static uint64_t attr_msg_size(const ipgc_entry *a, const char *name)
{
  uint64_t nsz = strlen(name) + 1;
  return 8 + pad8(nsz) + pad8(dtype_size(a)) + pad8(8 + 8 * (uint64_t)a->rank) + a->nbytes;
}
static void w_attr(Buf *B, const ipgc_entry *a, const char *name)
{
  uint64_t nsz = strlen(name) + 1, sz = attr_msg_size(a, name);
  w_msg_head(B, 0x0C, pad8(sz), 0);
  uint64_t start = bpos(B);
  wn(B, 1, 1);
  wn(B, 0, 1);
  wn(B, nsz, 2);
  wn(B, dtype_size(a), 2);
  wn(B, 8 + 8 * (uint64_t)a->rank, 2);
  wbytes(B, name, nsz);
  align8(B);
  w_dtype(B, a);
  align8(B);
  w_dspace(B, a);
  align8(B);
  uint64_t n;
  const void *d = payload(a, &n);
  wbytes(B, d, n);
  while (bpos(B) - start < pad8(sz)) wn(B, 0, 1);
}

/* object header version 1 (IV.A.1.a) with room for `body` bytes of messages */
static uint64_t w_ohdr_start(Buf *B, int nmsg, uint64_t body)
{
  align8(B);
  uint64_t at = bpos(B);
  wn(B, 1, 1);
  wn(B, 0, 1);
  wn(B, nmsg, 2);
  wn(B, 1, 4);
  wn(B, body, 4);
  wn(B, 0, 4);
  return at;
}

static void w_attrs(Buf *B, const WNode *w)
{
  for (int i = 0; i < w->nat; i++) {
    const char *nm = strchr(w->at[i]->path, '@') + 1;
    w_attr(B, w->at[i], nm);
  }
}
static uint64_t attrs_body(const WNode *w)
{
  uint64_t s = 0;
  for (int i = 0; i < w->nat; i++) s += 8 + pad8(attr_msg_size(w->at[i], strchr(w->at[i]->path, '@') + 1));
  return s;
}

static void w_dataset(Buf *B, WNode *w)
{
  const ipgc_entry *e = w->ds;
  uint64_t body = (8 + pad8(8 + 8 * (uint64_t)e->rank)) + (8 + pad8(dtype_size(e))) + (8 + 8) + (8 + 24) +
                  attrs_body(w);
  w->oh = w_ohdr_start(B, 4 + w->nat, body);
  w_msg_head(B, 0x01, pad8(8 + 8 * (uint64_t)e->rank), 0);
  w_dspace(B, e);
  align8(B);
  w_msg_head(B, 0x03, pad8(dtype_size(e)), 1); /* constant */
  w_dtype(B, e);
  align8(B);
  /* fill value version 2: allocation late, write on allocation, undefined */
  w_msg_head(B, 0x05, 8, 1);
  wn(B, 2, 1);
  wn(B, 2, 1);
  wn(B, 0, 1);
  wn(B, 0, 1);
  wn(B, 0, 4);
  /* layout version 3, contiguous */
  w_msg_head(B, 0x08, 24, 0);
  wn(B, 3, 1);
  wn(B, 1, 1);
  uint64_t addr_at = bpos(B);
  wn(B, UNDEF, 8);
  wn(B, e->nbytes, 8);
  wn(B, 0, 6);
  w_attrs(B, w);
  align8(B);
  if (e->nbytes) {
    uint64_t da = bpos(B);
    uint64_t n;
    const void *d = payload(e, &n);
    wbytes(B, d, n);
    align8(B);
    patch(B, addr_at, da, 8);
  }
}

#define LEAF_K_MIN 4
#define INTERNAL_K 16

static void w_group(Buf *B, WNode *w, int leafk)
{
  if (w->nkid > 1) qsort(w->kid, w->nkid, sizeof(WNode *), cmp_kid);
  /* object header: symbol-table message (IV.A.2.r) + attributes */
  w->oh = w_ohdr_start(B, 1 + w->nat, (8 + 16) + attrs_body(w));
  w_msg_head(B, 0x11, 16, 0);
  uint64_t stab_at = bpos(B);
  wn(B, UNDEF, 8);
  wn(B, UNDEF, 8);
  w_attrs(B, w);
  for (int i = 0; i < w->nkid; i++) {
    if (w->kid[i]->ds)
      w_dataset(B, w->kid[i]);
    else
      w_group(B, w->kid[i], leafk);
  }
  /* local heap (III.D): "" at 0, then the names, 8-byte aligned */
  uint64_t dsz = 8, *noff = (uint64_t *)malloc((w->nkid + 1) * sizeof(uint64_t));
  for (int i = 0; i < w->nkid; i++) {
    noff[i] = dsz;
    dsz += pad8(strlen(w->kid[i]->name) + 1);
  }
  align8(B);
  w->heap = bpos(B);
  wbytes(B, "HEAP", 4);
  wn(B, 0, 1);
  wn(B, 0, 3);
  wn(B, dsz, 8);
  wn(B, 1, 8); /* no free block */
  wn(B, w->heap + 32, 8);
  wn(B, 0, 8);
  for (int i = 0; i < w->nkid; i++) {
    uint64_t l = strlen(w->kid[i]->name) + 1;
    wbytes(B, w->kid[i]->name, l);
    wn(B, 0, pad8(l) - l);
  }
  /* symbol-table node (III.C) with 2K entries */
  uint64_t snod = bpos(B);
  wbytes(B, "SNOD", 4);
  wn(B, 1, 1);
  wn(B, 0, 1);
  wn(B, w->nkid, 2);
  for (int i = 0; i < 2 * leafk; i++) {
    if (i < w->nkid) {
      WNode *c = w->kid[i];
      wn(B, noff[i], 8);
      wn(B, c->oh, 8);
      if (c->ds) {
        wn(B, 0, 4);
        wn(B, 0, 4);
        wn(B, 0, 16);
      } else {
        wn(B, 1, 4);
        wn(B, 0, 4);
        wn(B, c->btree, 8);
        wn(B, c->heap, 8);
      }
    } else {
      wn(B, 0, 40);
    }
  }
  /* group B-tree (III.A.1): one leaf, key0 = "", key1 = the last name */
  w->btree = bpos(B);
  wbytes(B, "TREE", 4);
  wn(B, 0, 1);
  wn(B, 0, 1);
  wn(B, w->nkid ? 1 : 0, 2);
  wn(B, UNDEF, 8);
  wn(B, UNDEF, 8);
  wn(B, 0, 8);
  wn(B, w->nkid ? snod : 0, 8);
  wn(B, w->nkid ? noff[w->nkid - 1] : 0, 8);
  wn(B, 0, (2 * INTERNAL_K - 1) * 16);
  free(noff);
  patch(B, stab_at, w->btree, 8);
  patch(B, stab_at + 8, w->heap, 8);
}

static int max_kids(const WNode *w)
{
  int m = w->nkid;
  for (int i = 0; i < w->nkid; i++) {
    int k = max_kids(w->kid[i]);
    if (k > m) m = k;
  }
  return m;
}

int h5l_write(const char *fname, const ipgc_file *f)
{
  g_err[0] = 0;
  WNode *root = wnode_new("");
  for (size_t i = 0; i < f->n; i++) {
    const ipgc_entry *e = &f->e[i];
    const char *at = strchr(e->path, '@');
    if (at) {
      char obj[1024];
      snprintf(obj, sizeof(obj), "%.*s", (int)(at - e->path), e->path);
      WNode *w = wnode_path(root, obj);
      w->at = (const ipgc_entry **)realloc(w->at, (w->nat + 1) * sizeof(*w->at));
      w->at[w->nat++] = e;
    } else if (e->kind == IPGC_GROUP) {
      wnode_path(root, e->path);
    } else if (e->kind == IPGC_F64 || e->kind == IPGC_I32 || e->kind == IPGC_STR) {
      WNode *w = wnode_path(root, e->path);
      if (w == root || w->nkid) {
        wnode_free(root, 1);
        return fail(-1, "%s is both a group and a dataset", e->path);
      }
      w->ds = e;
    }
  }
  int leafk = (max_kids(root) + 1) / 2;
  if (leafk < LEAF_K_MIN) leafk = LEAF_K_MIN;
  if (leafk > 32767) {
    wnode_free(root, 1);
    return fail(-2, "group too large");
  }
  Buf B = {NULL, 0, 0};
  /* superblock version 0 (II.A); addresses patched at the end */
  wbytes(&B, SIG, 8);
  wn(&B, 0, 1); /* superblock version */
  wn(&B, 0, 1); /* free-space version */
  wn(&B, 0, 1); /* root group symbol-table entry version */
  wn(&B, 0, 1);
  wn(&B, 0, 1); /* shared header message format version */
  wn(&B, 8, 1); /* size of offsets */
  wn(&B, 8, 1); /* size of lengths */
  wn(&B, 0, 1);
  wn(&B, leafk, 2);
  wn(&B, INTERNAL_K, 2);
  wn(&B, 0, 4);     /* file consistency flags */
  wn(&B, 0, 8);     /* base address */
  wn(&B, UNDEF, 8); /* free-space info */
  uint64_t eof_at = bpos(&B);
  wn(&B, 0, 8);     /* end of file */
  wn(&B, UNDEF, 8); /* driver info */
  uint64_t ste = bpos(&B);
  wn(&B, 0, 40); /* root symbol-table entry */
  w_group(&B, root, leafk);
  patch(&B, eof_at, B.n, 8);
  patch(&B, ste, 0, 8);
  patch(&B, ste + 8, root->oh, 8);
  patch(&B, ste + 16, 1, 4);
  patch(&B, ste + 24, root->btree, 8);
  patch(&B, ste + 32, root->heap, 8);
  wnode_free(root, 1);
  FILE *fp = fopen(fname, "wb");
  int ok = fp && fwrite(B.b, 1, B.n, fp) == B.n;
  if (fp) ok = (fclose(fp) == 0) && ok;
  free(B.b);
  return ok ? 0 : fail(-1, "cannot write %s", fname);
}
