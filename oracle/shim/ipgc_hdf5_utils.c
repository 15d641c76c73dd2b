/*
 * Re-implementation of the reference's HDF5 wrapper API (src/hdf5_utils.h,
 * implemented upstream in src/hdf5_utils.c:53-574 over libhdf5) on top of the
 * IPGC keyed container, so that the unmodified reference sources can be
 * compiled and run as the CPU oracle on a machine without libhdf5.
 * Test infrastructure only.
 *
 * IPGC container (little endian), shared with ipole_b200/ipgc.py and the
 * product's host reader (ipole_b200/csrc/host/ipgc.c):
 *   char   magic[8] = "IPGC0001"
 *   uint32 n_entries
 *   n_entries x {
 *     uint16 path_len; char path[path_len]      absolute path, e.g. "/header/n1"
 *     uint8  kind                                0 group, 1 f64, 2 i32, 3 fixed string
 *     uint8  rank
 *     uint64 dims[rank]
 *     uint64 nbytes; uint8 data[nbytes]
 *   }
 * Attributes are stored as entries named "<object path>@<attribute name>".
 * HDF5 groups map to kind-0 entries; datasets keep HDF5's C (row-major)
 * element order, so a hyperslab read/write has the HDF5 semantics.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "hdf5_utils.h"

#define IPGC_GROUP 0
#define IPGC_F64 1
#define IPGC_I32 2
#define IPGC_STR 3
#define MAXRANK 8

typedef struct {
  char *path;
  int kind;
  int rank;
  uint64_t dims[MAXRANK];
  uint64_t nbytes;
  unsigned char *data;
} entry_t;

typedef struct {
  entry_t *e;
  size_t n, cap;
} store_t;

static store_t g_file = {0};
static char g_fname[4096];
static int g_writing = 0;
static int g_open = 0;
static char g_cwd[1024] = "/";

/* blobs: deep copies of subtrees (hdf5_get_blob / hdf5_write_blob) */
typedef struct {
  store_t s;
  char root[512];
} blob_t;
static blob_t g_blobs[16];
static int g_nblobs = 0;

static void store_clear(store_t *s)
{
  for (size_t i = 0; i < s->n; i++) {
    free(s->e[i].path);
    free(s->e[i].data);
  }
  free(s->e);
  s->e = NULL;
  s->n = s->cap = 0;
}

static entry_t *store_find(store_t *s, const char *path)
{
  for (size_t i = 0; i < s->n; i++)
    if (strcmp(s->e[i].path, path) == 0) return &s->e[i];
  return NULL;
}

static entry_t *store_put(store_t *s, const char *path, int kind, int rank, const uint64_t *dims,
                          const void *data, uint64_t nbytes)
{
  entry_t *e = store_find(s, path);
  if (!e) {
    if (s->n == s->cap) {
      s->cap = s->cap ? 2 * s->cap : 64;
      s->e = realloc(s->e, s->cap * sizeof(entry_t));
    }
    e = &s->e[s->n++];
    memset(e, 0, sizeof(*e));
    e->path = strdup(path);
  } else {
    free(e->data);
  }
  e->kind = kind;
  e->rank = rank;
  for (int i = 0; i < rank; i++) e->dims[i] = dims[i];
  e->nbytes = nbytes;
  e->data = nbytes ? malloc(nbytes) : NULL;
  if (nbytes && data) memcpy(e->data, data, nbytes);
  else if (nbytes) memset(e->data, 0, nbytes);
  return e;
}

static void join_path(const char *name, char *out, size_t outlen)
{
  char tmp[2048];
  if (name[0] == '/') snprintf(tmp, sizeof(tmp), "%s", name);
  else snprintf(tmp, sizeof(tmp), "%s%s%s", g_cwd,
                (g_cwd[strlen(g_cwd) - 1] == '/') ? "" : "/", name);
  /* collapse duplicate slashes, strip a trailing slash (except root) */
  size_t j = 0;
  for (size_t i = 0; tmp[i] && j + 1 < outlen; i++) {
    if (tmp[i] == '/' && j > 0 && out[j - 1] == '/') continue;
    out[j++] = tmp[i];
  }
  out[j] = 0;
  if (j > 1 && out[j - 1] == '/') out[j - 1] = 0;
}

static int type_kind(hsize_t t, size_t *elsize)
{
  if ((hid_t)t == H5T_IEEE_F64LE) { *elsize = 8; return IPGC_F64; }
  if ((hid_t)t == H5T_STD_I32LE) { *elsize = 4; return IPGC_I32; }
  if ((hid_t)t >= IPGC_STR_BASE) { *elsize = (size_t)((hid_t)t - IPGC_STR_BASE); return IPGC_STR; }
  fprintf(stderr, "ipgc shim: unknown type id %lld\n", (long long)t);
  exit(-1);
}

static int read_file(const char *fname, store_t *s)
{
  FILE *fp = fopen(fname, "rb");
  if (!fp) return -1;
  char magic[8];
  uint32_t n;
  if (fread(magic, 1, 8, fp) != 8 || memcmp(magic, "IPGC0001", 8) != 0 || fread(&n, 4, 1, fp) != 1) {
    fclose(fp);
    return -1;
  }
  for (uint32_t k = 0; k < n; k++) {
    uint16_t plen;
    char path[4096];
    uint8_t kind, rank;
    uint64_t dims[MAXRANK], nbytes;
    if (fread(&plen, 2, 1, fp) != 1 || plen >= sizeof(path) || fread(path, 1, plen, fp) != plen) goto bad;
    path[plen] = 0;
    if (fread(&kind, 1, 1, fp) != 1 || fread(&rank, 1, 1, fp) != 1 || rank > MAXRANK) goto bad;
    if (rank && fread(dims, 8, rank, fp) != rank) goto bad;
    if (fread(&nbytes, 8, 1, fp) != 1) goto bad;
    entry_t *e = store_put(s, path, kind, rank, dims, NULL, nbytes);
    if (nbytes && fread(e->data, 1, nbytes, fp) != nbytes) goto bad;
  }
  fclose(fp);
  return 0;
bad:
  fclose(fp);
  return -1;
}

static int write_file(const char *fname, store_t *s)
{
  FILE *fp = fopen(fname, "wb");
  if (!fp) return -1;
  uint32_t n = (uint32_t)s->n;
  fwrite("IPGC0001", 1, 8, fp);
  fwrite(&n, 4, 1, fp);
  for (size_t k = 0; k < s->n; k++) {
    entry_t *e = &s->e[k];
    uint16_t plen = (uint16_t)strlen(e->path);
    uint8_t kind = (uint8_t)e->kind, rank = (uint8_t)e->rank;
    fwrite(&plen, 2, 1, fp);
    fwrite(e->path, 1, plen, fp);
    fwrite(&kind, 1, 1, fp);
    fwrite(&rank, 1, 1, fp);
    if (rank) fwrite(e->dims, 8, rank, fp);
    fwrite(&e->nbytes, 8, 1, fp);
    if (e->nbytes) fwrite(e->data, 1, e->nbytes, fp);
  }
  fclose(fp);
  return 0;
}

static void ensure_parents(const char *path)
{
  char buf[2048];
  snprintf(buf, sizeof(buf), "%s", path);
  for (char *p = buf + 1; *p; p++) {
    if (*p == '/') {
      *p = 0;
      if (!store_find(&g_file, buf)) store_put(&g_file, buf, IPGC_GROUP, 0, NULL, NULL, 0);
      *p = '/';
    }
  }
}

/* ---- file ---- */
int hdf5_create(const char *fname)
{
  store_clear(&g_file);
  snprintf(g_fname, sizeof(g_fname), "%s", fname);
  g_writing = 1;
  g_open = 1;
  strcpy(g_cwd, "/");
  return 0;
}

int hdf5_open(const char *fname)
{
  store_clear(&g_file);
  if (read_file(fname, &g_file) != 0) {
    fprintf(stderr, "ipgc shim: could not open %s\n", fname);
    return -1;
  }
  snprintf(g_fname, sizeof(g_fname), "%s", fname);
  g_writing = 0;
  g_open = 1;
  strcpy(g_cwd, "/");
  return 0;
}

int hdf5_append(const char *fname)
{
  if (hdf5_open(fname) != 0) return -1;
  g_writing = 1;
  return 0;
}

int hdf5_set_file(hid_t fid) { (void)fid; return 0; }

int hdf5_close()
{
  int ret = 0;
  if (g_open && g_writing) ret = write_file(g_fname, &g_file);
  store_clear(&g_file);
  g_open = 0;
  g_writing = 0;
  strcpy(g_cwd, "/");
  return ret;
}

/* ---- directories ---- */
int hdf5_make_directory(const char *name)
{
  char p[2048];
  join_path(name, p, sizeof(p));
  ensure_parents(p);
  if (!store_find(&g_file, p)) store_put(&g_file, p, IPGC_GROUP, 0, NULL, NULL, 0);
  return 0;
}

void hdf5_set_directory(const char *path)
{
  snprintf(g_cwd, sizeof(g_cwd), "%s", path);
}

/* ---- blobs ---- */
hdf5_blob hdf5_get_blob(const char *name)
{
  char p[2048];
  join_path(name, p, sizeof(p));
  if (g_nblobs >= 16) { fprintf(stderr, "ipgc shim: too many blobs\n"); exit(-1); }
  blob_t *b = &g_blobs[g_nblobs];
  memset(b, 0, sizeof(*b));
  snprintf(b->root, sizeof(b->root), "%s", p);
  size_t rl = strlen(p);
  for (size_t i = 0; i < g_file.n; i++) {
    entry_t *e = &g_file.e[i];
    if (strncmp(e->path, p, rl) == 0 && (e->path[rl] == 0 || e->path[rl] == '/' || e->path[rl] == '@'))
      store_put(&b->s, e->path + rl, e->kind, e->rank, e->dims, e->data, e->nbytes);
  }
  return (hdf5_blob)(g_nblobs++);
}

int hdf5_write_blob(hdf5_blob blob, const char *name)
{
  char p[2048], q[4096];
  join_path(name, p, sizeof(p));
  blob_t *b = &g_blobs[blob];
  ensure_parents(p);
  for (size_t i = 0; i < b->s.n; i++) {
    entry_t *e = &b->s.e[i];
    snprintf(q, sizeof(q), "%s%s", p, e->path);
    store_put(&g_file, q, e->kind, e->rank, e->dims, e->data, e->nbytes);
  }
  return 0;
}

int hdf5_close_blob(hdf5_blob blob)
{
  store_clear(&g_blobs[blob].s);
  return 0;
}

/* ---- hyperslab copy between a file dataset and a memory array ---- */
static void slab_copy(int to_file, unsigned char *fbuf, unsigned char *mbuf, size_t elsize, size_t rank,
                      const hsize_t *fdims, const hsize_t *fstart, const hsize_t *fcount,
                      const hsize_t *mdims, const hsize_t *mstart)
{
  hsize_t idx[MAXRANK] = {0};
  size_t total = 1;
  for (size_t d = 0; d < rank; d++) total *= fcount[d];
  for (size_t n = 0; n < total; n++) {
    size_t fo = 0, mo = 0;
    for (size_t d = 0; d < rank; d++) {
      fo = fo * fdims[d] + (fstart[d] + idx[d]);
      mo = mo * mdims[d] + (mstart[d] + idx[d]);
    }
    if (to_file) memcpy(fbuf + fo * elsize, mbuf + mo * elsize, elsize);
    else memcpy(mbuf + mo * elsize, fbuf + fo * elsize, elsize);
    for (int d = (int)rank - 1; d >= 0; d--) {
      if (++idx[d] < fcount[d]) break;
      idx[d] = 0;
    }
  }
}

/* ---- write ---- */
int hdf5_write_single_val(const void *val, const char *name, hsize_t hdf5_type)
{
  char p[2048];
  size_t es;
  int kind = type_kind(hdf5_type, &es);
  join_path(name, p, sizeof(p));
  ensure_parents(p);
  if (kind == IPGC_STR) {
    char *buf = calloc(es + 1, 1);
    strncpy(buf, (const char *)val, es);
    store_put(&g_file, p, kind, 0, NULL, buf, es);
    free(buf);
  } else {
    store_put(&g_file, p, kind, 0, NULL, val, es);
  }
  return 0;
}

int hdf5_write_full_array(const void *data, const char *name, size_t rank, hsize_t *dims, hsize_t hdf5_type)
{
  char p[2048];
  size_t es;
  int kind = type_kind(hdf5_type, &es);
  uint64_t d64[MAXRANK];
  size_t n = 1;
  for (size_t i = 0; i < rank; i++) { d64[i] = dims[i]; n *= dims[i]; }
  join_path(name, p, sizeof(p));
  ensure_parents(p);
  store_put(&g_file, p, kind, (int)rank, d64, data, n * es);
  return 0;
}

int hdf5_write_array(const void *data, const char *name, size_t rank,
                     hsize_t *fdims, hsize_t *fstart, hsize_t *fcount, hsize_t *mdims, hsize_t *mstart,
                     hsize_t hdf5_type)
{
  char p[2048];
  size_t es;
  int kind = type_kind(hdf5_type, &es);
  join_path(name, p, sizeof(p));
  ensure_parents(p);
  entry_t *e = store_find(&g_file, p);
  if (!e) {
    uint64_t d64[MAXRANK];
    size_t n = 1;
    for (size_t i = 0; i < rank; i++) { d64[i] = fdims[i]; n *= fdims[i]; }
    e = store_put(&g_file, p, kind, (int)rank, d64, NULL, n * es);
  }
  slab_copy(1, e->data, (unsigned char *)data, es, rank, fdims, fstart, fcount, mdims, mstart);
  return 0;
}

int hdf5_write_chunked_array(const void *data, const char *name, size_t rank,
                             hsize_t *fdims, hsize_t *fstart, hsize_t *fcount, hsize_t *mdims, hsize_t *mstart,
                             hsize_t *chunk_size, hsize_t hdf5_type)
{
  (void)chunk_size;
  return hdf5_write_array(data, name, rank, fdims, fstart, fcount, mdims, mstart, hdf5_type);
}

/* ---- read ---- */
int hdf5_exists(const char *name)
{
  char p[2048];
  join_path(name, p, sizeof(p));
  return store_find(&g_file, p) != NULL;
}

int hdf5_read_single_val(void *val, const char *name, hsize_t hdf5_type)
{
  char p[2048];
  size_t es;
  int kind = type_kind(hdf5_type, &es);
  join_path(name, p, sizeof(p));
  entry_t *e = store_find(&g_file, p);
  if (!e) {
    fprintf(stderr, "ipgc shim: dataset %s not found\n", p);
    return -1;
  }
  if (kind == IPGC_STR) {
    size_t n = e->nbytes < es ? e->nbytes : es;
    memset(val, 0, es);
    memcpy(val, e->data, n);
    ((char *)val)[es - 1] = 0;
    return 0;
  }
  if (e->kind == kind) {
    memcpy(val, e->data, es);
  } else if (kind == IPGC_F64 && e->kind == IPGC_I32) {
    *(double *)val = (double)*(int32_t *)e->data;
  } else if (kind == IPGC_I32 && e->kind == IPGC_F64) {
    *(int32_t *)val = (int32_t) * (double *)e->data;
  } else {
    fprintf(stderr, "ipgc shim: type mismatch reading %s\n", p);
    return -1;
  }
  return 0;
}

int hdf5_read_full_array(void *data, const char *name, size_t rank, hsize_t *dims, hsize_t hdf5_type)
{
  char p[2048];
  size_t es;
  (void)rank; (void)dims;
  type_kind(hdf5_type, &es);
  join_path(name, p, sizeof(p));
  entry_t *e = store_find(&g_file, p);
  if (!e) return -1;
  memcpy(data, e->data, e->nbytes);
  return 0;
}

int hdf5_read_array(void *data, const char *name, size_t rank, hsize_t *fdims, hsize_t *fstart, hsize_t *fcount,
                    hsize_t *mdims, hsize_t *mstart, hsize_t hdf5_type)
{
  char p[2048];
  size_t es;
  type_kind(hdf5_type, &es);
  join_path(name, p, sizeof(p));
  entry_t *e = store_find(&g_file, p);
  if (!e) {
    fprintf(stderr, "ipgc shim: dataset %s not found\n", p);
    return -1;
  }
  slab_copy(0, e->data, (unsigned char *)data, es, rank, fdims, fstart, fcount, mdims, mstart);
  return 0;
}

int hdf5_read_array_multidim(void *data, const char *name, size_t frank, hsize_t *fdims, hsize_t *fstart,
                             hsize_t *fcount, size_t mrank, hsize_t *mdims, hsize_t *mstart, hsize_t *mcount,
                             hsize_t hdf5_type)
{
  (void)data; (void)name; (void)frank; (void)fdims; (void)fstart; (void)fcount;
  (void)mrank; (void)mdims; (void)mstart; (void)mcount; (void)hdf5_type;
  fprintf(stderr, "ipgc shim: hdf5_read_array_multidim is not provided (KORAL/HAMR readers)\n");
  exit(-1);
}

int hdf5_attr_exists(const char *data_name, const char *att_name)
{
  char p[2048], q[4096];
  join_path(data_name, p, sizeof(p));
  snprintf(q, sizeof(q), "%s@%s", p, att_name);
  return store_find(&g_file, q) != NULL;
}

int hdf5_read_attr_num(void *data, const char *att_name, const char *data_name, hsize_t hdf5_type)
{
  char p[2048], q[4096];
  size_t es;
  type_kind(hdf5_type, &es);
  join_path(data_name, p, sizeof(p));
  snprintf(q, sizeof(q), "%s@%s", p, att_name);
  entry_t *e = store_find(&g_file, q);
  if (!e) return -1;
  memcpy(data, e->data, es);
  return 0;
}

int hdf5_read_attr_arr(void *data, const char *att_name, const char *data_name)
{
  char p[2048], q[4096];
  join_path(data_name, p, sizeof(p));
  snprintf(q, sizeof(q), "%s@%s", p, att_name);
  entry_t *e = store_find(&g_file, q);
  if (!e) return -1;
  memcpy(data, e->data, e->nbytes);
  return 0;
}

/* ---- convenience ---- */
hid_t hdf5_make_str_type(size_t len) { return IPGC_STR_BASE + (hid_t)len; }

int hdf5_write_str_list(const void *data, const char *name, size_t strlen_, size_t len)
{
  char p[2048];
  uint64_t d = len;
  join_path(name, p, sizeof(p));
  ensure_parents(p);
  store_put(&g_file, p, IPGC_STR, 1, &d, data, strlen_ * len);
  return 0;
}

int hdf5_add_attr(const void *att, const char *att_name, const char *data_name, hsize_t hdf5_type)
{
  char p[2048], q[4096];
  size_t es;
  int kind = type_kind(hdf5_type, &es);
  join_path(data_name, p, sizeof(p));
  snprintf(q, sizeof(q), "%s@%s", p, att_name);
  if (kind == IPGC_STR) {
    char *buf = calloc(es + 1, 1);
    strncpy(buf, (const char *)att, es);
    store_put(&g_file, q, kind, 0, NULL, buf, es);
    free(buf);
  } else {
    store_put(&g_file, q, kind, 0, NULL, att, es);
  }
  return 0;
}

int hdf5_add_units(const char *name, const char *unit)
{
  return hdf5_add_attr(unit, "units", name, hdf5_make_str_type(strlen(unit) + 1));
}

void h5io_add_data_dbl_3ds(hid_t fid, const char *path, hsize_t n1, hsize_t n2, hsize_t n3, double data[])
{
  (void)fid; (void)path; (void)n1; (void)n2; (void)n3; (void)data;
  fprintf(stderr, "ipgc shim: emission histogram output is not provided\n");
}

hid_t H5Fcreate(const char *name, unsigned flags, hid_t fcpl, hid_t fapl)
{
  (void)name; (void)flags; (void)fcpl; (void)fapl;
  return -1;
}

herr_t H5Fclose(hid_t fid)
{
  (void)fid;
  return 0;
}
