/* IPGC keyed container: C reader/writer.  Layout (little endian):
 *   "IPGC0001", uint32 n, then n x {uint16 len, path, uint8 kind, uint8 rank,
 *   uint64 dims[rank], uint64 nbytes, data}. */
#include "ipgc.h"

#include "h5lite.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

void ipgc_free(ipgc_file *f)
{
  for (size_t i = 0; i < f->n; i++) {
    free(f->e[i].path);
    free(f->e[i].data);
  }
  free(f->e);
  f->e = NULL;
  f->n = f->cap = 0;
}

const ipgc_entry *ipgc_find(const ipgc_file *f, const char *path)
{
  for (size_t i = 0; i < f->n; i++)
    if (strcmp(f->e[i].path, path) == 0) return &f->e[i];
  return NULL;
}

static void ensure_parents(ipgc_file *f, const char *path)
{
  char buf[1024];
  snprintf(buf, sizeof(buf), "%s", path);
  char *at = strchr(buf, '@');
  if (at) *at = 0;
  for (char *p = buf + 1; *p; p++) {
    if (*p == '/') {
      *p = 0;
      if (!ipgc_find(f, buf)) ipgc_put(f, buf, IPGC_GROUP, 0, NULL, NULL, 0);
      *p = '/';
    }
  }
}

ipgc_entry *ipgc_put(ipgc_file *f, const char *path, int kind, int rank, const uint64_t *dims,
                     const void *data, uint64_t nbytes)
{
  ipgc_entry *e = (ipgc_entry *)ipgc_find(f, path);
  if (!e) {
    if (kind != IPGC_GROUP || strchr(path + 1, '/')) {
      /* parents first, so groups precede their members in the file */
      char tmp[1024];
      snprintf(tmp, sizeof(tmp), "%s", path);
      ensure_parents(f, tmp);
    }
    if (f->n == f->cap) {
      f->cap = f->cap ? 2 * f->cap : 64;
      f->e = (ipgc_entry *)realloc(f->e, f->cap * sizeof(ipgc_entry));
    }
    e = &f->e[f->n++];
    memset(e, 0, sizeof(*e));
    e->path = strdup(path);
  } else {
    free(e->data);
  }
  e->kind = kind;
  e->rank = rank;
  for (int i = 0; i < rank; i++) e->dims[i] = dims[i];
  e->nbytes = nbytes;
  e->data = nbytes ? (unsigned char *)malloc(nbytes) : NULL;
  if (nbytes && data) memcpy(e->data, data, nbytes);
  else if (nbytes) memset(e->data, 0, nbytes);
  return e;
}

int ipgc_read(const char *fname, ipgc_file *f)
{
  memset(f, 0, sizeof(*f));
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
    char path[1024];
    uint8_t kind, rank;
    uint64_t dims[IPGC_MAXRANK], nbytes;
    if (fread(&plen, 2, 1, fp) != 1 || plen >= sizeof(path) || fread(path, 1, plen, fp) != plen) goto bad;
    path[plen] = 0;
    if (fread(&kind, 1, 1, fp) != 1 || fread(&rank, 1, 1, fp) != 1 || rank > IPGC_MAXRANK) goto bad;
    if (rank && fread(dims, 8, rank, fp) != rank) goto bad;
    if (fread(&nbytes, 8, 1, fp) != 1) goto bad;
    if (f->n == f->cap) {
      f->cap = f->cap ? 2 * f->cap : 64;
      f->e = (ipgc_entry *)realloc(f->e, f->cap * sizeof(ipgc_entry));
    }
    ipgc_entry *e = &f->e[f->n++];
    memset(e, 0, sizeof(*e));
    e->path = strdup(path);
    e->kind = kind;
    e->rank = rank;
    for (int i = 0; i < rank; i++) e->dims[i] = dims[i];
    e->nbytes = nbytes;
    e->data = nbytes ? (unsigned char *)malloc(nbytes) : NULL;
    if (nbytes && fread(e->data, 1, nbytes, fp) != nbytes) goto bad;
  }
  fclose(fp);
  return 0;
bad:
  fclose(fp);
  ipgc_free(f);
  return -1;
}

int ipgc_write(const char *fname, const ipgc_file *f)
{
  FILE *fp = fopen(fname, "wb");
  if (!fp) return -1;
  uint32_t n = (uint32_t)f->n;
  int ok = fwrite("IPGC0001", 1, 8, fp) == 8 && fwrite(&n, 4, 1, fp) == 1;
  for (size_t k = 0; ok && k < f->n; k++) {
    const ipgc_entry *e = &f->e[k];
    uint16_t plen = (uint16_t)strlen(e->path);
    uint8_t kind = (uint8_t)e->kind, rank = (uint8_t)e->rank;
    ok = fwrite(&plen, 2, 1, fp) == 1 && fwrite(e->path, 1, plen, fp) == plen && fwrite(&kind, 1, 1, fp) == 1 &&
         fwrite(&rank, 1, 1, fp) == 1 && (!rank || fwrite(e->dims, 8, rank, fp) == rank) &&
         fwrite(&e->nbytes, 8, 1, fp) == 1 && (!e->nbytes || fwrite(e->data, 1, e->nbytes, fp) == e->nbytes);
  }
  if (fclose(fp) != 0) ok = 0;
  return ok ? 0 : -1;
}

int ipgc_get_f64(const ipgc_file *f, const char *path, double *v)
{
  const ipgc_entry *e = ipgc_find(f, path);
  if (!e) return -1;
  if (e->kind == IPGC_F64 && e->nbytes >= 8) memcpy(v, e->data, 8);
  else if (e->kind == IPGC_I32 && e->nbytes >= 4) { int32_t t; memcpy(&t, e->data, 4); *v = t; }
  else return -1;
  return 0;
}

int ipgc_get_i32(const ipgc_file *f, const char *path, int *v)
{
  const ipgc_entry *e = ipgc_find(f, path);
  if (!e) return -1;
  if (e->kind == IPGC_I32 && e->nbytes >= 4) { int32_t t; memcpy(&t, e->data, 4); *v = t; }
  else if (e->kind == IPGC_F64 && e->nbytes >= 8) { double t; memcpy(&t, e->data, 8); *v = (int)t; }
  else return -1;
  return 0;
}

int ipgc_get_str(const ipgc_file *f, const char *path, char *buf, size_t len)
{
  const ipgc_entry *e = ipgc_find(f, path);
  if (!e || e->kind != IPGC_STR || len == 0) return -1;
  size_t n = e->nbytes < len - 1 ? e->nbytes : len - 1;
  memcpy(buf, e->data, n);
  buf[n] = 0;
  return 0;
}

void ipgc_put_f64(ipgc_file *f, const char *path, double v) { ipgc_put(f, path, IPGC_F64, 0, NULL, &v, 8); }
void ipgc_put_i32(ipgc_file *f, const char *path, int v)
{
  int32_t t = v;
  ipgc_put(f, path, IPGC_I32, 0, NULL, &t, 4);
}
void ipgc_put_str(ipgc_file *f, const char *path, const char *s, size_t fixed_len)
{
  char *buf = (char *)calloc(fixed_len + 1, 1);
  strncpy(buf, s, fixed_len);
  ipgc_put(f, path, IPGC_STR, 0, NULL, buf, fixed_len);
  free(buf);
}
void ipgc_put_group(ipgc_file *f, const char *path)
{
  if (!ipgc_find(f, path)) ipgc_put(f, path, IPGC_GROUP, 0, NULL, NULL, 0);
}
void ipgc_put_array_f64(ipgc_file *f, const char *path, int rank, const uint64_t *dims, const double *data)
{
  uint64_t n = 1;
  for (int i = 0; i < rank; i++) n *= dims[i];
  ipgc_put(f, path, IPGC_F64, rank, dims, data, n * 8);
}

void ipgc_copy_subtree(const ipgc_file *src, const char *src_root, ipgc_file *dst, const char *dst_root)
{
  size_t rl = strlen(src_root);
  char q[2048];
  for (size_t i = 0; i < src->n; i++) {
    const ipgc_entry *e = &src->e[i];
    if (strncmp(e->path, src_root, rl) == 0 && (e->path[rl] == 0 || e->path[rl] == '/' || e->path[rl] == '@')) {
      snprintf(q, sizeof(q), "%s%s", dst_root, e->path + rl);
      ipgc_put(dst, q, e->kind, e->rank, e->dims, e->data, e->nbytes);
    }
  }
}

static char g_last[320];
const char *ipgc_error(void) { return g_last; }

int ipgc_load(const char *fname, ipgc_file *f)
{
  g_last[0] = 0;
  if (h5l_is_hdf5(fname)) {
    int rc = h5l_read(fname, f);
    if (rc) snprintf(g_last, sizeof(g_last), "%s: %s", fname, h5l_error());
    return rc;
  }
  int rc = ipgc_read(fname, f);
  if (rc) snprintf(g_last, sizeof(g_last), "%s: cannot open, or neither HDF5 nor an IPGC container", fname);
  return rc;
}

int ipgc_save(const char *fname, const ipgc_file *f)
{
  g_last[0] = 0;
  size_t n = strlen(fname);
  int rc;
  if (n >= 5 && strcmp(fname + n - 5, ".ipgc") == 0) {
    rc = ipgc_write(fname, f);
    if (rc) snprintf(g_last, sizeof(g_last), "%s: write error", fname);
  } else {
    rc = h5l_write(fname, f);
    if (rc) snprintf(g_last, sizeof(g_last), "%s: %s", fname, h5l_error());
  }
  return rc;
}
