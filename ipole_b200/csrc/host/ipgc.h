/* IPGC keyed container: C reader/writer (layout in ipole_b200/ipgc.py).
 * Used for iharm dumps (input) and images (output). */
#ifndef IPG_IPGC_H
#define IPG_IPGC_H
#include <stddef.h>
#include <stdint.h>

#define IPGC_GROUP 0
#define IPGC_F64 1
#define IPGC_I32 2
#define IPGC_STR 3
#define IPGC_MAXRANK 8

typedef struct {
  char *path;
  int kind, rank;
  uint64_t dims[IPGC_MAXRANK];
  uint64_t nbytes;
  unsigned char *data;
} ipgc_entry;

typedef struct {
  ipgc_entry *e;
  size_t n, cap;
} ipgc_file;

int ipgc_read(const char *fname, ipgc_file *f);            /* 0 ok, -1 error */
int ipgc_write(const char *fname, const ipgc_file *f);     /* 0 ok, -1 error */
/* either format: HDF5 (read by h5lite) when the file carries the HDF5
 * signature, else IPGC.  0 ok, -1 error, -2 HDF5 feature outside the subset */
int ipgc_load(const char *fname, ipgc_file *f);
/* IPGC when the name ends in ".ipgc", HDF5 otherwise (the reference's image
 * and dump files are HDF5).  0 ok, -1 error */
int ipgc_save(const char *fname, const ipgc_file *f);
/* message for the last failed ipgc_load/ipgc_save */
const char *ipgc_error(void);
void ipgc_free(ipgc_file *f);
const ipgc_entry *ipgc_find(const ipgc_file *f, const char *path);
ipgc_entry *ipgc_put(ipgc_file *f, const char *path, int kind, int rank, const uint64_t *dims,
                     const void *data, uint64_t nbytes);
/* typed helpers; parents groups are created on put */
int ipgc_get_f64(const ipgc_file *f, const char *path, double *v);
int ipgc_get_i32(const ipgc_file *f, const char *path, int *v);
int ipgc_get_str(const ipgc_file *f, const char *path, char *buf, size_t len);
void ipgc_put_f64(ipgc_file *f, const char *path, double v);
void ipgc_put_i32(ipgc_file *f, const char *path, int v);
void ipgc_put_str(ipgc_file *f, const char *path, const char *s, size_t fixed_len);
void ipgc_put_group(ipgc_file *f, const char *path);
void ipgc_put_array_f64(ipgc_file *f, const char *path, int rank, const uint64_t *dims, const double *data);
/* copy every entry under `src_root` of `src` to `dst_root` of `dst` */
void ipgc_copy_subtree(const ipgc_file *src, const char *src_root, ipgc_file *dst, const char *dst_root);
#endif
