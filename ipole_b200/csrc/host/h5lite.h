/* HDF5 files for ipole's dumps and images, without libhdf5.
 *
 * The reference reads iharm dumps and writes images through the HDF5 library
 * (src/hdf5_utils.c, src/io.c:140-273, model/iharm/model.c:848-1074,1876-1949).
 * This module reads and writes the part of the HDF5 file format
 * (The HDF Group, "HDF5 File Format Specification", version 3) that those
 * files use, into and from the same in-memory entry list as the IPGC container
 * (ipgc_file: groups, datasets "/a/b", attributes "/a/b@name").
 *
 * Written files: superblock version 0, version 1 object headers, groups as
 * symbol tables (one v1 B-tree leaf and one symbol-table node per group, local
 * heap for the names), contiguous datasets of little-endian IEEE doubles,
 * 32-bit signed integers and fixed-length null-terminated strings, version 1
 * attributes.  This is the layout libhdf5 itself writes by default.
 *
 * Read files: superblock versions 0-3; version 1 and 2 object headers with
 * continuation blocks; symbol-table groups and compact link-message groups
 * (dense groups, i.e. fractal heaps, are refused); datasets with contiguous,
 * compact or chunked (version 1 B-tree index) storage, the chunks optionally
 * deflate- and shuffle-filtered; integer and floating-point data of either
 * byte order (floats become doubles, integers 32-bit ints), fixed-length and
 * variable-length strings; attributes on groups and datasets. */
#ifndef IPG_H5LITE_H
#define IPG_H5LITE_H
#include "ipgc.h"

/* 1 if the file starts with the HDF5 signature */
int h5l_is_hdf5(const char *fname);
/* 0 ok, -1 I/O or malformed file, -2 a feature outside the subset (h5l_error() says which) */
int h5l_read(const char *fname, ipgc_file *f);
int h5l_write(const char *fname, const ipgc_file *f);
const char *h5l_error(void);
#endif
