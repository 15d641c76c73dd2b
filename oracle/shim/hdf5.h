/*
 * Minimal stand-in for <hdf5.h>, used ONLY to compile the reference ipole
 * sources as a CPU oracle on a machine without libhdf5.
 *
 * The reference touches HDF5 through its own wrapper API (src/hdf5_utils.h);
 * that wrapper is re-implemented in ipgc_hdf5_utils.c over the IPGC keyed
 * container (format described there).  This header supplies the types and
 * type-id constants the reference passes through that API, plus the two raw
 * calls made outside it (src/io.c:546,552, the emission histogram writer,
 * which is disabled by src/par.c:217-220).
 *
 * Test infrastructure: never linked into the product library.
 */
#ifndef IPG_ORACLE_HDF5_STUB_H
#define IPG_ORACLE_HDF5_STUB_H

#include <stdint.h>

typedef int64_t hid_t;
typedef unsigned long long hsize_t;
typedef int herr_t;

/* Type ids understood by the container shim.  String types are created by
 * hdf5_make_str_type(len) and encoded as IPGC_STR_BASE + len. */
#define H5T_IEEE_F64LE ((hid_t)1)
#define H5T_NATIVE_DOUBLE ((hid_t)1)
#define H5T_STD_I32LE ((hid_t)2)
#define IPGC_STR_BASE ((hid_t)1000)

#define H5P_DEFAULT ((hid_t)0)
#define H5F_ACC_TRUNC 2u

hid_t H5Fcreate(const char *name, unsigned flags, hid_t fcpl, hid_t fapl);
herr_t H5Fclose(hid_t fid);

#endif
