/* Stand-in for the subset of the HDF5 C API that the reference transport,
 * grid and atomic-data code call. Test infrastructure for the oracle
 * harness: reads are served from an in-memory store that the harness fills
 * with synthetic inputs (atomic data, fuzz line lists, 3-D models); writes are
 * accepted and dropped. */
#ifndef ORACLE_SHIM_HDF5_H
#define ORACLE_SHIM_HDF5_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int64_t hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
typedef long long hssize_t;
typedef int H5T_class_t;
typedef int H5S_seloper_t;

typedef struct { unsigned long fileno[2]; unsigned long objno[2]; unsigned nlink; int type; long mtime; size_t linklen; } H5G_stat_t;

#define H5P_DEFAULT ((hid_t)0)
#define H5S_ALL ((hid_t)0)
#define H5F_ACC_RDONLY 0u
#define H5F_ACC_RDWR 1u
#define H5F_ACC_TRUNC 2u
#define H5S_SELECT_SET 0
#define H5T_OPAQUE 5
#define H5T_VARIABLE ((size_t)-1)

/* native type ids */
#define H5T_NATIVE_INT ((hid_t)101)
#define H5T_NATIVE_DOUBLE ((hid_t)102)
#define H5T_NATIVE_FLOAT ((hid_t)103)
#define H5T_C_S1 ((hid_t)104)
#define H5T_NATIVE_CHAR ((hid_t)105)
#define H5T_NATIVE_LONG ((hid_t)106)
#define H5T_NATIVE_ULONG ((hid_t)107)

hid_t H5Fopen(const char* name, unsigned flags, hid_t fapl);
hid_t H5Fcreate(const char* name, unsigned flags, hid_t fcpl, hid_t fapl);
herr_t H5Fclose(hid_t f);
hid_t H5Gopen1(hid_t loc, const char* name);
hid_t H5Gopen2(hid_t loc, const char* name, hid_t gapl);
#define H5Gopen H5Gopen2
hid_t H5Gcreate1(hid_t loc, const char* name, size_t hint);
herr_t H5Gclose(hid_t g);
herr_t H5Gget_objinfo(hid_t loc, const char* name, int follow, H5G_stat_t* st);
hid_t H5Dopen1(hid_t loc, const char* name);
hid_t H5Dcreate1(hid_t loc, const char* name, hid_t type, hid_t space, hid_t dcpl);
herr_t H5Dclose(hid_t d);
herr_t H5Dwrite(hid_t d, hid_t mtype, hid_t mspace, hid_t fspace, hid_t xfer, const void* buf);
herr_t H5Dread(hid_t d, hid_t mtype, hid_t mspace, hid_t fspace, hid_t xfer, void* buf);
hid_t H5Dget_space(hid_t d);
hid_t H5Screate_simple(int rank, const hsize_t* dims, const hsize_t* maxdims);
herr_t H5Sclose(hid_t s);
herr_t H5Sselect_hyperslab(hid_t s, H5S_seloper_t op, const hsize_t* start, const hsize_t* stride, const hsize_t* count, const hsize_t* block);
int H5Sget_simple_extent_dims(hid_t s, hsize_t* dims, hsize_t* maxdims);
hid_t H5Tcreate(int cls, size_t size);
hid_t H5Tcopy(hid_t t);
herr_t H5Tset_size(hid_t t, size_t size);
herr_t H5Eset_auto1(void* func, void* client);

#ifdef __cplusplus
}
#endif
#endif
