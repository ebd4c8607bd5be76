/* Stand-in for the HDF5 "lite" API (H5LT*) used by the reference; served by
 * the oracle harness's in-memory store. Test infrastructure only. */
#ifndef ORACLE_SHIM_HDF5_HL_H
#define ORACLE_SHIM_HDF5_HL_H

#include "hdf5.h"

#ifdef __cplusplus
extern "C" {
#endif

herr_t H5LTread_dataset_double(hid_t loc, const char* name, double* buf);
herr_t H5LTread_dataset_int(hid_t loc, const char* name, int* buf);
herr_t H5LTread_dataset_float(hid_t loc, const char* name, float* buf);
herr_t H5LTmake_dataset(hid_t loc, const char* name, int rank, const hsize_t* dims, hid_t type, const void* buf);
herr_t H5LTfind_dataset(hid_t loc, const char* name);
herr_t H5LTget_attribute_int(hid_t loc, const char* obj, const char* attr, int* out);
herr_t H5LTget_dataset_info(hid_t loc, const char* name, hsize_t* dims, H5T_class_t* cls, size_t* size);

/* Harness-side registration of the in-memory store (not part of HDF5). A
 * "file" is any path string; datasets and attributes are keyed by the path
 * the reference code asks for. */
void oracle_h5_clear(void);
void oracle_h5_put_double(const char* file, const char* path, const double* v, size_t n, int rank, const hsize_t* dims);
void oracle_h5_put_int(const char* file, const char* path, const int* v, size_t n, int rank, const hsize_t* dims);
void oracle_h5_put_attr_int(const char* file, const char* obj, const char* attr, int v);

#ifdef __cplusplus
}
#endif
#endif
