/*
 * hdf5.h -- the part of the HDF5 C API the reference program calls, implemented on the
 * project's HDF5-subset library (h5lite), used only to compile the reference as the test
 * oracle in oracle/_ref.  TEST INFRASTRUCTURE ONLY.
 */
#ifndef CSP_HDF5_SHIM_H
#define CSP_HDF5_SHIM_H

#include <stddef.h>
#include <stdint.h>

typedef int64_t hid_t;
typedef unsigned long long hsize_t;
typedef int herr_t;
typedef enum { H5T_NO_CLASS = -1, H5T_INTEGER = 0, H5T_FLOAT = 1, H5T_TIME = 2, H5T_STRING = 3 } H5T_class_t;
typedef enum { H5T_STR_NULLTERM = 0, H5T_STR_NULLPAD = 1, H5T_STR_SPACEPAD = 2 } H5T_str_t;
typedef enum { H5S_SELECT_SET = 0 } H5S_seloper_t;
typedef enum { H5S_SCALAR = 0, H5S_SIMPLE = 1 } H5S_class_t;
typedef enum { H5FD_MPIO_INDEPENDENT = 0, H5FD_MPIO_COLLECTIVE = 1 } H5FD_mpio_xfer_t;

#define H5P_DEFAULT ((hid_t)0)
#define H5S_ALL ((hid_t)0)
#define H5P_FILE_ACCESS ((hid_t)1)
#define H5P_DATASET_CREATE ((hid_t)2)
#define H5P_DATASET_XFER ((hid_t)3)
#define H5F_ACC_RDONLY 0u
#define H5F_ACC_RDWR 1u
#define H5F_ACC_TRUNC 2u

/* predefined types: 1000 + h5lite type code (never equal to an H5T_class_t value) */
#define H5T_STD_U8LE ((hid_t)1001)
#define H5T_STD_U16LE ((hid_t)1002)
#define H5T_STD_U32LE ((hid_t)1003)
#define H5T_STD_U64LE ((hid_t)1004)
#define H5T_STD_I8LE ((hid_t)1005)
#define H5T_STD_I16LE ((hid_t)1006)
#define H5T_STD_I32LE ((hid_t)1007)
#define H5T_STD_I64LE ((hid_t)1008)
#define H5T_IEEE_F32LE ((hid_t)1009)
#define H5T_IEEE_F64LE ((hid_t)1010)
#define H5T_C_S1 ((hid_t)1011)
#define H5T_NATIVE_DOUBLE H5T_IEEE_F64LE
#define H5T_NATIVE_FLOAT H5T_IEEE_F32LE
#define H5T_NATIVE_INT H5T_STD_I32LE

hid_t H5Pcreate(hid_t cls);
herr_t H5Pclose(hid_t p);
herr_t H5Pset_fapl_mpio(hid_t p, int comm, int info);
herr_t H5Pset_dxpl_mpio(hid_t p, H5FD_mpio_xfer_t mode);
herr_t H5Pset_chunk(hid_t p, int rank, const hsize_t* dims);

hid_t H5Fopen(const char* name, unsigned flags, hid_t fapl);
hid_t H5Fcreate(const char* name, unsigned flags, hid_t fcpl, hid_t fapl);
herr_t H5Fclose(hid_t f);

hid_t H5Gopen(hid_t loc, const char* name, hid_t gapl);
hid_t H5Gcreate(hid_t loc, const char* name, hid_t lcpl, hid_t gcpl, hid_t gapl);
herr_t H5Gclose(hid_t g);

hid_t H5Aopen_by_name(hid_t loc, const char* obj_name, const char* attr_name, hid_t aapl, hid_t lapl);
hid_t H5Acreate2(hid_t loc, const char* name, hid_t type, hid_t space, hid_t acpl, hid_t aapl);
hid_t H5Aget_type(hid_t a);
herr_t H5Aread(hid_t a, hid_t mem_type, void* buf);
herr_t H5Awrite(hid_t a, hid_t mem_type, const void* buf);
herr_t H5Aclose(hid_t a);

H5T_class_t H5Tget_class(hid_t t);
size_t H5Tget_size(hid_t t);
hid_t H5Tcopy(hid_t t);
herr_t H5Tset_strpad(hid_t t, H5T_str_t pad);
herr_t H5Tset_size(hid_t t, size_t size);
herr_t H5Tclose(hid_t t);

hid_t H5Screate(H5S_class_t cls);
hid_t H5Screate_simple(int rank, const hsize_t* dims, const hsize_t* maxdims);
int H5Sget_simple_extent_dims(hid_t s, hsize_t* dims, hsize_t* maxdims);
herr_t H5Sselect_hyperslab(hid_t s, H5S_seloper_t op, const hsize_t* start, const hsize_t* stride,
                           const hsize_t* count, const hsize_t* block);
herr_t H5Sclose(hid_t s);

hid_t H5Dopen(hid_t loc, const char* name, hid_t dapl);
hid_t H5Dcreate(hid_t loc, const char* name, hid_t type, hid_t space, hid_t lcpl, hid_t dcpl, hid_t dapl);
hid_t H5Dget_space(hid_t d);
herr_t H5Dread(hid_t d, hid_t mem_type, hid_t mem_space, hid_t file_space, hid_t xfer, void* buf);
herr_t H5Dwrite(hid_t d, hid_t mem_type, hid_t mem_space, hid_t file_space, hid_t xfer, const void* buf);
herr_t H5Dclose(hid_t d);

#endif
