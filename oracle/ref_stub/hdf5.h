/* TEST ORACLE ONLY.  A stand-in for <hdf5.h> so that the reference's
 * execution-bucketing builders (src/io/csh5/execution_builders_part.hh),
 * which sit in a header chain that also opens HDF5 files, compile without
 * the HDF5 library.  The bridge calls none of the file functions; every
 * stand-in below returns -1 (an HDF5 failure) if anything did. */
#pragma once

typedef long long hid_t;
typedef int herr_t;
typedef int htri_t;
typedef unsigned long long hsize_t;
typedef long long hssize_t;
typedef int H5T_class_t;
typedef struct {
    int type;
} H5L_info_t;

#define H5P_DEFAULT ((hid_t) 0)
#define H5S_ALL ((hid_t) 0)
#define H5T_NATIVE_UINT32 ((hid_t) 1)
#define H5T_NATIVE_UINT64 ((hid_t) 2)
#define H5T_NATIVE_UINT16 ((hid_t) 3)
#define H5T_NATIVE_FLOAT ((hid_t) 4)
#define H5T_NATIVE_UCHAR ((hid_t) 5)
#define H5T_NATIVE_DOUBLE ((hid_t) 6)
#define H5T_NATIVE_CHAR ((hid_t) 7)
#define H5T_C_S1 ((hid_t) 8)
#define H5T_NATIVE_LLONG ((hid_t) 9)
#define H5T_VARIABLE ((unsigned long) -1)
#define H5F_ACC_RDONLY 0u
#define H5E_BEGIN_TRY {
#define H5E_END_TRY }
enum { H5S_SCALAR = 0, H5S_SELECT_SET = 0 };
enum { H5T_INTEGER = 0, H5T_FLOAT = 1, H5T_STRING = 3 };
enum { H5T_SGN_2 = 1, H5T_CSET_ASCII = 0, H5T_CSET_UTF8 = 1 };
enum { H5_INDEX_NAME = 0, H5_ITER_NATIVE = 2 };

#define CS_H5_STANDIN(name)                  \
    template <class... A>                   \
    inline long long name(A...) {           \
        return -1;                          \
    }
CS_H5_STANDIN(H5Aclose)
CS_H5_STANDIN(H5Acreate2)
CS_H5_STANDIN(H5Aexists)
CS_H5_STANDIN(H5Aget_type)
CS_H5_STANDIN(H5Aopen)
CS_H5_STANDIN(H5Aread)
CS_H5_STANDIN(H5Awrite)
CS_H5_STANDIN(H5Dclose)
CS_H5_STANDIN(H5Dcreate2)
CS_H5_STANDIN(H5Dget_space)
CS_H5_STANDIN(H5Dopen2)
CS_H5_STANDIN(H5Dread)
CS_H5_STANDIN(H5Dwrite)
CS_H5_STANDIN(H5Fclose)
CS_H5_STANDIN(H5Fopen)
CS_H5_STANDIN(H5Gclose)
CS_H5_STANDIN(H5Gcreate2)
CS_H5_STANDIN(H5Gopen2)
CS_H5_STANDIN(H5Lexists)
CS_H5_STANDIN(H5Sclose)
CS_H5_STANDIN(H5Screate)
CS_H5_STANDIN(H5Screate_simple)
CS_H5_STANDIN(H5Sget_simple_extent_dims)
CS_H5_STANDIN(H5Sselect_hyperslab)
CS_H5_STANDIN(H5Tclose)
CS_H5_STANDIN(H5Tcopy)
CS_H5_STANDIN(H5Tget_size)
CS_H5_STANDIN(H5Tset_size)
CS_H5_STANDIN(H5Aget_space)
CS_H5_STANDIN(H5Dget_type)
CS_H5_STANDIN(H5Dvlen_reclaim)
CS_H5_STANDIN(H5Literate)
CS_H5_STANDIN(H5Sget_simple_extent_ndims)
CS_H5_STANDIN(H5Sget_simple_extent_npoints)
CS_H5_STANDIN(H5Tget_class)
CS_H5_STANDIN(H5Tget_cset)
CS_H5_STANDIN(H5Tget_sign)
CS_H5_STANDIN(H5Tis_variable_str)
CS_H5_STANDIN(H5Tset_cset)
#undef CS_H5_STANDIN
