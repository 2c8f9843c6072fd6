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
#define H5F_ACC_RDONLY 0u
enum { H5S_SCALAR = 0, H5S_SELECT_SET = 0 };

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
#undef CS_H5_STANDIN
