/*
 * hdf5.h -- stand-in for the handful of HDF5 calls the reference's
 * FileManager makes (src/FileManager.cu:13-155), used only to build the
 * reference from its own sources into oracle/_ref/ (test infrastructure).
 *
 * A "file" here is a raw volume file as written by the oracle test helpers:
 * a 64-byte header ("VTVOL001", u32 version, u32 voxel type, i64 dims[3],
 * u64 data offset) followed by the voxels, x slowest and z fastest.  One
 * dataset per file; the dataset name is accepted and ignored.  Hyperslab
 * selections copy row by row exactly as H5Dread does for a contiguous
 * float32 dataset with matching file/memory selections.
 */
#ifndef VT_REF_HDF5_SHIM_H
#define VT_REF_HDF5_SHIM_H

#include <stdint.h>

typedef int64_t hid_t;
typedef unsigned long long hsize_t;
typedef int herr_t;

#define H5F_ACC_RDWR 1u
#define H5F_ACC_TRUNC 2u
#define H5P_DEFAULT ((hid_t)0)
#define H5S_ALL ((hid_t)0)
#define H5T_IEEE_F32LE ((hid_t)1)
#define H5T_ORDER_LE 0

typedef enum { H5S_SELECT_SET = 0 } H5S_seloper_t;
typedef int H5T_order_t;

#ifdef __cplusplus
extern "C" {
#endif
hid_t H5Fopen(const char* name, unsigned flags, hid_t fapl);
hid_t H5Fcreate(const char* name, unsigned flags, hid_t fcpl, hid_t fapl);
herr_t H5Fclose(hid_t f);
hid_t H5Dopen1(hid_t f, const char* name);
hid_t H5Dget_space(hid_t d);
herr_t H5Dclose(hid_t d);
int H5Sget_simple_extent_dims(hid_t s, hsize_t dims[], hsize_t maxdims[]);
herr_t H5Sselect_hyperslab(hid_t s, H5S_seloper_t op, const hsize_t start[], const hsize_t stride[],
                           const hsize_t count[], const hsize_t block[]);
hid_t H5Screate_simple(int rank, const hsize_t dims[], const hsize_t maxdims[]);
herr_t H5Sclose(hid_t s);
herr_t H5Dread(hid_t d, hid_t memtype, hid_t memspace, hid_t filespace, hid_t plist, void* buf);
hid_t H5Tcopy(hid_t t);
herr_t H5Tset_order(hid_t t, H5T_order_t order);
herr_t H5Tclose(hid_t t);
hid_t H5Dcreate2(hid_t f, const char* name, hid_t type, hid_t space, hid_t lcpl, hid_t dcpl, hid_t dapl);
herr_t H5Dwrite(hid_t d, hid_t memtype, hid_t memspace, hid_t filespace, hid_t plist, const void* buf);
#ifdef __cplusplus
}
#endif
#endif
