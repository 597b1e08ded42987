/*
 * hdf5.h -- minimal HDF5 stand-in used to build and run the reference's own C
 * sources on a machine without HDF5.  TEST INFRASTRUCTURE only.
 *
 * A "file" NAME is the directory NAME.d; a dataset "/x" in it is the raw
 * little-endian file NAME.d/x.bin holding the whole dataset in C (row-major)
 * order.  Hyperslab selections (start/count/block, stride 1, count 1 per
 * dimension, as the reference uses them) map to pread/pwrite runs, so several
 * ranks can write disjoint parts of one dataset.
 */
#ifndef LBRB_SHIM_HDF5_H
#define LBRB_SHIM_HDF5_H

#include "mpi.h"

typedef long long hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;

#define H5P_DEFAULT 0
#define H5P_FILE_ACCESS 1
#define H5P_DATASET_XFER 2
#define H5F_ACC_TRUNC 1
#define H5F_ACC_RDWR 2
#define H5FD_MPIO_COLLECTIVE 1
#define H5S_SELECT_SET 0
#define H5T_NATIVE_DOUBLE 1
#define H5T_NATIVE_INT 2
#define H5E_DEFAULT 0

herr_t H5Eset_current_stack(hid_t stack);
hid_t H5Pcreate(hid_t cls);
herr_t H5Pset_fapl_mpio(hid_t plist, MPI_Comm comm, MPI_Info info);
herr_t H5Pset_dxpl_mpio(hid_t plist, int mode);
herr_t H5Pclose(hid_t plist);
hid_t H5Screate_simple(int rank, const hsize_t dims[], const hsize_t maxdims[]);
herr_t H5Sselect_hyperslab(hid_t space, int op, const hsize_t start[], const hsize_t stride[],
                           const hsize_t count[], const hsize_t block[]);
herr_t H5Sclose(hid_t space);
hid_t H5Fcreate(const char *name, unsigned flags, hid_t fcpl, hid_t fapl);
hid_t H5Fopen(const char *name, unsigned flags, hid_t fapl);
herr_t H5Fclose(hid_t file);
hid_t H5Dcreate(hid_t file, const char *name, hid_t type, hid_t space, hid_t lcpl, hid_t dcpl,
                hid_t dapl);
hid_t H5Dopen(hid_t file, const char *name, hid_t dapl);
herr_t H5Dwrite(hid_t dset, hid_t memtype, hid_t memspace, hid_t filespace, hid_t xfer,
                const void *buf);
herr_t H5Dread(hid_t dset, hid_t memtype, hid_t memspace, hid_t filespace, hid_t xfer, void *buf);
herr_t H5Dclose(hid_t dset);

#endif
