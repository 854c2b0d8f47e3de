/*
 * oracle/shim/hdf5.h -- the HDF5 API subset the reference's sources call
 * (Solver/src/hdf5_funcs.c, utils.c, solver.c:1800-1807), for building the
 * reference program against single-rank stand-ins.  Test infrastructure only:
 * oracle/shim/h5log.c records every group, attribute and dataset written into
 * a plain log file (read by tests/h5log.py) instead of an HDF5 file, so the
 * reference's outputs can be compared with the GPU program's HDF5 files.
 */
#ifndef NS2D_SHIM_HDF5_H
#define NS2D_SHIM_HDF5_H
#include <stdbool.h> /* libhdf5's public headers bring in bool */
#include <stddef.h>
#include <stdint.h>
#include "mpi.h"
typedef int64_t hid_t;
typedef int herr_t;
typedef int htri_t;
typedef unsigned long long hsize_t;
#define H5F_ACC_RDONLY 0u
#define H5F_ACC_RDWR 1u
#define H5F_ACC_TRUNC 2u
#define H5P_DEFAULT ((hid_t)0)
#define H5P_FILE_ACCESS ((hid_t)1)
#define H5P_DATASET_XFER ((hid_t)2)
#define H5S_ALL ((hid_t)0)
#define H5T_NATIVE_DOUBLE ((hid_t)101)
#define H5T_NATIVE_INT ((hid_t)102)
#define H5T_COMPOUND 6
#define H5S_SELECT_SET 0
#define H5FD_MPIO_COLLECTIVE 1
#ifndef MPI_INFO_NULL
#define MPI_INFO_NULL 0
#endif
hid_t H5Fcreate(const char* name, unsigned flags, hid_t fcpl, hid_t fapl);
hid_t H5Fopen(const char* name, unsigned flags, hid_t fapl);
herr_t H5Fclose(hid_t f);
hid_t H5Pcreate(hid_t cls);
herr_t H5Pset_fapl_mpio(hid_t p, int comm, int info);
herr_t H5Pset_dxpl_mpio(hid_t p, int mode);
herr_t H5Pclose(hid_t p);
htri_t H5Lexists(hid_t loc, const char* name, hid_t lapl);
hid_t H5Gcreate(hid_t loc, const char* name, hid_t lcpl, hid_t gcpl, hid_t gapl);
hid_t H5Gopen(hid_t loc, const char* name, hid_t gapl);
herr_t H5Gclose(hid_t g);
hid_t H5Screate_simple(int rank, const hsize_t* dims, const hsize_t* maxdims);
herr_t H5Sselect_hyperslab(hid_t space, int op, const hsize_t* start, const hsize_t* stride, const hsize_t* count,
                           const hsize_t* block);
herr_t H5Sclose(hid_t s);
hid_t H5Dcreate(hid_t loc, const char* name, hid_t type, hid_t space, hid_t lcpl, hid_t dcpl, hid_t dapl);
herr_t H5Dwrite(hid_t dset, hid_t memtype, hid_t memspace, hid_t filespace, hid_t plist, const void* buf);
herr_t H5Dclose(hid_t d);
hid_t H5Acreate(hid_t loc, const char* name, hid_t type, hid_t space, hid_t acpl, hid_t aapl);
herr_t H5Awrite(hid_t attr, hid_t type, const void* buf);
herr_t H5Aclose(hid_t a);
hid_t H5Tcreate(int cls, size_t size);
herr_t H5Tinsert(hid_t type, const char* name, size_t offset, hid_t member);
herr_t H5Tclose(hid_t t);
#endif
