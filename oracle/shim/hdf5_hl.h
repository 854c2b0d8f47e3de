/* oracle/shim/hdf5_hl.h -- see hdf5.h in this folder (test infrastructure only). */
#ifndef NS2D_SHIM_HDF5_HL_H
#define NS2D_SHIM_HDF5_HL_H
#include "hdf5.h"
herr_t H5LTmake_dataset(hid_t loc, const char* name, int rank, const hsize_t* dims, hid_t type, const void* buf);
herr_t H5LTread_dataset_double(hid_t loc, const char* name, double* buf);
herr_t H5LTread_dataset(hid_t loc, const char* name, hid_t type, void* buf);
#endif
