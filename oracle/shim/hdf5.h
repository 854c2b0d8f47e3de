/*
 * oracle/shim/hdf5.h -- type stand-ins for the HDF5 names that appear in the
 * reference's data_types.h and solver.c (MAX_PALIN input, :1800-1807).  Test
 * infrastructure only: file I/O is not part of the compiled path, so the
 * functions report failure.
 */
#ifndef NS2D_SHIM_HDF5_H
#define NS2D_SHIM_HDF5_H
#include <stdint.h>
typedef int64_t hid_t;
typedef int herr_t;
typedef unsigned long long hsize_t;
#define H5F_ACC_RDONLY 0u
#define H5F_ACC_RDWR 1u
#define H5P_DEFAULT ((hid_t)0)
static inline hid_t H5Fopen(const char* n, unsigned f, hid_t p) { (void)n; (void)f; (void)p; return (hid_t)-1; }
static inline herr_t H5Fclose(hid_t f) { (void)f; return 0; }
#endif
