/*
 * oracle/shim/hooks.c -- no-op bodies of the reference's output functions
 * (Solver/src/hdf5_funcs.h, utils.h) for the library builds of the solver,
 * which leave hdf5_funcs.c out (test infrastructure only).  The program build
 * (`make cli`) compiles the reference's own hdf5_funcs.c against h5log.c
 * instead.
 */
#include "fftw3-mpi.h"

/* Output hooks of Solver/src/hdf5_funcs.h and utils.h: no file I/O here. */
void CreateOutputFilesWriteICs(const long int* N, double dt) { (void)N; (void)dt; }
/* A harness may watch the saves (e.g. to keep the state SpectralSolve saves). */
void (*shim_write_hook)(double t, long int iters) = 0;
void WriteDataToFile(double t, double dt, long int iters) {
    (void)dt;
    if (shim_write_hook) shim_write_hook(t, iters);
}
void FinalWriteAndCloseOutputFiles(const long int* N, int iters, int save_data_indx) {
    (void)N; (void)iters; (void)save_data_indx;
}
void OpenTestingFile(void) {}
void WriteTestDataReal(double* data, char* dset_name, int dset_rank, int* dset_dims, int local_dim_x) {
    (void)data; (void)dset_name; (void)dset_rank; (void)dset_dims; (void)local_dim_x;
}
void WriteTestDataFourier(fftw_complex* data, char* dset_name, int dim_x, int dim_y, int local_dim_x) {
    (void)data; (void)dset_name; (void)dim_x; (void)dim_y; (void)local_dim_x;
}
