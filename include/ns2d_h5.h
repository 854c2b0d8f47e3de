/*
 * ns2d_h5.h -- a self-contained HDF5 writer for the solver's output files
 * (lib/libns2d_h5.so, no libhdf5 needed).
 *
 * Replaces, for the program's own output, the HDF5 calls of
 * Solver/src/hdf5_funcs.c (H5Fcreate / H5Gcreate / H5Acreate+H5Awrite /
 * H5Dcreate+H5Dwrite / H5LTmake_dataset, hdf5_funcs.c:33-1870): groups,
 * scalar double attributes ("TimeValue", "TimeStep"), and contiguous datasets
 * of native doubles, native ints and the complex compound {r, i} of
 * CreateComplexDatatype (hdf5_funcs.c:1837-1868).
 *
 * Files use the layout libhdf5 writes by default: superblock version 0,
 * version-1 object headers, groups as symbol tables (v1 B-tree + local heap +
 * symbol-table nodes), contiguous storage.  Raw data is appended as each
 * dataset is written; the metadata is written by ns2d_h5_close (or
 * ns2d_h5_flush), so a file is readable once closed.
 *
 * Not thread-safe per file.  Errors return -1 and leave a message readable
 * with ns2d_h5_error.
 */
#ifndef NS2D_H5_H
#define NS2D_H5_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ns2d_h5_file ns2d_h5_file;

enum {
    NS2D_H5_F64 = 0,  /* H5T_NATIVE_DOUBLE (IEEE little-endian)              */
    NS2D_H5_I32 = 1,  /* H5T_NATIVE_INT (32-bit signed little-endian)        */
    NS2D_H5_C128 = 2  /* compound {"r": double at 0, "i": double at 8}       */
};

/* Create (truncate) a file.  NULL on failure (ns2d_h5_error(NULL) says why). */
ns2d_h5_file* ns2d_h5_create(const char* path);

/* Create group `path` ("/Iter_00001"); its parent must exist.  Creating a
   group that exists returns 0 (H5Lexists + H5Gopen of CreateGroup,
   hdf5_funcs.c:1066-1071). */
int ns2d_h5_group(ns2d_h5_file* f, const char* path);

/* Does an object (group or dataset) exist at `path`? 1 / 0. */
int ns2d_h5_exists(ns2d_h5_file* f, const char* path);

/* Attach a double attribute of dataspace [1] to the group or dataset at
   `path` (H5Acreate + H5Awrite, hdf5_funcs.c:1075-1110). */
int ns2d_h5_attr_double(ns2d_h5_file* f, const char* path, const char* name, double value);

/* Write a dataset at `path` (parent group must exist) of `rank` (1..8)
   dimensions `dims`, element type NS2D_H5_*, from `data` in C order. */
int ns2d_h5_dataset(ns2d_h5_file* f, const char* path, int type, int rank, const uint64_t* dims, const void* data);

/* Write the metadata now; the file is a complete HDF5 file afterwards.  Later
   writes are still allowed (the next flush supersedes this one's metadata). */
int ns2d_h5_flush(ns2d_h5_file* f);

/* Flush and close.  Returns -1 (after releasing f) if the flush failed. */
int ns2d_h5_close(ns2d_h5_file* f);

/* Reading existing files in libhdf5's default layout (superblock 0/1,
   symbol-table groups, v1 object headers, contiguous or compact storage) --
   input files (MAX_PALIN, Solver/src/solver.c:1775-1853) and saved runs for
   post-processing (PostProcessing/src/hdf5_funcs.c:33-170).  All return 0 (or
   a count) on success and -1 with ns2d_h5_error(NULL) set otherwise; each call
   opens and closes the file. */

/* Element type (NS2D_H5_*, -1 for others), rank and dimensions (<= 8) of a dataset. */
int ns2d_h5_dataset_info(const char* path, const char* dataset, int* type, int* rank, uint64_t* dims);
/* `count` elements of type NS2D_H5_* (H5LTread_dataset) into out, C order. */
int ns2d_h5_read(const char* path, const char* dataset, int type, void* out, uint64_t count);
/* ns2d_h5_read of doubles (H5LTread_dataset_double). */
int ns2d_h5_read_double(const char* path, const char* dataset, double* out, uint64_t count);
/* A one-double attribute of the object at `object` (H5LTget_attribute_double). */
int ns2d_h5_read_attr_double(const char* path, const char* object, const char* name, double* value);
/* The link names of group `group`, each followed by '\n', into buf (cap
   bytes, NUL-terminated); returns how many. */
int ns2d_h5_list(const char* path, const char* group, char* buf, size_t cap);

/* Message of the last failure on f (or, for NULL, of the last failed create,
   close or read). */
const char* ns2d_h5_error(const ns2d_h5_file* f);

#ifdef __cplusplus
}
#endif
#endif
