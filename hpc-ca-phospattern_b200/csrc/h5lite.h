/*
 * h5lite -- a small HDF5 reader/writer for the files calcium_sparks reads and writes.
 *
 * Reads: superblock version 0/1, version-1 object headers (with continuation blocks),
 * symbol-table groups (v1 B-trees, symbol nodes, local heaps), attributes (version 1-3
 * messages) and datasets with compact, contiguous or chunked (v1 B-tree, deflate /
 * shuffle filters) layout, of fixed-point, floating-point and fixed-length string types.
 * This is the subset h5py / libhdf5 use for the reference's geometry and species files
 * (the geometry files under createdgeometries and the parameter files under parameters).
 *
 * Writes: the same subset (superblock version 0, symbol-table groups, contiguous
 * datasets, version-1 attribute messages).  A file is held in memory as an object tree;
 * h5l_close writes the whole tree when the file was created or modified.
 */
#ifndef H5LITE_H
#define H5LITE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* type codes */
enum {
  H5L_U8 = 1, H5L_U16, H5L_U32, H5L_U64, H5L_I8, H5L_I16, H5L_I32, H5L_I64,
  H5L_F32, H5L_F64, H5L_STR
};

#define H5L_MAX_DIMS 8

typedef struct h5l_type {
  int code;          /* H5L_* */
  size_t size;       /* bytes per element (string: its fixed length) */
  int strpad;        /* strings: 0 null-terminated, 1 null-padded, 2 space-padded */
} h5l_type;

typedef struct h5l_attr {
  char* name;
  h5l_type type;
  int ndims;
  uint64_t dims[H5L_MAX_DIMS];
  unsigned char* data;
  size_t nbytes;
} h5l_attr;

typedef struct h5l_obj {
  char* name;                 /* link name within its parent ("" for the root) */
  int is_group;
  struct h5l_obj* parent;
  struct h5l_obj** children;  /* groups / datasets (groups only) */
  int nchildren, capchildren;
  h5l_attr* attrs;
  int nattrs, capattrs;
  /* datasets */
  h5l_type type;
  int ndims;
  uint64_t dims[H5L_MAX_DIMS];
  unsigned char* data;        /* the whole dataset, file byte order (little endian) */
  size_t nbytes;
  uint64_t file_addr;         /* created files: where the raw data were written (all ones: not yet) */
} h5l_obj;

typedef struct h5l_file {
  char* path;
  int writable;
  int dirty;
  h5l_obj* root;
  /* Files made by h5l_create are flushed incrementally: every dataset's raw data are
   * written once, at data_end, and only the metadata (after the raw data) and the
   * superblock are rewritten; a dataset's data must not change after the flush that
   * wrote them.  Files opened for writing are rewritten whole. */
  int incremental;
  int flushed;
  uint64_t data_end;
} h5l_file;

/* last error message (thread local) */
const char* h5l_error(void);

h5l_file* h5l_open(const char* path, int writable);
h5l_file* h5l_create(const char* path);
int h5l_flush(h5l_file* f);
int h5l_close(h5l_file* f);

/* object lookup by path relative to `base` (NULL = root); "/" separators, leading and
 * trailing slashes ignored */
h5l_obj* h5l_lookup(h5l_file* f, h5l_obj* base, const char* path);
/* create a group (parents must exist); returns the existing group if present */
h5l_obj* h5l_group_create(h5l_file* f, h5l_obj* base, const char* path);
/* create a dataset with zero-filled data */
h5l_obj* h5l_dset_create(h5l_file* f, h5l_obj* base, const char* path, h5l_type type, int ndims,
                         const uint64_t* dims);
uint64_t h5l_dset_nelem(const h5l_obj* d);

h5l_attr* h5l_attr_find(h5l_obj* o, const char* name);
/* create or replace an attribute (data copied, file byte layout) */
h5l_attr* h5l_attr_write(h5l_file* f, h5l_obj* o, const char* name, h5l_type type, int ndims,
                         const uint64_t* dims, const void* data);

h5l_type h5l_type_of(int code);
h5l_type h5l_type_str(size_t len);

/* convert n elements between numeric types (src/dst codes H5L_U8..H5L_F64) */
int h5l_convert(const void* src, int src_code, void* dst, int dst_code, size_t n);

#ifdef __cplusplus
}
#endif
#endif
