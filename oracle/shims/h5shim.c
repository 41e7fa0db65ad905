/* h5shim.c -- implementation of oracle/shims/hdf5.h on h5lite.  TEST INFRASTRUCTURE ONLY:
 * compiled into the reference program built as the oracle (oracle/_ref). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "hdf5.h"
#include "h5lite.h"

enum { K_FREE = 0, K_FILE, K_OBJ, K_ATTR, K_TYPE, K_SPACE, K_PLIST };

typedef struct {
  int kind;
  h5l_file* file;
  h5l_obj* obj;
  char* attr;
  h5l_type type;
  int ndims;
  uint64_t dims[H5L_MAX_DIMS];
  int sel;
  uint64_t start[H5L_MAX_DIMS], extent[H5L_MAX_DIMS];
} handle_t;

#define MAXH 4096
static handle_t H[MAXH];

static hid_t newh(int kind) {
  for (int i = 100; i < MAXH; i++)
    if (H[i].kind == K_FREE) { memset(&H[i], 0, sizeof H[i]); H[i].kind = kind; return (hid_t)i + 100000; }
  fprintf(stderr, "h5shim: out of handles\n");
  exit(3);
}
static handle_t* geth(hid_t h) {
  if (h >= 100000 && h < 100000 + MAXH && H[h - 100000].kind != K_FREE) return &H[h - 100000];
  return NULL;
}
static void freeh(hid_t h) {
  handle_t* p = geth(h);
  if (!p) return;
  free(p->attr);
  p->kind = K_FREE;
}

static int type_from(hid_t t, h5l_type* out) {
  if (t >= 1001 && t <= 1010) { *out = h5l_type_of((int)(t - 1000)); return 0; }
  if (t == 1011) { *out = h5l_type_str(1); return 0; }
  handle_t* p = geth(t);
  if (p && p->kind == K_TYPE) { *out = p->type; return 0; }
  return -1;
}

/* object (group or file root) a location handle refers to */
static h5l_obj* loc_obj(hid_t loc, h5l_file** f) {
  handle_t* p = geth(loc);
  if (!p) return NULL;
  *f = p->file;
  if (p->kind == K_FILE) return p->file->root;
  if (p->kind == K_OBJ) return p->obj;
  return NULL;
}

hid_t H5Pcreate(hid_t cls) { (void)cls; return newh(K_PLIST); }
herr_t H5Pclose(hid_t p) { freeh(p); return 0; }
herr_t H5Pset_fapl_mpio(hid_t p, int comm, int info) { (void)p; (void)comm; (void)info; return 0; }
herr_t H5Pset_dxpl_mpio(hid_t p, H5FD_mpio_xfer_t mode) { (void)p; (void)mode; return 0; }
herr_t H5Pset_chunk(hid_t p, int rank, const hsize_t* dims) { (void)p; (void)rank; (void)dims; return 0; }

hid_t H5Fopen(const char* name, unsigned flags, hid_t fapl) {
  (void)fapl;
  h5l_file* f = h5l_open(name, flags == H5F_ACC_RDWR);
  if (!f) { fprintf(stderr, "H5Fopen: %s\n", h5l_error()); return -1; }
  hid_t h = newh(K_FILE);
  geth(h)->file = f;
  return h;
}
hid_t H5Fcreate(const char* name, unsigned flags, hid_t fcpl, hid_t fapl) {
  (void)flags; (void)fcpl; (void)fapl;
  h5l_file* f = h5l_create(name);
  hid_t h = newh(K_FILE);
  geth(h)->file = f;
  return h;
}
herr_t H5Fclose(hid_t fh) {
  handle_t* p = geth(fh);
  if (!p || p->kind != K_FILE) return -1;
  int rc = h5l_close(p->file);
  if (rc) fprintf(stderr, "H5Fclose: %s\n", h5l_error());
  /* invalidate every handle of this file */
  for (int i = 0; i < MAXH; i++)
    if (H[i].kind != K_FREE && H[i].file == p->file && &H[i] != p) { free(H[i].attr); H[i].kind = K_FREE; }
  freeh(fh);
  return rc;
}

static hid_t obj_handle(h5l_file* f, h5l_obj* o) {
  hid_t h = newh(K_OBJ);
  geth(h)->file = f;
  geth(h)->obj = o;
  return h;
}

hid_t H5Gopen(hid_t loc, const char* name, hid_t gapl) {
  (void)gapl;
  h5l_file* f;
  h5l_obj* base = loc_obj(loc, &f);
  if (!base) return -1;
  h5l_obj* o = h5l_lookup(f, base, name);
  if (!o || !o->is_group) return -1;
  return obj_handle(f, o);
}
hid_t H5Gcreate(hid_t loc, const char* name, hid_t lcpl, hid_t gcpl, hid_t gapl) {
  (void)lcpl; (void)gcpl; (void)gapl;
  h5l_file* f;
  h5l_obj* base = loc_obj(loc, &f);
  if (!base) return -1;
  h5l_obj* o = h5l_group_create(f, base, name);
  if (!o) { fprintf(stderr, "H5Gcreate %s: %s\n", name, h5l_error()); return -1; }
  return obj_handle(f, o);
}
herr_t H5Gclose(hid_t g) { freeh(g); return 0; }

hid_t H5Aopen_by_name(hid_t loc, const char* obj_name, const char* attr_name, hid_t aapl, hid_t lapl) {
  (void)aapl; (void)lapl;
  h5l_file* f;
  h5l_obj* base = loc_obj(loc, &f);
  if (!base) return -1;
  h5l_obj* o = h5l_lookup(f, base, obj_name);
  if (!o || !h5l_attr_find(o, attr_name)) return -1;
  hid_t h = newh(K_ATTR);
  handle_t* p = geth(h);
  p->file = f;
  p->obj = o;
  p->attr = strdup(attr_name);
  return h;
}
hid_t H5Acreate2(hid_t loc, const char* name, hid_t type, hid_t space, hid_t acpl, hid_t aapl) {
  (void)acpl; (void)aapl;
  h5l_file* f;
  h5l_obj* o = loc_obj(loc, &f);
  handle_t* sp = geth(space);
  h5l_type t;
  if (!o || !sp || type_from(type, &t)) return -1;
  uint64_t n = 1;
  for (int i = 0; i < sp->ndims; i++) n *= sp->dims[i];
  void* zero = calloc(1, n * t.size + 1);
  h5l_attr_write(f, o, name, t, sp->ndims, sp->dims, zero);
  free(zero);
  hid_t h = newh(K_ATTR);
  handle_t* p = geth(h);
  p->file = f;
  p->obj = o;
  p->attr = strdup(name);
  return h;
}
hid_t H5Aget_type(hid_t a) {
  handle_t* p = geth(a);
  if (!p || p->kind != K_ATTR) return -1;
  h5l_attr* at = h5l_attr_find(p->obj, p->attr);
  hid_t h = newh(K_TYPE);
  geth(h)->type = at->type;
  return h;
}
herr_t H5Aread(hid_t a, hid_t mem_type, void* buf) {
  handle_t* p = geth(a);
  if (!p || p->kind != K_ATTR) return -1;
  h5l_attr* at = h5l_attr_find(p->obj, p->attr);
  h5l_type mt;
  if (type_from(mem_type, &mt)) return -1;
  if (mt.code == at->type.code || mt.code == H5L_STR) { memcpy(buf, at->data, at->nbytes); return 0; }
  return h5l_convert(at->data, at->type.code, buf, mt.code, at->nbytes / at->type.size);
}
herr_t H5Awrite(hid_t a, hid_t mem_type, const void* buf) {
  handle_t* p = geth(a);
  if (!p || p->kind != K_ATTR) return -1;
  h5l_attr* at = h5l_attr_find(p->obj, p->attr);
  h5l_type mt;
  if (type_from(mem_type, &mt)) return -1;
  if (mt.code == at->type.code || at->type.code == H5L_STR) { memcpy(at->data, buf, at->nbytes); }
  else h5l_convert(buf, mt.code, at->data, at->type.code, at->nbytes / at->type.size);
  p->file->dirty = 1;
  return 0;
}
herr_t H5Aclose(hid_t a) { freeh(a); return 0; }

H5T_class_t H5Tget_class(hid_t t) {
  h5l_type ty;
  if (type_from(t, &ty)) return H5T_NO_CLASS;
  if (ty.code == H5L_STR) return H5T_STRING;
  if (ty.code == H5L_F32 || ty.code == H5L_F64) return H5T_FLOAT;
  return H5T_INTEGER;
}
size_t H5Tget_size(hid_t t) {
  h5l_type ty;
  return type_from(t, &ty) ? 0 : ty.size;
}
hid_t H5Tcopy(hid_t t) {
  h5l_type ty;
  if (type_from(t, &ty)) return -1;
  hid_t h = newh(K_TYPE);
  geth(h)->type = ty;
  return h;
}
herr_t H5Tset_strpad(hid_t t, H5T_str_t pad) {
  handle_t* p = geth(t);
  if (!p || p->kind != K_TYPE) return -1;
  p->type.strpad = (int)pad;
  return 0;
}
herr_t H5Tset_size(hid_t t, size_t size) {
  handle_t* p = geth(t);
  if (!p || p->kind != K_TYPE) return -1;
  p->type.size = size;
  return 0;
}
herr_t H5Tclose(hid_t t) { freeh(t); return 0; }

hid_t H5Screate(H5S_class_t cls) {
  (void)cls;
  return newh(K_SPACE);
}
hid_t H5Screate_simple(int rank, const hsize_t* dims, const hsize_t* maxdims) {
  (void)maxdims;
  hid_t h = newh(K_SPACE);
  handle_t* p = geth(h);
  p->ndims = rank;
  for (int i = 0; i < rank; i++) p->dims[i] = dims[i];
  return h;
}
int H5Sget_simple_extent_dims(hid_t s, hsize_t* dims, hsize_t* maxdims) {
  handle_t* p = geth(s);
  if (!p || p->kind != K_SPACE) return -1;
  for (int i = 0; i < p->ndims; i++) {
    if (dims) dims[i] = p->dims[i];
    if (maxdims) maxdims[i] = p->dims[i];
  }
  return p->ndims;
}
herr_t H5Sselect_hyperslab(hid_t s, H5S_seloper_t op, const hsize_t* start, const hsize_t* stride,
                           const hsize_t* count, const hsize_t* block) {
  (void)op; (void)stride;
  handle_t* p = geth(s);
  if (!p || p->kind != K_SPACE) return -1;
  p->sel = 1;
  for (int i = 0; i < p->ndims; i++) {
    p->start[i] = start[i];
    p->extent[i] = block ? count[i] * block[i] : count[i];
  }
  return 0;
}
herr_t H5Sclose(hid_t s) { freeh(s); return 0; }

hid_t H5Dopen(hid_t loc, const char* name, hid_t dapl) {
  (void)dapl;
  h5l_file* f;
  h5l_obj* base = loc_obj(loc, &f);
  if (!base) return -1;
  h5l_obj* o = h5l_lookup(f, base, name);
  if (!o || o->is_group) return -1;
  return obj_handle(f, o);
}
hid_t H5Dcreate(hid_t loc, const char* name, hid_t type, hid_t space, hid_t lcpl, hid_t dcpl, hid_t dapl) {
  (void)lcpl; (void)dcpl; (void)dapl;
  h5l_file* f;
  h5l_obj* base = loc_obj(loc, &f);
  handle_t* sp = geth(space);
  h5l_type t;
  if (!base || !sp || type_from(type, &t)) return -1;
  h5l_obj* o = h5l_dset_create(f, base, name, t, sp->ndims, sp->dims);
  if (!o) { fprintf(stderr, "H5Dcreate %s: %s\n", name, h5l_error()); return -1; }
  return obj_handle(f, o);
}
hid_t H5Dget_space(hid_t d) {
  handle_t* p = geth(d);
  if (!p || p->kind != K_OBJ) return -1;
  hid_t h = newh(K_SPACE);
  handle_t* s = geth(h);
  s->ndims = p->obj->ndims;
  for (int i = 0; i < s->ndims; i++) s->dims[i] = p->obj->dims[i];
  return h;
}

/* copy between the dataset and a dense buffer over the file-space selection */
static herr_t transfer(hid_t d, hid_t mem_type, hid_t file_space, void* rbuf, const void* wbuf) {
  handle_t* p = geth(d);
  if (!p || p->kind != K_OBJ) return -1;
  h5l_obj* o = p->obj;
  h5l_type mt;
  if (type_from(mem_type, &mt)) return -1;
  handle_t* fs = geth(file_space);
  const int nd = o->ndims;
  uint64_t start[H5L_MAX_DIMS], ext[H5L_MAX_DIMS];
  for (int i = 0; i < nd; i++) {
    start[i] = (fs && fs->sel) ? fs->start[i] : 0;
    ext[i] = (fs && fs->sel) ? fs->extent[i] : o->dims[i];
    if (start[i] + ext[i] > o->dims[i]) return -1;
  }
  uint64_t n = 1;
  for (int i = 0; i < nd; i++) n *= ext[i];
  const size_t fes = o->type.size, mes = mt.size;
  uint64_t idx[H5L_MAX_DIMS] = {0};
  for (uint64_t k = 0; k < n; k++) {
    uint64_t rem = k, lin = 0;
    for (int i = nd - 1; i >= 0; i--) { idx[i] = rem % ext[i]; rem /= ext[i]; }
    for (int i = 0; i < nd; i++) lin = lin * o->dims[i] + start[i] + idx[i];
    unsigned char* fp = o->data + lin * fes;
    if (rbuf) h5l_convert(fp, o->type.code, (unsigned char*)rbuf + k * mes, mt.code, 1);
    else h5l_convert((const unsigned char*)wbuf + k * mes, mt.code, fp, o->type.code, 1);
  }
  if (wbuf) p->file->dirty = 1;
  return 0;
}

herr_t H5Dread(hid_t d, hid_t mem_type, hid_t mem_space, hid_t file_space, hid_t xfer, void* buf) {
  (void)mem_space; (void)xfer;
  return transfer(d, mem_type, file_space, buf, NULL);
}
herr_t H5Dwrite(hid_t d, hid_t mem_type, hid_t mem_space, hid_t file_space, hid_t xfer, const void* buf) {
  (void)mem_space; (void)xfer;
  return transfer(d, mem_type, file_space, NULL, buf);
}
herr_t H5Dclose(hid_t d) { freeh(d); return 0; }
