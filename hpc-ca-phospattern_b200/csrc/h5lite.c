/* h5lite.c -- see h5lite.h.  Format: the HDF5 file format specification (superblock
 * version 0, object header version 1, v1 B-trees, local heaps, symbol nodes). */
#define _GNU_SOURCE
#include "h5lite.h"

#include <errno.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/types.h>
#include <unistd.h>
#include <zlib.h>

#define UNDEF 0xffffffffffffffffULL

static __thread char g_err[512];
const char* h5l_error(void) { return g_err; }
static void seterr(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}

/* ------------------------------------------------------------------ types */
h5l_type h5l_type_of(int code) {
  h5l_type t = {code, 0, 0};
  switch (code) {
    case H5L_U8: case H5L_I8: t.size = 1; break;
    case H5L_U16: case H5L_I16: t.size = 2; break;
    case H5L_U32: case H5L_I32: case H5L_F32: t.size = 4; break;
    default: t.size = 8; break;
  }
  return t;
}

h5l_type h5l_type_str(size_t len) {
  h5l_type t = {H5L_STR, len, 0};
  return t;
}

static double get_as_double(const unsigned char* p, int code) {
  switch (code) {
    case H5L_U8: return *(const uint8_t*)p;
    case H5L_I8: return *(const int8_t*)p;
    case H5L_U16: { uint16_t v; memcpy(&v, p, 2); return v; }
    case H5L_I16: { int16_t v; memcpy(&v, p, 2); return v; }
    case H5L_U32: { uint32_t v; memcpy(&v, p, 4); return v; }
    case H5L_I32: { int32_t v; memcpy(&v, p, 4); return v; }
    case H5L_U64: { uint64_t v; memcpy(&v, p, 8); return (double)v; }
    case H5L_I64: { int64_t v; memcpy(&v, p, 8); return (double)v; }
    case H5L_F32: { float v; memcpy(&v, p, 4); return v; }
    default: { double v; memcpy(&v, p, 8); return v; }
  }
}

static void put_from_double(unsigned char* p, int code, double x) {
  switch (code) {
    case H5L_U8: *(uint8_t*)p = (uint8_t)x; break;
    case H5L_I8: *(int8_t*)p = (int8_t)x; break;
    case H5L_U16: { uint16_t v = (uint16_t)x; memcpy(p, &v, 2); break; }
    case H5L_I16: { int16_t v = (int16_t)x; memcpy(p, &v, 2); break; }
    case H5L_U32: { uint32_t v = (uint32_t)x; memcpy(p, &v, 4); break; }
    case H5L_I32: { int32_t v = (int32_t)x; memcpy(p, &v, 4); break; }
    case H5L_U64: { uint64_t v = (uint64_t)x; memcpy(p, &v, 8); break; }
    case H5L_I64: { int64_t v = (int64_t)x; memcpy(p, &v, 8); break; }
    case H5L_F32: { float v = (float)x; memcpy(p, &v, 4); break; }
    default: memcpy(p, &x, 8); break;
  }
}

int h5l_convert(const void* src, int src_code, void* dst, int dst_code, size_t n) {
  const size_t ss = h5l_type_of(src_code).size, ds = h5l_type_of(dst_code).size;
  if (src_code == H5L_STR || dst_code == H5L_STR) { seterr("no string conversion"); return -1; }
  if (src_code == dst_code) { memmove(dst, src, n * ss); return 0; }
  const int is_int64 = (src_code == H5L_U64 || src_code == H5L_I64) && (dst_code == H5L_U64 || dst_code == H5L_I64);
  for (size_t i = 0; i < n; i++) {
    if (is_int64) { memcpy((unsigned char*)dst + i * ds, (const unsigned char*)src + i * ss, 8); continue; }
    put_from_double((unsigned char*)dst + i * ds, dst_code, get_as_double((const unsigned char*)src + i * ss, src_code));
  }
  return 0;
}

/* ------------------------------------------------------------------ tree */
static h5l_obj* obj_new(const char* name, int is_group) {
  h5l_obj* o = (h5l_obj*)calloc(1, sizeof(h5l_obj));
  o->name = strdup(name ? name : "");
  o->is_group = is_group;
  o->file_addr = UNDEF;
  return o;
}

static void obj_free(h5l_obj* o) {
  if (!o) return;
  for (int i = 0; i < o->nchildren; i++) obj_free(o->children[i]);
  free(o->children);
  for (int i = 0; i < o->nattrs; i++) { free(o->attrs[i].name); free(o->attrs[i].data); }
  free(o->attrs);
  free(o->data);
  free(o->name);
  free(o);
}

static void obj_add_child(h5l_obj* p, h5l_obj* c) {
  if (p->nchildren == p->capchildren) {
    p->capchildren = p->capchildren ? 2 * p->capchildren : 8;
    p->children = (h5l_obj**)realloc(p->children, sizeof(h5l_obj*) * p->capchildren);
  }
  p->children[p->nchildren++] = c;
  c->parent = p;
}

static h5l_obj* child_named(h5l_obj* p, const char* name, size_t len) {
  for (int i = 0; i < p->nchildren; i++)
    if (strlen(p->children[i]->name) == len && strncmp(p->children[i]->name, name, len) == 0) return p->children[i];
  return NULL;
}

h5l_obj* h5l_lookup(h5l_file* f, h5l_obj* base, const char* path) {
  h5l_obj* o = base ? base : f->root;
  if (path && path[0] == '/') o = f->root;
  const char* p = path ? path : "";
  while (*p) {
    while (*p == '/') p++;
    if (!*p) break;
    const char* e = strchr(p, '/');
    size_t len = e ? (size_t)(e - p) : strlen(p);
    if (len == 1 && p[0] == '.') { p += len; continue; }
    if (!o->is_group) return NULL;
    o = child_named(o, p, len);
    if (!o) return NULL;
    p += len;
  }
  return o;
}

static h5l_obj* parent_for(h5l_file* f, h5l_obj* base, const char* path, const char** leaf) {
  /* split path into parent path and leaf name */
  static __thread char buf[1024];
  snprintf(buf, sizeof buf, "%s", path);
  size_t n = strlen(buf);
  while (n > 1 && buf[n - 1] == '/') buf[--n] = 0;
  char* slash = strrchr(buf, '/');
  h5l_obj* par;
  if (!slash) { par = base ? base : f->root; *leaf = buf; return par; }
  *slash = 0;
  par = (slash == buf) ? f->root : h5l_lookup(f, buf[0] == '/' ? NULL : base, buf);
  *leaf = slash + 1;
  return par;
}

h5l_obj* h5l_group_create(h5l_file* f, h5l_obj* base, const char* path) {
  const char* leaf;
  h5l_obj* par = parent_for(f, base, path, &leaf);
  if (!par || !par->is_group) { seterr("parent group of \"%s\" does not exist", path); return NULL; }
  if (!*leaf) return par;
  h5l_obj* o = child_named(par, leaf, strlen(leaf));
  if (o) return o->is_group ? o : NULL;
  o = obj_new(leaf, 1);
  obj_add_child(par, o);
  f->dirty = 1;
  return o;
}

uint64_t h5l_dset_nelem(const h5l_obj* d) {
  uint64_t n = 1;
  for (int i = 0; i < d->ndims; i++) n *= d->dims[i];
  return n;
}

h5l_obj* h5l_dset_create(h5l_file* f, h5l_obj* base, const char* path, h5l_type type, int ndims,
                         const uint64_t* dims) {
  const char* leaf;
  h5l_obj* par = parent_for(f, base, path, &leaf);
  if (!par || !par->is_group || !*leaf) { seterr("parent group of \"%s\" does not exist", path); return NULL; }
  if (ndims < 0 || ndims > H5L_MAX_DIMS) { seterr("too many dimensions"); return NULL; }
  if (child_named(par, leaf, strlen(leaf))) { seterr("\"%s\" exists", path); return NULL; }
  h5l_obj* o = obj_new(leaf, 0);
  o->type = type;
  o->ndims = ndims;
  for (int i = 0; i < ndims; i++) o->dims[i] = dims[i];
  o->nbytes = h5l_dset_nelem(o) * type.size;
  o->data = (unsigned char*)calloc(1, o->nbytes ? o->nbytes : 1);
  obj_add_child(par, o);
  f->dirty = 1;
  return o;
}

h5l_attr* h5l_attr_find(h5l_obj* o, const char* name) {
  for (int i = 0; i < o->nattrs; i++)
    if (strcmp(o->attrs[i].name, name) == 0) return &o->attrs[i];
  return NULL;
}

h5l_attr* h5l_attr_write(h5l_file* f, h5l_obj* o, const char* name, h5l_type type, int ndims,
                         const uint64_t* dims, const void* data) {
  h5l_attr* a = h5l_attr_find(o, name);
  if (!a) {
    if (o->nattrs == o->capattrs) {
      o->capattrs = o->capattrs ? 2 * o->capattrs : 8;
      o->attrs = (h5l_attr*)realloc(o->attrs, sizeof(h5l_attr) * o->capattrs);
    }
    a = &o->attrs[o->nattrs++];
    memset(a, 0, sizeof *a);
    a->name = strdup(name);
  }
  free(a->data);
  a->type = type;
  a->ndims = ndims;
  uint64_t n = 1;
  for (int i = 0; i < ndims; i++) { a->dims[i] = dims[i]; n *= dims[i]; }
  a->nbytes = n * type.size;
  a->data = (unsigned char*)malloc(a->nbytes ? a->nbytes : 1);
  if (a->nbytes) memcpy(a->data, data, a->nbytes);
  if (f) f->dirty = 1;
  return a;
}

/* ------------------------------------------------------------------ reader */
typedef struct {
  const unsigned char* b;
  size_t n;
  int fail;
} rd_t;

static int chk(rd_t* r, uint64_t off, uint64_t len) {
  if (off > r->n || len > r->n - off) {
    if (!r->fail) seterr("read past the end of the file (offset %llu, %llu bytes)", (unsigned long long)off,
                         (unsigned long long)len);
    r->fail = 1;
    return 0;
  }
  return 1;
}
static uint64_t rdu(rd_t* r, uint64_t off, int nb) {
  if (!chk(r, off, nb)) return 0;
  uint64_t v = 0;
  for (int i = nb - 1; i >= 0; i--) v = (v << 8) | r->b[off + i];
  return v;
}

static int parse_dtype(rd_t* r, uint64_t off, size_t msize, h5l_type* t) {
  if (!chk(r, off, 8)) return -1;
  const int cls = r->b[off] & 0x0f;
  const unsigned bf0 = r->b[off + 1];
  const uint32_t size = (uint32_t)rdu(r, off + 4, 4);
  (void)msize;
  t->size = size;
  t->strpad = 0;
  if (cls == 0) {              /* fixed point */
    if (bf0 & 1) { seterr("big-endian integers are not supported"); return -1; }
    const int sgn = (bf0 >> 3) & 1;
    switch (size) {
      case 1: t->code = sgn ? H5L_I8 : H5L_U8; break;
      case 2: t->code = sgn ? H5L_I16 : H5L_U16; break;
      case 4: t->code = sgn ? H5L_I32 : H5L_U32; break;
      case 8: t->code = sgn ? H5L_I64 : H5L_U64; break;
      default: seterr("integer size %u not supported", size); return -1;
    }
  } else if (cls == 1) {       /* floating point */
    if (bf0 & 1) { seterr("big-endian floats are not supported"); return -1; }
    if (size == 4) t->code = H5L_F32;
    else if (size == 8) t->code = H5L_F64;
    else { seterr("float size %u not supported", size); return -1; }
  } else if (cls == 3) {       /* string */
    t->code = H5L_STR;
    t->strpad = bf0 & 0x0f;
  } else {
    seterr("datatype class %d not supported", cls);
    return -1;
  }
  return 0;
}

static int parse_dspace(rd_t* r, uint64_t off, int* ndims, uint64_t* dims) {
  const int ver = (int)rdu(r, off, 1);
  const int nd = (int)rdu(r, off + 1, 1);
  if (nd > H5L_MAX_DIMS) { seterr("rank %d too large", nd); return -1; }
  uint64_t p;
  if (ver == 1) p = off + 8;
  else if (ver == 2) {
    const int type = (int)rdu(r, off + 3, 1);
    if (type == 2) { *ndims = 0; return 0; }
    p = off + 4;
  } else { seterr("dataspace version %d not supported", ver); return -1; }
  *ndims = nd;
  for (int i = 0; i < nd; i++) dims[i] = rdu(r, p + 8 * i, 8);
  return r->fail ? -1 : 0;
}

typedef struct {
  int layout;              /* 0 compact, 1 contiguous, 2 chunked, -1 none */
  uint64_t addr, size;
  uint64_t cdata_off;      /* compact data offset */
  int cndims;
  uint32_t cdims[H5L_MAX_DIMS + 1];
  int nfilters;
  int filters[8];
  int shuffle_size;
} layout_t;

static int parse_layout(rd_t* r, uint64_t off, layout_t* L) {
  const int ver = (int)rdu(r, off, 1);
  if (ver == 3) {
    L->layout = (int)rdu(r, off + 1, 1);
    if (L->layout == 0) { L->size = rdu(r, off + 2, 2); L->cdata_off = off + 4; }
    else if (L->layout == 1) { L->addr = rdu(r, off + 2, 8); L->size = rdu(r, off + 10, 8); }
    else if (L->layout == 2) {
      L->cndims = (int)rdu(r, off + 2, 1);
      if (L->cndims > H5L_MAX_DIMS + 1) { seterr("chunk rank too large"); return -1; }
      L->addr = rdu(r, off + 3, 8);
      for (int i = 0; i < L->cndims; i++) L->cdims[i] = (uint32_t)rdu(r, off + 11 + 4 * i, 4);
    } else { seterr("layout class %d not supported", L->layout); return -1; }
  } else if (ver == 1 || ver == 2) {
    const int nd = (int)rdu(r, off + 1, 1);
    L->layout = (int)rdu(r, off + 2, 1);
    uint64_t p = off + 8;
    if (L->layout != 0) { L->addr = rdu(r, p, 8); p += 8; }
    if (nd > H5L_MAX_DIMS + 1) { seterr("layout rank too large"); return -1; }
    L->cndims = nd;
    for (int i = 0; i < nd; i++) L->cdims[i] = (uint32_t)rdu(r, p + 4 * i, 4);
    p += 4 * nd;
    if (L->layout == 0) { L->size = rdu(r, p, 4); L->cdata_off = p + 4; }
    if (L->layout == 1) {
      uint64_t s = 1;
      for (int i = 0; i < nd; i++) s *= L->cdims[i];
      L->size = s;  /* element count x element size is checked against the dataspace later */
    }
  } else { seterr("layout version %d not supported", ver); return -1; }
  return r->fail ? -1 : 0;
}

static int parse_filters(rd_t* r, uint64_t off, layout_t* L) {
  const int ver = (int)rdu(r, off, 1);
  const int nf = (int)rdu(r, off + 1, 1);
  uint64_t p = (ver == 1) ? off + 8 : off + 2;
  L->nfilters = 0;
  for (int i = 0; i < nf && i < 8; i++) {
    const int id = (int)rdu(r, p, 2);
    int namelen = 0;
    if (ver == 1 || id >= 256) { namelen = (int)rdu(r, p + 2, 2); p += 4; } else p += 2;
    p += 2;  /* flags */
    const int nvals = (int)rdu(r, p, 2);
    p += 2;
    if (ver == 1) namelen = (namelen + 7) & ~7;
    p += namelen;
    if (id == 2 && nvals > 0) L->shuffle_size = (int)rdu(r, p, 4);
    p += 4 * nvals;
    if (ver == 1 && (nvals & 1)) p += 4;
    if (id != 1 && id != 2 && id != 3) { seterr("filter %d not supported", id); return -1; }
    L->filters[L->nfilters++] = id;
  }
  return r->fail ? -1 : 0;
}

static int unfilter(const layout_t* L, unsigned char* raw, size_t rawlen, unsigned char* out, size_t outlen,
                    uint32_t mask) {
  unsigned char* cur = (unsigned char*)malloc(rawlen ? rawlen : 1);
  memcpy(cur, raw, rawlen);
  size_t curlen = rawlen;
  for (int i = L->nfilters - 1; i >= 0; i--) {
    if (mask & (1u << i)) continue;
    const int id = L->filters[i];
    if (id == 1) {
      unsigned char* o = (unsigned char*)malloc(outlen ? outlen : 1);
      uLongf dl = (uLongf)outlen;
      if (uncompress(o, &dl, cur, (uLong)curlen) != Z_OK) { free(o); free(cur); seterr("deflate failed"); return -1; }
      free(cur);
      cur = o;
      curlen = dl;
    } else if (id == 2) {
      const int es = L->shuffle_size > 0 ? L->shuffle_size : 1;
      const size_t ne = curlen / es;
      unsigned char* o = (unsigned char*)malloc(curlen ? curlen : 1);
      for (size_t e = 0; e < ne; e++)
        for (int b = 0; b < es; b++) o[e * es + b] = cur[b * ne + e];
      memcpy(o + ne * es, cur + ne * es, curlen - ne * es);
      free(cur);
      cur = o;
    } else if (id == 3) {
      if (curlen >= 4) curlen -= 4;
    }
  }
  if (curlen < outlen) { free(cur); seterr("chunk shorter than expected"); return -1; }
  memcpy(out, cur, outlen);
  free(cur);
  return 0;
}

static int read_chunks(rd_t* r, uint64_t addr, const layout_t* L, h5l_obj* d, int depth) {
  if (depth > 32) { seterr("chunk B-tree too deep"); return -1; }
  if (!chk(r, addr, 24) || memcmp(r->b + addr, "TREE", 4) != 0) { seterr("bad chunk B-tree node"); return -1; }
  const int level = r->b[addr + 5];
  const int used = (int)rdu(r, addr + 6, 2);
  const int nd = L->cndims;            /* dataset rank + 1 */
  const uint64_t keysz = 8 + 8 * (uint64_t)nd;
  uint64_t p = addr + 24;
  const size_t es = d->type.size;
  uint64_t chunk_elems = 1;
  for (int i = 0; i < nd - 1; i++) chunk_elems *= L->cdims[i];
  const size_t chunk_bytes = chunk_elems * es;
  unsigned char* buf = (unsigned char*)malloc(chunk_bytes ? chunk_bytes : 1);
  for (int e = 0; e < used; e++) {
    const uint32_t csize = (uint32_t)rdu(r, p, 4);
    const uint32_t fmask = (uint32_t)rdu(r, p + 4, 4);
    uint64_t offs[H5L_MAX_DIMS + 1];
    for (int i = 0; i < nd; i++) offs[i] = rdu(r, p + 8 + 8 * i, 8);
    const uint64_t child = rdu(r, p + keysz, 8);
    p += keysz + 8;
    if (r->fail) { free(buf); return -1; }
    if (level > 0) {
      if (read_chunks(r, child, L, d, depth + 1)) { free(buf); return -1; }
      continue;
    }
    if (!chk(r, child, csize)) { free(buf); return -1; }
    if (L->nfilters) {
      if (unfilter(L, (unsigned char*)r->b + child, csize, buf, chunk_bytes, fmask)) { free(buf); return -1; }
    } else {
      if (csize < chunk_bytes) { free(buf); seterr("chunk too small"); return -1; }
      memcpy(buf, r->b + child, chunk_bytes);
    }
    /* scatter the chunk into the dataset (row-major, clipped at the edges) */
    const int rank = d->ndims;
    uint64_t idx[H5L_MAX_DIMS] = {0};
    for (uint64_t c = 0; c < chunk_elems; c++) {
      uint64_t rem = c;
      for (int i = rank - 1; i >= 0; i--) { idx[i] = rem % L->cdims[i]; rem /= L->cdims[i]; }
      uint64_t lin = 0;
      int inside = 1;
      for (int i = 0; i < rank; i++) {
        const uint64_t g = offs[i] + idx[i];
        if (g >= d->dims[i]) { inside = 0; break; }
        lin = lin * d->dims[i] + g;
      }
      if (inside) memcpy(d->data + lin * es, buf + c * es, es);
    }
  }
  free(buf);
  return 0;
}

static h5l_obj* read_object(rd_t* r, uint64_t addr, const char* name, int depth);

static int read_group_entries(rd_t* r, uint64_t btree, uint64_t heap_data, h5l_obj* g, int depth) {
  if (depth > 32) { seterr("group B-tree too deep"); return -1; }
  if (!chk(r, btree, 24) || memcmp(r->b + btree, "TREE", 4) != 0) { seterr("bad group B-tree node"); return -1; }
  const int level = r->b[btree + 5];
  const int used = (int)rdu(r, btree + 6, 2);
  uint64_t p = btree + 24 + 8;  /* skip key 0 */
  for (int e = 0; e < used; e++) {
    const uint64_t child = rdu(r, p, 8);
    p += 16;
    if (r->fail) return -1;
    if (level > 0) {
      if (read_group_entries(r, child, heap_data, g, depth + 1)) return -1;
      continue;
    }
    if (!chk(r, child, 8) || memcmp(r->b + child, "SNOD", 4) != 0) { seterr("bad symbol node"); return -1; }
    const int nsym = (int)rdu(r, child + 6, 2);
    for (int s = 0; s < nsym; s++) {
      const uint64_t ent = child + 8 + 40 * (uint64_t)s;
      const uint64_t noff = rdu(r, ent, 8);
      const uint64_t oaddr = rdu(r, ent + 8, 8);
      if (r->fail || !chk(r, heap_data + noff, 1)) return -1;
      const char* nm = (const char*)r->b + heap_data + noff;
      h5l_obj* c = read_object(r, oaddr, nm, depth + 1);
      if (!c) return -1;
      obj_add_child(g, c);
    }
  }
  return 0;
}

static h5l_obj* read_object(rd_t* r, uint64_t addr, const char* name, int depth) {
  if (depth > 64) { seterr("object nesting too deep"); return NULL; }
  if (!chk(r, addr, 16)) return NULL;
  if (r->b[addr] != 1) { seterr("object header version %d not supported (only version 1)", r->b[addr]); return NULL; }
  const int nmsgs = (int)rdu(r, addr + 2, 2);
  const uint64_t hsize = rdu(r, addr + 8, 4);
  uint64_t blocks[64][2];
  int nblocks = 1;
  blocks[0][0] = addr + 16;
  blocks[0][1] = hsize;
  h5l_obj* o = obj_new(name, 0);
  int have_space = 0, have_type = 0, is_group = 0;
  uint64_t st_btree = UNDEF, st_heap = UNDEF;
  layout_t L;
  memset(&L, 0, sizeof L);
  L.layout = -1;
  int seen = 0;
  for (int b = 0; b < nblocks && seen < nmsgs; b++) {
    uint64_t p = blocks[b][0];
    const uint64_t end = blocks[b][0] + blocks[b][1];
    while (p + 8 <= end && seen < nmsgs) {
      const int type = (int)rdu(r, p, 2);
      const uint64_t msize = rdu(r, p + 2, 2);
      const int flags = (int)rdu(r, p + 4, 1);
      const uint64_t d = p + 8;
      if (r->fail || !chk(r, d, msize)) { obj_free(o); return NULL; }
      seen++;
      if ((flags & 2) && type != 0) { seterr("shared object header messages are not supported"); obj_free(o); return NULL; }
      switch (type) {
        case 0x0001: if (parse_dspace(r, d, &o->ndims, o->dims)) { obj_free(o); return NULL; } have_space = 1; break;
        case 0x0003: if (parse_dtype(r, d, msize, &o->type)) { obj_free(o); return NULL; } have_type = 1; break;
        case 0x0008: if (parse_layout(r, d, &L)) { obj_free(o); return NULL; } break;
        case 0x000B: if (parse_filters(r, d, &L)) { obj_free(o); return NULL; } break;
        case 0x0011: is_group = 1; st_btree = rdu(r, d, 8); st_heap = rdu(r, d + 8, 8); break;
        case 0x0010:
          if (nblocks < 64) { blocks[nblocks][0] = rdu(r, d, 8); blocks[nblocks][1] = rdu(r, d + 8, 8); nblocks++; }
          break;
        case 0x000C: {
          const int ver = (int)rdu(r, d, 1);
          const uint64_t nsz = rdu(r, d + 2, 2), tsz = rdu(r, d + 4, 2), ssz = rdu(r, d + 6, 2);
          uint64_t q = d + (ver == 3 ? 9 : 8);
          const uint64_t nsz_p = ver == 1 ? ((nsz + 7) & ~7ull) : nsz;
          const uint64_t tsz_p = ver == 1 ? ((tsz + 7) & ~7ull) : tsz;
          const uint64_t ssz_p = ver == 1 ? ((ssz + 7) & ~7ull) : ssz;
          if (!chk(r, q, nsz)) { obj_free(o); return NULL; }
          char* an = strndup((const char*)r->b + q, nsz);
          h5l_type at;
          int and_ = 0;
          uint64_t adims[H5L_MAX_DIMS];
          if (parse_dtype(r, q + nsz_p, tsz, &at) || parse_dspace(r, q + nsz_p + tsz_p, &and_, adims)) {
            free(an); obj_free(o); return NULL;
          }
          uint64_t ne = 1;
          for (int i = 0; i < and_; i++) ne *= adims[i];
          const uint64_t dq = q + nsz_p + tsz_p + ssz_p;
          if (!chk(r, dq, ne * at.size)) { free(an); obj_free(o); return NULL; }
          h5l_attr_write(NULL, o, an, at, and_, adims, r->b + dq);
          free(an);
          break;
        }
        default: break;
      }
      p = d + ((msize + 7) & ~7ull);
    }
  }
  if (is_group) {
    o->is_group = 1;
    if (!chk(r, st_heap, 32) || memcmp(r->b + st_heap, "HEAP", 4) != 0) { seterr("bad local heap"); obj_free(o); return NULL; }
    const uint64_t heap_data = rdu(r, st_heap + 24, 8);
    if (read_group_entries(r, st_btree, heap_data, o, depth)) { obj_free(o); return NULL; }
    return o;
  }
  if (!have_space || !have_type || L.layout < 0) {
    /* neither a group nor a dataset we understand (e.g. a committed datatype): keep it empty */
    o->is_group = 1;
    return o;
  }
  const uint64_t ne = h5l_dset_nelem(o);
  o->nbytes = ne * o->type.size;
  o->data = (unsigned char*)calloc(1, o->nbytes ? o->nbytes : 1);
  if (L.layout == 0) {
    if (!chk(r, L.cdata_off, o->nbytes)) { obj_free(o); return NULL; }
    memcpy(o->data, r->b + L.cdata_off, o->nbytes);
  } else if (L.layout == 1) {
    if (L.addr != UNDEF && o->nbytes) {
      if (!chk(r, L.addr, o->nbytes)) { obj_free(o); return NULL; }
      memcpy(o->data, r->b + L.addr, o->nbytes);
    }
  } else if (L.layout == 2) {
    if (L.addr != UNDEF && read_chunks(r, L.addr, &L, o, 0)) { obj_free(o); return NULL; }
  }
  return o;
}

h5l_file* h5l_open(const char* path, int writable) {
  FILE* fp = fopen(path, "rb");
  if (!fp) { seterr("cannot open %s: %s", path, strerror(errno)); return NULL; }
  fseek(fp, 0, SEEK_END);
  long n = ftell(fp);
  fseek(fp, 0, SEEK_SET);
  unsigned char* b = (unsigned char*)malloc(n > 0 ? n : 1);
  if (n > 0 && fread(b, 1, n, fp) != (size_t)n) { fclose(fp); free(b); seterr("cannot read %s", path); return NULL; }
  fclose(fp);
  rd_t r = {b, (size_t)n, 0};
  static const unsigned char sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  uint64_t base = UNDEF;
  for (uint64_t off = 0; off + 8 <= (uint64_t)n; off = off ? off * 2 : 512)
    if (memcmp(b + off, sig, 8) == 0) { base = off; break; }
  if (base == UNDEF) { free(b); seterr("%s is not an HDF5 file", path); return NULL; }
  const int ver = b[base + 8];
  if (ver > 1) { free(b); seterr("%s: superblock version %d not supported (0 or 1)", path, ver); return NULL; }
  if (b[base + 13] != 8 || b[base + 14] != 8) { free(b); seterr("%s: only 8-byte offsets and lengths", path); return NULL; }
  const uint64_t entry = base + (ver == 0 ? 56 : 60);
  const uint64_t root_addr = rdu(&r, entry + 8, 8);
  h5l_obj* root = read_object(&r, root_addr, "", 0);
  free(b);
  if (!root) return NULL;
  root->is_group = 1;
  h5l_file* f = (h5l_file*)calloc(1, sizeof(h5l_file));
  f->path = strdup(path);
  f->writable = writable;
  f->root = root;
  return f;
}

h5l_file* h5l_create(const char* path) {
  h5l_file* f = (h5l_file*)calloc(1, sizeof(h5l_file));
  f->path = strdup(path);
  f->writable = 1;
  f->dirty = 1;
  f->root = obj_new("", 1);
  f->incremental = 1;
  f->data_end = 96;                    /* after the superblock */
  return f;
}

/* ------------------------------------------------------------------ writer */
#define SYM_LEAF_K 32           /* symbol nodes of 64 entries */
#define SYM_INT_K 32            /* B-tree nodes of 64 children */

/* A byte buffer holding file addresses [base, n): b[0] is the byte at address base.
 * place_data: datasets' raw data go into the buffer (whole-file writes), else they are
 * already in the file at their file_addr (incremental flushes). */
typedef struct {
  unsigned char* b;
  size_t n, cap;
  uint64_t base;
  int place_data;
} wb_t;
#define WB(w, at) ((w)->b + ((at) - (w)->base))

static void wb_reserve(wb_t* w, size_t extra) {
  const size_t used = w->n - w->base;
  if (used + extra > w->cap) {
    size_t c = w->cap ? w->cap : 4096;
    while (c < used + extra) c *= 2;
    w->b = (unsigned char*)realloc(w->b, c);
    w->cap = c;
  }
}
static uint64_t wb_alloc(wb_t* w, size_t len) {   /* 8-byte aligned, zeroed */
  const size_t pad = (8 - (w->n & 7)) & 7;
  wb_reserve(w, pad + len);
  memset(WB(w, w->n), 0, pad + len);
  w->n += pad;
  const uint64_t at = w->n;
  w->n += len;
  return at;
}
static void put(wb_t* w, uint64_t at, uint64_t v, int nb) {
  for (int i = 0; i < nb; i++) WB(w, at)[i] = (unsigned char)(v >> (8 * i));
}

static size_t dtype_size(const h5l_type* t) { return t->code == H5L_STR ? 8 : (t->code >= H5L_F32 && t->code <= H5L_F64) ? 20 : 12; }

static void dtype_encode(unsigned char* p, const h5l_type* t) {
  memset(p, 0, dtype_size(t));
  if (t->code == H5L_STR) {
    p[0] = 0x13;
    p[1] = (unsigned char)(t->strpad & 0x0f);
    put(&(wb_t){p, 8, 8}, 4, t->size, 4);
    return;
  }
  if (t->code == H5L_F32 || t->code == H5L_F64) {
    const int dbl = t->code == H5L_F64;
    p[0] = 0x11;
    p[1] = 0x20;                       /* little endian, mantissa normalisation: implied */
    p[2] = dbl ? 63 : 31;              /* sign bit */
    wb_t w = {p, 20, 20};
    put(&w, 4, dbl ? 8 : 4, 4);
    put(&w, 8, 0, 2);                  /* bit offset */
    put(&w, 10, dbl ? 64 : 32, 2);     /* precision */
    p[12] = dbl ? 52 : 23;             /* exponent location */
    p[13] = dbl ? 11 : 8;              /* exponent size */
    p[14] = 0;                         /* mantissa location */
    p[15] = dbl ? 52 : 23;             /* mantissa size */
    put(&w, 16, dbl ? 1023 : 127, 4);  /* exponent bias */
    return;
  }
  const int sgn = t->code >= H5L_I8 && t->code <= H5L_I64;
  p[0] = 0x10;
  p[1] = sgn ? 0x08 : 0x00;
  wb_t w = {p, 12, 12};
  put(&w, 4, t->size, 4);
  put(&w, 8, 0, 2);
  put(&w, 10, 8 * t->size, 2);
}

static size_t dspace_size(int ndims) { return 8 + 8 * (size_t)ndims; }

static void dspace_encode(unsigned char* p, int ndims, const uint64_t* dims) {
  memset(p, 0, dspace_size(ndims));
  p[0] = 1;
  p[1] = (unsigned char)ndims;
  wb_t w = {p, dspace_size(ndims), dspace_size(ndims)};
  for (int i = 0; i < ndims; i++) put(&w, 8 + 8 * i, dims[i], 8);
}

#define A8(x) (((x) + 7) & ~(size_t)7)

typedef struct { int type; size_t size; unsigned char* data; } msg_t;

static uint64_t write_header(wb_t* w, msg_t* m, int nm) {
  size_t total = 0;
  for (int i = 0; i < nm; i++) total += 8 + A8(m[i].size);
  if (total < 24) total = 24;          /* room for at least one continuation-sized message */
  const uint64_t at = wb_alloc(w, 16 + total);
  int nmsgs = nm;
  uint64_t p = at + 16;
  for (int i = 0; i < nm; i++) {
    put(w, p, m[i].type, 2);
    put(w, p + 2, A8(m[i].size), 2);
    memcpy(WB(w, p + 8), m[i].data, m[i].size);
    p += 8 + A8(m[i].size);
  }
  if (p < at + 16 + total) {           /* fill the rest with a NIL message */
    put(w, p, 0, 2);
    put(w, p + 2, at + 16 + total - p - 8, 2);
    nmsgs++;
  }
  WB(w, at)[0] = 1;
  put(w, at + 2, nmsgs, 2);
  put(w, at + 4, 1, 4);
  put(w, at + 8, total, 4);
  return at;
}

static msg_t attr_msg(const h5l_attr* a) {
  const size_t nl = strlen(a->name) + 1;
  const size_t ts = dtype_size(&a->type), ss = dspace_size(a->ndims);
  msg_t m;
  m.type = 0x000C;
  m.size = 8 + A8(nl) + A8(ts) + A8(ss) + a->nbytes;
  m.data = (unsigned char*)calloc(1, m.size);
  wb_t w = {m.data, m.size, m.size, 0, 0};
  m.data[0] = 1;
  put(&w, 2, nl, 2);
  put(&w, 4, ts, 2);
  put(&w, 6, ss, 2);
  memcpy(m.data + 8, a->name, nl);
  dtype_encode(m.data + 8 + A8(nl), &a->type);
  dspace_encode(m.data + 8 + A8(nl) + A8(ts), a->ndims, a->dims);
  if (a->nbytes) memcpy(m.data + 8 + A8(nl) + A8(ts) + A8(ss), a->data, a->nbytes);
  return m;
}

static int cmp_child(const void* a, const void* b) {
  return strcmp((*(h5l_obj* const*)a)->name, (*(h5l_obj* const*)b)->name);
}

typedef struct { uint64_t header, btree, heap; } written_t;

static int write_object(wb_t* w, h5l_obj* o, written_t* out);

static int write_group(wb_t* w, h5l_obj* g, written_t* out) {
  const int n = g->nchildren;
  if (n > 2 * SYM_LEAF_K * 2 * SYM_INT_K) { seterr("group %s has too many members", g->name); return -1; }
  qsort(g->children, n, sizeof(h5l_obj*), cmp_child);
  written_t* cw = (written_t*)calloc(n ? n : 1, sizeof(written_t));
  for (int i = 0; i < n; i++)
    if (write_object(w, g->children[i], &cw[i])) { free(cw); return -1; }
  /* local heap: "" at offset 0, then every name */
  size_t hsz = 8;
  for (int i = 0; i < n; i++) hsz += A8(strlen(g->children[i]->name) + 1);
  const uint64_t heap = wb_alloc(w, 32);
  const uint64_t hdata = wb_alloc(w, hsz);
  uint64_t* noff = (uint64_t*)calloc(n ? n : 1, sizeof(uint64_t));
  size_t q = 8;
  for (int i = 0; i < n; i++) {
    noff[i] = q;
    memcpy(WB(w, hdata + q), g->children[i]->name, strlen(g->children[i]->name) + 1);
    q += A8(strlen(g->children[i]->name) + 1);
  }
  memcpy(WB(w, heap), "HEAP", 4);
  WB(w, heap)[4] = 0;
  put(w, heap + 8, hsz, 8);
  put(w, heap + 16, UNDEF, 8);
  put(w, heap + 24, hdata, 8);
  /* symbol nodes of up to 2*SYM_LEAF_K entries */
  const int per = 2 * SYM_LEAF_K;
  const int nsnod = n ? (n + per - 1) / per : 1;
  uint64_t snod[2 * SYM_INT_K];
  for (int s = 0; s < nsnod; s++) {
    const size_t sz = 8 + 40 * (size_t)per;
    snod[s] = wb_alloc(w, sz);
    memcpy(WB(w, snod[s]), "SNOD", 4);
    WB(w, snod[s])[4] = 1;
    const int first = s * per, cnt = (n - first) < per ? (n - first) : per;
    put(w, snod[s] + 6, cnt > 0 ? cnt : 0, 2);
    for (int k = 0; k < cnt; k++) {
      const int i = first + k;
      const uint64_t e = snod[s] + 8 + 40 * (uint64_t)k;
      put(w, e, noff[i], 8);
      put(w, e + 8, cw[i].header, 8);
      if (g->children[i]->is_group) {
        put(w, e + 16, 1, 4);
        put(w, e + 24, cw[i].btree, 8);
        put(w, e + 32, cw[i].heap, 8);
      }
    }
  }
  /* one leaf-level B-tree node over the symbol nodes */
  const size_t bsz = 24 + (2 * SYM_INT_K + 1) * 8 + 2 * SYM_INT_K * 8;
  const uint64_t bt = wb_alloc(w, bsz);
  memcpy(WB(w, bt), "TREE", 4);
  WB(w, bt)[4] = 0;
  WB(w, bt)[5] = 0;
  put(w, bt + 6, n ? nsnod : 0, 2);
  put(w, bt + 8, UNDEF, 8);
  put(w, bt + 16, UNDEF, 8);
  uint64_t p = bt + 24;
  put(w, p, 0, 8);                      /* key 0: "" */
  p += 8;
  for (int s = 0; s < (n ? nsnod : 0); s++) {
    put(w, p, snod[s], 8);
    const int last = ((s + 1) * per < n ? (s + 1) * per : n) - 1;
    put(w, p + 8, noff[last], 8);
    p += 16;
  }
  /* group object header: symbol table message + attributes */
  msg_t* m = (msg_t*)calloc(1 + g->nattrs, sizeof(msg_t));
  unsigned char st[16];
  wb_t sw = {st, 16, 16, 0, 0};
  put(&sw, 0, bt, 8);
  put(&sw, 8, heap, 8);
  m[0].type = 0x0011; m[0].size = 16; m[0].data = st;
  for (int i = 0; i < g->nattrs; i++) m[1 + i] = attr_msg(&g->attrs[i]);
  out->header = write_header(w, m, 1 + g->nattrs);
  out->btree = bt;
  out->heap = heap;
  for (int i = 0; i < g->nattrs; i++) free(m[1 + i].data);
  free(m);
  free(noff);
  free(cw);
  return 0;
}

static int write_dataset(wb_t* w, h5l_obj* d, written_t* out) {
  uint64_t addr = UNDEF;
  if (d->nbytes) {
    if (w->place_data) {
      addr = wb_alloc(w, d->nbytes);
      memcpy(WB(w, addr), d->data, d->nbytes);
    } else {
      addr = d->file_addr;
    }
  }
  msg_t* m = (msg_t*)calloc(4 + d->nattrs, sizeof(msg_t));
  unsigned char ds[8 + 8 * H5L_MAX_DIMS], dt[20], fill[4] = {2, 1, 0, 0}, lay[18];
  dspace_encode(ds, d->ndims, d->dims);
  dtype_encode(dt, &d->type);
  memset(lay, 0, sizeof lay);
  lay[0] = 3;
  lay[1] = 1;
  wb_t lw = {lay, 18, 18};
  put(&lw, 2, addr, 8);
  put(&lw, 10, d->nbytes, 8);
  m[0].type = 0x0001; m[0].size = dspace_size(d->ndims); m[0].data = ds;
  m[1].type = 0x0003; m[1].size = dtype_size(&d->type); m[1].data = dt;
  m[2].type = 0x0005; m[2].size = 4; m[2].data = fill;
  m[3].type = 0x0008; m[3].size = 18; m[3].data = lay;
  for (int i = 0; i < d->nattrs; i++) m[4 + i] = attr_msg(&d->attrs[i]);
  out->header = write_header(w, m, 4 + d->nattrs);
  out->btree = out->heap = UNDEF;
  for (int i = 0; i < d->nattrs; i++) free(m[4 + i].data);
  free(m);
  return 0;
}

static int write_object(wb_t* w, h5l_obj* o, written_t* out) {
  return o->is_group ? write_group(w, o, out) : write_dataset(w, o, out);
}

/* The 96-byte version-0 superblock: root group entry and end-of-file address. */
static void superblock(unsigned char* sb, const written_t* root, uint64_t eof) {
  static const unsigned char sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  wb_t w = {sb, 96, 96, 0, 0};
  memset(sb, 0, 96);
  memcpy(sb, sig, 8);
  sb[13] = 8; sb[14] = 8;
  put(&w, 16, SYM_LEAF_K, 2);
  put(&w, 18, SYM_INT_K, 2);
  put(&w, 20, 0, 4);
  put(&w, 24, 0, 8);                  /* base address */
  put(&w, 32, UNDEF, 8);              /* free-space info */
  put(&w, 40, eof, 8);                /* end of file */
  put(&w, 48, UNDEF, 8);              /* driver info */
  put(&w, 56, 0, 8);                  /* root entry: name offset */
  put(&w, 64, root->header, 8);
  put(&w, 72, 1, 4);                  /* cache type 1: symbol table scratch */
  put(&w, 80, root->btree, 8);
  put(&w, 88, root->heap, 8);
}

/* Raw data of every dataset not yet in the file, appended at *end. */
static int place_new_data(FILE* fp, h5l_obj* o, uint64_t* end) {
  if (o->is_group) {
    for (int i = 0; i < o->nchildren; i++)
      if (place_new_data(fp, o->children[i], end)) return -1;
    return 0;
  }
  if (!o->nbytes || o->file_addr != UNDEF) return 0;
  const uint64_t at = (*end + 7) & ~(uint64_t)7;
  if (fseeko(fp, (off_t)at, SEEK_SET) || fwrite(o->data, 1, o->nbytes, fp) != o->nbytes) return -1;
  o->file_addr = at;
  *end = at + o->nbytes;
  return 0;
}

static int flush_incremental(h5l_file* f) {
  FILE* fp = fopen(f->path, f->flushed ? "r+b" : "w+b");
  if (!fp) { seterr("cannot write %s: %s", f->path, strerror(errno)); return -1; }
  uint64_t end = f->data_end;
  if (place_new_data(fp, f->root, &end)) {
    fclose(fp);
    seterr("short write to %s", f->path);
    return -1;
  }
  f->data_end = end;
  wb_t w = {NULL, 0, 0, 0, 0};
  w.base = w.n = (end + 7) & ~(uint64_t)7;
  written_t root;
  if (write_group(&w, f->root, &root)) { free(w.b); fclose(fp); return -1; }
  unsigned char sb[96];
  superblock(sb, &root, w.n);
  const size_t len = w.n - w.base;
  int bad = fseeko(fp, (off_t)w.base, SEEK_SET) || fwrite(w.b, 1, len, fp) != len;
  bad = bad || fseeko(fp, 0, SEEK_SET) || fwrite(sb, 1, 96, fp) != 96;
  bad = bad || fflush(fp) || ftruncate(fileno(fp), (off_t)w.n);
  fclose(fp);
  free(w.b);
  if (bad) { seterr("short write to %s", f->path); return -1; }
  f->flushed = 1;
  f->dirty = 0;
  return 0;
}

int h5l_flush(h5l_file* f) {
  if (!f->writable || !f->dirty) return 0;
  if (f->incremental) return flush_incremental(f);
  wb_t w = {NULL, 0, 0, 0, 1};
  const uint64_t sb = wb_alloc(&w, 96);
  written_t root;
  if (write_group(&w, f->root, &root)) { free(w.b); return -1; }
  superblock(WB(&w, sb), &root, w.n);
  FILE* fp = fopen(f->path, "wb");
  if (!fp) { free(w.b); seterr("cannot write %s: %s", f->path, strerror(errno)); return -1; }
  const size_t wr = fwrite(w.b, 1, w.n, fp);
  fclose(fp);
  free(w.b);
  if (wr != w.n) { seterr("short write to %s", f->path); return -1; }
  f->dirty = 0;
  return 0;
}

int h5l_close(h5l_file* f) {
  if (!f) return 0;
  int rc = h5l_flush(f);
  obj_free(f->root);
  free(f->path);
  free(f);
  return rc;
}

/* ------------------------------------------------------------------ flat helpers
 * Path-based accessors for foreign-function callers (Python ctypes). */
int h5l_get_attr(h5l_file* f, const char* obj, const char* name, int* code, size_t* size, int* ndims,
                 uint64_t* dims, const void** data, size_t* nbytes) {
  h5l_obj* o = h5l_lookup(f, NULL, obj);
  if (!o) { seterr("no object \"%s\"", obj); return -1; }
  h5l_attr* a = h5l_attr_find(o, name);
  if (!a) { seterr("no attribute \"%s\" on \"%s\"", name, obj); return -1; }
  *code = a->type.code; *size = a->type.size; *ndims = a->ndims;
  for (int i = 0; i < a->ndims; i++) dims[i] = a->dims[i];
  *data = a->data; *nbytes = a->nbytes;
  return 0;
}

int h5l_get_dset(h5l_file* f, const char* path, int* code, size_t* size, int* ndims, uint64_t* dims,
                 const void** data, size_t* nbytes) {
  h5l_obj* o = h5l_lookup(f, NULL, path);
  if (!o || o->is_group) { seterr("no dataset \"%s\"", path); return -1; }
  *code = o->type.code; *size = o->type.size; *ndims = o->ndims;
  for (int i = 0; i < o->ndims; i++) dims[i] = o->dims[i];
  *data = o->data; *nbytes = o->nbytes;
  return 0;
}

/* names of the members of a group, '\n' separated, each prefixed 'g' or 'd' */
int h5l_list(h5l_file* f, const char* path, char* buf, size_t n) {
  h5l_obj* o = h5l_lookup(f, NULL, path);
  if (!o || !o->is_group) { seterr("no group \"%s\"", path); return -1; }
  size_t q = 0;
  if (n) buf[0] = 0;
  for (int i = 0; i < o->nchildren; i++) {
    int k = snprintf(buf + q, q < n ? n - q : 0, "%c%s\n", o->children[i]->is_group ? 'g' : 'd', o->children[i]->name);
    q += k;
  }
  return (int)q;
}

/* attribute names of an object, '\n' separated */
int h5l_list_attrs(h5l_file* f, const char* path, char* buf, size_t n) {
  h5l_obj* o = h5l_lookup(f, NULL, path);
  if (!o) { seterr("no object \"%s\"", path); return -1; }
  size_t q = 0;
  if (n) buf[0] = 0;
  for (int i = 0; i < o->nattrs; i++) q += snprintf(buf + q, q < n ? n - q : 0, "%s\n", o->attrs[i].name);
  return (int)q;
}

int h5l_put_attr(h5l_file* f, const char* obj, const char* name, int code, size_t size, int ndims,
                 const uint64_t* dims, const void* data) {
  h5l_obj* o = h5l_lookup(f, NULL, obj);
  if (!o) o = h5l_group_create(f, NULL, obj);
  if (!o) return -1;
  h5l_type t = code == H5L_STR ? h5l_type_str(size) : h5l_type_of(code);
  return h5l_attr_write(f, o, name, t, ndims, dims, data) ? 0 : -1;
}

int h5l_put_dset(h5l_file* f, const char* path, int code, int ndims, const uint64_t* dims, const void* data) {
  h5l_obj* o = h5l_dset_create(f, NULL, path, h5l_type_of(code), ndims, dims);
  if (!o) return -1;
  if (o->nbytes) memcpy(o->data, data, o->nbytes);
  return 0;
}

int h5l_put_group(h5l_file* f, const char* path) { return h5l_group_create(f, NULL, path) ? 0 : -1; }
