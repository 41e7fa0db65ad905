/*
 * csp_io.c -- inputs and output of the calcium_sparks driver (see csp_io.h), on the
 * project's HDF5 subset (h5lite).
 */
#include "csp_io.h"

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "h5lite.h"

/* ---------------------------------------------------------------- inputs ---- */

typedef struct rd {
  h5l_file* f;
  const char* file;
  char* err;
  size_t nerr;
  int failed;
} rd;

static void rd_fail(rd* r, const char* fmt, ...) {
  if (r->failed) return;
  r->failed = 1;
  va_list ap;
  va_start(ap, fmt);
  char buf[400];
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  snprintf(r->err, r->nerr, "%s: %s", r->file, buf);
}

static h5l_attr* rd_attr(rd* r, const char* obj, const char* name) {
  if (r->failed) return NULL;
  h5l_obj* o = h5l_lookup(r->f, NULL, obj);
  h5l_attr* a = o ? h5l_attr_find(o, name) : NULL;
  if (!a) rd_fail(r, "Could not open attr \"%s%s\"", obj, name);
  return a;
}

static size_t attr_nelem(const h5l_attr* a) {
  size_t n = 1;
  for (int i = 0; i < a->ndims; i++) n *= a->dims[i];
  return n;
}

/* numeric attribute as doubles (up to maxn); returns the element count */
static int rd_doubles(rd* r, const char* obj, const char* name, double* out, int maxn) {
  h5l_attr* a = rd_attr(r, obj, name);
  if (!a) return 0;
  if (a->type.code == H5L_STR) { rd_fail(r, "attr \"%s%s\" is a string", obj, name); return 0; }
  size_t n = attr_nelem(a);
  if ((int)n > maxn) { rd_fail(r, "attr \"%s%s\" has %zu values (max %d)", obj, name, n, maxn); return 0; }
  h5l_convert(a->data, a->type.code, out, H5L_F64, n);
  return (int)n;
}

static double rd_double(rd* r, const char* obj, const char* name) {
  double v = 0.0;
  rd_doubles(r, obj, name, &v, 1);
  return v;
}

static void rd_string(rd* r, const char* obj, const char* name, char* out, size_t n) {
  out[0] = '\0';
  h5l_attr* a = rd_attr(r, obj, name);
  if (!a) return;
  if (a->type.code != H5L_STR) { rd_fail(r, "attr \"%s%s\" is not a string", obj, name); return; }
  size_t len = a->nbytes < n - 1 ? a->nbytes : n - 1;
  memcpy(out, a->data, len);
  out[len] = '\0';
  char* z = memchr(out, '\0', len + 1);
  if (z) *z = '\0';
  /* space padding */
  for (int i = (int)strlen(out) - 1; i >= 0 && out[i] == ' '; i--) out[i] = '\0';
}

static h5l_obj* rd_dset(rd* r, const char* path) {
  if (r->failed) return NULL;
  h5l_obj* d = h5l_lookup(r->f, NULL, path);
  if (!d || d->is_group) rd_fail(r, "Could not open dataset \"%s\"", path);
  return d && !d->is_group ? d : NULL;
}

static int read_geometry(rd* r, csp_model* m, cs_model_mem* mem) {
  m->h_geom = rd_double(r, "/", "h");
  rd_doubles(r, "/", "global_size", m->global_size, 3);
  m->num_domains = (int32_t)rd_double(r, "/domains", "num");
  if (!r->failed && (m->num_domains < 1 || m->num_domains > CSP_MAX_DOMAINS))
    rd_fail(r, "%d domains (max %d)", m->num_domains, CSP_MAX_DOMAINS);
  for (int i = 0; i < m->num_domains && !r->failed; i++) {
    char key[32];
    snprintf(key, sizeof key, "name_%d", i);
    rd_string(r, "/domains", key, m->domain_names[i], CSP_NAME_LEN);
    m->domain_indices[i] = (uint8_t)i;
  }
  h5l_obj* v = rd_dset(r, "/domains/voxels");
  if (v) {
    if (v->ndims != 3) { rd_fail(r, "/domains/voxels is not 3-D"); return -1; }
    for (int a = 0; a < 3; a++) m->N[a] = (int32_t)v->dims[a];
    size_t n = (size_t)h5l_dset_nelem(v);
    mem->voxels = malloc(n);
    if (!mem->voxels) { rd_fail(r, "out of memory"); return -1; }
    h5l_convert(v->data, v->type.code, mem->voxels, H5L_U8, n);
    m->voxels = mem->voxels;
  }
  h5l_obj* c = rd_dset(r, "/domains/domain_connections");
  if (c) {
    size_t n = (size_t)h5l_dset_nelem(c);
    if (n != (size_t)(m->num_domains * m->num_domains)) { rd_fail(r, "domain_connections size %zu", n); return -1; }
    h5l_convert(c->data, c->type.code, m->domain_connections, H5L_U8, n);
  }
  m->num_boundaries = (int32_t)rd_double(r, "/boundaries", "num");
  if (!r->failed && (m->num_boundaries < 0 || m->num_boundaries > CSP_MAX_BOUNDARIES))
    rd_fail(r, "%d boundaries (max %d)", m->num_boundaries, CSP_MAX_BOUNDARIES);
  for (int i = 0; i < m->num_boundaries && !r->failed; i++) {
    char key[32], type[32], path[64];
    csp_boundary* b = &m->boundaries[i];
    snprintf(key, sizeof key, "name_%d", i);
    rd_string(r, "/boundaries", key, b->name, CSP_NAME_LEN);
    snprintf(key, sizeof key, "type_%d", i);
    rd_string(r, "/boundaries", key, type, sizeof type);
    b->type = strcmp(type, "discrete") == 0 ? CSP_BOUNDARY_DISCRETE : CSP_BOUNDARY_DENSITY;
    snprintf(path, sizeof path, "/boundaries/%s", b->name);
    h5l_obj* d = rd_dset(r, path);
    if (!d) break;
    size_t n = (size_t)h5l_dset_nelem(d);
    if (n % 6) { rd_fail(r, "%s has %zu values (not pairs of 3-D voxels)", path, n); break; }
    mem->pairs[i] = malloc((n ? n : 1) * sizeof(uint16_t));
    if (!mem->pairs[i]) { rd_fail(r, "out of memory"); break; }
    h5l_convert(d->data, d->type.code, mem->pairs[i], H5L_U16, n);
    b->num_pairs = (int32_t)(n / 6);
    b->pairs = mem->pairs[i];
  }
  return r->failed ? -1 : 0;
}

static void read_ryr(rd* r, const char* grp, csp_ryr_params* p) {
  p->Kd_open = rd_double(r, grp, "Kd_open");
  p->k_min_open = rd_double(r, grp, "k_min_open");
  p->k_max_open = rd_double(r, grp, "k_max_open");
  p->n_open = rd_double(r, grp, "n_open");
  p->Kd_close = rd_double(r, grp, "Kd_close");
  p->k_min_close = rd_double(r, grp, "k_min_close");
  p->k_max_close = rd_double(r, grp, "k_max_close");
  p->n_close = rd_double(r, grp, "n_close");
  p->i_unitary = rd_double(r, grp, "i_unitary");
  rd_string(r, grp, "boundary", p->boundary, CSP_NAME_LEN);
  rd_string(r, grp, "species", p->species, CSP_NAME_LEN);
}

static int read_species(rd* r, csp_model* m) {
  m->num_species = (int32_t)rd_double(r, "/", "num_species");
  if (!r->failed && (m->num_species < 1 || m->num_species > CSP_MAX_SPECIES))
    rd_fail(r, "%d species (max %d)", m->num_species, CSP_MAX_SPECIES);
  for (int i = 0; i < m->num_species && !r->failed; i++) {
    char key[32];
    snprintf(key, sizeof key, "species_name_%d", i);
    rd_string(r, "/", key, m->species_names[i], CSP_NAME_LEN);
  }
  for (int di = 0; di < m->num_domains && !r->failed; di++) {
    const char* d = m->domain_names[di];
    csp_domain_species* ds = &m->domain[di];
    double tmp[CSP_MAX_SPECIES];
    int n = rd_doubles(r, d, "init", ds->init, CSP_MAX_SPECIES);
    if (!r->failed && n < m->num_species) rd_fail(r, "/%s init has %d values", d, n);
    ds->num_diffusive = (int32_t)rd_double(r, d, "num_diffusive");
    if (ds->num_diffusive > 0) {
      n = rd_doubles(r, d, "diffusive", tmp, CSP_MAX_SPECIES);
      for (int k = 0; k < n; k++) ds->diffusive[k] = (uint8_t)tmp[k];
      rd_doubles(r, d, "sigma", ds->sigma, CSP_MAX_SPECIES);
    }
    ds->num_buffers = (int32_t)rd_double(r, d, "num_buffers");
    if (!r->failed && (ds->num_buffers < 0 || ds->num_buffers > CSP_MAX_BUFFERS))
      rd_fail(r, "/%s has %d buffers", d, ds->num_buffers);
    for (int bi = 0; bi < ds->num_buffers && !r->failed; bi++) {
      char grp[64];
      snprintf(grp, sizeof grp, "/%s/buffer_%d", d, bi);
      ds->k_off[bi] = rd_double(r, grp, "k_off");
      ds->k_on[bi] = rd_double(r, grp, "k_on");
      ds->tot[bi] = rd_double(r, grp, "tot");
      double sp[2] = {0, 0};
      rd_doubles(r, grp, "species", sp, 2);
      ds->bsp0[bi] = (uint8_t)sp[0];
      ds->bsp1[bi] = (uint8_t)sp[1];
    }
  }
  m->num_fixed_domain_species = (int32_t)rd_double(r, "/", "num_fixed_domain_species");
  if (m->num_fixed_domain_species > 0) {
    double fx[2 * CSP_MAX_FIXED];
    int n = rd_doubles(r, "/", "fixed_domain_species", fx, 2 * CSP_MAX_FIXED);
    for (int k = 0; k < n; k++) m->fixed_domain_species[k] = (uint8_t)fx[k];
  }
  if (rd_doubles(r, "/", "convolution_constants", m->convolution_constants, 3) != 3 && !r->failed)
    rd_fail(r, "convolution_constants needs 3 values");
  m->use_ryr = (uint8_t)rd_double(r, "/", "use_ryr");
  m->use_p_ryr = (uint8_t)rd_double(r, "/", "use_p_ryr");
  m->use_serca = (uint8_t)rd_double(r, "/", "use_serca");
  if (m->use_ryr) read_ryr(r, "/ryr", &m->ryr);
  if (m->use_p_ryr) read_ryr(r, "/p_ryr", &m->p_ryr);
  if (m->use_serca) {
    m->serca.v_cyt_to_A_sr = rd_double(r, "/serca", "v_cyt_to_A_sr");
    m->serca.density = rd_double(r, "/serca", "density");
    m->serca.scale = rd_double(r, "/serca", "scale");
    rd_string(r, "/serca", "boundary", m->serca.boundary, CSP_NAME_LEN);
    /* the reference takes the SERCA species from the /ryr group (boundaryfluxes.c:511) */
    rd_string(r, "/ryr", "species", m->serca.species, CSP_NAME_LEN);
  }
  return r->failed ? -1 : 0;
}

int cs_read_model(const char* geometry_file, const char* species_file, csp_model* m, cs_model_mem* mem,
                  char* err, size_t nerr) {
  memset(m, 0, sizeof *m);
  memset(mem, 0, sizeof *mem);
  rd r = {0};
  r.err = err;
  r.nerr = nerr;
  r.file = geometry_file;
  r.f = h5l_open(geometry_file, 0);
  if (!r.f) {
    snprintf(err, nerr, "%s: %s", geometry_file, h5l_error());
    return -1;
  }
  int rc = read_geometry(&r, m, mem);
  h5l_close(r.f);
  if (rc) return rc;
  r.file = species_file;
  r.f = h5l_open(species_file, 0);
  if (!r.f) {
    snprintf(err, nerr, "%s: %s", species_file, h5l_error());
    return -1;
  }
  rc = read_species(&r, m);
  h5l_close(r.f);
  return rc;
}

void cs_model_mem_free(cs_model_mem* mem) {
  free(mem->voxels);
  for (int i = 0; i < CSP_MAX_BOUNDARIES; i++) free(mem->pairs[i]);
  memset(mem, 0, sizeof *mem);
}

/* ---------------------------------------------------------------- output ---- */

struct cs_output {
  h5l_file* f;
  h5l_obj* group;      /* current /data_%07d */
};

static char out_err[512];

const char* cs_output_error(void) { return out_err; }

static int out_fail(const char* what) {
  snprintf(out_err, sizeof out_err, "%s: %s", what, h5l_error());
  return -1;
}

static int attr_f64(cs_output* o, h5l_obj* obj, const char* name, const double* v, uint64_t n) {
  return h5l_attr_write(o->f, obj, name, h5l_type_of(H5L_F64), 1, &n, v) ? 0 : out_fail(name);
}

static int attr_u64(cs_output* o, h5l_obj* obj, const char* name, const uint64_t* v, uint64_t n) {
  return h5l_attr_write(o->f, obj, name, h5l_type_of(H5L_U64), 1, &n, v) ? 0 : out_fail(name);
}

/* fixed-length, null-terminated string of strlen bytes in a scalar dataspace
 * (write_h5_attr, utils.c:101-130) */
static int attr_str(cs_output* o, h5l_obj* obj, const char* name, const char* s) {
  return h5l_attr_write(o->f, obj, name, h5l_type_str(strlen(s)), 0, NULL, s) ? 0 : out_fail(name);
}

cs_output* cs_output_create(const char* path, double h, const uint64_t N[3], const char* geometry_file,
                            const char* species_file) {
  cs_output* o = calloc(1, sizeof *o);
  if (!o) return NULL;
  o->f = h5l_create(path);
  if (!o->f) {
    out_fail(path);
    free(o);
    return NULL;
  }
  h5l_obj* root = o->f->root;
  if (attr_f64(o, root, "h", &h, 1) || attr_u64(o, root, "N", N, 3) ||
      attr_str(o, root, "geometry_file", geometry_file) || attr_str(o, root, "species_file", species_file)) {
    h5l_close(o->f);
    free(o);
    return NULL;
  }
  return o;
}

int cs_output_group(cs_output* o, unsigned output_ind, double t, uint64_t time_ind) {
  char name[32];
  snprintf(name, sizeof name, "/data_%07u", output_ind);
  o->group = h5l_group_create(o->f, NULL, name);
  if (!o->group) return out_fail(name);
  if (attr_f64(o, o->group, "time", &t, 1) || attr_u64(o, o->group, "time_index", &time_ind, 1)) return -1;
  return 0;
}

int cs_output_scalar(cs_output* o, const char* domain, const char* species, double mn, double mx, double avg) {
  h5l_obj* d = h5l_group_create(o->f, o->group, domain);
  if (!d) return out_fail(domain);
  h5l_obj* s = h5l_group_create(o->f, d, species);
  if (!s) return out_fail(species);
  /* attribute order of species.c:3039-3050 */
  if (attr_f64(o, s, "max", &mx, 1) || attr_f64(o, s, "min", &mn, 1) || attr_f64(o, s, "average", &avg, 1))
    return -1;
  return 0;
}

int cs_output_dataset(cs_output* o, const char* name, int ndims, const uint64_t* dims, const double* data) {
  h5l_obj* d = h5l_dset_create(o->f, o->group, name, h5l_type_of(H5L_F64), ndims, dims);
  if (!d) return out_fail(name);
  if (d->nbytes) memcpy(d->data, data, d->nbytes);
  o->f->dirty = 1;
  return 0;
}

int cs_output_flush(cs_output* o) { return h5l_flush(o->f) ? out_fail("flush") : 0; }

int cs_output_close(cs_output* o) {
  if (!o) return 0;
  int rc = h5l_close(o->f) ? out_fail("close") : 0;
  free(o);
  return rc;
}
