/*
 * csparks_oracle.c -- FP64 CPU restatement of the reference calcium_sparks time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the parity tests, smoke() and
 * bench.py's cpu_baseline leg compare the CUDA path against.  Nothing in the product
 * (libcsparks_cuda.so, the calcium_sparks CLI) links, loads or calls it.
 *
 * It restates, serially and in FP64, what the reference (fvm_mpi/src/) does on one MPI
 * rank: setup (species.c:95-884, geometry.c:96-344, boundaryfluxes.c:361-605), the loop
 * body (calcium_sparks.c:190-228) and the scalar outputs (species.c:2785-2880).  Each
 * function cites the reference lines it follows.  Its own correctness is pinned against
 * the reference program itself, compiled from the reference sources with the shims in
 * oracle/shims (oracle/Makefile.ref), by tests/test_oracle_pin.py.
 *
 * Random numbers: the reference draws channel transitions from MT19937 (mtwist.c); this
 * oracle draws them from the same counter-based Philox4x32-10 stream as the GPU path
 * (key = (seed, realisation), counter = (channel, boundary, step)), so stochastic
 * trajectories can be compared draw for draw with the GPU.  Runs with every channel
 * forced (-O / -C) use no random numbers and match the reference itself.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../include/csparks.h"

#define ND CSP_MAX_DOMAINS
#define NS CSP_MAX_SPECIES

enum { FLUX_NONE = 0, FLUX_RYR, FLUX_P_RYR, FLUX_SERCA };

typedef struct {
  int type, inner;            /* density/discrete, inner (from != to) / outer */
  int npairs;                 /* species-voxel pairs (subdivision-expanded) */
  uint32_t* vox;              /* [npairs][6] species voxel coords from, to */
  int flux;                   /* FLUX_* */
  int flux_dsi;
  double params[10];          /* RyR_model::params layout, boundaryfluxes.h:54 */
  uint8_t* state;             /* discrete: channel state per pair */
  double t_close;
} obnd_t;

typedef struct {
  csp_info info;
  int nx, ny, nz;
  size_t nvox;
  int S;                      /* subdivisions */
  double h, h_geom, dt, dV;
  int nd, ns;
  uint8_t* dom;
  double* u1[NS];
  double* du[NS];
  double init[ND][NS];
  int ndiff, diff_species[NS], substeps[NS];
  double coef[NS][ND][ND];
  int nbuf;
  double konT[CSP_MAX_BUFFERS * ND], koffT[CSP_MAX_BUFFERS * ND], totT[CSP_MAX_BUFFERS * ND];
  uint8_t bsp0T[CSP_MAX_BUFFERS * ND], bsp1T[CSP_MAX_BUFFERS * ND];
  uint8_t bsp0[ND][NS], bsp1[ND][NS];
  int reaction_substep, stochastic_substep;
  int nb;
  obnd_t b[CSP_MAX_BOUNDARIES];
  size_t nfixed[NS];
  size_t* fixed[NS];
  int force_dirichlet;
  uint8_t update[NS];
  long domain_num[ND];
  double volumes[ND];
  uint64_t seed;
  uint32_t realisation;
  double tabort, last_closed;
  int64_t time_ind;           /* next step index (the reference's time_ind) */
} oracle_t;

/* ---------------- Philox4x32-10 (Salmon et al., SC'11) ---------------- */
static void philox4x32(uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int i = 0; i < 10; i++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    c0 = hi1 ^ c1 ^ k0; c1 = lo1; c2 = hi0 ^ c3 ^ k1; c3 = lo0;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Uniform double in [0,1) with 53 random bits, for (channel, boundary, step). */
static double channel_uniform(const oracle_t* o, uint32_t channel, uint32_t boundary, int64_t step) {
  uint32_t ctr[4] = {channel, boundary, (uint32_t)step, (uint32_t)((uint64_t)step >> 32)};
  uint32_t key[2] = {(uint32_t)o->seed, o->realisation ^ (uint32_t)(o->seed >> 32)};
  uint32_t r[4];
  philox4x32(ctr, key, r);
  return ((double)(r[0] >> 5) * 67108864.0 + (double)(r[1] >> 6)) * (1.0 / 9007199254740992.0);
}

/* ---------------- flux laws (boundaryfluxes.c:12-141) ---------------- */
static double serca_flux(double dt, double h, double u0, double u1, const double* params) {
  /* boundaryfluxes.c:12-85 */
  const double Ca_sr = u1 / 1000, Ca_i = u0 / 1000;
  const double k_p1 = 25900, k_p2 = 2540, k_p3 = 20.5, k_m1 = 16, k_m2 = 67200, k_m3 = 149;
  const double kdcai = 0.9, kdcasr = 2.24, kdh1 = 1.09e-5, kdhi = 3.54e-3, kdhsr = 1.05e-8,
               kdh = 7.24e-5, H_i = 1e-4, ATP = 5, ADP = 36.3e-3, P_i = 1;
  double T_Cai = Ca_i / kdcai, T_Casr = Ca_sr / kdcasr;
  double T_Cai2 = T_Cai * T_Cai, T_Casr2 = T_Casr * T_Casr;
  double T_H1 = H_i / kdh1, T_Hi = (H_i * H_i) / kdhi, T_Hsr = (H_i * H_i) / kdhsr, T_H = H_i / kdh;
  double a_p1 = k_p1 * ATP;
  double a_p2 = k_p2 * T_Cai2 / (T_Cai2 + T_Cai2 * T_Hi + T_Hi * (1 + T_H1));
  double a_p3 = k_p3 * T_Hsr / (T_Casr2 * T_H + T_H + T_Hsr * (1 + T_H));
  double a_m1 = k_m1 * T_Hi / (T_Cai2 + T_Cai2 * T_Hi + T_Hi * (1 + T_H1));
  double a_m2 = k_m2 * ADP * T_Casr2 * T_H / (T_Casr2 * T_H + T_H + T_Hsr * (1 + T_H));
  double a_m3 = k_m3 * P_i;
  double s1 = a_p2 * a_p3 + a_m1 * a_p3 + a_m1 * a_m2;
  double s2 = a_p1 * a_p3 + a_m2 * a_p1 + a_m2 * a_m3;
  double s3 = a_p1 * a_p2 + a_m3 * a_m1 + a_m3 * a_p2;
  double v_cycle = (a_p1 * a_p2 * a_p3 - a_m1 * a_m2 * a_m3) / (s1 + s2 + s3);
  double density = params[1];
  double Q = 1e-3 / 6e17, S = v_cycle * Q, I = density * S, A = h * h, J = A * I;
  double V = 1e-24 * h * h * h;
  return dt * (J / V);
}

static double ryr_flux(double dt, double h, double u0, double u1, const double* params) {
  /* boundaryfluxes.c:87-141 */
  double i_c = params[6];
  double K_0 = exp(-2 * dt * 1e15 / (2 * 96485.) * i_c / (1300. - 0.1) / (h * h * h));
  return (u0 - u1) * (1 - K_0) / 2;
}

static double flux_eval(const obnd_t* b, double dt, double h, double u0, double u1) {
  return b->flux == FLUX_SERCA ? serca_flux(dt, h, u0, u1, b->params) : ryr_flux(dt, h, u0, u1, b->params);
}

/* ---------------- setup ---------------- */
static int find_name(const char names[][CSP_NAME_LEN], int n, const char* s) {
  for (int i = 0; i < n; i++)
    if (strncmp(names[i], s, CSP_NAME_LEN) == 0) return i;
  return -1;
}

static int boundary_id(const csp_model* m, const char* name) {
  for (int i = 0; i < m->num_boundaries; i++)
    if (strncmp(m->boundaries[i].name, name, CSP_NAME_LEN) == 0) return i;
  return -1;
}

static int diffusive_id(const oracle_t* o, const csp_model* m, const char* species) {
  int si = find_name(m->species_names, m->num_species, species);
  for (int d = 0; d < o->ndiff; d++)
    if (o->diff_species[d] == si) return d;
  return -1;
}

/* Species_init_boundary_voxels, species.c:938-1035 (one rank: every pair is local). */
static int init_boundary_voxels(oracle_t* o, const csp_model* m, int bi) {
  const csp_boundary* gb = &m->boundaries[bi];
  obnd_t* b = &o->b[bi];
  const int S = o->S;
  const int sub = gb->type == CSP_BOUNDARY_DISCRETE ? 1 : S;
  b->type = gb->type;
  b->npairs = sub * sub * gb->num_pairs;
  b->vox = (uint32_t*)calloc((size_t)b->npairs * 6 + 6, sizeof(uint32_t));
  if (!b->vox) return -1;
  /* boundary position from the first pair, geometry.c:619-629 */
  b->inner = 0;
  if (gb->num_pairs > 0) {
    const uint16_t* p = gb->pairs;
    b->inner = !(p[0] == p[3] && p[1] == p[4] && p[2] == p[5]);
  }
  for (int j = 0; j < gb->num_pairs; j++) {
    const uint16_t* lb = &gb->pairs[6 * j];
    /* Geometry_get_boundary_dir, geometry.c:1490-1530 */
    int dim2 = 0;
    for (int dim = 0; dim < 3; dim++) {
      if (lb[dim] != lb[dim + 3]) { dim2 = lb[dim] < lb[dim + 3] ? dim * 2 : dim * 2 + 1; break; }
    }
    int dim = dim2 / 2, left_right = dim2 % 2;
    int odim = dim != 0 ? 0 : 1;
    int idim = dim != 2 ? 2 : 1;
    unsigned from_ind = lb[dim] * S + (left_right == 0 ? S - 1 : 0);
    unsigned to_ind = lb[dim + 3] * S + (left_right == 0 ? 0 : S - 1);
    for (int oi = 0; oi < sub; oi++) {
      unsigned o_ind = S * lb[odim] + oi;
      if (gb->type == CSP_BOUNDARY_DISCRETE) o_ind += S / 2;
      for (int ii = 0; ii < sub; ii++) {
        unsigned i_ind = S * lb[idim] + ii;
        if (gb->type == CSP_BOUNDARY_DISCRETE) i_ind += S / 2;
        uint32_t* v = &b->vox[((size_t)j * sub * sub + oi * sub + ii) * 6];
        v[dim] = from_ind; v[odim] = o_ind; v[idim] = i_ind;
        v[dim + 3] = to_ind; v[odim + 3] = o_ind; v[idim + 3] = i_ind;
      }
    }
  }
  return 0;
}

static size_t vidx(const oracle_t* o, const uint32_t* c) {
  return ((size_t)c[0] * o->ny + c[1]) * o->nz + c[2];
}

static void set_ryr_params(obnd_t* b, const csp_ryr_params* p, double t_close) {
  /* parameter layout set at boundaryfluxes.c:445-454 */
  b->params[0] = p->Kd_close; b->params[1] = p->k_max_close; b->params[2] = p->n_open;
  b->params[3] = p->k_max_open; b->params[4] = p->k_min_open; b->params[5] = p->n_close;
  b->params[6] = p->i_unitary; b->params[7] = p->k_min_close; b->params[8] = t_close;
  b->params[9] = p->Kd_open;
  b->t_close = t_close;
}

static double get_t_close(const csp_options* opt, const char* name) {
  /* arguments_get_t_close, options.c:592-601 */
  for (int i = 0; i < opt->num_t_close; i++)
    if (strncmp(opt->t_close[i].name, name, CSP_NAME_LEN) == 0) return opt->t_close[i].time;
  return -1;
}

static const csp_open_list* get_open_list(const csp_options* opt, const char* name) {
  for (int i = 0; i < opt->num_open_lists; i++)
    if (strncmp(opt->open[i].name, name, CSP_NAME_LEN) == 0) return &opt->open[i];
  return NULL;
}

/* Initial channel state draws: init_RyR_model_states_stochastically,
 * boundaryfluxes.c:229-272, with the Philox stream at step 0. */
static void init_states_stochastic(oracle_t* o, int bi, const double* c0_of_channel) {
  obnd_t* b = &o->b[bi];
  const double* p = b->params;
  for (int i = 0; i < b->npairs; i++) {
    double c0 = c0_of_channel[i];
    double ko = fmax(fmin(pow(c0 / p[9], p[2]), p[3]), p[4]);
    double kc = fmax(fmin(pow(c0 / p[0], p[5]), p[1]), p[7]);
    double r = channel_uniform(o, (uint32_t)i, (uint32_t)bi, 0);
    b->state[i] = r <= kc / (ko + kc) ? 0 : 1;
  }
}

void* oracle_create(const csp_model* m, const csp_options* opt, uint32_t realisation) {
  oracle_t* o = (oracle_t*)calloc(1, sizeof(oracle_t));
  if (!o) return NULL;
  o->nd = m->num_domains;
  o->ns = m->num_species;
  o->realisation = realisation;
  o->seed = opt->seed;
  /* subdivisions and resolution, geometry.c:104-105 */
  o->S = (int)fmax(1., floor(m->h_geom / opt->h));
  o->S &= 0xff; /* stored in a domain_id (uint8) */
  if (o->S == 0) o->S = 1;
  o->h_geom = m->h_geom;
  o->h = m->h_geom / o->S;
  o->dV = o->h * o->h * o->h;
  o->nx = m->N[0] * o->S; o->ny = m->N[1] * o->S; o->nz = m->N[2] * o->S;
  o->nvox = (size_t)o->nx * o->ny * o->nz;
  /* species voxel domains, species.c:596-605 */
  o->dom = (uint8_t*)malloc(o->nvox);
  for (int x = 0; x < o->nx; x++)
    for (int y = 0; y < o->ny; y++)
      for (int z = 0; z < o->nz; z++)
        o->dom[((size_t)x * o->ny + y) * o->nz + z] =
            m->voxels[((size_t)(x / o->S) * m->N[1] + y / o->S) * m->N[2] + z / o->S];
  for (int d = 0; d < o->nd; d++) o->domain_num[d] = 0;
  for (size_t i = 0; i < (size_t)m->N[0] * m->N[1] * m->N[2]; i++)
    if (m->voxels[i] < o->nd) o->domain_num[m->voxels[i]]++;
  for (int d = 0; d < o->nd; d++) o->volumes[d] = o->domain_num[d] * m->h_geom * m->h_geom * m->h_geom;

  /* diffusive species, max sigma, species.c:181-201 */
  double max_sigma = 0, max_sigma_species[NS] = {0};
  uint8_t all_diffusive[NS] = {0};
  for (int d = 0; d < o->nd; d++) {
    const csp_domain_species* ds = &m->domain[d];
    for (int k = 0; k < ds->num_diffusive; k++) {
      int s = ds->diffusive[k];
      all_diffusive[s] = 1;
      max_sigma = fmax(max_sigma, ds->sigma[k]);
      max_sigma_species[s] = fmax(ds->sigma[k], max_sigma_species[s]);
    }
    for (int s = 0; s < o->ns; s++) o->init[d][s] = ds->init[s];
  }
  /* time step, species.c:265 */
  o->dt = opt->dt > 0 ? opt->dt : 0.95 * (1. / 6) * o->h * o->h / max_sigma;
  /* per-species substeps, species.c:281-294 */
  o->ndiff = 0;
  for (int s = 0; s < o->ns; s++) {
    if (!all_diffusive[s]) continue;
    double sdt = fabs(max_sigma - max_sigma_species[s]) < 1e-12 ? o->dt
                                                               : 0.95 * (1. / 6) * o->h * o->h / max_sigma_species[s];
    int sub = (int)fmax(1., floor(sdt / o->dt));
    o->substeps[o->ndiff] = sub & 0xff; /* species_substeps is a domain_id (uint8) */
    o->diff_species[o->ndiff] = s;
    o->ndiff++;
  }
  /* coefficient tables, species.c:1545-1560 (sigma indexed by the diffusive index) */
  for (int dsi = 0; dsi < o->ndiff; dsi++) {
    memset(o->coef[dsi], 0, sizeof(o->coef[dsi]));
    for (int di = 0; di < o->nd; di++) {
      const csp_domain_species* a = &m->domain[di];
      if (!(dsi < a->num_diffusive && a->sigma[dsi] != 0)) continue;
      for (int dn = 0; dn < di; dn++) {
        const csp_domain_species* b = &m->domain[dn];
        if (m->domain_connections[di * o->nd + dn] && dsi < b->num_diffusive && b->sigma[dsi] != 0)
          o->coef[dsi][di][dn] = o->coef[dsi][dn][di] =
              o->dt * 0.5 * (a->sigma[dsi] + b->sigma[dsi]) / (o->h * o->h) * o->substeps[dsi];
      }
      o->coef[dsi][di][di] = o->dt * a->sigma[dsi] / (o->h * o->h) * o->substeps[dsi];
    }
  }
  /* buffer tables, species.c:216-241, 304-313 */
  uint8_t is_buf[NS] = {0};
  memset(o->bsp0, 0, sizeof(o->bsp0));
  memset(o->bsp1, 0, sizeof(o->bsp1));
  for (int d = 0; d < o->nd; d++) {
    const csp_domain_species* ds = &m->domain[d];
    for (int bi = 0; bi < ds->num_buffers; bi++) {
      o->bsp0[d][bi] = ds->bsp0[bi];
      o->bsp1[d][bi] = ds->bsp1[bi];
      o->bsp0T[bi * o->nd + d] = ds->bsp0[bi];
      o->bsp1T[bi * o->nd + d] = ds->bsp1[bi];
      o->konT[bi * o->nd + d] = ds->k_on[bi];
      o->koffT[bi * o->nd + d] = ds->k_off[bi];
      o->totT[bi * o->nd + d] = ds->tot[bi];
      is_buf[ds->bsp0[bi]] = 1;
    }
  }
  o->nbuf = 0;
  for (int s = 0; s < o->ns; s++) o->nbuf += is_buf[s];
  /* sub-stepping of channels and reactions, species.c:784-787 */
  o->stochastic_substep = (int)fmax(1., floor(opt->dt_update_stoch / o->dt));
  o->reaction_substep = (int)fmax(1., floor(opt->dt_update_react / o->dt));

  /* fields, species.c:322-329 and Species_init_values species.c:887-935 */
  for (int s = 0; s < o->ns; s++) {
    o->u1[s] = (double*)malloc(o->nvox * sizeof(double));
    o->du[s] = (double*)malloc(o->nvox * sizeof(double));
    for (size_t i = 0; i < o->nvox; i++) o->u1[s][i] = o->init[o->dom[i]][s];
  }
  /* fixed domain species, species.c:3095-3207 (domain based: every voxel of the domain) */
  for (int s = 0; s < o->ns; s++) { o->nfixed[s] = 0; o->fixed[s] = NULL; }
  for (int i = 0; i < m->num_fixed_domain_species; i++) {
    int d = m->fixed_domain_species[2 * i], s = m->fixed_domain_species[2 * i + 1];
    size_t cnt = 0;
    for (size_t v = 0; v < o->nvox; v++) cnt += o->dom[v] == d;
    o->fixed[s] = (size_t*)realloc(o->fixed[s], (o->nfixed[s] + cnt + 1) * sizeof(size_t));
    for (size_t v = 0; v < o->nvox; v++)
      if (o->dom[v] == d) o->fixed[s][o->nfixed[s]++] = v;
  }
  o->force_dirichlet = opt->force_dirichlet;

  /* boundaries and flux map, boundaryfluxes.c:361-542 */
  o->nb = m->num_boundaries;
  for (int bi = 0; bi < o->nb; bi++) {
    if (init_boundary_voxels(o, m, bi)) return NULL;
    o->b[bi].flux = FLUX_NONE;
  }
  /* BoundaryFluxes_get_flux_info returns the first match in the order ryr, p_ryr, serca */
  int bmap[3] = {-1, -1, -1};
  if (m->use_ryr) bmap[0] = boundary_id(m, m->ryr.boundary);
  if (m->use_p_ryr) bmap[1] = boundary_id(m, m->p_ryr.boundary);
  if (m->use_serca) bmap[2] = boundary_id(m, m->serca.boundary);
  for (int k = 2; k >= 0; k--) {
    int bi = bmap[k];
    if (bi < 0) continue;
    obnd_t* b = &o->b[bi];
    if (k == 0) { b->flux = FLUX_RYR; set_ryr_params(b, &m->ryr, get_t_close(opt, "ryr")); b->flux_dsi = diffusive_id(o, m, m->ryr.species); }
    if (k == 1) { b->flux = FLUX_P_RYR; set_ryr_params(b, &m->p_ryr, get_t_close(opt, "p_ryr")); b->flux_dsi = diffusive_id(o, m, m->p_ryr.species); }
    if (k == 2) {
      b->flux = FLUX_SERCA;
      b->params[0] = m->serca.v_cyt_to_A_sr; b->params[1] = m->serca.density; b->params[2] = m->serca.scale;
      b->flux_dsi = diffusive_id(o, m, m->serca.species);
    }
    if (b->flux_dsi < 0) return NULL;
  }
  /* channel states, boundaryfluxes.c:544-605 */
  for (int bi = 0; bi < o->nb; bi++)
    if (o->b[bi].type == CSP_BOUNDARY_DISCRETE) o->b[bi].state = (uint8_t*)calloc(o->b[bi].npairs + 1, 1);
  int nd_discrete = 0;
  for (int bi = 0; bi < o->nb; bi++) nd_discrete += o->b[bi].type == CSP_BOUNDARY_DISCRETE;
  if (m->use_ryr && nd_discrete > 0) {
    int ryr_bi = bmap[0];
    /* Ca at the "to" voxel of each ryr channel (index i*2+1 of the gathered array) */
    obnd_t* rb = &o->b[ryr_bi];
    double* c0 = (double*)malloc(sizeof(double) * (rb->npairs + 1));
    for (int i = 0; i < rb->npairs; i++) c0[i] = o->u1[0][vidx(o, &rb->vox[6 * i + 3])];
    const csp_open_list* ol = get_open_list(opt, m->ryr.boundary);
    if (ol) {
      for (int i = 0; i < ol->count; i++) rb->state[ol->indices[i]] = 1;
    } else {
      init_states_stochastic(o, ryr_bi, c0);
    }
    if (m->use_p_ryr && bmap[1] >= 0) {
      obnd_t* pb = &o->b[bmap[1]];
      const csp_open_list* pl = get_open_list(opt, m->p_ryr.boundary);
      if (pl) {
        for (int i = 0; i < pl->count; i++) pb->state[pl->indices[i]] = 1;
      } else {
        /* the reference evaluates the p_ryr draw with the ryr boundary's Ca array
           (boundaryfluxes.c:595-597); past its end this uses the channel's own voxel */
        double* pc = (double*)malloc(sizeof(double) * (pb->npairs + 1));
        for (int i = 0; i < pb->npairs; i++)
          pc[i] = i < rb->npairs ? c0[i] : o->u1[0][vidx(o, &pb->vox[6 * i + 3])];
        init_states_stochastic(o, bmap[1], pc);
        free(pc);
      }
    }
    free(c0);
  }
  /* du := u, species.c:22-32 */
  for (int s = 0; s < o->ns; s++) memcpy(o->du[s], o->u1[s], o->nvox * sizeof(double));
  memset(o->update, 0, sizeof(o->update));
  o->tabort = opt->tabort;
  o->last_closed = -1.0;
  o->time_ind = 1;

  /* info */
  csp_info* in = &o->info;
  memset(in, 0, sizeof(*in));
  in->n[0] = o->nx; in->n[1] = o->ny; in->n[2] = o->nz;
  in->subdivisions = o->S; in->h = o->h; in->dt = o->dt;
  in->num_species = o->ns; in->num_diffusive = o->ndiff;
  for (int d = 0; d < o->ndiff; d++) { in->diffusive_species[d] = o->diff_species[d]; in->substeps[d] = o->substeps[d]; }
  in->num_buffers = o->nbuf;
  in->stochastic_substep = o->stochastic_substep;
  in->reaction_substep = o->reaction_substep;
  int64_t steps = 0;
  for (double t = 0.; t < opt->tstop; t += o->dt) steps++;  /* calcium_sparks.c:190 */
  in->total_steps = steps;
  for (int bi = 0; bi < o->nb; bi++) in->num_channels[bi] = o->b[bi].type == CSP_BOUNDARY_DISCRETE ? o->b[bi].npairs : 0;
  return o;
}

/* ---------------- one step (calcium_sparks.c:190-228) ---------------- */

/* Species_step_diffusion, species.c:1501-1650 on one rank: du = u + sum over in-box
 * neighbours of coef[d(v)][d(n)]*(u_n - u); neighbours outside the box are dropped. */
static void step_diffusion(oracle_t* o) {
  const int nx = o->nx, ny = o->ny, nz = o->nz;
  const size_t sx = (size_t)ny * nz, sy = nz;
  for (int dsi = 0; dsi < o->ndiff; dsi++) {
    if (o->time_ind % o->substeps[dsi] != 0) continue;
    int si = o->diff_species[dsi];
    const double* u1 = o->u1[si];
    double* du = o->du[si];
    o->update[si] = 1;
    for (int x = 0; x < nx; x++)
      for (int y = 0; y < ny; y++)
        for (int z = 0; z < nz; z++) {
          size_t v = x * sx + y * sy + z;
          double u = u1[v];
          const double* c = o->coef[dsi][o->dom[v]];
          double d = u;
          if (z > 0) d += c[o->dom[v - 1]] * (u1[v - 1] - u);
          if (z < nz - 1) d += c[o->dom[v + 1]] * (u1[v + 1] - u);
          if (y > 0) d += c[o->dom[v - sy]] * (u1[v - sy] - u);
          if (y < ny - 1) d += c[o->dom[v + sy]] * (u1[v + sy] - u);
          if (x > 0) d += c[o->dom[v - sx]] * (u1[v - sx] - u);
          if (x < nx - 1) d += c[o->dom[v + sx]] * (u1[v + sx] - u);
          du[v] = d;
        }
  }
}

/* Species_evaluate_stochastic_events species.c:1910-1957 +
 * evaluate_RyR_stochastically boundaryfluxes.c:295-359. */
static void step_stochastic(oracle_t* o) {
  int nd_discrete = 0;
  for (int bi = 0; bi < o->nb; bi++) nd_discrete += o->b[bi].type == CSP_BOUNDARY_DISCRETE;
  if (nd_discrete == 0 || o->time_ind % o->stochastic_substep != 0) return;
  const double t = o->time_ind * o->dt, dts = o->dt * o->stochastic_substep;
  for (int bi = 0; bi < o->nb; bi++) {
    obnd_t* b = &o->b[bi];
    if (b->type != CSP_BOUNDARY_DISCRETE || b->flux == FLUX_NONE || b->flux == FLUX_SERCA) continue;
    const double* p = b->params;
    for (int i = 0; i < b->npairs; i++) {
      if (p[8] > 0) {
        if (p[8] <= t + dts) b->state[i] = 0;
        continue;
      }
      double c0 = o->u1[0][vidx(o, &b->vox[6 * i + 3])];
      double kc = fmax(fmin(pow(c0 / p[0], p[5]), p[1]), p[7]);
      double ko = fmax(fmin(pow(c0 / p[9], p[2]), p[3]), p[4]);
      double r = channel_uniform(o, (uint32_t)i, (uint32_t)bi, o->time_ind);
      if (b->state[i] == 0) { if (r <= dts * ko) b->state[i] = 1; }
      else if (b->state[i] == 1) { if (r <= dts * kc) b->state[i] = 0; }
    }
  }
}

/* Species_step_boundary_fluxes, species.c:1704-1810 (no ghost pairs on one rank). */
static void step_fluxes(oracle_t* o) {
  for (int bi = 0; bi < o->nb; bi++) {
    obnd_t* b = &o->b[bi];
    if (b->flux == FLUX_NONE) continue;
    if (o->time_ind % o->substeps[b->flux_dsi] != 0) continue;
    int si = o->diff_species[b->flux_dsi];
    o->update[si] = 1;
    for (int i = 0; i < b->npairs; i++) {
      if (b->type == CSP_BOUNDARY_DISCRETE && !(b->state[i] == 1)) continue;
      size_t v0 = vidx(o, &b->vox[6 * i]), v1 = vidx(o, &b->vox[6 * i + 3]);
      double J = flux_eval(b, o->dt, o->h, o->u1[si][v0], o->u1[si][v1]);
      o->du[si][v1] += J;
      if (b->inner) o->du[si][v0] -= J;
    }
  }
}

/* Species_step_reaction species.c:1653-1702 + reaction_SIMD kernel_generic.cpp:397-509. */
static void step_reaction(oracle_t* o) {
  if (o->nbuf == 0 || o->time_ind % o->reaction_substep != 0) return;
  const double dt = o->dt * o->reaction_substep;
  const int nd = o->nd;
  for (size_t v = 0; v < o->nvox; v++) {
    int di = o->dom[v];
    for (int bi = 0; bi < o->nbuf; bi++) {
      int s0 = o->bsp0T[bi * nd + di], s1 = o->bsp1T[bi * nd + di];
      double b0 = o->u1[s0][v], b1 = o->u1[s1][v];
      double J = o->konT[bi * nd + di] * (o->totT[bi * nd + di] - b0) * b1 - o->koffT[bi * nd + di] * b0;
      if (o->update[s0]) o->du[s0][v] += dt * J; else o->du[s0][v] = b0 + dt * J;
      if (o->update[s1]) o->du[s1][v] -= dt * J; else o->du[s1][v] = b1 - dt * J;
    }
  }
  for (int di = 0; di < nd; di++)
    for (int bi = 0; bi < o->nbuf; bi++) {
      o->update[o->bsp0[di][bi]] = 1;
      o->update[o->bsp1[di][bi]] = 1;
    }
}

/* Species_apply_du species.c:1080-1121 and Species_apply_fixed_values :1066-1077. */
static void step_apply(oracle_t* o) {
  for (int s = 0; s < o->ns; s++) {
    if (!o->update[s]) continue;
    memcpy(o->u1[s], o->du[s], o->nvox * sizeof(double));
    o->update[s] = 0;
  }
  if (o->force_dirichlet) {
    for (int x = 0; x < o->nx; x++)
      for (int y = 0; y < o->ny; y++)
        for (int z = 0; z < o->nz; z++) {
          if (!(x == 0 || x == o->nx - 1 || y == 0 || y == o->ny - 1 || z == 0 || z == o->nz - 1)) continue;
          size_t v = ((size_t)x * o->ny + y) * o->nz + z;
          o->u1[0][v] = o->init[o->dom[v]][0];
        }
  }
  for (int s = 0; s < o->ns; s++)
    for (size_t k = 0; k < o->nfixed[s]; k++) {
      size_t v = o->fixed[s][k];
      o->u1[s][v] = o->init[o->dom[v]][s];
    }
}

/* Abort rule on the current channel openness: all channels of the discrete boundaries
 * closed for tabort ms (the rule of Species_check_open_discrete_boundaries,
 * species.c:3384-3488, evaluated every step). */
static void step_abort(oracle_t* o) {
  if (o->tabort == 0) return;
  int open = 0, nd = 0;
  for (int bi = 0; bi < o->nb; bi++) {
    if (o->b[bi].type != CSP_BOUNDARY_DISCRETE) continue;
    nd++;
    for (int i = 0; i < o->b[bi].npairs; i++) open += o->b[bi].state[i] == 1;
  }
  if (nd == 0) return;
  double t = o->time_ind * o->dt;  /* t+dt of the reference loop after time_ind steps */
  if (open) { o->last_closed = -1.0; return; }
  if (o->tabort >= 0) {
    if (o->last_closed < 0) o->last_closed = t;
    if (t - o->last_closed >= o->tabort) o->info.stopped = 1;
  }
}

int oracle_step(void* h, int64_t nsteps) {
  oracle_t* o = (oracle_t*)h;
  for (int64_t k = 0; k < nsteps; k++) {
    if (o->info.stopped || o->info.step >= o->info.total_steps) { o->info.stopped = 1; break; }
    step_diffusion(o);
    step_stochastic(o);
    step_fluxes(o);
    step_reaction(o);
    step_apply(o);
    o->info.step++;
    step_abort(o);
    o->time_ind++;
  }
  return 0;
}

int oracle_get_state(void* h, double* u) {
  oracle_t* o = (oracle_t*)h;
  for (int s = 0; s < o->ns; s++) memcpy(u + (size_t)s * o->nvox, o->u1[s], o->nvox * sizeof(double));
  return 0;
}

int oracle_set_state(void* h, const double* u) {
  oracle_t* o = (oracle_t*)h;
  for (int s = 0; s < o->ns; s++) {
    memcpy(o->u1[s], u + (size_t)s * o->nvox, o->nvox * sizeof(double));
    memcpy(o->du[s], o->u1[s], o->nvox * sizeof(double));
  }
  return 0;
}

int oracle_get_info(void* h, csp_info* info) {
  *info = ((oracle_t*)h)->info;
  return 0;
}

int oracle_get_channel_states(void* h, int32_t bi, int32_t* states) {
  oracle_t* o = (oracle_t*)h;
  if (bi < 0 || bi >= o->nb || o->b[bi].type != CSP_BOUNDARY_DISCRETE) return CSP_ERANGE;
  for (int i = 0; i < o->b[bi].npairs; i++) states[i] = o->b[bi].state[i];
  return 0;
}

int oracle_set_channel_states(void* h, int32_t bi, const int32_t* states) {
  oracle_t* o = (oracle_t*)h;
  if (bi < 0 || bi >= o->nb || o->b[bi].type != CSP_BOUNDARY_DISCRETE) return CSP_ERANGE;
  for (int i = 0; i < o->b[bi].npairs; i++) o->b[bi].state[i] = (uint8_t)states[i];
  return 0;
}

/* Species_output_scalar_data, species.c:2785-2880: min (init FLT_MAX), max (init
 * FLT_MIN), sum(u*dV) per (domain, species). */
int oracle_reduce(void* h, double* mn, double* mx, double* tot) {
  oracle_t* o = (oracle_t*)h;
  const int n = o->nd * o->ns;
  for (int i = 0; i < n; i++) { mn[i] = 3.40282346638528859812e+38; mx[i] = 1.17549435082228750797e-38; tot[i] = 0; }
  for (int s = 0; s < o->ns; s++)
    for (size_t v = 0; v < o->nvox; v++) {
      int k = o->dom[v] * o->ns + s;
      double val = o->u1[s][v];
      mn[k] = val < mn[k] ? val : mn[k];
      mx[k] = val > mx[k] ? val : mx[k];
      tot[k] += val * o->dV;
    }
  return 0;
}

double oracle_domain_volume(void* h, int d) { return ((oracle_t*)h)->volumes[d]; }

void oracle_destroy(void* h) {
  oracle_t* o = (oracle_t*)h;
  if (!o) return;
  for (int s = 0; s < o->ns; s++) { free(o->u1[s]); free(o->du[s]); free(o->fixed[s]); }
  for (int bi = 0; bi < o->nb; bi++) { free(o->b[bi].vox); free(o->b[bi].state); }
  free(o->dom);
  free(o);
}
