/*
 * calcium_sparks.c -- the reference's calcium_sparks program on one B200.
 *
 * A drop-in for fvm_mpi/src/calcium_sparks.c: the same command line (csp_options.c), the
 * same geometry / species HDF5 inputs and <casename>.h5 output (csp_io.c) and the same
 * console tables, with the time step of the whole domain run by libcsparks_cuda.so
 * through its C ABI (include/csparks.h).  The run itself follows calcium_sparks.c:
 * 150-229: initial output at t = 0, then steps in chunks between outputs; an output
 * every save_interval = max(1, floor(dt_save/dt)) steps (time t + dt of the step, with t
 * accumulated as `t += dt` in FP64); after every step the abort rule of
 * Species_check_open_discrete_boundaries (species.c:3384-3486), evaluated here on the
 * host on the channel states of the last output as the reference does, so that the
 * library's own abort rule is switched off (tabort = 0).
 */
#define _GNU_SOURCE
#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "csp_io.h"
#include "csp_options.h"
#include "csparks.h"

/* ------------------------------------------------------------ timings ---- */
/* the reference's timing table (utils.c:10-75).  The step's buckets come from the
 * library's per-phase device times (csp_get_phase_times, estimated from a timed sample of
 * every advance call): "Diffusion stencil" = the voxel kernel, which also does the buffer
 * reactions and fixed values ("Reaction stencil" holds only the learned surrogate's
 * kernel, "Fixed Domains" / "Apply du" stay 0: no separate pass), "Boundary fluxes" =
 * density-boundary rows + step epilogue, "Stochastic evaluation" = RyR/pRyR gating with
 * the channel fluxes; "Diffusion Total" = "Diffusion stencil".  Ghost exchange and the
 * border stencils have no counterpart on one GPU and stay 0. */
enum {
  T_SETUP = 0, T_INIT, T_GEOM, T_SPECIES, T_GHOST, T_DIFF, T_BORDERS, T_BOUNDARIES, T_STOCH, T_REACT, T_FIXED,
  T_APPLYDU, T_CONV, T_WRITE, T_BORDERSX, T_BORDERSY, T_BORDERSZ, T_MAINLOOP, T_DIFFTOT, T_SIM, T_NUM
};
static const char* tnames[T_NUM] = {
    "Setup", "Init species", "Construct geometry", "Construct species", "Communicate ghost values",
    "Diffusion stencil", "Diffusion stencil borders", "Boundary fluxes", "Stochastic evaluation",
    "Reaction stencil", "Fixed Domains", "Apply du", "Convolution", "Write", "Diffusion stencil borders X",
    "Diffusion stencil borders Y", "Diffusion stencil borders Z", "Main Loop time", "Diffusion Total",
    "Simulation time"};
static double tval[T_NUM];
static unsigned tcalls[T_NUM];

static double now(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + ts.tv_nsec * 1e-9;
}
static void push_time(int w) { tval[w] -= now(); }
static void pop_time(int w) {
  tval[w] += now();
  tcalls[w]++;
}

static void output_timings(void) {
  printf("\n");
  printf("%30s %10s %10s %10s %10s\n", "Timings", "avg", "max", "min", "Num");
  printf("---------------------------------------------------------------\n");
  double s = 0;
  for (int i = 0; i < T_NUM; i++) {
    if (i <= T_WRITE) s += tval[i];
    printf("%30s|%10.1f|%10.1f|%10.1f|%10d\n", tnames[i], tval[i], tval[i], tval[i], tcalls[i]);
  }
  printf("%30s|%10.1f|%10.1f|%10.1f|%10d\n", "sum", s, s, s, 0);
}

static void die(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vfprintf(stderr, fmt, ap);
  va_end(ap);
  fflush(stdout);
  exit(1);
}

static void check(csp_handle* h, int rc, const char* what) {
  if (rc == CSP_OK) return;
  char msg[512];
  csp_status(h, msg, sizeof msg);
  die("*** ERROR: %s failed (%d): %s\n", what, rc, msg);
}

/* ------------------------------------------------------------ the run ---- */

typedef struct run {
  cs_arguments* a;
  csp_model m;
  cs_model_mem mem;
  csp_handle* h;
  csp_info info;
  int ns, nd;
  double h_sim;                      /* species resolution */
  double volumes[CSP_MAX_DOMAINS];   /* geometry voxels x h_geom^3 (geometry.c:160-200) */
  long long domain_num[CSP_MAX_DOMAINS];
  /* discrete boundaries, in boundary order */
  int ndisc, disc_b[CSP_MAX_BOUNDARIES], disc_n[CSP_MAX_BOUNDARIES];
  int32_t* snapshot;                 /* channel states of the last output, concatenated */
  int nchan;
  /* outputs */
  cs_output* out;
  int save_sp[CSP_MAX_SPECIES * 4], nsave;      /* -s species indices */
  int sheets[3], sheet_idx[3][64];              /* per axis: global indices */
  int all_sp[CSP_MAX_SPECIES * 4], nall;
  int ls_species, ls_dom_ids[CSP_MAX_DOMAINS];
  double ls_offsets_nm[3];
  int fields_pending;                            /* an output waits for its sheets / all_data */
  /* abort rule */
  double last_opened;
} run;

static int species_id(run* R, const char* name) {
  for (int s = 0; s < R->m.num_species; s++)
    if (strcmp(R->m.species_names[s], name) == 0) return s;
  return -1;
}

static int domain_id(run* R, const char* name) {
  for (int d = 0; d < R->m.num_domains; d++)
    if (strcmp(R->m.domain_names[d], name) == 0) return d;
  return -1;
}

static int boundary_id(run* R, const char* name) {
  for (int b = 0; b < R->m.num_boundaries; b++)
    if (strcmp(R->m.boundaries[b].name, name) == 0) return b;
  return -1;
}

static void species_list(run* R, char* buf, size_t n) {
  buf[0] = '\0';
  for (int s = 0; s < R->m.num_species; s++) {
    size_t l = strlen(buf);
    snprintf(buf + l, n - l, s == 0 ? "\"%s\"" : ", \"%s\"", R->m.species_names[s]);
  }
}

/* ---- verbose listings ---- */

static void output_geometry(run* R) {
  const csp_model* m = &R->m;
  printf("Process neigbors (%d -> no neighbor)\n", -2);
  printf("-----------------------------------------------------------------------------\n");
  printf("  process %2d: coord(%d,%d,%d); X[%d,%d], Y[%d,%d], Z[%d,%d]\n", 0, 0, 0, 0, -2, -2, -2, -2, -2, -2);
  printf("\nGeometry attributs:\n");
  printf("-----------------------------------------------------------------------------\n");
  printf("  Global sizes:          (%.1f, %.1f, %.1f) um\n", m->global_size[0] / 1000., m->global_size[1] / 1000.,
         m->global_size[2] / 1000.);
  printf("  Resolution:            %.3f nm\n", m->h_geom);
  const int sub = (int)fmax(1., floor(m->h_geom / R->a->h));   /* geometry.c:104 */
  printf("  Simulation resolution: %.3f nm\n", m->h_geom / sub);
  printf("  Subdivisions 1D (3D):  %d (%d)\n", sub, sub * sub * sub);
  printf("\n");
  printf("Domains: %d\n", m->num_domains);
  printf("-----------------------------------------------------------------------------\n");
  for (int i = 0; i < m->num_domains; i++) {
    printf(" %2d : \"%s\", V: %.4e nm^3, Voxels: %zu", i, m->domain_names[i], R->volumes[i],
           (size_t)R->domain_num[i]);
    int ncon = 0;
    for (int j = 0; j < m->num_domains; j++)
      if (i != j) ncon += m->domain_connections[i * m->num_domains + j];
    if (ncon) {
      printf(", Connections: ");
      int k = 0;
      for (int j = 0; j < m->num_domains; j++) {
        if (i == j || !m->domain_connections[i * m->num_domains + j]) continue;
        printf("%s\"%s\"", k ? ", " : "", m->domain_names[j]);
        k++;
      }
    }
    printf("\n");
  }
  printf("\n");
  printf("  Voxel distributions (%zu,%zu,%zu) : %.2e\n", (size_t)m->N[0], (size_t)m->N[1], (size_t)m->N[2],
         (double)m->N[0] * m->N[1] * m->N[2]);
  printf("\n");
  printf("Boundaries: %d\n", m->num_boundaries);
  printf("-----------------------------------------------------------------------------\n");
  for (int b = 0; b < m->num_boundaries; b++)
    printf(" %2d : \"%s\", type: %s, pairs: %d\n", b, m->boundaries[b].name,
           m->boundaries[b].type == CSP_BOUNDARY_DISCRETE ? "discrete" : "density", m->boundaries[b].num_pairs);
  fflush(stdout);
}

/* Model parameters (Species_output_init_values, species.c:2105-2250) */
static void output_init_values(run* R) {
  const csp_model* m = &R->m;
  printf("\n");
  printf("Model parameters:\n");
  printf("-----------------------------------------------------------------------------\n");
  printf("%8s", "Init:");
  for (int s = 0; s < m->num_species; s++) printf("%13s", m->species_names[s]);
  printf("\n");
  for (int d = 0; d < m->num_domains; d++) {
    printf("%7s:", m->domain_names[d]);
    for (int s = 0; s < m->num_species; s++) {
      if (m->domain[d].init[s] > 0) printf("%13.2e", m->domain[d].init[s]);
      else printf("%13s", "-");
    }
    printf("\n");
  }
  printf("\n");
  printf("%8s", "Sigma:");
  for (int k = 0; k < R->info.num_diffusive; k++) printf("%13s", m->species_names[R->info.diffusive_species[k]]);
  printf("\n");
  for (int d = 0; d < m->num_domains; d++) {
    printf("%7s:", m->domain_names[d]);
    for (int k = 0; k < R->info.num_diffusive; k++) {
      const int s = R->info.diffusive_species[k];
      int found = 0;
      for (int j = 0; j < m->domain[d].num_diffusive; j++)
        if (m->domain[d].diffusive[j] == s) {
          printf("%13.2e", m->domain[d].sigma[j]);
          found = 1;
        }
      if (!found) printf("%13s", "-");
    }
    printf("\n");
  }
  int is_buf[CSP_MAX_SPECIES] = {0}, nbuf = 0;
  for (int d = 0; d < m->num_domains; d++)
    for (int b = 0; b < m->domain[d].num_buffers; b++) {
      nbuf += !is_buf[m->domain[d].bsp0[b]];
      is_buf[m->domain[d].bsp0[b]] = 1;
    }
  if (nbuf > 0) {
    const char* head[3] = {"B_tot:", "k_off:", "k_on:"};
    for (int t = 0; t < 3; t++) {
      printf("\n");
      printf("%8s", head[t]);
      for (int s = 0; s < m->num_species; s++) printf("%13s", is_buf[s] ? m->species_names[s] : "");
      printf("\n");
      for (int d = 0; d < m->num_domains; d++) {
        const csp_domain_species* ds = &m->domain[d];
        printf("%7s:", m->domain_names[d]);
        int bi = 0;
        for (int s = 0; s < m->num_species; s++) {
          if (!is_buf[s]) {
            printf("%13s", "");
          } else if (bi < ds->num_buffers && ds->bsp0[bi] == s) {
            const double v = t == 0 ? ds->tot[bi] : t == 1 ? ds->k_off[bi] : ds->k_on[bi];
            printf("%13.2e", v);
            bi++;
          } else {
            printf("%13s", "-");
          }
        }
        printf("\n");
      }
    }
  }
  if (m->num_fixed_domain_species > 0) {
    printf("\n");
    printf("%8s\n", "Fixed domain species:");
    for (int i = 0; i < m->num_fixed_domain_species; i++)
      printf("%8s:%8s\n", m->domain_names[m->fixed_domain_species[2 * i]],
             m->species_names[m->fixed_domain_species[2 * i + 1]]);
  }
}

/* Boundary fluxes (BoundaryFluxes_output_init_data, boundaryfluxes.c:607-672) */
static void output_fluxes(run* R) {
  const csp_model* m = &R->m;
  if (!m->use_ryr && !m->use_p_ryr && !m->use_serca) return;
  printf("\n");
  printf("Boundary fluxes:\n");
  printf("-----------------------------------------------------------------------------\n");
  const csp_ryr_params* P[2] = {&m->ryr, &m->p_ryr};
  const int use[2] = {m->use_ryr, m->use_p_ryr};
  const char* title[2] = {"RyR", "pRyR"};
  for (int k = 0; k < 2; k++) {
    if (!use[k]) continue;
    const csp_ryr_params* p = P[k];
    printf("  %s:\n", title[k]);
    printf("  Open:  kd: %4.2f, N: %.2f, k_min: %.2f, k_max: %.2f\n", p->Kd_open, p->n_open, p->k_min_open,
           p->k_max_open);
    printf("  Close:  kd: %4.2f, N: %.2f, k_min: %.2f, k_max: %.2f\n", p->Kd_close, p->n_close, p->k_min_close,
           p->k_max_close);
    printf("  Flux:        i_c: %.2f pA\n", p->i_unitary);
    const int b = boundary_id(R, p->boundary);
    int open = 0, n = 0;
    if (b >= 0 && m->boundaries[b].type == CSP_BOUNDARY_DISCRETE) {
      n = m->boundaries[b].num_pairs;
      int32_t* st = malloc(sizeof(int32_t) * (size_t)(n ? n : 1));
      check(R->h, csp_get_channel_states(R->h, 0, b, st), "csp_get_channel_states");
      for (int i = 0; i < n; i++) open += st[i] == 1;
      free(st);
    }
    printf("  Num open %ss: %d/%d\n", title[k], open, n);
    printf("\n");
  }
  if (m->use_serca) {
    printf("  SERCA:\n");
    printf("  v_cyt_to_A_sr: %4.2g\n", m->serca.v_cyt_to_A_sr);
    printf("        density: %4.2g\n", m->serca.density);
    printf("          scale: %4.2g\n", m->serca.scale);
  }
}

/* Time stepping (Species_output_time_stepping_information, species.c:3210-3241) */
static void output_time_stepping(run* R, double tstop, size_t save_interval) {
  const csp_info* I = &R->info;
  printf("\n");
  printf("Time stepping:\n");
  printf("-----------------------------------------------------------------------------\n");
  printf("%13s %10.2g ms\n%13s%10.3g ms\n%13s%10zu\n%13s%10zu\n\n", "tstop", tstop, "dt", I->dt, "num dt",
         (size_t)(tstop / I->dt), "save interval", save_interval);
  printf("%13s%13s%10s\n", "Diffusion", "dt [ms]", "substeps");
  for (int k = 0; k < I->num_diffusive; k++)
    printf("%13s%13.3g%10d\n", R->m.species_names[I->diffusive_species[k]], I->dt * I->substeps[k], I->substeps[k]);
  printf("\n%13s%13s%10s\n", "", "dt [ms]", "substeps");
  printf("%13s%13.3g%10d\n", "Discr bound", I->stochastic_substep * I->dt, I->stochastic_substep);
  printf("\n%13s%13s%10s\n", "", "dt [ms]", "substeps");
  printf("%13s%13.3g%10d\n", "Reaction", I->reaction_substep * I->dt, I->reaction_substep);
}

/* ------------------------------------------------------------ outputs ---- */

static void print_table(run* R, const char* title, const double* v, int divide) {
  const csp_model* m = &R->m;
  printf("%8s", title);
  for (int s = 0; s < m->num_species; s++) printf("%13s", m->species_names[s]);
  printf("\n");
  for (int d = 0; d < m->num_domains; d++) {
    printf("%7s:", m->domain_names[d]);
    for (int s = 0; s < m->num_species; s++) {
      const double x = v[d * m->num_species + s];
      printf("%13.2e", divide ? x / R->volumes[d] : x);
    }
    printf("\n");
  }
  printf("\n");
}

/* One output (Species_output_data, species.c:2253-2340, with the linescan computed
 * first as calcium_sparks.c:177/208 do), in two parts.  begin_output: linescan,
 * reductions, console tables, the group with its scalars, channel states and linescan,
 * and -- when sheets or all_data are asked for -- an asynchronous copy of those species'
 * fields (csp_snapshot_async).  finish_output: the sheets and all_data datasets from that
 * copy and the file write; the main loop runs it while the device takes the next cycle's
 * steps (csp_advance_async ... csp_advance_wait). */
static void finish_output(run* R);

static void begin_output(run* R, unsigned output_ind, double t, uint64_t time_ind) {
  cs_arguments* a = R->a;
  const csp_model* m = &R->m;
  const int ns = m->num_species, nd = m->num_domains;
  double* ls = NULL;
  if (a->linescan) {
    push_time(T_CONV);
    ls = malloc(sizeof(double) * (size_t)R->info.n[a->linescan->axis]);
    check(R->h, csp_linescan(R->h, 0, R->ls_species, a->linescan->axis, R->ls_offsets_nm, m->convolution_constants,
                             a->linescan->num_domains, ls), "csp_linescan");
    pop_time(T_CONV);
  }
  push_time(T_WRITE);
  double mn[CSP_MAX_DOMAINS * CSP_MAX_SPECIES], mx[CSP_MAX_DOMAINS * CSP_MAX_SPECIES];
  double tot[CSP_MAX_DOMAINS * CSP_MAX_SPECIES];
  int32_t* open = malloc(sizeof(int32_t) * (size_t)(R->nchan ? R->nchan : 1));
  check(R->h, csp_reduce_outputs(R->h, 0, mn, mx, tot, open), "csp_reduce_outputs");
  memcpy(R->snapshot, open, sizeof(int32_t) * (size_t)R->nchan);
  if (!a->silent) {
    double conservation = 0.;
    for (int i = 0; i < nd * ns; i++) conservation += tot[i];
    printf("\n%u: time: %.2f ms, time_index: %zu, conservation: %g\n", output_ind, t, (size_t)time_ind, conservation);
    printf("-----------------------------------------------------------------------------\n");
    print_table(R, "Average:", tot, 1);
    print_table(R, "Min:", mn, 0);
    print_table(R, "Max:", mx, 0);
    if (R->ndisc > 0) {
      printf("%8s", "Channels:\n");
      int off = 0;
      for (int k = 0; k < R->ndisc; k++) {
        printf("%7s: ", m->boundaries[R->disc_b[k]].name);
        int sum = 0;
        /* the line-break test indexes the boundary sizes by the discrete index, as the
           reference does (species.c:2995-3003) */
        const int size_k = m->boundaries[k].num_pairs;
        for (int i = 0; i < R->disc_n[k]; i++) {
          sum += open[off + i];
          printf("%d:%d", i, open[off + i]);
          if (i < size_k - 1) {
            printf(", ");
            if (i % 14 == 0 && i != 0) printf("\n         ");
          }
        }
        printf(" | %d/%d\n", sum, R->disc_n[k]);
        off += R->disc_n[k];
      }
      printf("\n");
    }
  }
  if (cs_output_group(R->out, output_ind, t, time_ind)) die("*** ERROR: output: %s\n", cs_output_error());
  for (int d = 0; d < nd; d++)
    for (int s = 0; s < ns; s++) {
      const int i = d * ns + s;
      if (cs_output_scalar(R->out, m->domain_names[d], m->species_names[s], mn[i], mx[i], tot[i] / R->volumes[d]))
        die("*** ERROR: output: %s\n", cs_output_error());
    }
  for (int k = 0, off = 0; k < R->ndisc; k++) {
    char name[64];
    snprintf(name, sizeof name, "discrete_%s", m->boundaries[R->disc_b[k]].name);
    uint64_t n = (uint64_t)R->disc_n[k];
    double* v = malloc(sizeof(double) * (size_t)(n ? n : 1));
    for (uint64_t i = 0; i < n; i++) v[i] = open[off + i];
    if (cs_output_dataset(R->out, name, 1, &n, v)) die("*** ERROR: output: %s\n", cs_output_error());
    free(v);
    off += R->disc_n[k];
  }
  if (ls) {
    int one, two;
    cs_linescan_axes(a->linescan->axis, &one, &two);
    char doms[64] = "", name[128];
    for (int i = 0; i < a->linescan->num_domains; i++) {
      size_t l = strlen(doms);
      snprintf(doms + l, sizeof doms - l, "%d_", R->ls_dom_ids[i]);
    }
    const char axc[3] = {'x', 'y', 'z'};
    snprintf(name, sizeof name, "linescan_%s_%s%c_%d_%c_%d", a->linescan->species, doms, axc[one],
             a->linescan->offsets[one], axc[two], a->linescan->offsets[two]);
    uint64_t n = (uint64_t)R->info.n[a->linescan->axis];
    if (cs_output_dataset(R->out, name, 1, &n, ls)) die("*** ERROR: output: %s\n", cs_output_error());
    free(ls);
  }
  free(open);
  if (R->nsave || R->nall) {
    uint32_t mask = 0;
    for (int q = 0; q < R->nsave; q++) mask |= 1u << R->save_sp[q];
    for (int q = 0; q < R->nall; q++) mask |= 1u << R->all_sp[q];
    check(R->h, csp_snapshot_async(R->h, 0, mask), "csp_snapshot_async");
    R->fields_pending = 1;
  } else {
    if (cs_output_flush(R->out)) die("*** ERROR: output: %s\n", cs_output_error());
  }
  pop_time(T_WRITE);
}

static void finish_output(run* R) {
  if (!R->fields_pending) return;
  R->fields_pending = 0;
  push_time(T_WRITE);
  const csp_model* m = &R->m;
  const int* n = R->info.n;
  const size_t nvox = (size_t)n[0] * n[1] * n[2];
  const double* state = NULL;
  check(R->h, csp_snapshot_wait(R->h, &state), "csp_snapshot_wait");
  const char axc[3] = {'x', 'y', 'z'};
  for (int q = 0; q < R->nsave; q++) {
    const int s = R->save_sp[q];
    const double* u = state + (size_t)s * nvox;
    for (int ax = 0; ax < 3; ax++) {
      const int lx = (ax + 1) % 3, ly = (ax + 2) % 3;
      uint64_t dims[2] = {(uint64_t)n[lx], (uint64_t)n[ly]};
      double* sheet = malloc(sizeof(double) * (size_t)(n[lx] * n[ly]));
      for (int k = 0; k < R->sheets[ax]; k++) {
        const int idx = R->sheet_idx[ax][k];
        for (int i = 0; i < n[lx]; i++)
          for (int j = 0; j < n[ly]; j++) {
            int c[3];
            c[ax] = idx; c[lx] = i; c[ly] = j;
            sheet[(size_t)i * n[ly] + j] = u[((size_t)c[0] * n[1] + c[1]) * n[2] + c[2]];
          }
        char name[64];
        snprintf(name, sizeof name, "%s_%c_sheet_%d", m->species_names[s], axc[ax], idx);
        if (cs_output_dataset(R->out, name, 2, dims, sheet)) die("*** ERROR: output: %s\n", cs_output_error());
      }
      free(sheet);
    }
  }
  for (int q = 0; q < R->nall; q++) {
    const int s = R->all_sp[q];
    char name[64];
    snprintf(name, sizeof name, "%s_all_data", m->species_names[s]);
    uint64_t dims[3] = {(uint64_t)n[0], (uint64_t)n[1], (uint64_t)n[2]};
    if (cs_output_dataset(R->out, name, 3, dims, state + (size_t)s * nvox))
      die("*** ERROR: output: %s\n", cs_output_error());
  }
  if (cs_output_flush(R->out)) die("*** ERROR: output: %s\n", cs_output_error());
  pop_time(T_WRITE);
}

/* Species_check_open_discrete_boundaries (species.c:3384-3486) after a step at time t:
 * whether every channel of the boundaries named "ryr" / "p_ryr" was closed in the last
 * output, for tabort ms.  Without -X, or without discrete boundaries, the reference
 * prints "aborting" and goes on. */
static int abort_check(run* R, double t) {
  const double tabort = R->a->tabort;
  if (tabort == 0.0 || R->ndisc == 0) {
    fputs("aborting", stdout);
    return 0;
  }
  int sum_ryr = 0, sum_p = 0, has_ryr = 0, has_p = 0;
  for (int k = 0, off = 0; k < R->ndisc; k++) {
    const char* nm = R->m.boundaries[R->disc_b[k]].name;
    int sum = 0;
    for (int i = 0; i < R->disc_n[k]; i++) sum += R->snapshot[off + i];
    if (strcmp(nm, "ryr") == 0) { has_ryr = 1; sum_ryr = sum; }
    if (strcmp(nm, "p_ryr") == 0) { has_p = 1; sum_p = sum; }
    off += R->disc_n[k];
  }
  int all_closed = 0;
  if (has_ryr && !has_p) all_closed = sum_ryr == 0;
  else if (!has_ryr && has_p) all_closed = sum_p == 0;
  else if (has_ryr && has_p) all_closed = sum_ryr == 0 && sum_p == 0;
  if (!all_closed) {
    R->last_opened = -1.0;
    return 0;
  }
  if (tabort >= 0) {
    if (R->last_opened < 0) R->last_opened = t;
    if (t - R->last_opened >= tabort) return 1;
  }
  return 0;
}

/* ------------------------------------------------------------ main ---- */

int main(int argc, char** argv) {
  push_time(T_SIM);
  push_time(T_SETUP);
  static cs_arguments a;
  cs_arguments_default(&a);
  cs_parse_arguments(argc, argv, &a);
  static run R;
  memset(&R, 0, sizeof R);
  R.a = &a;
  R.last_opened = -1.0;
  const uint64_t seed = a.seed_given ? (uint64_t)a.seed
                                     : ((uint64_t)time(NULL) << 20) ^ (uint64_t)getpid() ^ (uint64_t)clock();
  cs_arguments_output(&a);
  pop_time(T_SETUP);

  push_time(T_GEOM);
  char err[512];
  if (cs_read_model(a.geometry_file, a.model_file, &R.m, &R.mem, err, sizeof err)) die("*** ERROR: %s\n", err);
  const csp_model* m = &R.m;
  const double dVg = m->h_geom * m->h_geom * m->h_geom;
  for (size_t i = 0, n = (size_t)m->N[0] * m->N[1] * m->N[2]; i < n; i++)
    if (m->voxels[i] < m->num_domains) R.domain_num[m->voxels[i]]++;
  for (int d = 0; d < m->num_domains; d++) R.volumes[d] = R.domain_num[d] * dVg;
  if (a.verbose) output_geometry(&R);
  pop_time(T_GEOM);

  push_time(T_SETUP);
  /* -O lists against the boundary sizes (calcium_sparks.c:126-146) */
  for (int i = 0; i < a.states_info_length; i++) {
    const int b = boundary_id(&R, a.states_info[i].name);
    if (b < 0) die("*** ERROR: \"%s\" is not a valid boundary name.\n", a.states_info[i].name);
    if (a.states_info[i].max_ind >= m->boundaries[b].num_pairs)
      die("*** ERROR: Expected max %s indices given by option --force_discrete_boundaries_open: %d to be lower "
          "than the number of %s boundaries: %d\n", a.states_info[i].name, a.states_info[i].max_ind,
          a.states_info[i].name, m->boundaries[b].num_pairs);
  }
  pop_time(T_SETUP);

  push_time(T_SPECIES);
  char all[1024];
  species_list(&R, all, sizeof all);
  for (int i = 0; i < a.num_save_species; i++) {
    const int s = species_id(&R, a.species[i]);
    if (s < 0)
      die("*** ERROR: Expected given save species to be present in the model loaded from file. \n\"%s\" cannot "
          "be found in [%s].\n", a.species[i], all);
    if (R.nsave < (int)(sizeof R.save_sp / sizeof R.save_sp[0])) R.save_sp[R.nsave++] = s;
  }
  for (int i = 0; i < a.all_data_num_species; i++) {
    const int s = species_id(&R, a.all_data_species[i]);
    if (s < 0)
      die("*** ERROR: Expected given save species to be present in the model loaded from file. \n\"%s\" cannot "
          "be found in [%s].\n", a.all_data_species[i], all);
    if (R.nall < (int)(sizeof R.all_sp / sizeof R.all_sp[0])) R.all_sp[R.nall++] = s;
  }
  csp_options o;
  csp_options_default(&o);
  o.h = a.h;
  o.dt = a.dt;
  o.tstop = a.tstop;
  o.dt_save = a.dt_save;
  o.dt_update_react = a.dt_update_react;
  o.dt_update_stoch = a.dt_update_stoch;
  o.tabort = 0.0;                  /* the abort rule runs here, on the output snapshots */
  o.force_dirichlet = a.force_dirichlet;
  o.seed_given = 1;
  o.seed = seed;
  if (a.states_info_length > CSP_MAX_BOUNDARIES || a.num_t_close > CSP_MAX_BOUNDARIES)
    die("*** ERROR: more than %d -O / -C boundary lists\n", CSP_MAX_BOUNDARIES);
  o.num_open_lists = a.states_info_length;
  for (int i = 0; i < a.states_info_length; i++) {
    snprintf(o.open[i].name, CSP_NAME_LEN, "%s", a.states_info[i].name);
    o.open[i].count = a.states_info[i].count;
    o.open[i].indices = a.states_info[i].idx;
  }
  o.num_t_close = a.num_t_close;
  for (int i = 0; i < a.num_t_close; i++) {
    snprintf(o.t_close[i].name, CSP_NAME_LEN, "%s", a.t_close[i].name);
    o.t_close[i].time = a.t_close[i].time;
  }
  check(NULL, csp_create(m, &o, 1, &R.h), "csp_create");
  check(R.h, csp_get_info(R.h, 0, &R.info), "csp_get_info");
  {
    /* the voxel kernel's tile shape for this grid, timed once (the fields are the same
       for every shape); without a fitting shape the default stays */
    csp_tune_report tr;
    (void)csp_autotune(R.h, 3, &tr);
  }
  const int* n = R.info.n;
  R.h_sim = R.info.h;
  /* sheets (species.c:790-830): default z = (N_z/2 - subdivisions/2) h */
  if (a.num_save_species) {
    if (a.num_ax_points[0] + a.num_ax_points[1] + a.num_ax_points[2] == 0) {
      a.num_ax_points[2] = 1;
      a.ax_points[2] = malloc(sizeof(double));
      a.ax_points[2][0] = (double)(n[2] / 2 - R.info.subdivisions / 2) * R.h_sim;
    }
    for (int ax = 0; ax < 3; ax++) {
      if (a.num_ax_points[ax] > 64) die("*** ERROR: more than 64 sheets along one axis\n");
      R.sheets[ax] = a.num_ax_points[ax];
      for (int i = 0; i < a.num_ax_points[ax]; i++) {
        const double c = a.ax_points[ax][i];
        if (c <= 0 || c >= n[ax] * R.h_sim)
          die("*** ERROR: Expected given z coordinate for save species to be within: (0,%f), got: %f.\n",
              n[ax] * R.h_sim, c);
        R.sheet_idx[ax][i] = (int)floor(c / R.h_sim);
      }
    }
  }
  /* linescan (species.c:838-880) */
  if (a.linescan) {
    R.ls_species = species_id(&R, a.linescan->species);
    if (R.ls_species < 0) die("*** ERROR: \"%s\" is not a valid species name.\n", a.linescan->species);
    for (int i = 0; i < a.linescan->num_domains; i++) {
      R.ls_dom_ids[i] = domain_id(&R, a.linescan->domains[i]);
      if (R.ls_dom_ids[i] < 0) die("*** ERROR: \"%s\" is not a valid domain name.\n", a.linescan->domains[i]);
    }
    for (int ax = 0; ax < 3; ax++) {
      const int lim0 = n[ax] / 2, lim1 = n[ax] - lim0 - 1;
      if (ax != a.linescan->axis && (a.linescan->offsets[ax] < -lim0 || a.linescan->offsets[ax] > lim1))
        die("*** ERROR: Expected given relative positions for convolution to be within: [%d, %d], got: %d.\n",
            -lim0, lim1, a.linescan->offsets[ax]);
      R.ls_offsets_nm[ax] = (lim0 + a.linescan->offsets[ax]) * R.h_sim;
    }
  }
  /* discrete boundaries in boundary order (the order of csp_reduce_outputs' openness) */
  for (int b = 0; b < m->num_boundaries; b++)
    if (m->boundaries[b].type == CSP_BOUNDARY_DISCRETE) {
      R.disc_b[R.ndisc] = b;
      R.disc_n[R.ndisc] = m->boundaries[b].num_pairs;
      R.nchan += R.disc_n[R.ndisc];
      R.ndisc++;
    }
  R.snapshot = calloc((size_t)(R.nchan ? R.nchan : 1), sizeof(int32_t));
  pop_time(T_SPECIES);

  push_time(T_SETUP);
  const double dt = R.info.dt;
  const long long save_interval = (long long)fmax(1., floor(a.dt_save / dt));
  if (a.verbose) {
    output_init_values(&R);
    output_fluxes(&R);
    output_time_stepping(&R, a.tstop, (size_t)save_interval);
  }
  char path[1024];
  snprintf(path, sizeof path, "%s.h5", a.casename);
  const uint64_t N[3] = {(uint64_t)n[0], (uint64_t)n[1], (uint64_t)n[2]};
  R.out = cs_output_create(path, R.h_sim, N, a.geometry_file, a.model_file);
  if (!R.out) die("*** ERROR: cannot create %s: %s\n", path, cs_output_error());
  pop_time(T_SETUP);

  begin_output(&R, 0, 0.0, 0);
  finish_output(&R);
  unsigned output_ind = 0;

  if (a.verbose) check(R.h, csp_set_phase_timing(R.h, 1), "csp_set_phase_timing");
  push_time(T_MAINLOOP);
  const long long total = R.info.total_steps;
  long long k = 0;       /* steps taken */
  double t = 0.0;        /* the reference's loop variable: t of step k+1 is the sum of k dt */
  int stop = 0;
  while (k < total && !stop) {
    const long long next_out = (k / save_interval + 1) * save_interval;
    const long long end = next_out < total ? next_out : total;
    /* steps before an output step check the rule on the current snapshot */
    const long long scan_end = end == next_out ? end - 1 : end;
    long long run_to = end;
    double tt = t;
    for (long long j = k + 1; j <= scan_end; j++) {
      tt += dt;
      if (abort_check(&R, tt)) {
        run_to = j;
        stop = 1;
        break;
      }
    }
    int32_t flag = 0;
    check(R.h, csp_advance_async(R.h, run_to - k), "csp_advance_async");
    finish_output(&R);          /* the previous output's fields and file, while the device steps */
    check(R.h, csp_advance_wait(R.h, &flag), "csp_advance_wait");
    for (long long j = k; j < run_to; j++) t += dt;
    k = run_to;
    if (stop) break;
    if (k == next_out) {
      begin_output(&R, ++output_ind, t, (uint64_t)k);
      if (abort_check(&R, t)) break;
    }
  }
  finish_output(&R);
  fflush(stdout);
  pop_time(T_MAINLOOP);

  if (cs_output_close(R.out)) die("*** ERROR: output: %s\n", cs_output_error());
  if (a.verbose) {
    double ph[CSP_NUM_PHASES];
    int64_t nst = 0;
    check(R.h, csp_get_phase_times(R.h, ph, &nst), "csp_get_phase_times");
    const struct { int bucket; double ms; } map[] = {
        {T_DIFF, ph[CSP_PHASE_VOXELS]}, {T_BOUNDARIES, ph[CSP_PHASE_DENSITY] + ph[CSP_PHASE_EPILOGUE]},
        {T_STOCH, ph[CSP_PHASE_CHANNELS]}, {T_REACT, ph[CSP_PHASE_SURROGATE]}, {T_DIFFTOT, ph[CSP_PHASE_VOXELS]}};
    for (size_t i = 0; i < sizeof map / sizeof map[0]; i++) {
      tval[map[i].bucket] = map[i].ms / 1e3;
      tcalls[map[i].bucket] = (unsigned)nst;
    }
  }
  csp_destroy(R.h);
  free(R.snapshot);
  cs_model_mem_free(&R.mem);
  pop_time(T_SIM);
  if (a.verbose) output_timings();
  cs_arguments_free(&a);
  return 0;
}
