/*
 * csp_options.c -- the calcium_sparks command line (see csp_options.h).
 *
 * Multi-token options consume the following arguments up to the next one that starts
 * with '-' (options.c:68-80, 85-100, 211-214); -l also takes negative numbers as its
 * offsets.  -O groups its tokens into boundary names (tokens that atoi reads as 0 and
 * that are not "0") followed by their increasing, non-negative channel indices
 * (options.c:221-311).  -C takes name / time pairs (options.c:161-214).
 */
#define _GNU_SOURCE
#include "csp_options.h"

#include <argp.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

const char* argp_program_version = "calcium_sparks (B200) 0.1";

static void die(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vfprintf(stderr, fmt, ap);
  va_end(ap);
  fflush(stdout);
  exit(1);
}

static void* xmalloc(size_t n) {
  void* p = malloc(n ? n : 1);
  if (!p) die("Error: Malloc failed for process 0\n");
  return p;
}

int cs_mod(int dividend, int divisor) {
  return dividend - divisor * (int)floor(1.0 * dividend / divisor);
}

void cs_linescan_axes(int axis, int* one, int* two) {
  const int sgn = (axis % 2 == 0) ? 1 : -1;   /* (int)pow(-1, axis) */
  *one = cs_mod(axis + sgn, 3);
  *two = cs_mod(axis + 2 * sgn, 3);
}

void cs_arguments_default(cs_arguments* a) {
  memset(a, 0, sizeof *a);
  a->casename = "casename";
  a->tstop = 10.;
  a->h = 6.;
  a->dt_save = .5;
  a->dt = -1.;
  a->dt_update_react = -1.;
  a->dt_update_stoch = -1.;
  a->split_plane = CS_SPLIT_XY;
}

/* a token atoi reads as 0 that is not "0": a name (options.c:228-231) */
static int is_name(const char* s) { return atoi(s) == 0 && s[0] != '0'; }

/* number of tokens after the current option argument up to the next '-' token */
static int count_following(struct argp_state* st) {
  int off = 0;
  while (st->argv[st->next + off] != NULL && st->argv[st->next + off][0] != '-') off++;
  return off;
}

static void parse_open(struct argp_state* st, cs_arguments* a) {
  char** first = &st->argv[st->next - 1];
  if (!is_name(first[0]))
    die("*** Error: Expected a string as the first argument for --open option. Instead got: %s.\n", first[0]);
  const int off = count_following(st);
  const int ntok = off + 1;
  if (atoi(first[ntok - 1]) == 0 && strcmp(first[ntok - 1], "0") != 0)
    die("*** Error: Expected an integer as the last argument for --force_discrete_boundaries_open "
        "option.Instead got: %s.\n", first[ntok - 1]);
  int nlists = 0;
  for (int i = 0; i < ntok; i++) nlists += is_name(first[i]);
  cs_open_info* lists = xmalloc(sizeof(cs_open_info) * (size_t)(a->states_info_length + nlists));
  if (a->states_info_length) memcpy(lists, a->states_info, sizeof(cs_open_info) * (size_t)a->states_info_length);
  free(a->states_info);
  a->states_info = lists;
  int i = 0;
  while (i < ntok) {
    cs_open_info* L = &a->states_info[a->states_info_length++];
    L->name = first[i++];
    int j = i;
    while (j < ntok && !is_name(first[j])) j++;
    L->count = j - i;
    L->idx = xmalloc(sizeof(int) * (size_t)L->count);
    L->max_ind = 0;
    for (int k = 0; k < L->count; k++) {
      L->idx[k] = atoi(first[i + k]);
      if (L->idx[k] < 0)
        die("***Error: Expected a positive number for the open indices given by "
            "--force_discrete_boundaries_open option. For %s got %d.\n", L->name, L->idx[k]);
      if (L->idx[k] > L->max_ind) L->max_ind = L->idx[k];
      if (k > 0 && L->idx[k] <= L->idx[k - 1])
        die("***Error: Expected a monotonicly increasing numbers for the open states indices given by "
            "--force_discrete_boundaries_open option. For %s got %d and %d.\n", L->name, L->idx[k - 1],
            L->idx[k]);
    }
    i = j;
  }
  st->next += off;
}

static void parse_t_close(struct argp_state* st, cs_arguments* a) {
  char** first = &st->argv[st->next - 1];
  const int off = count_following(st);
  const int nargs = off + 1;
  if (nargs % 2 != 0)
    die("*** Error: Incorrect number of provided arguments for --t_close option. Expects an even "
        "positive number. Instead found %d provided arguments.\n", nargs);
  const int n = nargs / 2;
  a->t_close = realloc(a->t_close, sizeof(cs_action_time) * (size_t)(a->num_t_close + n));
  if (!a->t_close) die("Error: Malloc failed for process 0\n");
  for (int k = 0; k < nargs; k++) {
    if (k % 2 == 0) {
      if (!is_name(first[k]))
        die("Error: Expected a string on the  %d arguments for --t_close option. Instead got: %s.\n", k + 1,
            first[k]);
      a->t_close[a->num_t_close + k / 2].name = first[k];
    } else {
      double v = atof(first[k]);
      if (v == 0.0 && strcmp(first[k], "0") != 0 && strcmp(first[k], "0.0") != 0)
        die("Error: Expected a REAL number on the %d arguments for --t_close option. Instead got: %s.\n", k + 1,
            first[k]);
      a->t_close[a->num_t_close + k / 2].time = v;
    }
  }
  a->num_t_close += n;
  st->next += off;
}

static void parse_linescan(struct argp_state* st, cs_arguments* a) {
  char** args = &st->argv[st->next - 1];
  int off = 0;
  /* further tokens: anything not starting with '-', or a negative number */
  while (st->argv[st->next + off] != NULL &&
         (st->argv[st->next + off][0] != '-' ||
          (st->argv[st->next + off][1] >= '0' && st->argv[st->next + off][1] <= '9')))
    off++;
  const int nargs = off + 1;
  if (nargs < 4)
    die("*** Error: Incorrect number of provided arguments for --linescan option. Expects at least 4, but"
        "instead found %d.\n", nargs);
  if (strlen(args[0]) != 1 || (args[0][0] != 'x' && args[0][0] != 'y' && args[0][0] != 'z'))
    die("*** Error: Expects axis x,y or z as the first argument passed to --linescan (-l). Instead got: %s\n",
        args[0]);
  cs_linescan* L = xmalloc(sizeof(cs_linescan));
  memset(L, 0, sizeof *L);
  L->axis = args[0][0] - 'x';
  L->species = args[1];
  L->num_domains = nargs - 4;
  L->domains = L->num_domains ? xmalloc(sizeof(char*) * (size_t)L->num_domains) : NULL;
  for (int i = 0; i < L->num_domains; i++) L->domains[i] = args[2 + i];
  int one, two;
  cs_linescan_axes(L->axis, &one, &two);
  L->offsets[one] = atoi(args[2 + L->num_domains]);
  L->offsets[two] = atoi(args[3 + L->num_domains]);
  if (a->linescan) {
    free(a->linescan->domains);
    free(a->linescan);
  }
  a->linescan = L;
  st->next += off;
}

static void parse_mpi_dist(struct argp_state* st, cs_arguments* a) {
  a->mpi_dist_given = 1;
  a->mpi_prod = 1;
  for (int k = 0; k < 3; k++) {
    const char* s = st->argv[st->next - 1 + k];
    if (s == NULL || s[0] == '-')
      die("*** Error: Excpected three positive integers after the --mpi_dist option. Found only %d\n", k);
    a->mpi_dist[k] = (unsigned)atoi(s);
    if (atoi(s) < 1)
      die("*** Error: Encountered a wrong number at position %d for the --mpi_dist option. Expected an "
          "integer > 0.\n", k + 1);
    a->mpi_prod *= a->mpi_dist[k];
  }
  st->next += 2;
}

enum { OPT_ALL_DATA = 777, OPT_MPI_DIST = 778 };

static struct argp_option options[] = {
    {"casename", 'c', "CASENAME", 0, "Sets the name of the run to CASENAME. Default (\"casename\")", 0},
    {"dt", 'd', "TIME", 0, "Forced minimal timestep. If negative time step will be deducted from diffusion "
                           "constants. Default(-1.)", 0},
    {"force_dirichlet", 'f', 0, 0, "Force to use Dirichlet boundary condition.", 0},
    {"geometry_file", 'g', "FILE", 0, "Read the geometry from FILE. Expects a .h5 file.", 0},
    {"resolution", 'h', "RES", 0, "Run simulation with RES nm as the spatial resolution. Default(6.)", 0},
    {"species_file", 'm', "FILE", 0, "Read the species model from FILE. Expects a .h5 file.", 0},
    {"dt_save", 'o', "TIME", 0, "Save solution for each dt_save. Default(.5)", 0},
    {"split_processes", 'p', "PLANE", 0, "Split processes in given directions {XY, YZ, XZ}. Default(XY). "
                                         "Checked and ignored: one GPU holds the whole domain.", 0},
    {"quiet", 'q', 0, 0, "Don't produce any output", 0},
    {"save_species", 's', "SPECIES", 0, "A list of species that should be saved in 2D sheets at given "
                                        "z-coordinates.", 0},
    {"tstop", 't', "TIME", 0, "Run simulation for TIME number of ms. Default(10.)", 0},
    {"verbose", 'v', 0, 0, "Produce verbose output", 0},
    {"save_x_coords", 'x', "COORD", 0, "X coordinates for the 2D sheet that will be saved.", 0},
    {"save_y_coords", 'y', "COORD", 0, "Y coordinates for the 2D sheet that will be saved.", 0},
    {"save_z_coords", 'z', "COORD", 0, "Z coordinates for the 2D sheet that will be saved.", 0},
    {"linescan", 'l', "DIR_SPCECIES_COORD", 0, "Computes convolution of the species with 3-D Gaussian "
                                               "function.", 0},
    {"t_close", 'C', "TIME", 0, "Time for closing currents. If negative, they are closed stochastically. "
                                "Default (-1)", 0},
    {"dt_update_stoch", 'D', "TIME", 0, "Time step for updating the stochastics. If negative it will be the "
                                        "same as global timestep. Default (-1)", 0},
    {"open", 'O', "OPEN_STATES", 0, "Initialize given discrete fluxes to open. Otherwise they are randomly "
                                    "initialized.", 0},
    {"seed", 'S', "SEED", 0, "Provide a seed for the random generator. If not given the seed will be random "
                             "each run.", 0},
    {"dt_update_react", 'T', "TIME", 0, "Time step for updating the reactions. If negative it will be the "
                                        "same as global timestep. Default (-1)", 0},
    {"abort", 'X', "TYPE TIME", 0, "Abort simulations after TIME ms after the last RyR channel has been "
                                   "closed. By default it is inactive.", 0},
    {"all_data", OPT_ALL_DATA, "SPECIES", 0, "Save species values of all points (3D)", 0},
    {"mpi_dist", OPT_MPI_DIST, "MPI_DIST", 0, "An mpi distribution for processor splitting in XYZ "
                                              "directions. Checked and ignored on one GPU.", 0},
    {0}};

static error_t parse_opt(int key, char* arg, struct argp_state* st) {
  cs_arguments* a = st->input;
  int off, ax;
  switch (key) {
    case 'c': a->casename = arg; break;
    case 'd': a->dt = atof(arg); break;
    case 'f': a->force_dirichlet = 1; break;
    case 'g': a->geometry_file = arg; break;
    case 'h': a->h = atof(arg); break;
    case 'm': a->model_file = arg; break;
    case 'o': a->dt_save = atof(arg); break;
    case 'p':
      if (strcmp(arg, "XY") == 0) a->split_plane = CS_SPLIT_XY;
      else if (strcmp(arg, "YZ") == 0) a->split_plane = CS_SPLIT_YZ;
      else if (strcmp(arg, "XZ") == 0) a->split_plane = CS_SPLIT_XZ;
      else if (strcmp(arg, "XYZ") == 0) a->split_plane = CS_SPLIT_XYZ;
      else die("***Error: Expected argument for option -p is one of {XY, XZ, YZ}. Instead got %s\n", arg);
      break;
    case 'q': a->silent = 1; break;
    case 's':
      off = count_following(st);
      a->species = &st->argv[st->next - 1];
      a->num_save_species = off + 1;
      st->next += off;
      break;
    case 't': a->tstop = atof(arg); break;
    case 'v': a->verbose = 1; break;
    case 'x': case 'y': case 'z':
      ax = key - 'x';
      off = count_following(st);
      free(a->ax_points[ax]);
      a->num_ax_points[ax] = off + 1;
      a->ax_points[ax] = xmalloc(sizeof(double) * (size_t)(off + 1));
      for (int i = 0; i <= off; i++) a->ax_points[ax][i] = atof(st->argv[st->next - 1 + i]);
      st->next += off;
      break;
    case 'l': parse_linescan(st, a); break;
    case 'C': parse_t_close(st, a); break;
    case 'D': a->dt_update_stoch = atof(arg); break;
    case 'O': parse_open(st, a); break;
    case 'S': a->seed = (uint32_t)atoi(arg); a->seed_given = 1; break;
    case 'T': a->dt_update_react = atof(arg); break;
    case 'X': a->tabort = atof(arg); break;
    case OPT_ALL_DATA:
      off = count_following(st);
      a->all_data_species = &st->argv[st->next - 1];
      a->all_data_num_species = off + 1;
      st->next += off;
      break;
    case OPT_MPI_DIST: parse_mpi_dist(st, a); break;
    case ARGP_KEY_ARG: argp_usage(st); break;
    default: return ARGP_ERR_UNKNOWN;
  }
  return 0;
}

static struct argp argp_def = {options, parse_opt, 0,
                               "calcium_spark -- A finite volume program modeling a calcium spark simulation", 0, 0,
                               0};

void cs_parse_arguments(int argc, char** argv, cs_arguments* a) {
  argp_parse(&argp_def, argc, argv, 0, 0, a);
  /* one process: the reference's process-count checks (calcium_sparks.c:75-97) for size 1 */
  if (a->mpi_dist_given && a->mpi_prod != 1)
    die("*** Error: --mpi_dist option was used. Expected the number of processes to be equal to %d. "
        "Instead got %d.\n", a->mpi_prod, 1);
  if (!a->geometry_file) die("*** ERROR: Expected a geometry file passed as argument: --geometry_file or -g\n");
  if (!a->model_file) die("*** ERROR: Expected a species file passed as argument: --species_file or -m\n");
  if (a->verbose) a->silent = 0;
}

void cs_arguments_output(const cs_arguments* a) {
  if (a->silent) return;
  const char coord[3] = {'x', 'y', 'z'};
  printf("\n");
  printf("Arguments:\n");
  printf("-----------------------------------------------------------------------------\n");
  printf("  casename:          \"%s\"\n", a->casename);
  printf("  geometry_file:     \"%s\"\n", a->geometry_file);
  printf("  species_file:      \"%s\"\n", a->model_file);
  printf("  tstop:             %.6f ms\n", a->tstop);
  printf("  h:                 %.1f nm\n", a->h);
  printf("  dt:                %.3g\n", a->dt);
  printf("  dt_save:           %.3g\n", a->dt_save);
  printf("  dt_update_stoch:   %.3g\n", a->dt_update_stoch);
  printf("  dt_update_react:   %.3g\n", a->dt_update_react);
  printf("  t_close:           %s", a->num_t_close ? "" : "-");
  for (int i = 0; i < a->num_t_close; i++) {
    printf("%s %.3g", a->t_close[i].name, a->t_close[i].time);
    if (i < a->num_t_close - 1) printf(", ");
  }
  printf("\n");
  printf("  linescan:          %s", a->linescan ? "" : "-\n");
  if (a->linescan) {
    int one, two;
    cs_linescan_axes(a->linescan->axis, &one, &two);
    printf("%c, %s, %d, %d\n", coord[a->linescan->axis], a->linescan->species, a->linescan->offsets[one],
           a->linescan->offsets[two]);
  }
  printf("  abort simulations:%s", a->tabort != 0.0 ? "" : "-\n");
  if (a->tabort != 0.0) printf("%.3g\n", a->tabort);
  printf("  save_2D_species:   %s", a->num_save_species ? "" : "-");
  for (int i = 0; i < a->num_save_species; i++) {
    printf("%s", a->species[i]);
    if (i < a->num_save_species - 1) printf(", ");
  }
  printf("\n");
  if (a->num_save_species) {
    if (a->num_ax_points[0] + a->num_ax_points[1] + a->num_ax_points[2] == 0) {
      printf("   z-coords (nm):   center\n");
    } else {
      for (int ax = 0; ax < 3; ax++)
        if (a->num_ax_points[ax]) {
          printf("    %c-coords (nm):   ", coord[ax]);
          for (int i = 0; i < a->num_ax_points[ax]; i++) {
            printf("%.2f", a->ax_points[ax][i]);
            if (i < a->num_ax_points[ax] - 1) printf(", ");
          }
          printf("\n");
        }
    }
  }
  printf("  save_all_data:     %s", a->all_data_num_species ? "" : "-");
  for (int i = 0; i < a->all_data_num_species; i++) {
    printf("%s", a->all_data_species[i]);
    if (i < a->all_data_num_species - 1) printf(", ");
  }
  printf("\n");
  printf("  open states:       %s", a->states_info_length ? "" : "-");
  for (int i = 0; i < a->states_info_length; i++) {
    if (i > 0) printf("                   ");
    printf("%s: ", a->states_info[i].name);
    for (int j = 0; j < a->states_info[i].count; j++) {
      printf("%d", a->states_info[i].idx[j]);
      if (j < a->states_info[i].count - 1) printf(", ");
    }
    printf("\n");
  }
  printf("\n\n");
}

void cs_arguments_free(cs_arguments* a) {
  for (int i = 0; i < 3; i++) free(a->ax_points[i]);
  free(a->t_close);
  for (int i = 0; i < a->states_info_length; i++) free(a->states_info[i].idx);
  free(a->states_info);
  if (a->linescan) {
    free(a->linescan->domains);
    free(a->linescan);
  }
  memset(a, 0, sizeof *a);
}
