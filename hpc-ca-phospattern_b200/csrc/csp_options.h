/*
 * csp_options.h -- command line of the calcium_sparks driver (bin/calcium_sparks).
 *
 * The option set, defaults and multi-token rules are those of the reference program
 * (fvm_mpi/src/calcium_sparks.c:19-45, options.c:13-393, defaults options.c:502-542):
 *   -c CASENAME  -d TIME  -f  -g FILE  -h RES  -m FILE  -o TIME  -p PLANE  -q  -v
 *   -s SP ...   -t TIME  -x C ...  -y C ...  -z C ...  -l AXIS SP [DOMAINS...] OFF1 OFF2
 *   -C NAME T ...  -D TIME  -O NAME I J ... [NAME I ...]  -S SEED  -T TIME  -X TIME
 *   --all_data SP ...   --mpi_dist NX NY NZ
 * A run uses one GPU: -p and --mpi_dist are checked as the reference checks them for a
 * single process and otherwise ignored.  Errors print the reference's message to stderr
 * and exit with status 1 (the reference's MPI_Abort(comm, 1)).
 */
#ifndef CSP_OPTIONS_H
#define CSP_OPTIONS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { CS_SPLIT_XY = 0, CS_SPLIT_YZ, CS_SPLIT_XZ, CS_SPLIT_XYZ };

/* one "-O name i j ..." list (options.h:21-26) */
typedef struct cs_open_info {
  char* name;
  int count;
  int max_ind;
  int* idx;
} cs_open_info;

/* one "-C name t" pair (options.h:30-34) */
typedef struct cs_action_time {
  char* name;
  double time;
} cs_action_time;

/* "-l axis species [domains...] off1 off2" (options.h:38-45) */
typedef struct cs_linescan {
  int axis;                /* 0 x, 1 y, 2 z */
  char* species;
  char** domains;
  int num_domains;
  int offsets[3];          /* relative positions of the two fixed axes (voxels from the centre) */
} cs_linescan;

typedef struct cs_arguments {
  double tstop, h;
  int silent, verbose, force_dirichlet;
  double dt_save;
  int seed_given;
  uint32_t seed;
  int split_plane;
  cs_action_time* t_close;
  int num_t_close;
  double dt_update_react, dt_update_stoch, dt, tabort;
  char** species;          /* -s */
  int num_save_species;
  char** all_data_species; /* --all_data */
  int all_data_num_species;
  int num_ax_points[3];    /* -x / -y / -z */
  double* ax_points[3];
  char* geometry_file;
  char* model_file;
  char* casename;
  cs_open_info* states_info;
  int states_info_length;
  cs_linescan* linescan;
  int mpi_dist_given;
  unsigned mpi_dist[3];
  unsigned mpi_prod;
} cs_arguments;

void cs_arguments_default(cs_arguments* a);
/* parse argv; exits with status 1 on the errors the reference reports */
void cs_parse_arguments(int argc, char** argv, cs_arguments* a);
/* the "Arguments:" listing (arguments_output, options.c:395-500) */
void cs_arguments_output(const cs_arguments* a);
void cs_arguments_free(cs_arguments* a);
/* floored modulo (utils.c:215-218) */
int cs_mod(int dividend, int divisor);
/* the two fixed axes of a linescan along `axis`, in the reference's order */
void cs_linescan_axes(int axis, int* one, int* two);

#ifdef __cplusplus
}
#endif
#endif
