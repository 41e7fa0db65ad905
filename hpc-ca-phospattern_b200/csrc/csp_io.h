/*
 * csp_io.h -- the calcium_sparks driver's files: the reference's geometry and species
 * HDF5 inputs read into a csp_model, and the <casename>.h5 output it writes.
 *
 * Inputs (geometry.c:96-344, species.c:103-258, boundaryfluxes.c:377-527):
 *   geometry: root attrs h, global_size; /domains (num, name_i, indices; datasets voxels,
 *   domain_connections); /boundaries (num, name_i, type_i; one uint16 [n][6] dataset per
 *   boundary).
 *   species: root attrs num_species, species_name_i, num_fixed_domain_species,
 *   fixed_domain_species, convolution_constants, use_ryr / use_p_ryr / use_serca; one
 *   group per domain (init, num_diffusive, diffusive, sigma, num_buffers, buffer_i/{k_on,
 *   k_off, tot, species}); /ryr, /p_ryr, /serca parameter groups.
 * Output (species.c:2253-2551, 2785-3092):
 *   root attrs h (f64[1]), N (u64[3]), geometry_file, species_file (strings);
 *   /data_%07d with attrs time (f64[1]), time_index (u64[1]); <domain>/<species> groups
 *   with min, max, average (f64[1]); discrete_<boundary> (f64[n]); optional
 *   <sp>_<x|y|z>_sheet_<i> (f64 2-D), <sp>_all_data (f64 3-D) and
 *   linescan_<sp>_<doms><a>_<o1>_<b>_<o2> (f64 1-D).
 */
#ifndef CSP_IO_H
#define CSP_IO_H

#include <stdint.h>

#include "csparks.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Arrays a csp_model points to. */
typedef struct cs_model_mem {
  uint8_t* voxels;
  uint16_t* pairs[CSP_MAX_BOUNDARIES];
} cs_model_mem;

/* Read both files; returns 0, or -1 with a message in err. */
int cs_read_model(const char* geometry_file, const char* species_file, csp_model* m, cs_model_mem* mem,
                  char* err, size_t nerr);
void cs_model_mem_free(cs_model_mem* mem);

typedef struct cs_output cs_output;

/* Create <path> with the root attributes (species.c:2272-2281). */
cs_output* cs_output_create(const char* path, double h, const uint64_t N[3], const char* geometry_file,
                            const char* species_file);
/* Start group /data_%07d (species.c:2287-2292). */
int cs_output_group(cs_output* o, unsigned output_ind, double t, uint64_t time_ind);
/* <group>/<domain>/<species> with max, min, average */
int cs_output_scalar(cs_output* o, const char* domain, const char* species, double mn, double mx, double avg);
/* a 1-D .. 3-D f64 dataset in the current group */
int cs_output_dataset(cs_output* o, const char* name, int ndims, const uint64_t* dims, const double* data);
/* write the file as it stands (the reference closes the file after every output) */
int cs_output_flush(cs_output* o);
int cs_output_close(cs_output* o);
const char* cs_output_error(void);

#ifdef __cplusplus
}
#endif
#endif
