/*
 * csparks.h -- C ABI of the B200 calcium_sparks time step (libcsparks_cuda.so).
 *
 * The reference program (ComputationalPhysiology/hpc-ca-phospattern, fvm_mpi/) advances
 * its reaction-diffusion state through the host-memory FP64 kernels declared in
 * fvm_mpi/src/kernel.h:2-18 and the step drivers of fvm_mpi/src/species.c.  This
 * library replaces that step with sm_100a CUDA kernels: the whole domain (or an
 * ensemble of independent realisations) lives in HBM, and one call advances it by any
 * number of steps.  The host owns every input array; the library owns device memory.
 *
 * Conventions
 *   - every int-returning call returns 0 (CSP_OK) or a negative CSP_E* code; nothing
 *     aborts the process.  csp_status() gives a message for the last error.
 *   - calls on one handle are ordered on one internal CUDA stream; the handle is not
 *     thread safe.
 *   - fields are C order [x][y][z] with z fastest, index x*ny*nz + y*nz + z
 *     (species.c:1513), one array per species, species-major ([species][x][y][z]).
 *   - units: concentration uM, time ms, length nm, sigma nm^2/ms.
 */
#ifndef CSPARKS_H
#define CSPARKS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CSP_MAX_DOMAINS    5   /* max_num_domains, kernel_generic.cpp:11 */
#define CSP_MAX_SPECIES    8
#define CSP_MAX_BUFFERS    8
#define CSP_MAX_BOUNDARIES 8
#define CSP_MAX_FIXED      8
#define CSP_NAME_LEN       20  /* MAX_SPECIES_NAME, types.h:10 */

enum {
  CSP_OK = 0,
  CSP_EINVAL = -1,      /* bad argument / inconsistent model */
  CSP_ENOMEM = -2,      /* device or host allocation failed */
  CSP_ECUDA = -3,       /* CUDA runtime error */
  CSP_ERANGE = -4,      /* index out of range (realisation, channel, -O index) */
  CSP_EDEVICE = -5,     /* device-side error word set (bounds / timeout) */
  CSP_ENOTSUP = -6      /* a model feature this build does not support */
};

enum { CSP_BOUNDARY_DENSITY = 0, CSP_BOUNDARY_DISCRETE = 1 };  /* geometry.h:46 */

/* One boundary of the geometry file: /boundaries/<name>, uint16 [n][6] voxel pairs
 * (x0,y0,z0,x1,y1,z1) in geometry voxels (geometry.c:239-259, 576-620). */
typedef struct csp_boundary {
  char name[CSP_NAME_LEN];
  int32_t type;                 /* CSP_BOUNDARY_DENSITY | CSP_BOUNDARY_DISCRETE */
  int32_t num_pairs;
  const uint16_t* pairs;        /* [num_pairs][6] */
} csp_boundary;

/* Per-domain part of the species file, group /<domain_name> (species.c:171-241). */
typedef struct csp_domain_species {
  int32_t num_diffusive;
  uint8_t diffusive[CSP_MAX_SPECIES];   /* species indices */
  double sigma[CSP_MAX_SPECIES];        /* sigma[k] belongs to diffusive[k] */
  double init[CSP_MAX_SPECIES];         /* initial value of every species */
  int32_t num_buffers;
  double k_on[CSP_MAX_BUFFERS];
  double k_off[CSP_MAX_BUFFERS];
  double tot[CSP_MAX_BUFFERS];
  uint8_t bsp0[CSP_MAX_BUFFERS];        /* bound buffer species (attr "species"[0]) */
  uint8_t bsp1[CSP_MAX_BUFFERS];        /* free ligand species (attr "species"[1]) */
} csp_domain_species;

/* RyR / pRyR group of the species file (boundaryfluxes.c:421-503). */
typedef struct csp_ryr_params {
  double Kd_open, k_min_open, k_max_open, n_open;
  double Kd_close, k_min_close, k_max_close, n_close;
  double i_unitary;                     /* pA */
  char boundary[CSP_NAME_LEN];
  char species[CSP_NAME_LEN];
} csp_ryr_params;

/* SERCA group of the species file (boundaryfluxes.c:506-527).  The reference reads the
 * SERCA species name from the /ryr group (boundaryfluxes.c:511); loaders fill
 * `species` the same way. */
typedef struct csp_serca_params {
  double v_cyt_to_A_sr, density, scale;
  char boundary[CSP_NAME_LEN];
  char species[CSP_NAME_LEN];
} csp_serca_params;

/* Everything the geometry file and the species file of one realisation hold. */
typedef struct csp_model {
  /* geometry file (geometry.c:96-344) */
  double h_geom;                        /* root attr "h" */
  double global_size[3];                /* root attr "global_size" */
  int32_t N[3];                         /* shape of /domains/voxels */
  int32_t num_domains;
  char domain_names[CSP_MAX_DOMAINS][CSP_NAME_LEN];
  uint8_t domain_indices[CSP_MAX_DOMAINS];
  const uint8_t* voxels;                /* [N0][N1][N2] domain ids */
  uint8_t domain_connections[CSP_MAX_DOMAINS * CSP_MAX_DOMAINS];  /* [num][num] */
  int32_t num_boundaries;
  csp_boundary boundaries[CSP_MAX_BOUNDARIES];
  /* species file (species.c:103-258, boundaryfluxes.c:377-527) */
  int32_t num_species;
  char species_names[CSP_MAX_SPECIES][CSP_NAME_LEN];
  csp_domain_species domain[CSP_MAX_DOMAINS];
  int32_t num_fixed_domain_species;
  uint8_t fixed_domain_species[2 * CSP_MAX_FIXED];  /* (domain, species) pairs */
  uint8_t use_ryr, use_p_ryr, use_serca;
  csp_ryr_params ryr, p_ryr;
  csp_serca_params serca;
  double convolution_constants[3];
} csp_model;

/* One "-O name i j ..." list (options.c:221-311). */
typedef struct csp_open_list {
  char name[CSP_NAME_LEN];
  int32_t count;
  const int32_t* indices;
} csp_open_list;

/* One "-C name t" pair (options.c:161-214). */
typedef struct csp_t_close {
  char name[CSP_NAME_LEN];
  double time;
} csp_t_close;

/* The command-line arguments that reach the time step (options.h:47-137,
 * defaults options.c:502-542). */
typedef struct csp_options {
  double h;                 /* -h requested resolution, nm (default 6) */
  double dt;                /* -d; <= 0 selects 0.95*h^2/(6*sigma_max) */
  double tstop;             /* -t, ms (default 10) */
  double dt_save;           /* -o, ms (default 0.5) */
  double dt_update_react;   /* -T (default -1) */
  double dt_update_stoch;   /* -D (default -1) */
  double tabort;            /* -X value; 0 = inactive */
  int32_t force_dirichlet;  /* -f */
  int32_t seed_given;       /* -S given */
  uint64_t seed;            /* -S; realisation r draws from Philox key (seed, r) */
  int32_t num_open_lists;
  csp_open_list open[CSP_MAX_BOUNDARIES];
  int32_t num_t_close;
  csp_t_close t_close[CSP_MAX_BOUNDARIES];
  /* Philox stream of the realisation's channel draws = its index in the csp_create batch +
   * stream_offset (0: the batch index).  A realisation run in another batch (a shard of an
   * ensemble on another GPU) draws the same channel trajectory when the offsets make the
   * stream its index in the whole ensemble.  No counterpart in the reference: one MT19937
   * stream per run, seeded by -S (calcium_sparks.c:113-116). */
  int64_t stream_offset;
} csp_options;

/* Fills `o` with the reference defaults (options.c:502-542). */
void csp_options_default(csp_options* o);

/* Derived per-realisation constants (species.c:265-294, 784-787). */
typedef struct csp_info {
  int32_t n[3];             /* species voxels per axis */
  int32_t subdivisions;
  double h;                 /* species resolution, nm */
  double dt;                /* ms */
  int32_t num_species;
  int32_t num_diffusive;
  int32_t diffusive_species[CSP_MAX_SPECIES];
  int32_t substeps[CSP_MAX_SPECIES];
  int32_t num_buffers;      /* num_all_buffers */
  int32_t stochastic_substep;
  int32_t reaction_substep;
  int64_t total_steps;      /* iterations of `for (t=0; t<tstop; t+=dt)` */
  int64_t step;             /* steps already taken */
  int32_t num_channels[CSP_MAX_BOUNDARIES];   /* discrete boundaries, in boundary order */
  int32_t stopped;          /* 1 once the -X rule or total_steps ended the run */
  int64_t fused_pairs;      /* boundary pairs evaluated inside the voxel kernels */
  int64_t flux_rows;        /* voxels updated by the boundary / channel kernel */
} csp_info;

typedef struct csp_handle csp_handle;

/* Select the CUDA device of the calling thread for the handles it creates next (one
 * process per GPU: rank i calls csp_set_device(i) before csp_create). */
int csp_set_device(int32_t device);

/* Build device state for n independent realisations (models[r], options[r]) and set
 * the initial state exactly as the reference does before its time loop
 * (calcium_sparks.c:150-178: Species_init_values, channel init, du := u).
 * Replaces Species_construct + BoundaryFluxes_construct + Species_init_values +
 * BoundaryFluxes_init_stochastic_boundaries + Species_init_du
 * (species.c:95, 887, 22; boundaryfluxes.c:361, 544). */
int csp_create(const csp_model* models, const csp_options* options, int32_t n,
               csp_handle** out);

/* Derived constants and progress of realisation r. */
int csp_get_info(const csp_handle* h, int32_t r, csp_info* info);

/* Overwrite / read the fields of realisation r: u[num_species][nx][ny][nz], FP64 on the
 * host, FP32 on the device.  (The reference keeps these fields in Species_t::u1,
 * species.h:52.) */
int csp_upload_state(csp_handle* h, int32_t r, const double* u);
int csp_download_state(csp_handle* h, int32_t r, double* u);
/* The same for every realisation in one call: u[r] is realisation r's state (n pointers).
 * The copies run back to back with one wait at the end (use page-locked host memory for
 * full link speed). */
int csp_upload_states(csp_handle* h, const double* const* u);
int csp_download_states(csp_handle* h, double* const* u);

/* The same transfers with FP32 host fields (the device precision: the values are those of
 * the FP64 calls, with half the bytes over PCIe).  u[r]: float [num_species][nx][ny][nz]. */
int csp_upload_states_f32(csp_handle* h, const float* const* u);
int csp_download_states_f32(csp_handle* h, float* const* u);

/* One ensemble job from host memory: every realisation's state uploaded from u_in[r],
 * advanced by nsteps steps, downloaded into u_out[r] (u_out may alias u_in), in the layout
 * of csp_upload_states with host_dtype CSP_HOST_F64 or of csp_upload_states_f32 with
 * CSP_HOST_F32.  The fields equal those of upload + csp_advance(nsteps) + download: the
 * realisations are independent, so the call advances them in groups of consecutive
 * realisations (about equal voxels, at most 8 groups) and pipelines the groups on three
 * streams -- the input copies of group g+1 and the output copies of group g-1 overlap the
 * steps of group g.  Use page-locked host memory for the copies to overlap.  stop_flags
 * (nullable, n entries) as csp_advance; step_flags (nullable, [nsteps][n]) receives every
 * realisation's stop flag after every step.  (The reference has no ensemble: its host
 * loop, calcium_sparks.c:190-228, advances one domain held in Species_t::u1,
 * species.h:52.) */
enum { CSP_HOST_F64 = 0, CSP_HOST_F32 = 1 };
int csp_run_states(csp_handle* h, int32_t host_dtype, const void* const* u_in, int64_t nsteps, void* const* u_out,
                   int32_t* stop_flags, int32_t* step_flags);

/* Advance every still-running realisation by up to nsteps steps: diffusion, channel
 * gating, boundary fluxes, reactions, apply and fixed values, in the order of the
 * reference loop body calcium_sparks.c:190-228 (Species_step_diffusion species.c:1501,
 * Species_evaluate_stochastic_events :1910, Species_step_boundary_fluxes :1704,
 * Species_step_reaction :1653, Species_apply_du :1080, Species_apply_fixed_values
 * :1066).  A realisation stops at its total_steps.  stop_flags (nullable, n entries)
 * receives 1 for stopped realisations. */
int csp_advance(csp_handle* h, int64_t nsteps, int32_t* stop_flags);

/* csp_advance in two halves: launch nsteps steps and return at once, then wait for them
 * and read the stop flags.  Between the two a caller may do host work (write the previous
 * output) while the device steps; no other call of this handle may come between them but
 * csp_snapshot_wait.  (The reference's loop body is synchronous, calcium_sparks.c:190-228;
 * the split lets the output path of species.c:2253-2551 overlap the next cycle.) */
int csp_advance_async(csp_handle* h, int64_t nsteps);
int csp_advance_wait(csp_handle* h, int32_t* stop_flags);

/* Start a copy of realisation r's fields to the host without waiting: the species in
 * species_mask (bit s) are converted to FP64 on the handle stream, in the layout of
 * csp_download_state ([num_species][nx][ny][nz]; species outside the mask are left
 * unset), and copied on a second stream into a page-locked buffer owned by the handle, so
 * the copy overlaps a csp_advance_async launched next.  csp_snapshot_wait waits for the
 * copy and returns that buffer in *u, valid until the next csp_snapshot_async or
 * csp_destroy.  Replaces the field reads of Species_output_data (species.c:2263-2298,
 * 3027-3081: sheets and <sp>_all_data). */
int csp_snapshot_async(csp_handle* h, int32_t r, uint32_t species_mask);
int csp_snapshot_wait(csp_handle* h, const double** u);

/* Per (domain, species) min / max / sum(u*dV) in FP64, and the channel openness of
 * every discrete boundary in boundary order (Species_output_scalar_data,
 * species.c:2785-2880).  min/max/total: [num_domains][num_species]; openness: all
 * channels of all discrete boundaries, concatenated. */
int csp_reduce_outputs(csp_handle* h, int32_t r, double* min_values, double* max_values,
                       double* total_values, int32_t* openness);

/* Channel states (0 closed / 1 open) of discrete boundary `boundary` (index into
 * model.boundaries) of realisation r (ModelStates::s0, basefluxinfo.h:9-16). */
int csp_get_channel_states(const csp_handle* h, int32_t r, int32_t boundary, int32_t* states);
int csp_set_channel_states(csp_handle* h, int32_t r, int32_t boundary, const int32_t* states);

/* Message of the last error and the device error word (bounds / timeout). */
int csp_status(const csp_handle* h, char* msg, size_t n);

/* The CUDA stream (cudaStream_t) every call of this handle is ordered on. */
int csp_get_stream(const csp_handle* h, void** stream);

/* Device time in ms of the last csp_advance call (CUDA events on the handle stream). */
int csp_last_advance_ms(const csp_handle* h, float* ms);

/* Advance like csp_advance, but launch the two kernels of every step one by one with CUDA
 * events around each launch (no graph); voxel_ms / boundary_ms receive the summed device
 * times of the voxel kernel and of the boundary / gating kernel. */
int csp_profile_advance(csp_handle* h, int64_t nsteps, float* voxel_ms, float* boundary_ms);

/* Per-phase device times of the step (the counterpart of the reference's -v timing buckets
 * Diffusion stencil / Boundary fluxes / Stochastic evaluation / Reaction stencil,
 * utils.c:11-75).  The step's kernels fuse several of the reference's phases, so a phase
 * here is one kernel family: CSP_PHASE_VOXELS = diffusion of every species with the buffer
 * reactions and fixed values (species.c:1501-1702), CSP_PHASE_DENSITY = density-boundary
 * (SERCA) fluxes, CSP_PHASE_CHANNELS = RyR/pRyR gating with the channel fluxes
 * (species.c:1704-1957), CSP_PHASE_SURROGATE = the learned reaction increments,
 * CSP_PHASE_EPILOGUE = step counter and abort rule.  While enabled, the first 16 steps of
 * every csp_advance / csp_advance_async call run as direct launches with CUDA events
 * between the kernels; their per-phase time, scaled to the call's steps, is accumulated
 * (an estimate: the other steps replay the captured graph untimed).  ms[CSP_NUM_PHASES]
 * receives the accumulated milliseconds, steps the steps they stand for. */
enum { CSP_PHASE_VOXELS = 0, CSP_PHASE_DENSITY, CSP_PHASE_CHANNELS, CSP_PHASE_SURROGATE, CSP_PHASE_EPILOGUE,
       CSP_NUM_PHASES };
int csp_set_phase_timing(csp_handle* h, int32_t on);
int csp_get_phase_times(const csp_handle* h, double* ms, int64_t* steps);

/* Test hook for the failure path of the staged voxel kernel's bounded waits.  While armed
 * (on != 0), every launch of the staged kernel makes one thread of its first CTA wait on an
 * mbarrier that nothing completes, with a 1 ms limit; that CTA then leaves its x loop as
 * one (the decision is taken at the end-of-plane barrier), waits for its own bulk copies
 * in flight, sets the timeout bit of the device error word and returns, and csp_advance
 * returns CSP_EDEVICE with csp_status naming the timeout.  The handle's fields are
 * undefined afterwards and the error stays set; the device and other handles stay usable.
 * No counterpart in the reference: it has no device and aborts on any error
 * (fvm_mpi/src/utils.h:21-27). */
int csp_test_wait_timeout(csp_handle* h, int32_t on);

/* Select the voxel kernel: 0 = staged (TMA bulk copies into shared memory, default),
 * 1 = direct (one thread per voxel, global loads).  Both give bitwise equal results. */
int csp_set_kernel(csp_handle* h, int32_t which);

/* Linescan of species `species` of realisation r along physical axis `axis` (0 x, 1 y,
 * 2 z): out[a] = sum over species voxels of u * g(o_x - x h) g(o_y - y h) g(o_z - z h) with
 * o_axis = a*h, the other two offsets_nm[] fixed (nm), g(d, s) = exp(-d^2/2s)/sqrt(2 pi s)
 * with s = conv[axis of d] (the species file's convolution_constants).  num_domains > 0
 * keeps only voxels whose domain id is below num_domains, the reference's test.  out has
 * n[axis] entries.  Replaces Species_compute_convolution_with_gaussian_function_locally
 * (species.c:1960-2037; gauss, utils.c:209-213). */
int csp_linescan(csp_handle* h, int32_t r, int32_t species, int32_t axis, const double* offsets_nm,
                 const double* conv, int32_t num_domains, double* out);

/* ---- learned reaction surrogate ----
 * With dt_update_react = n*dt the reference advances the buffer reactions every n steps
 * by one explicit step of dt_r = n*dt (Species_step_reaction, species.c:1653-1702).  The
 * surrogate replaces that increment by a small MLP (8 inputs: log Ca, the bound fractions
 * of the buffer species 1..5, log dt_r, the domain id; two ReLU layers of 64; 5 outputs)
 * that predicts the correction of the explicit step towards the plain integrator (the
 * same reaction update taken n times at the step dt).  Every voxel's increment must pass
 * a trapezoidal-rule residual test (relative to the buffer totals, tolerance tol), else
 * the voxel takes the plain integrator; voxels within 1e-8 of equilibrium take the
 * explicit step without evaluating the network.  Needs every buffer bound to species 0 and bound
 * species among 1..5. */
#define CSP_MLP_NPARAM 5061   /* w1[8][64] b1[64] w2[64][64] b2[64] w3[64][5] b3[5] */

typedef struct csp_mlp_config {
  int64_t samples;          /* training pairs (default 1e6) */
  int64_t val_samples;      /* held-out pairs (default 65536) */
  int32_t epochs;           /* default 10 */
  int32_t batch;            /* default 16384 */
  float lr;                 /* Adam learning rate, cosine decay (default 1e-3) */
  double tol;               /* acceptance tolerance reported on the held-out pairs (default 1e-4) */
  uint64_t seed;            /* Philox key of the pair sampler */
  int32_t source;           /* CSP_MLP_SOURCE_SAMPLED (default) or CSP_MLP_SOURCE_HARVEST */
} csp_mlp_config;
enum { CSP_MLP_SOURCE_SAMPLED = 0, CSP_MLP_SOURCE_HARVEST = 1 };

typedef struct csp_mlp_report {
  float val_loss_first, val_loss_last;   /* held-out mean squared error before / after */
  double val_accept_rate;                /* held-out pairs passing the residual test */
  float train_ms;                        /* device time of the training loop */
  int32_t steps;
  int64_t samples;
} csp_mlp_report;

/* Initial parameters: He-uniform hidden layers from `seed`, zero output layer (the
 * untrained network reproduces the single explicit step). */
void csp_mlp_init(uint64_t seed, float* params);
/* Train on device: pairs sampled from realisation r's buffer constants (Ca log-uniform in
 * 0.1-500 uM in the cytosol, 10-2000 uM in SR domains; targets from the plain integrator),
 * Adam on the mean squared error; params in (start) / out (trained). */
int csp_mlp_train(csp_handle* h, int32_t r, const csp_mlp_config* cfg, float* params, csp_mlp_report* rep);
/* Training pairs from the simulation's own states.  Every voxel of the surrogate's domains
 * with Ca in 0.1-500 uM, in every realisation, at the current step, is a candidate; each
 * is taken with a probability for its log10-Ca bin (32 bins) chosen so that about n pairs
 * are taken, as near log-uniform in Ca as the states allow (bins with fewer candidates
 * give all they have).  A pair is the features of the voxel's state and the target from
 * the plain integrator, as for sampled states.  Pairs accumulate in the handle (device
 * memory for `capacity` pairs, allocated by the first call) across calls at different
 * steps; *taken / *held receive the pairs of this call / all held.  csp_mlp_train with
 * cfg->source = CSP_MLP_SOURCE_HARVEST trains on every held pair (a tenth at most, up to
 * val_samples, held out), shuffled.  The reaction these pairs stand for is the
 * reference's Species_step_reaction (species.c:1653-1702). */
int csp_mlp_harvest(csp_handle* h, int64_t n, uint64_t seed, int64_t capacity, int64_t* taken, int64_t* held);
/* Copy held pairs [first, first + n) to the host: x[n][8] features, t[n][5] targets. */
int csp_mlp_harvested(const csp_handle* h, int64_t first, int64_t n, float* x, float* t);
/* Loss and gradient of the mean squared error of params on n host pairs x[n][8], t[n][5]
 * with the device kernels used in training (for checks against a CPU implementation). */
int csp_mlp_gradient(const float* params, const float* x, const float* t, int64_t n, float* grad, float* loss);
/* Network outputs y[n][5] of inputs x[n][8]: the FP32 pass of training (tensor_cores = 0),
 * the TF32 tensor-core pass the simulation uses (tensor_cores = 1: warp mma.sync tiles of
 * 32 samples) or the same on the 5th-generation tensor cores (tensor_cores = 2: tcgen05
 * MMAs on tiles of 128 samples with the accumulators in tensor memory). */
int csp_mlp_forward(const float* params, const float* x, int64_t n, int32_t tensor_cores, float* y);
/* Use params (NULL: switch off) for the reaction steps of every realisation. */
int csp_set_surrogate(csp_handle* h, const float* params, double tol);
/* Since csp_set_surrogate: voxel reaction increments taken, those the network was
 * evaluated for (the others were at equilibrium to within 1e-8 of their buffer totals, or
 * in a stiff domain), and those that took the plain integrator. */
int csp_surrogate_counts(const csp_handle* h, int64_t* voxels, int64_t* network, int64_t* fallbacks);
/* The tensor cores the surrogate's network tiles use: kind = 1 (the default) warp mma.sync
 * tiles of 32 voxels; kind = 2 tcgen05 MMAs on tiles of 128 voxels with the accumulators in
 * tensor memory (the same TF32 operands; at the surrogate's tile counts the serial
 * per-layer MMA waits make it slower than kind 1).  No counterpart in the reference. */
int csp_set_surrogate_tensor_cores(csp_handle* h, int32_t kind);

/* ---- autotuner ----
 * Times candidate tile shapes of the staged voxel kernel (threads per CTA, x planes per
 * work unit) and the direct kernel (segment = -1: one thread per voxel, every plane at
 * once, which wins on batches too small to give the staged kernel's work units to every
 * CTA slot) at the current step and keeps the fastest; fields are the same for every
 * candidate.  No counterpart in the reference (its OpenMP loops have no tile parameters). */
#define CSP_TUNE_MAX 10
typedef struct csp_tune_report {
  int32_t n;                       /* candidates tried */
  int32_t threads[CSP_TUNE_MAX];
  int32_t segment[CSP_TUNE_MAX];   /* x planes per work unit */
  float ms[CSP_TUNE_MAX];          /* voxel-kernel time per launch (-1: did not fit) */
  int32_t chosen;                  /* index of the plan in use */
} csp_tune_report;
int csp_autotune(csp_handle* h, int32_t repeats, csp_tune_report* report);

void csp_destroy(csp_handle* h);

/* ---- allocation-free reduction ----
 * No counterpart in the reference.  For callers that cannot allocate device memory: a
 * plugin inside a framework that has reserved the device memory for its own pool, or
 * code that must not call cudaMalloc (it synchronises the device) in a latency-bound
 * loop.  Computes, for one FP32 field of n voxels already on the device with its uint8
 * domain ids (bits 0-2), the per-domain min (from FLT_MAX), max (from FLT_MIN) and
 * sum(u)*dV in FP64 -- the reductions of csp_reduce_outputs -- into the caller's device
 * array out[3][num_domains] (min, max, total), on `stream` (NULL = default stream).
 * It allocates nothing: block partials live in a file-scope device array of
 * CSP_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until exit.
 *  - the first call on a device looks the array's address up (cudaGetSymbolAddress) and
 *    keeps it for the life of the process; make that first call before any stream
 *    capture; after a cudaDeviceReset of that device the call is not supported (the
 *    array may move when the module is loaded again);
 *  - all calls share the array: calls that overlap on the GPU race; each call overwrites
 *    every partial it reads, so no clearing is needed;
 *  - num_domains above CSP_NOALLOC_MAX_DOMAINS or n above CSP_NOALLOC_MAX_VOXELS return
 *    CSP_ERANGE (with a message on stderr). */
#define CSP_NOALLOC_MAX_DOMAINS 5
#define CSP_NOALLOC_MAX_VOXELS (1LL << 40)
#define CSP_NOALLOC_SCRATCH_BYTES (592 * 3 * CSP_MAX_DOMAINS * 8)
int csp_reduce_field_noalloc(const float* field, const uint8_t* domains, int64_t n, int32_t num_domains,
                             double dV, double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CSPARKS_H */
