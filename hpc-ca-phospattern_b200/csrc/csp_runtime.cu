// csp_runtime.cu -- libcsparks_cuda.so: the C ABI of include/csparks.h.
//
// Host side: derive every per-realisation constant from the model and options exactly
// as the reference setup does (species.c:95-884, geometry.c:96-344,
// boundaryfluxes.c:361-605), build the boundary-flux rows, allocate HBM, and drive the
// step kernels (direct launches, or replay of a captured CUDA graph of STEPS_PER_GRAPH
// steps: the kernels read the step index from device memory, so one graph serves
// every cycle).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <map>
#include <unordered_map>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <random>
#include <string>
#include <vector>

#include "csp_kernels.cuh"
#include "csp_staged.cuh"
#include "csp_mlp.cuh"

using namespace csp;

namespace {

constexpr int STEPS_PER_GRAPH = 16;
constexpr int PHASE_SAMPLE = 16;            // steps timed per advance call (csp_set_phase_timing)
thread_local char g_create_error[512];

struct HostReal {
  RealDesc desc;                  // host copy (device pointers filled in)
  csp_info info;
  int nd;
  double dV;
  double volumes[ND];
  std::vector<int> boundary_channel_base;   // per boundary: first global channel, or -1
  std::vector<int> boundary_nch;
  size_t field_elems;             // n0*P
  int perm[3];                    // device axis i holds physical axis perm[i]
  int nphys[3];                   // species voxels per physical axis
  std::vector<unsigned char> cls; // chunk class table (RealDesc::cls)
  // padded linear device index of physical species voxel (x, y, z)
  long long dev_index(int x, int y, int z) const {
    const int c[3] = {x, y, z};
    return (long long)c[perm[0]] * desc.P + (long long)c[perm[1]] * desc.nz + c[perm[2]];
  }
};

// Device axis order of one realisation.  The stencil is isotropic and every face has the
// same no-flux rule, so the kernels may hold the field in any axis order.  The marching
// axis (device axis 0) is the physical axis crossed by the most domain changes, so that
// domain-boundary sheets (cleft, jSR, network SR at fixed z in a dyad) become whole
// planes and the voxels sharing a warp share a neighbourhood type.
static void choose_axes(const csp_model& m, int perm[3]) {
  long long ch[3] = {0, 0, 0};
  const int N0 = m.N[0], N1 = m.N[1], N2 = m.N[2];
  for (int x = 0; x < N0; x++)
    for (int y = 0; y < N1; y++)
      for (int z = 0; z < N2; z++) {
        const size_t v = ((size_t)x * N1 + y) * N2 + z;
        if (x + 1 < N0 && m.voxels[v] != m.voxels[v + (size_t)N1 * N2]) ch[0]++;
        if (y + 1 < N1 && m.voxels[v] != m.voxels[v + N2]) ch[1]++;
        if (z + 1 < N2 && m.voxels[v] != m.voxels[v + 1]) ch[2]++;
      }
  int a0 = 0;
  for (int a = 1; a < 3; a++)
    if (ch[a] > ch[a0]) a0 = a;
  int rest[2], k = 0;
  for (int a = 0; a < 3; a++)
    if (a != a0) rest[k++] = a;
  // contiguous last: a length that is a multiple of 4 (4-voxel groups then never straddle
  // a row), then the fewest changes; on a tie keep the physical order
  const int n[3] = {N0, N1, N2};
  const bool a4 = n[rest[0]] % 4 == 0, b4 = n[rest[1]] % 4 == 0;
  const bool swap = a4 != b4 ? a4 : ch[rest[0]] < ch[rest[1]];
  perm[0] = a0;
  perm[1] = swap ? rest[1] : rest[0];
  perm[2] = swap ? rest[0] : rest[1];
}

// Chunk class table of one realisation from its device-layout domain bytes (see
// RealDesc::cls).
static void chunk_classes(const RealDesc& D, const std::vector<unsigned char>& dom, std::vector<unsigned char>& cls) {
  const int nch = (D.plane + CLASS_L - 1) / CLASS_L;
  cls.assign((size_t)D.nx * nch, CLASS_MIXED);
  std::vector<unsigned char> pu((size_t)D.nx * nch, CLASS_MIXED);
  for (int q = 0; q < D.nx; q++)
    for (int c = 0; c < nch; c++) {
      const int lo = std::max(0, c * CLASS_L - D.nz), hi = std::min(D.plane, c * CLASS_L + CLASS_L + D.nz);
      const unsigned char* row = dom.data() + (size_t)q * D.P;
      const unsigned char d = row[lo];
      bool same = d <= DOMAIN_BITS;
      for (int p = lo + 1; same && p < hi; p++) same = row[p] == d;
      if (same) pu[(size_t)q * nch + c] = d;
    }
  for (int x = 0; x < D.nx; x++)
    for (int c = 0; c < nch; c++) {
      const unsigned char d = pu[(size_t)x * nch + c];
      if (d == CLASS_MIXED) continue;
      if (x > 0 && pu[(size_t)(x - 1) * nch + c] != d) continue;
      if (x + 1 < D.nx && pu[(size_t)(x + 1) * nch + c] != d) continue;
      cls[(size_t)x * nch + c] = d;
    }
}

}  // namespace

struct csp_handle {
  int n = 0;
  std::vector<HostReal> real;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.f;
  // device memory
  float* d_fields = nullptr;
  unsigned char* d_dom = nullptr;
  unsigned char* d_cls = nullptr;
  RealDesc* d_desc = nullptr;
  RealCtl* d_ctl = nullptr;
  FluxRow* d_rows = nullptr;
  FluxEntry* d_entries = nullptr;
  FluxPair* d_pairs = nullptr;
  FluxParams* d_params = nullptr;
  unsigned char* d_states = nullptr;
  int* d_err = nullptr;
  double* d_red = nullptr;
  double* d_red_out = nullptr;
  void* d_stage = nullptr;           // host-state staging of upload / download (one realisation)
  size_t stage_bytes = 0;
  // asynchronous snapshots: FP64 fields converted on the handle stream into d_snap, copied
  // on snap_stream into the page-locked h_snap (ev_snap: converted, ev_copy: copied)
  double* d_snap = nullptr;
  double* h_snap = nullptr;
  size_t snap_elems = 0;
  cudaStream_t snap_stream = nullptr;
  cudaEvent_t ev_snap = nullptr, ev_copy = nullptr;
  bool snap_pending = false;
  bool advance_pending = false;
  int nrows = 0, nch = 0;
  int nrows_density = 0;             // rows [0, nrows_density) have density pairs only
  DensityRow* d_drows = nullptr;     // the density rows in 32 bytes (null: k_boundaries<false>)
  int ndrows = 0;                    // compact rows (pair rows count once)
  // rows are realisation-major: the rows of realisation r are [first[r], first[r+1]) of the
  // compact density rows, the density-only FluxRows and the channel FluxRows
  std::vector<int> drow_first, krow_first, crow_first;
  // csp_run_states: host-to-device stream, staging (two input and two output slots), per
  // step stop flags
  cudaStream_t in_stream = nullptr;
  void* d_pipe = nullptr;
  size_t pipe_bytes = 0;
  int* d_stepflags = nullptr;
  size_t stepflags_elems = 0;
  StepRec* d_rec = nullptr;          // per realisation: what its running step does
  int max_plane_vox = 0;
  long long max_vox = 0;
  long long max_field = 0;           // max n0*P (padded planes)
  int kernel = 0;                 // 0 staged, 1 direct
  int inject_wait = 0;            // csp_test_wait_timeout armed (direct launches, no graph)
  // csp_set_phase_timing: the first steps of every advance call run as direct launches
  // with events between the step's kernels; the sample's per-phase device time, scaled to
  // the steps of the call, is added to phase_ms at the call's wait
  int phase_timing = 0;
  cudaEvent_t phase_ev[PHASE_SAMPLE * (CSP_NUM_PHASES + 1)] = {};
  int phase_sampled = 0;
  int64_t phase_call_steps = 0;
  double phase_ms[CSP_NUM_PHASES] = {};
  int64_t phase_steps = 0;
  StagedPlan plan;
  cudaGraphExec_t graph = nullptr;
  int graph_kernel = -1;
  int graph_plan = -1;
  int plan_epoch = 0;                       // bumped when the autotuner replaces the plan
  int graph_surrogate = 0;
  int graph_sur_tc = 0;
  // learned reaction surrogate (csp_set_surrogate)
  int surrogate = 0;
  float surrogate_tol = 1e-4f;
  unsigned surrogate_fq = 0;         // k_react_network<FQ> of the ensemble's fixed-point species
  float* d_mlp = nullptr;                   // MLP_NPARAM parameters
  unsigned long long* d_mlp_cnt = nullptr;  // voxels, network evaluations, fallbacks
  unsigned short* d_sur_list = nullptr;     // per k_react_surrogate CTA: its network voxels
  unsigned* d_sur_counts = nullptr;         // per segment: listed network / plain-integrator voxels
  unsigned* d_sur_tiles = nullptr;          // tiles of 32 listed voxels: network half, then plain half
  long long sur_tile_cap = 0;               // tiles per half
  unsigned* d_sur_queue = nullptr;          // network tiles, k_react_network CTAs done, plain tiles, k_react_plain CTAs done
  unsigned char* d_rx_class = nullptr;      // surrogate class bytes (RealDesc::rx_class), layout of d_dom
  int sur_network_ctas = 0;                 // persistent CTAs of k_react_network
  int sur_plain_ctas = 0;                   // persistent CTAs of k_react_plain
  int sur_umma_ctas = 0;                    // persistent CTAs of k_react_network_umma
  int sur_tc = 1;                           // network tiles: 1 warp mma.sync, 2 tcgen05 (csp_set_surrogate_tensor_cores)
  // training pairs harvested from the fields (csp_mlp_harvest): features [cap][8], targets [cap][5]
  float* d_hx = nullptr;
  float* d_ht = nullptr;
  long long harvest_cap = 0, harvest_n = 0;
  std::string msg;
};

static int fail(csp_handle* h, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (h) h->msg = buf; else snprintf(g_create_error, sizeof g_create_error, "%s", buf);
  return code;
}

// Calls that touch the device state of a handle are refused while an asynchronous advance
// is pending: they would queue behind it and break csp_advance_wait's contract.
#define CSP_NOT_PENDING(h)                                                                    \
  do {                                                                                        \
    if ((h)->advance_pending)                                                                 \
      return fail(h, CSP_EINVAL, "an asynchronous advance is pending (csp_advance_wait)");    \
  } while (0)

#define CUDA_TRY(h, call)                                                                     \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) return fail(h, CSP_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

static int name_index(const char names[][CSP_NAME_LEN], int n, const char* s) {
  for (int i = 0; i < n; i++)
    if (strncmp(names[i], s, CSP_NAME_LEN) == 0) return i;
  return -1;
}

static int boundary_index(const csp_model& m, const char* name) {
  for (int i = 0; i < m.num_boundaries; i++)
    if (strncmp(m.boundaries[i].name, name, CSP_NAME_LEN) == 0) return i;
  return -1;
}

extern "C" void csp_options_default(csp_options* o) {
  // arguments_construct, options.c:502-542
  memset(o, 0, sizeof(*o));
  o->h = 6.;
  o->dt = -1.;
  o->tstop = 10.;
  o->dt_save = .5;
  o->dt_update_react = -1.;
  o->dt_update_stoch = -1.;
  o->tabort = 0.;
}

namespace {

// Per-realisation constants (species.c:181-313, 784-787; geometry.c:104-105).
struct Derived {
  int S, nx, ny, nz;
  double h, dt;
  int ndiff;
  int diff_species[NS], substeps[NS];
  double coef[NS][ND][ND];
  int nbuf;
  double kon[NB * ND], koff[NB * ND], tot[NB * ND];
  unsigned char bsp0[NB * ND], bsp1[NB * ND];
  unsigned reaction_flag_mask;
  int reaction_substep, stochastic_substep;
  long long total_steps;
};

int derive(const csp_model& m, const csp_options& o, Derived& dv, std::string& err) {
  if (m.num_domains < 1 || m.num_domains > ND) { err = "num_domains out of range (max 5)"; return CSP_EINVAL; }
  if (m.num_species < 1 || m.num_species > NS) { err = "num_species out of range (max 8)"; return CSP_EINVAL; }
  if (m.num_boundaries < 0 || m.num_boundaries > CSP_MAX_BOUNDARIES) { err = "num_boundaries out of range"; return CSP_EINVAL; }
  if (!m.voxels) { err = "voxels is NULL"; return CSP_EINVAL; }
  if (!(o.h > 0)) { err = "resolution -h must be positive"; return CSP_EINVAL; }
  for (int a = 0; a < 3; a++)
    if (m.N[a] < 1) { err = "geometry size must be positive"; return CSP_EINVAL; }
  int S = (int)std::fmax(1., std::floor(m.h_geom / o.h));
  S &= 0xff;  // Geometry_t::subdivisions is a domain_id
  if (S == 0) { err = "subdivisions overflow (h_geom/h >= 256)"; return CSP_EINVAL; }
  dv.S = S;
  dv.h = m.h_geom / S;
  dv.nx = m.N[0] * S; dv.ny = m.N[1] * S; dv.nz = m.N[2] * S;
  const int nd = m.num_domains;
  double max_sigma = 0, max_sigma_species[NS] = {0};
  bool is_diff[NS] = {false};
  for (int d = 0; d < nd; d++) {
    const csp_domain_species& ds = m.domain[d];
    if (ds.num_diffusive < 0 || ds.num_diffusive > NS || ds.num_buffers < 0 || ds.num_buffers > NB) {
      err = "per-domain species counts out of range"; return CSP_EINVAL;
    }
    for (int k = 0; k < ds.num_diffusive; k++) {
      const int s = ds.diffusive[k];
      if (s >= m.num_species) { err = "diffusive species index out of range"; return CSP_EINVAL; }
      is_diff[s] = true;
      max_sigma = std::fmax(max_sigma, ds.sigma[k]);
      max_sigma_species[s] = std::fmax(ds.sigma[k], max_sigma_species[s]);
    }
  }
  dv.dt = o.dt > 0 ? o.dt : 0.95 * (1. / 6) * dv.h * dv.h / max_sigma;  // species.c:265
  if (!(dv.dt > 0) || !std::isfinite(dv.dt)) { err = "time step is not positive (no diffusive species and no -d?)"; return CSP_EINVAL; }
  dv.ndiff = 0;
  for (int s = 0; s < m.num_species; s++) {  // species.c:281-294
    if (!is_diff[s]) continue;
    const double sdt = std::fabs(max_sigma - max_sigma_species[s]) < 1e-12
                           ? dv.dt : 0.95 * (1. / 6) * dv.h * dv.h / max_sigma_species[s];
    dv.substeps[dv.ndiff] = ((int)std::fmax(1., std::floor(sdt / dv.dt))) & 0xff;
    if (dv.substeps[dv.ndiff] == 0) { err = "species substeps overflow"; return CSP_EINVAL; }
    dv.diff_species[dv.ndiff++] = s;
  }
  // coefficient tables, species.c:1545-1560: sigma[di][dsi] is indexed by the diffusive
  // index dsi, i.e. a domain's diffusive list is expected to follow the global order.
  for (int dsi = 0; dsi < dv.ndiff; dsi++) {
    for (int a = 0; a < ND; a++)
      for (int b = 0; b < ND; b++) dv.coef[dsi][a][b] = 0.0;
    for (int di = 0; di < nd; di++) {
      const csp_domain_species& A = m.domain[di];
      if (!(dsi < A.num_diffusive && A.sigma[dsi] != 0)) continue;
      for (int dn = 0; dn < di; dn++) {
        const csp_domain_species& B = m.domain[dn];
        if (m.domain_connections[di * nd + dn] && dsi < B.num_diffusive && B.sigma[dsi] != 0)
          dv.coef[dsi][di][dn] = dv.coef[dsi][dn][di] =
              dv.dt * 0.5 * (A.sigma[dsi] + B.sigma[dsi]) / (dv.h * dv.h) * dv.substeps[dsi];
      }
      dv.coef[dsi][di][di] = dv.dt * A.sigma[dsi] / (dv.h * dv.h) * dv.substeps[dsi];
    }
  }
  // buffer tables (species.c:134-145, 216-241, 304-313)
  memset(dv.kon, 0, sizeof dv.kon); memset(dv.koff, 0, sizeof dv.koff); memset(dv.tot, 0, sizeof dv.tot);
  memset(dv.bsp0, 0, sizeof dv.bsp0); memset(dv.bsp1, 0, sizeof dv.bsp1);
  bool is_buf[NS] = {false};
  unsigned char bsp0_dom[ND][NS] = {{0}}, bsp1_dom[ND][NS] = {{0}};
  for (int d = 0; d < nd; d++) {
    const csp_domain_species& ds = m.domain[d];
    for (int bi = 0; bi < ds.num_buffers; bi++) {
      if (ds.bsp0[bi] >= m.num_species || ds.bsp1[bi] >= m.num_species) { err = "buffer species index out of range"; return CSP_EINVAL; }
      dv.bsp0[bi * nd + d] = ds.bsp0[bi]; dv.bsp1[bi * nd + d] = ds.bsp1[bi];
      dv.kon[bi * nd + d] = ds.k_on[bi]; dv.koff[bi * nd + d] = ds.k_off[bi]; dv.tot[bi * nd + d] = ds.tot[bi];
      bsp0_dom[d][bi] = ds.bsp0[bi]; bsp1_dom[d][bi] = ds.bsp1[bi];
      is_buf[ds.bsp0[bi]] = true;
    }
  }
  dv.nbuf = 0;
  for (int s = 0; s < m.num_species; s++) dv.nbuf += is_buf[s];
  for (int d = 0; d < nd; d++)
    if (m.domain[d].num_buffers > dv.nbuf) { err = "a domain holds more buffers than there are buffer species"; return CSP_EINVAL; }
  dv.reaction_flag_mask = 0;  // species.c:1695-1699
  for (int d = 0; d < nd; d++)
    for (int bi = 0; bi < dv.nbuf; bi++) dv.reaction_flag_mask |= (1u << bsp0_dom[d][bi]) | (1u << bsp1_dom[d][bi]);
  dv.stochastic_substep = (int)std::fmax(1., std::floor(o.dt_update_stoch / dv.dt));  // species.c:784
  dv.reaction_substep = (int)std::fmax(1., std::floor(o.dt_update_react / dv.dt));    // species.c:787
  long long steps = 0;
  for (double t = 0.; t < o.tstop; t += dv.dt) steps++;  // calcium_sparks.c:190
  dv.total_steps = steps;
  return CSP_OK;
}

struct PairHost {
  FluxPair p;
};

}  // namespace

// Species voxel pairs of one geometry boundary (Species_init_boundary_voxels,
// species.c:938-1035); coordinates in species voxels, [n][6].
static void boundary_species_pairs(const csp_boundary& gb, int S, std::vector<unsigned>& out) {
  const int sub = gb.type == CSP_BOUNDARY_DISCRETE ? 1 : S;
  out.assign((size_t)gb.num_pairs * sub * sub * 6, 0u);
  for (int j = 0; j < gb.num_pairs; j++) {
    const uint16_t* lb = &gb.pairs[6 * j];
    int dim2 = 0;  // Geometry_get_boundary_dir, geometry.c:1490-1530
    for (int dim = 0; dim < 3; dim++)
      if (lb[dim] != lb[dim + 3]) { dim2 = lb[dim] < lb[dim + 3] ? 2 * dim : 2 * dim + 1; break; }
    const int dim = dim2 / 2, lr = dim2 % 2;
    const int odim = dim != 0 ? 0 : 1, idim = dim != 2 ? 2 : 1;
    const unsigned from_ind = lb[dim] * S + (lr == 0 ? S - 1 : 0);
    const unsigned to_ind = lb[dim + 3] * S + (lr == 0 ? 0 : S - 1);
    for (int oi = 0; oi < sub; oi++) {
      unsigned o_ind = S * lb[odim] + oi;
      if (gb.type == CSP_BOUNDARY_DISCRETE) o_ind += S / 2;
      for (int ii = 0; ii < sub; ii++) {
        unsigned i_ind = S * lb[idim] + ii;
        if (gb.type == CSP_BOUNDARY_DISCRETE) i_ind += S / 2;
        unsigned* v = &out[((size_t)j * sub * sub + oi * sub + ii) * 6];
        v[dim] = from_ind; v[odim] = o_ind; v[idim] = i_ind;
        v[dim + 3] = to_ind; v[odim + 3] = o_ind; v[idim + 3] = i_ind;
      }
    }
  }
}

static const csp_open_list* open_list(const csp_options& o, const char* name) {
  for (int i = 0; i < o.num_open_lists; i++)
    if (strncmp(o.open[i].name, name, CSP_NAME_LEN) == 0) return &o.open[i];
  return nullptr;
}

static double t_close_of(const csp_options& o, const char* name) {
  for (int i = 0; i < o.num_t_close; i++)
    if (strncmp(o.t_close[i].name, name, CSP_NAME_LEN) == 0) return o.t_close[i].time;
  return -1;
}

static void ryr_params(FluxParams& fp, const csp_ryr_params& p, double t_close) {
  // RyR_model::params layout, boundaryfluxes.c:445-454
  fp.p[0] = p.Kd_close; fp.p[1] = p.k_max_close; fp.p[2] = p.n_open; fp.p[3] = p.k_max_open;
  fp.p[4] = p.k_min_open; fp.p[5] = p.n_close; fp.p[6] = p.i_unitary; fp.p[7] = p.k_min_close;
  fp.p[8] = t_close; fp.p[9] = p.Kd_open;
  fp.t_close = t_close;
}

static int round_up(int a, int b) { return (a + b - 1) / b * b; }

extern "C" int csp_create(const csp_model* models, const csp_options* options, int32_t n, csp_handle** out) {
  if (!out) return fail(nullptr, CSP_EINVAL, "out is NULL");
  *out = nullptr;
  if (!models || !options || n < 1) return fail(nullptr, CSP_EINVAL, "models/options NULL or n < 1");
  csp_handle* h = new csp_handle();
  h->n = n;
  h->real.resize(n);
  std::vector<Derived> dv(n);
  size_t field_total = 0, dom_total = 0;
  for (int r = 0; r < n; r++) {
    std::string err;
    int rc = derive(models[r], options[r], dv[r], err);
    if (rc) { delete h; return fail(nullptr, rc, "realisation %d: %s", r, err.c_str()); }
    HostReal& hr0 = h->real[r];
    choose_axes(models[r], hr0.perm);
    hr0.nphys[0] = dv[r].nx; hr0.nphys[1] = dv[r].ny; hr0.nphys[2] = dv[r].nz;
    const int n0 = hr0.nphys[hr0.perm[0]], n1 = hr0.nphys[hr0.perm[1]], n2 = hr0.nphys[hr0.perm[2]];
    const int plane = n1 * n2;
    const int P = round_up(plane, PLANE_ALIGN);
    if ((long long)n0 * P >= (1ll << 31)) { delete h; return fail(nullptr, CSP_EINVAL, "realisation %d: grid too large (2^31 voxels per field)", r); }
    hr0.field_elems = (size_t)n0 * P;
    field_total += hr0.field_elems * 2 * models[r].num_species;
    dom_total += hr0.field_elems;
    h->max_plane_vox = std::max(h->max_plane_vox, plane);
    h->max_vox = std::max(h->max_vox, (long long)n0 * plane);
    h->max_field = std::max(h->max_field, (long long)n0 * P);
  }
  // -- device allocation (one arena for all fields) --
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreate(&h->ev0)) != cudaSuccess || (e = cudaEventCreate(&h->ev1)) != cudaSuccess) {
    csp_destroy(h);
    return fail(nullptr, CSP_ECUDA, "stream/event creation: %s", cudaGetErrorString(e));
  }
  if (cudaMalloc(&h->d_fields, field_total * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&h->d_dom, dom_total + 256) != cudaSuccess ||
      cudaMalloc(&h->d_desc, n * sizeof(RealDesc)) != cudaSuccess ||
      cudaMalloc(&h->d_ctl, n * sizeof(RealCtl)) != cudaSuccess ||
      cudaMalloc(&h->d_err, sizeof(int)) != cudaSuccess) {
    csp_destroy(h);
    return fail(nullptr, CSP_ENOMEM, "device allocation of %.3f GB failed",
                (field_total * 4.0 + dom_total) / 1e9);
  }
  cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream);
  cudaMemsetAsync(h->d_fields, 0, field_total * sizeof(float), h->stream);
  cudaMemsetAsync(h->d_dom, 0, dom_total + 256, h->stream);

  std::vector<FluxPair> pairs;
  std::vector<char> fused;           // pair evaluated inside the voxel kernels
  std::vector<FluxParams> params;
  std::vector<unsigned char> states0;
  std::vector<RealCtl> ctl(n);
  size_t foff = 0, doff = 0;
  std::vector<float> hostf;
  std::vector<unsigned char> hostd;
  for (int r = 0; r < n; r++) {
    const csp_model& m = models[r];
    const csp_options& o = options[r];
    const Derived& d = dv[r];
    HostReal& hr = h->real[r];
    RealDesc& D = hr.desc;
    memset(&D, 0, sizeof D);
    const int nd = m.num_domains;
    hr.nd = nd;
    // device axes (choose_axes): nx / ny / nz below are device axes 0 / 1 / 2
    D.nx = hr.nphys[hr.perm[0]]; D.ny = hr.nphys[hr.perm[1]]; D.nz = hr.nphys[hr.perm[2]];
    D.plane = D.ny * D.nz;
    D.P = round_up(D.plane, PLANE_ALIGN);
    D.ns = m.num_species; D.nd = nd; D.ndiff = d.ndiff; D.nbuf = d.nbuf;
    D.reaction_substep = d.reaction_substep; D.stochastic_substep = d.stochastic_substep;
    D.dirichlet = o.force_dirichlet ? 1 : 0;
    for (int k = 0; k < d.ndiff; k++) { D.substeps[k] = d.substeps[k]; D.diff_species[k] = d.diff_species[k]; }
    D.reaction_flag_mask = d.reaction_flag_mask;
    D.dt_r = (float)(d.dt * d.reaction_substep);
    for (int k = 0; k < d.ndiff; k++)
      for (int a = 0; a < ND; a++)
        for (int b = 0; b < ND; b++) D.coef[k][a * ND + b] = (float)d.coef[k][a][b];
    for (int t = 0; t < NB * ND; t++) {
      D.kon_dt[t] = (float)(d.kon[t] * (d.dt * d.reaction_substep));
      D.koff_dt[t] = (float)(d.koff[t] * (d.dt * d.reaction_substep));
      D.tot[t] = (float)d.tot[t];
      D.bsp0[t] = d.bsp0[t]; D.bsp1[t] = d.bsp1[t];
    }
    // per-species lookup tables of the voxel kernels
    for (int s = 0; s < NS; s++) D.dsi_of[s] = -1;
    for (int k = 0; k < d.ndiff; k++) D.dsi_of[d.diff_species[k]] = (signed char)k;
    D.react_fast = 1;
    for (int dd = 0; dd < ND; dd++)
      for (int s = 0; s < NS; s++) D.rtab[dd][s] = -1;
    for (int dd = 0; dd < nd; dd++)
      for (int bi = 0; bi < m.domain[dd].num_buffers; bi++) {
        const int s0 = m.domain[dd].bsp0[bi], s1 = m.domain[dd].bsp1[bi];
        if (s1 != 0 || s0 == 0 || D.rtab[dd][s0] >= 0) D.react_fast = 0;
        else D.rtab[dd][s0] = (signed char)bi;
      }
    // field bases (RealDesc::base): for a diffusing species the initial value of the first
    // domain of each set of domains it diffuses between (coefficient tables, species.c:
    // 1547-1560), else each domain's own initial value
    for (int s = 0; s < m.num_species; s++) {
      int comp[ND];
      for (int a = 0; a < nd; a++) comp[a] = a;
      const int k = D.dsi_of[s];
      for (bool changed = k >= 0; changed;) {
        changed = false;
        for (int a = 0; a < nd; a++)
          for (int b = 0; b < nd; b++)
            if (a != b && d.coef[k][a][b] != 0.0 && comp[a] < comp[b]) { comp[b] = comp[a]; changed = true; }
      }
      for (int a = 0; a < nd; a++) {
        D.base[a][s] = m.domain[comp[a]].init[s];
        D.fbase[a][s] = (float)D.base[a][s];
        D.dinit[a][s] = (float)(m.domain[a].init[s] - D.base[a][s]);
      }
    }
    // fixed-point species (RealDesc::fixq): never diffusive, the bound form of some buffer
    // and the ligand of none; unit a power of two with 2 tot below 2^31 units
    {
      unsigned bound = 0, ligand = 0;
      for (int dd = 0; dd < nd; dd++)
        for (int bi = 0; bi < m.domain[dd].num_buffers; bi++) {
          bound |= 1u << m.domain[dd].bsp0[bi];
          ligand |= 1u << m.domain[dd].bsp1[bi];
        }
      for (int s = 1; s < m.num_species; s++)
        if (D.dsi_of[s] < 0 && (bound >> s & 1u) && !(ligand >> s & 1u)) D.fixq |= 1u << s;
      for (int dd = 0; dd < ND; dd++)
        for (int s = 0; s < NS; s++) {
          double range = 0.0;
          if (dd < nd && s < m.num_species) {
            range = std::fabs(m.domain[dd].init[s]) + std::fabs(D.base[dd][s]);
            for (int bi = 0; bi < m.domain[dd].num_buffers; bi++)
              if (m.domain[dd].bsp0[bi] == s) range = std::max(range, m.domain[dd].tot[bi]);
          }
          const int e = range > 0.0 ? (int)std::ceil(std::log2(range)) : 0;
          D.qunit[dd][s] = std::ldexp(1.0f, e - 30);
          D.qinv[dd][s] = std::ldexp(1.0f, 30 - e);
        }
    }
    // buffer reactions about the bases (buffer_dj): a_dt = dt_r k_on (tot - base_s0),
    // j0_dt = dt_r (k_on (tot - base_s0) base_s1 - k_off base_s0), FP64 before rounding
    for (int bi = 0; bi < d.nbuf; bi++)
      for (int dd = 0; dd < nd; dd++) {
        const int t = bi * nd + dd;
        const double dtr = d.dt * d.reaction_substep;
        const double b0 = D.base[dd][d.bsp0[t]], b1 = D.base[dd][d.bsp1[t]];
        D.a_dt[t] = (float)(dtr * d.kon[t] * (d.tot[t] - b0));
        D.j0_dt[t] = (float)(dtr * (d.kon[t] * (d.tot[t] - b0) * b1 - d.koff[t] * b0));
      }
    for (int dd = 0; dd < ND; dd++)
      for (int s = 0; s < NS; s++) {
        D.cdiag[dd][s] = (dd < nd && D.dsi_of[s] >= 0) ? D.coef[D.dsi_of[s]][dd * ND + dd] : 0.f;
        const int bi = D.rtab[dd][s];
        if (bi >= 0) {
          const int t = bi * nd + dd;
          D.rk[dd][s] = make_float4(-D.kon_dt[t], -D.koff_dt[t], D.a_dt[t], D.j0_dt[t]);
          D.rmask[dd] |= (unsigned char)(1u << s);
        } else {
          D.rk[dd][s] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
    for (int i = 0; i < m.num_fixed_domain_species; i++) {
      const int dd = m.fixed_domain_species[2 * i], s = m.fixed_domain_species[2 * i + 1];
      if (dd >= nd || s >= m.num_species) { csp_destroy(h); return fail(nullptr, CSP_EINVAL, "fixed_domain_species out of range"); }
      D.fixed_mask[dd] |= (unsigned char)(1u << s);
    }
    for (int dd = 0; dd < nd; dd++)
      for (int s = 0; s < m.num_species; s++) D.init[dd][s] = (float)m.domain[dd].init[s];
    D.total_steps = d.total_steps;
    D.dt = d.dt; D.h = d.h; D.tabort = o.tabort;
    D.seed = o.seed;
    D.stream = (unsigned)(r + o.stream_offset);
    for (int b = 0; b < 2; b++)
      for (int s = 0; s < m.num_species; s++) {
        D.u[b][s] = h->d_fields + foff;
        foff += hr.field_elems;
      }
    D.dom = h->d_dom + doff;
    doff += hr.field_elems;
    hr.dV = d.h * d.h * d.h;
    // species voxel domains (species.c:596-605) and the initial state (species.c:887-935)
    hostd.assign(hr.field_elems, 0);
    long gcount[ND] = {0};
    for (int x = 0; x < d.nx; x++)
      for (int y = 0; y < d.ny; y++)
        for (int z = 0; z < d.nz; z++) {
          const unsigned char dd =
              m.voxels[((size_t)(x / d.S) * m.N[1] + y / d.S) * m.N[2] + z / d.S];
          if (dd >= nd) { csp_destroy(h); return fail(nullptr, CSP_EINVAL, "voxel domain id %d >= num_domains", dd); }
          hostd[hr.dev_index(x, y, z)] = dd;
        }
    for (size_t i = 0; i < (size_t)m.N[0] * m.N[1] * m.N[2]; i++) gcount[m.voxels[i]]++;
    for (int dd = 0; dd < ND; dd++) hr.volumes[dd] = dd < nd ? gcount[dd] * m.h_geom * m.h_geom * m.h_geom : 0.0;
    hostf.assign(hr.field_elems, 0.f);
    for (int s = 0; s < m.num_species; s++) {
      for (size_t i = 0; i < hr.field_elems; i++) {
        const int dd = hostd[i];
        hostf[i] = D.dinit[dd][s];                                                   // init - base
        if (D.fixq >> s & 1u) {
          const int32_t q = (int32_t)std::lrint((double)D.dinit[dd][s] * D.qinv[dd][s]);
          memcpy(&hostf[i], &q, sizeof q);
        }
      }
      cudaMemcpyAsync(D.u[0][s], hostf.data(), hr.field_elems * sizeof(float), cudaMemcpyHostToDevice, h->stream);
      cudaStreamSynchronize(h->stream);
    }
    // -- boundaries, flux map and channels (boundaryfluxes.c:361-605) --
    hr.boundary_channel_base.assign(m.num_boundaries, -1);
    hr.boundary_nch.assign(m.num_boundaries, 0);
    int bmap[3] = {-1, -1, -1};
    if (m.use_ryr) bmap[0] = boundary_index(m, m.ryr.boundary);
    if (m.use_p_ryr) bmap[1] = boundary_index(m, m.p_ryr.boundary);
    if (m.use_serca) bmap[2] = boundary_index(m, m.serca.boundary);
    for (int k = 0; k < 3; k++)
      if ((k == 0 ? m.use_ryr : k == 1 ? m.use_p_ryr : m.use_serca) && bmap[k] < 0) {
        csp_destroy(h);
        return fail(nullptr, CSP_EINVAL, "flux boundary \"%s\" not in the geometry",
                    k == 0 ? m.ryr.boundary : k == 1 ? m.p_ryr.boundary : m.serca.boundary);
      }
    std::vector<std::vector<unsigned>> bvox(m.num_boundaries);
    for (int bi = 0; bi < m.num_boundaries; bi++) {
      const csp_boundary& gb = m.boundaries[bi];
      if (gb.num_pairs > 0 && !gb.pairs) { csp_destroy(h); return fail(nullptr, CSP_EINVAL, "boundary %d pairs NULL", bi); }
      for (int j = 0; j < gb.num_pairs * 6; j++)
        if (gb.pairs[j] >= m.N[j % 3]) { csp_destroy(h); return fail(nullptr, CSP_EINVAL, "boundary %s voxel out of the geometry", gb.name); }
      boundary_species_pairs(gb, d.S, bvox[bi]);
      if (gb.type == CSP_BOUNDARY_DISCRETE) {
        hr.boundary_channel_base[bi] = (int)states0.size();
        hr.boundary_nch[bi] = gb.num_pairs;
        states0.resize(states0.size() + gb.num_pairs, 0);
        D.has_channels = 1;
      }
    }
    auto lin = [&](const unsigned* c) -> long long { return hr.dev_index((int)c[0], (int)c[1], (int)c[2]); };
    // flux info per boundary: first of ryr, p_ryr, serca (BoundaryFluxes_get_flux_info)
    for (int bi = 0; bi < m.num_boundaries; bi++) {
      int kind = FLUX_NONE;
      for (int k = 0; k < 3; k++)
        if (bmap[k] == bi) { kind = k + 1; break; }
      if (kind == FLUX_NONE) continue;
      const char* spname = kind == FLUX_RYR ? m.ryr.species : kind == FLUX_P_RYR ? m.p_ryr.species : m.serca.species;
      const int si = name_index(m.species_names, m.num_species, spname);
      int dsi = -1;
      for (int k = 0; k < d.ndiff; k++)
        if (d.diff_species[k] == si) dsi = k;
      if (si < 0 || dsi < 0) { csp_destroy(h); return fail(nullptr, CSP_EINVAL, "\"%s\" is not a valid diffusive species name", spname); }
      FluxParams fp;
      memset(&fp, 0, sizeof fp);
      if (kind == FLUX_RYR) ryr_params(fp, m.ryr, t_close_of(o, "ryr"));
      else if (kind == FLUX_P_RYR) ryr_params(fp, m.p_ryr, t_close_of(o, "p_ryr"));
      else {
        fp.p[0] = m.serca.v_cyt_to_A_sr; fp.p[1] = m.serca.density; fp.p[2] = m.serca.scale; fp.t_close = -1;
        // serca_flux (boundaryfluxes.c:73-84): dt * density*v*Q * h^2 / (1e-24 h^3)
        fp.p[9] = d.dt * (m.serca.density * (1e-3 / 6e17)) / (1e-24 * d.h);
      }
      const int pidx = (int)params.size();
      params.push_back(fp);
      const csp_boundary& gb = m.boundaries[bi];
      const std::vector<unsigned>& bv = bvox[bi];
      const int np = (int)(bv.size() / 6);
      const bool inner = gb.num_pairs > 0 && !(gb.pairs[0] == gb.pairs[3] && gb.pairs[1] == gb.pairs[4] && gb.pairs[2] == gb.pairs[5]);
      for (int i = 0; i < np; i++) {
        FluxPair p;
        memset(&p, 0, sizeof p);
        p.r = r; p.species = si; p.dsi = dsi; p.kind = kind; p.boundary = bi; p.inner = inner ? 1 : 0;
        p.param = pidx;
        p.channel = gb.type == CSP_BOUNDARY_DISCRETE ? hr.boundary_channel_base[bi] + i : -1;
        p.local_channel = i;
        p.v0 = lin(&bv[6 * i]);
        p.v1 = lin(&bv[6 * i + 3]);
        p.doms = (hostd[p.v0] & DOMAIN_BITS) | (hostd[p.v1] & DOMAIN_BITS) << 3;
        pairs.push_back(p);
        fused.push_back(0);
      }
    }
    int64_t nfused = 0;
    // -- density-boundary pairs joining two face-adjacent voxels are evaluated inside the
    // voxel kernels: per voxel a 6-direction code vector, deduplicated into <= 31 patterns
    // stored in the domain byte (bits 3-7).  Anything that does not fit stays a flux row.
    {
      std::vector<size_t> cand;
      for (size_t i = 0; i < pairs.size(); i++) {
        const FluxPair& p = pairs[i];
#ifdef CSP_FUSE_DENSITY
        if (p.r == r && p.kind == FLUX_SERCA && p.inner && p.channel < 0) cand.push_back(i);
#endif
      }
      int nslot = 0;
      int slot_boundary[4] = {-1, -1, -1, -1};
      auto dev_coords = [&](long long v, int c[3]) {
        c[0] = (int)(v / D.P);
        const int rem = (int)(v - (long long)c[0] * D.P);
        c[1] = rem / D.nz;
        c[2] = rem - c[1] * D.nz;
      };
      bool ok = true;
      // candidate pairs that can be fused: (pair, slot, k_from, k_to)
      struct Cand { size_t i; int slot, kf, kt; };
      std::vector<Cand> cands;
      for (size_t i : cand) {
        const FluxPair& p = pairs[i];
        int a[3], b[3];
        dev_coords(p.v0, a);
        dev_coords(p.v1, b);
        int axis = -1, nd_ = 0;
        for (int q = 0; q < 3; q++)
          if (a[q] != b[q]) { nd_++; axis = q; }
        if (nd_ != 1 || std::abs(a[axis] - b[axis]) != 1) continue;   // not face-adjacent
        int slot = -1;
        for (int q = 0; q < nslot; q++)
          if (slot_boundary[q] == p.boundary) slot = q;
        if (slot < 0) {
          if (nslot == 4) continue;
          slot = nslot++;
          slot_boundary[slot] = p.boundary;
          D.fslot_species[slot] = p.species;
          D.fslot_kind[slot] = p.kind;
          for (int q = 0; q < 10; q++) D.fslot_p[slot][q] = params[p.param].p[q];
        }
        // direction k: device axis 2 -> 0/1, axis 1 -> 2/3, axis 0 -> 4/5 (minus / plus)
        const int kbase = 2 * (2 - axis);
        cands.push_back({i, slot, kbase + (b[axis] > a[axis] ? 1 : 0), kbase + (b[axis] > a[axis] ? 0 : 1)});
      }
      // per-voxel code vectors; pairs touching voxels whose pattern is not among the 31
      // most frequent ones go back to the boundary kernel, until the patterns fit
      std::vector<char> keep(cands.size(), 1);
      std::unordered_map<long long, std::array<unsigned char, 6>> vc;
      std::map<std::array<unsigned char, 6>, int> patterns;
      for (int iter = 0; iter < 64; iter++) {
        vc.clear();
        for (size_t q = 0; q < cands.size(); q++) {
          if (!keep[q]) continue;
          const FluxPair& p = pairs[cands[q].i];
          auto& c0 = vc[p.v0];
          auto& c1 = vc[p.v1];
          if (c0[cands[q].kf] || c1[cands[q].kt]) { keep[q] = 0; continue; }   // face already used
          c0[cands[q].kf] = (unsigned char)(cands[q].slot + 1);
          c1[cands[q].kt] = (unsigned char)((cands[q].slot + 1) | 0x80);
        }
        std::map<std::array<unsigned char, 6>, long long> freq;
        for (auto& kv : vc) freq[kv.second]++;
        patterns.clear();
        if ((int)freq.size() <= 31) {
          for (auto& kv : freq) patterns.emplace(kv.first, (int)patterns.size() + 1);
          break;
        }
        std::vector<std::pair<long long, std::array<unsigned char, 6>>> byf;
        for (auto& kv : freq) byf.push_back({kv.second, kv.first});
        std::stable_sort(byf.begin(), byf.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
        std::map<std::array<unsigned char, 6>, int> top;
        for (int q = 0; q < 31; q++) top.emplace(byf[q].second, 1);
        for (size_t q = 0; q < cands.size(); q++) {
          if (!keep[q]) continue;
          const FluxPair& p = pairs[cands[q].i];
          if (!top.count(vc[p.v0]) || !top.count(vc[p.v1])) keep[q] = 0;
        }
      }
      std::vector<size_t> taken;
      for (size_t q = 0; q < cands.size(); q++)
        if (keep[q]) taken.push_back(cands[q].i);
      if (patterns.empty() && !vc.empty()) ok = false;
      if (getenv("CSP_DEBUG"))
        fprintf(stderr, "csp: realisation %d: %zu density pairs, %zu fused, %zu flux patterns\n", r, cand.size(),
                ok ? taken.size() : (size_t)0, patterns.size());
      if (ok && !taken.empty()) {
        memset(D.fpat, 0, sizeof D.fpat);
        for (auto& kv : patterns)
          for (int k = 0; k < 6; k++) D.fpat[kv.second][k] = kv.first[k];
        for (auto& kv : vc) hostd[kv.first] = (unsigned char)(hostd[kv.first] | (patterns[kv.second] << 3));
        for (size_t i : taken) fused[i] = 1;
        nfused = (int64_t)taken.size();
      }
    }
    cudaMemcpyAsync((void*)D.dom, hostd.data(), hr.field_elems, cudaMemcpyHostToDevice, h->stream);
    chunk_classes(D, hostd, hr.cls);
    D.ncls = (D.plane + CLASS_L - 1) / CLASS_L;
    cudaStreamSynchronize(h->stream);
    // initial channel states (BoundaryFluxes_init_stochastic_boundaries, boundaryfluxes.c:544-605)
    int ndiscrete = 0;
    for (int bi = 0; bi < m.num_boundaries; bi++) ndiscrete += m.boundaries[bi].type == CSP_BOUNDARY_DISCRETE;
    if (m.use_ryr && ndiscrete > 0) {
      const int rb = bmap[0];
      const std::vector<unsigned>& rv = bvox[rb];
      const int nr = (int)(rv.size() / 6);
      auto c0_at = [&](const std::vector<unsigned>& bv, int i) -> double {
        const unsigned* c = &bv[6 * i + 3];
        const int x = c[0], y = c[1], z = c[2];
        const unsigned char dd = m.voxels[((size_t)(x / d.S) * m.N[1] + y / d.S) * m.N[2] + z / d.S];
        return m.domain[dd].init[0];
      };
      auto init_boundary = [&](int bi, const csp_ryr_params& rp, const char* bname, bool use_ryr_values) -> int {
        const int base = hr.boundary_channel_base[bi];
        if (base < 0) return CSP_OK;
        const int nchb = hr.boundary_nch[bi];
        const csp_open_list* ol = open_list(o, bname);
        if (ol) {
          for (int i = 0; i < ol->count; i++) {
            if (ol->indices[i] < 0 || ol->indices[i] >= nchb) return CSP_ERANGE;
            states0[base + ol->indices[i]] = 1;
          }
          return CSP_OK;
        }
        FluxParams fp;
        ryr_params(fp, rp, -1);
        const double* p = fp.p;
        for (int i = 0; i < nchb; i++) {
          // the reference reads the ryr boundary's Ca for the p_ryr draw (boundaryfluxes.c:595-597)
          const double c0 = use_ryr_values && i < nr ? c0_at(rv, i) : c0_at(bvox[bi], i);
          const double ko = std::fmax(std::fmin(std::pow(c0 / p[9], p[2]), p[3]), p[4]);
          const double kc = std::fmax(std::fmin(std::pow(c0 / p[0], p[5]), p[1]), p[7]);
          const double rv_ = channel_uniform(o.seed, (unsigned)(r + o.stream_offset), (unsigned)i, (unsigned)bi, 0);
          states0[base + i] = rv_ <= kc / (ko + kc) ? 0 : 1;
        }
        return CSP_OK;
      };
      if (init_boundary(rb, m.ryr, m.ryr.boundary, false)) { csp_destroy(h); return fail(nullptr, CSP_ERANGE, "-O index out of range for %s", m.ryr.boundary); }
      if (m.use_p_ryr && bmap[1] >= 0 &&
          init_boundary(bmap[1], m.p_ryr, m.p_ryr.boundary, true)) {
        csp_destroy(h);
        return fail(nullptr, CSP_ERANGE, "-O index out of range for %s", m.p_ryr.boundary);
      }
    }
    // info
    csp_info& in = hr.info;
    memset(&in, 0, sizeof in);
    in.fused_pairs = nfused;
    in.n[0] = d.nx; in.n[1] = d.ny; in.n[2] = d.nz;
    in.subdivisions = d.S; in.h = d.h; in.dt = d.dt;
    in.num_species = m.num_species; in.num_diffusive = d.ndiff;
    for (int k = 0; k < d.ndiff; k++) { in.diffusive_species[k] = d.diff_species[k]; in.substeps[k] = d.substeps[k]; }
    in.num_buffers = d.nbuf;
    in.stochastic_substep = d.stochastic_substep;
    in.reaction_substep = d.reaction_substep;
    in.total_steps = d.total_steps;
    for (int bi = 0; bi < m.num_boundaries; bi++) in.num_channels[bi] = hr.boundary_nch[bi];
    RealCtl& c = ctl[r];
    memset(&c, 0, sizeof c);
    c.last_closed = -1.0;
    c.stopped = d.total_steps <= 0 ? 1 : 0;
  }
  h->nch = (int)states0.size();
  // -- flux rows: group pair sides by (realisation, species, voxel), pair order kept --
  struct Side { int r, s; long long v; int pair; float sign; int owner; };
  std::vector<Side> sides;
  for (int i = 0; i < (int)pairs.size(); i++) {
    const FluxPair& p = pairs[i];
    if (fused[i]) continue;
    sides.push_back({p.r, p.species, p.v1, i, 1.f, p.channel >= 0 ? 1 : 0});
    if (p.inner) sides.push_back({p.r, p.species, p.v0, i, -1.f, 0});
  }
  std::stable_sort(sides.begin(), sides.end(), [](const Side& a, const Side& b) {
    if (a.r != b.r) return a.r < b.r;
    if (a.s != b.s) return a.s < b.s;
    if (a.v != b.v) return a.v < b.v;
    return a.pair < b.pair;
  });
  std::vector<FluxRow> rows;
  std::vector<FluxEntry> entries;
  for (size_t i = 0; i < sides.size();) {
    size_t j = i;
    FluxRow row;
    memset(&row, 0, sizeof row);
    row.r = sides[i].r; row.v = sides[i].v;
    row.species = (unsigned char)sides[i].s;
    {
      const FluxPair& p0 = pairs[sides[i].pair];
      row.v0 = p0.v0; row.v1 = p0.v1; row.param = p0.param; row.channel = p0.channel;
      row.local_channel = p0.local_channel; row.sign = sides[i].sign;
      row.dsi = (unsigned char)p0.dsi; row.kind = (unsigned char)p0.kind; row.owner = (unsigned char)sides[i].owner;
      row.boundary = (unsigned char)p0.boundary;
      row.doms = (unsigned char)p0.doms;
    }
    j = i + 1;
    row.more_begin = (int)entries.size();
    while (j < sides.size() && sides[j].r == row.r && sides[j].s == row.species && sides[j].v == row.v) {
      FluxEntry en;
      en.pair = sides[j].pair; en.sign = sides[j].sign; en.owner = sides[j].owner; en.pad = 0;
      entries.push_back(en);
      j++;
    }
    row.more_end = (int)entries.size();
    // a voxel reset by the fixed-value rules after the step keeps its reset value
    const HostReal& rr = h->real[row.r];
    const RealDesc& D = rr.desc;
    const int c0 = (int)(row.v / D.P), p = (int)(row.v - (long long)c0 * D.P);
    const int c1 = p / D.nz, c2 = p - c1 * D.nz;
    int ph[3];
    ph[rr.perm[0]] = c0; ph[rr.perm[1]] = c1; ph[rr.perm[2]] = c2;
    const int S = dv[row.r].S;
    const unsigned char dd = models[row.r].voxels[((size_t)(ph[0] / S) * models[row.r].N[1] + ph[1] / S) * models[row.r].N[2] + ph[2] / S];
    const bool face = c0 == 0 || c0 == D.nx - 1 || c1 == 0 || c1 == D.ny - 1 || c2 == 0 || c2 == D.nz - 1;
    row.apply = !((D.fixed_mask[dd] >> row.species) & 1u) && !(D.dirichlet && row.species == 0 && face);
    rows.push_back(row);
    h->real[row.r].info.flux_rows++;
    i = j;
  }
  h->nrows = (int)rows.size();
  // rows touched by density pairs only first (gating-free launch), channel rows after
  auto has_channel = [&](const FluxRow& rw) {
    if (rw.channel >= 0) return true;
    for (int e = rw.more_begin; e < rw.more_end; e++)
      if (pairs[entries[e].pair].channel >= 0) return true;
    return false;
  };
  std::stable_partition(rows.begin(), rows.end(), [&](const FluxRow& rw) { return !has_channel(rw); });
  h->nrows_density = 0;
  while (h->nrows_density < h->nrows && !has_channel(rows[h->nrows_density])) h->nrows_density++;
  // the density rows in 32 bytes, when every one fits the compact form
  std::vector<DensityRow> drows;
  for (int i = 0; i < h->nrows_density; i++) {
    const FluxRow& rw = rows[i];
    const RealDesc& D = h->real[rw.r].desc;
    const long long lim = 0x7fffffffll;
    const bool to = rw.v == rw.v1 && rw.sign > 0.f, from = rw.v == rw.v0 && rw.sign < 0.f;
    const long long vo = to ? rw.v0 : rw.v1;
    if (!(to || from) || rw.v > lim || vo > lim || rw.v < 0 || vo < 0 || rw.param < 0 || rw.param > 0xffff ||
        rw.species >= NS || rw.dsi >= D.ndiff || rw.more_end - rw.more_begin > 0xff) {
      drows.clear();
      break;
    }
    DensityRow d;
    d.v = (int)rw.v;
    d.vo = (int)vo;
    d.r = rw.r;
    d.more_begin = rw.more_begin;
    d.scale = rw.kind == FLUX_SERCA ? params[rw.param].p[9] : 0.0;
    d.meta0 = (unsigned)rw.param | ((unsigned)rw.species << 16) | ((unsigned)rw.dsi << 24);
    const unsigned d0 = rw.doms & DOMAIN_BITS, d1 = (rw.doms >> 3) & DOMAIN_BITS;
    d.meta1 = (rw.apply ? DROW_APPLY : 0u) | (to ? DROW_TO : 0u) | (rw.kind == FLUX_SERCA ? DROW_SERCA : 0u) |
              ((unsigned)(rw.more_end - rw.more_begin) << 8) | (to ? d1 : d0) << 16 | (to ? d0 : d1) << 19;
    drows.push_back(d);
  }
  // pairs whose two voxels have single-pair rows: one pair row instead of two rows
  if (!drows.empty()) {
    std::vector<int> byv(drows.size());
    for (size_t i = 0; i < byv.size(); i++) byv[i] = (int)i;
    std::sort(byv.begin(), byv.end(), [&](int x, int y) {
      return drows[x].r != drows[y].r ? drows[x].r < drows[y].r : drows[x].v < drows[y].v;
    });
    std::vector<char> gone(drows.size(), 0);
    for (size_t i = 0; i < drows.size(); i++) {
      DensityRow& t = drows[i];
      if (!(t.meta1 & DROW_TO) || ((t.meta1 >> 8) & 0xffu) != 0u) continue;
      auto it = std::lower_bound(byv.begin(), byv.end(), 0, [&](int x, int) {
        return drows[x].r != t.r ? drows[x].r < t.r : drows[x].v < t.vo;
      });
      if (it == byv.end() || drows[*it].r != t.r || drows[*it].v != t.vo) continue;
      const DensityRow& f = drows[*it];
      if ((f.meta1 & (DROW_TO | DROW_PAIR)) || ((f.meta1 >> 8) & 0xffu) != 0u || f.vo != t.v || f.meta0 != t.meta0 ||
          gone[*it])
        continue;
      t.meta1 |= DROW_PAIR | ((f.meta1 & DROW_APPLY) ? DROW_APPLY_FROM : 0u);
      gone[*it] = 1;
    }
    size_t k = 0;
    for (size_t i = 0; i < drows.size(); i++)
      if (!gone[i]) drows[k++] = drows[i];
    drows.resize(k);
  }
  h->ndrows = (int)drows.size();
  {
    auto firsts = [&](std::vector<int>& f, int count, auto r_of) {
      f.assign(n + 1, count);
      for (int i = count - 1; i >= 0; i--) f[r_of(i)] = i;
      for (int r = n - 1; r >= 0; r--) f[r] = std::min(f[r], f[r + 1]);
    };
    firsts(h->drow_first, h->ndrows, [&](int i) { return drows[i].r; });
    firsts(h->krow_first, h->nrows_density, [&](int i) { return rows[i].r; });
    firsts(h->crow_first, h->nrows - h->nrows_density, [&](int i) { return rows[h->nrows_density + i].r; });
  }
  auto upload = [&](void** dst, const void* src, size_t bytes) -> bool {
    if (bytes == 0) bytes = 16;
    if (cudaMalloc(dst, bytes) != cudaSuccess) return false;
    if (src) cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, h->stream);
    return cudaStreamSynchronize(h->stream) == cudaSuccess;
  };
  std::vector<unsigned char> st2(2 * (size_t)std::max(h->nch, 1), 0);
  std::copy(states0.begin(), states0.end(), st2.begin());
  size_t cls_total = 0;
  for (int r = 0; r < n; r++) cls_total += h->real[r].cls.size();
  std::vector<unsigned char> cls_all;
  cls_all.reserve(cls_total);
  for (int r = 0; r < n; r++) cls_all.insert(cls_all.end(), h->real[r].cls.begin(), h->real[r].cls.end());
  if (!upload((void**)&h->d_cls, cls_all.empty() ? nullptr : cls_all.data(), cls_all.size())) {
    csp_destroy(h);
    return fail(nullptr, CSP_ENOMEM, "device allocation of the chunk class table failed");
  }
  std::vector<RealDesc> descs(n);
  for (int r = 0, off = 0; r < n; r++) {
    h->real[r].desc.cls = h->d_cls + off;
    off += (int)h->real[r].cls.size();
    descs[r] = h->real[r].desc;
  }
  std::vector<StepRec> recs(n);
  for (int r = 0; r < n; r++) write_steprec(descs[r], ctl[r], recs[r]);
  bool ok = upload((void**)&h->d_rec, recs.data(), recs.size() * sizeof(StepRec)) &&
            (drows.empty() || upload((void**)&h->d_drows, drows.data(), drows.size() * sizeof(DensityRow))) &&
            upload((void**)&h->d_rows, rows.empty() ? nullptr : rows.data(), rows.size() * sizeof(FluxRow)) &&
            upload((void**)&h->d_entries, entries.empty() ? nullptr : entries.data(), entries.size() * sizeof(FluxEntry)) &&
            upload((void**)&h->d_pairs, pairs.empty() ? nullptr : pairs.data(), pairs.size() * sizeof(FluxPair)) &&
            upload((void**)&h->d_params, params.empty() ? nullptr : params.data(), params.size() * sizeof(FluxParams)) &&
            upload((void**)&h->d_states, st2.data(), st2.size());
  if (!ok) { csp_destroy(h); return fail(nullptr, CSP_ENOMEM, "device allocation of flux tables failed"); }
  if ((e = cudaMemcpyAsync(h->d_desc, descs.data(), n * sizeof(RealDesc), cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(h->d_ctl, ctl.data(), n * sizeof(RealCtl), cudaMemcpyHostToDevice, h->stream)) != cudaSuccess) {
    csp_destroy(h);
    return fail(nullptr, CSP_ECUDA, "descriptor upload: %s", cudaGetErrorString(e));
  }
  const int red_blocks = 296;
  if (cudaMalloc(&h->d_red, red_blocks * 3 * ND * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&h->d_red_out, 3 * ND * sizeof(double)) != cudaSuccess) {
    csp_destroy(h);
    return fail(nullptr, CSP_ENOMEM, "device allocation of reduction buffers failed");
  }
  h->plan = staged_plan(descs);
  if (staged_prepare(h->plan) != cudaSuccess) h->kernel = 1;
  e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) { csp_destroy(h); return fail(nullptr, CSP_ECUDA, "setup: %s", cudaGetErrorString(e)); }
  *out = h;
  return CSP_OK;
}

// The kernels of one step, for the realisations [r0, r1) (r1 < 0: all of them, the
// launches csp_advance captures).  Realisations are independent, so stepping a range
// gives that range exactly what a step of the whole batch gives it.
static void launch_voxels(csp_handle* h, int r0 = 0, int r1 = -1) {
  if (r1 < 0) r1 = h->n;
  if (h->kernel == 1) {
    dim3 grid((unsigned)((h->max_vox + 255) / 256), (unsigned)(r1 - r0));
    k_voxels_direct<<<grid, 256, 0, h->stream>>>(h->d_desc + r0, h->d_ctl + r0, h->d_err);
  } else {
    staged_launch(h->plan, h->d_desc, h->d_ctl, h->d_err, h->stream, h->inject_wait != 0, r0, r1, h->surrogate != 0);
  }
}

// The flux-row kernels of one step: density-boundary rows (SERCA), then the channel rows
// (gating + RyR flux), for the realisations [r0, r1).
static void launch_density_rows(csp_handle* h, int r0, int r1) {
  const int nd = h->nrows_density;
  const int dr0 = h->drow_first[r0], dr1 = h->drow_first[r1];
  const int kr0 = h->krow_first[r0], kr1 = h->krow_first[r1];
  if (nd > 0 && h->d_drows) {
    if (dr1 > dr0)
      k_density_rows<<<(dr1 - dr0 + 255) / 256, 256, 0, h->stream>>>(h->d_desc, h->d_rec, h->d_drows + dr0,
                                                                     dr1 - dr0, h->d_entries, h->d_pairs,
                                                                     h->d_params);
  } else if (kr1 > kr0) {
    k_boundaries<false><<<(kr1 - kr0 + 255) / 256, 256, 0, h->stream>>>(h->d_desc, h->d_ctl, h->d_rows + kr0,
                                                                         kr1 - kr0, h->d_entries, h->d_pairs,
                                                                         h->d_params, h->d_states,
                                                                         std::max(h->nch, 1));
  }
}

static void launch_channel_rows(csp_handle* h, int r0, int r1) {
  const int nd = h->nrows_density;
  const int cr0 = h->crow_first[r0], cr1 = h->crow_first[r1];
  if (cr1 > cr0)
    k_boundaries<true><<<(cr1 - cr0 + 255) / 256, 256, 0, h->stream>>>(h->d_desc, h->d_ctl, h->d_rows + nd + cr0,
                                                                        cr1 - cr0, h->d_entries, h->d_pairs,
                                                                        h->d_params, h->d_states,
                                                                        std::max(h->nch, 1));
}

// The network kernel's instantiations for the fixed-point species of the ensemble (none,
// TRPN's slot alone, or any slot).
using NetworkKernel = void (*)(const RealDesc*, const RealCtl*, const float*, float, const unsigned short*,
                               const unsigned*, const unsigned*, unsigned*, int, unsigned long long*);
static NetworkKernel network_kernel(unsigned fq) {
  return fq == 0u ? k_react_network<0u> : fq == 0x10u ? k_react_network<0x10u> : k_react_network<0x3Eu>;
}
using NetworkUmmaKernel = void (*)(const RealDesc*, const RealCtl*, const float*, float, const unsigned short*,
                                   const unsigned*, const unsigned*, unsigned*, int, unsigned long long*, int*);
static NetworkUmmaKernel network_kernel_umma(unsigned fq) {
  return fq == 0u ? k_react_network_umma<0u> : fq == 0x10u ? k_react_network_umma<0x10u> : k_react_network_umma<0x3Eu>;
}
using PlainKernel = void (*)(const RealDesc*, const RealCtl*, const unsigned short*, const unsigned*,
                             const unsigned*, unsigned*, int, unsigned long long*);
static PlainKernel plain_kernel(unsigned fq) {
  return fq == 0u ? k_react_plain<0u> : fq == 0x10u ? k_react_plain<0x10u> : k_react_plain<0x3Eu>;
}

static void launch_surrogate(csp_handle* h, int r0, int r1) {
  if (!h->surrogate) return;
  const int chunks = (int)((h->max_field + MLP_DEPLOY_SPAN - 1) / MLP_DEPLOY_SPAN);
  const long long nseg = (long long)chunks * (r1 - r0);
  unsigned* tiles_plain = h->d_sur_tiles + h->sur_tile_cap;
  k_react_surrogate<<<(unsigned)std::min<long long>(nseg, 2 * h->sur_network_ctas), MLP_DEPLOY_T, 0, h->stream>>>(
      h->d_desc + r0, h->d_ctl + r0, chunks, r1 - r0, h->d_sur_list, h->d_sur_counts, h->d_sur_tiles, tiles_plain,
      h->d_sur_queue,
      h->d_mlp_cnt);
  plain_kernel(h->surrogate_fq)<<<h->sur_plain_ctas, MLP_DEPLOY_T, 0, h->stream>>>(
      h->d_desc + r0, h->d_ctl + r0, h->d_sur_list, h->d_sur_counts, tiles_plain, h->d_sur_queue + 2, chunks,
      h->d_mlp_cnt);
  if (h->sur_tc == 2)
    network_kernel_umma(h->surrogate_fq)<<<h->sur_umma_ctas, UM_T * UM_NET_WGS, UM_NET_SMEM, h->stream>>>(
        h->d_desc + r0, h->d_ctl + r0, h->d_mlp, h->surrogate_tol, h->d_sur_list, h->d_sur_counts, h->d_sur_tiles,
        h->d_sur_queue, chunks, h->d_mlp_cnt, h->d_err);
  else
    network_kernel(h->surrogate_fq)<<<h->sur_network_ctas, MLP_DEPLOY_T, MLP_NETWORK_SMEM, h->stream>>>(
        h->d_desc + r0, h->d_ctl + r0, h->d_mlp, h->surrogate_tol, h->d_sur_list, h->d_sur_counts, h->d_sur_tiles,
        h->d_sur_queue, chunks, h->d_mlp_cnt);
}

static void launch_epilogue(csp_handle* h, int r0, int r1, int* step_flags) {
  k_epilogue<<<(r1 - r0 + 127) / 128, 128, 0, h->stream>>>(h->d_desc + r0, h->d_ctl + r0, h->d_rec + r0, r1 - r0,
                                                           step_flags, h->surrogate ? h->d_sur_queue : nullptr);
}

static void launch_boundaries(csp_handle* h, int r0 = 0, int r1 = -1, int* step_flags = nullptr) {
  if (r1 < 0) r1 = h->n;
  launch_density_rows(h, r0, r1);
  launch_channel_rows(h, r0, r1);
  launch_surrogate(h, r0, r1);
  launch_epilogue(h, r0, r1, step_flags);
}

// One step of every realisation with an event before and after each phase (CSP_PHASE_*).
static void launch_step_timed(csp_handle* h, cudaEvent_t* ev) {
  cudaEventRecord(ev[0], h->stream);
  launch_voxels(h);
  cudaEventRecord(ev[1 + CSP_PHASE_VOXELS], h->stream);
  launch_density_rows(h, 0, h->n);
  cudaEventRecord(ev[1 + CSP_PHASE_DENSITY], h->stream);
  launch_channel_rows(h, 0, h->n);
  cudaEventRecord(ev[1 + CSP_PHASE_CHANNELS], h->stream);
  launch_surrogate(h, 0, h->n);
  cudaEventRecord(ev[1 + CSP_PHASE_SURROGATE], h->stream);
  launch_epilogue(h, 0, h->n, nullptr);
  cudaEventRecord(ev[1 + CSP_PHASE_EPILOGUE], h->stream);
}

static cudaError_t launch_step(csp_handle* h, int r0 = 0, int r1 = -1, int* step_flags = nullptr) {
  launch_voxels(h, r0, r1);
  launch_boundaries(h, r0, r1, step_flags);
  return cudaGetLastError();
}

static int ensure_graph(csp_handle* h) {
  if (h->graph && h->graph_kernel == h->kernel && h->graph_surrogate == h->surrogate && h->graph_sur_tc == h->sur_tc &&
      h->graph_plan == h->plan_epoch)
    return CSP_OK;
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
  cudaGraph_t g;
  CUDA_TRY(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < STEPS_PER_GRAPH; i++) {
    cudaError_t e = launch_step(h);
    if (e != cudaSuccess) {
      cudaStreamEndCapture(h->stream, &g);
      return fail(h, CSP_ECUDA, "capture: %s", cudaGetErrorString(e));
    }
  }
  CUDA_TRY(h, cudaStreamEndCapture(h->stream, &g));
  cudaError_t e = cudaGraphInstantiate(&h->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) { h->graph = nullptr; return fail(h, CSP_ECUDA, "graph instantiate: %s", cudaGetErrorString(e)); }
  h->graph_kernel = h->kernel;
  h->graph_plan = h->plan_epoch;
  h->graph_surrogate = h->surrogate;
  h->graph_sur_tc = h->sur_tc;
  return CSP_OK;
}

// The timed sample of the last advance call, scaled to the call's steps, into phase_ms.
static void add_phase_sample(csp_handle* h) {
  if (!h->phase_sampled) return;
  double ms[CSP_NUM_PHASES] = {};
  for (int i = 0; i < h->phase_sampled; i++) {
    const cudaEvent_t* ev = &h->phase_ev[i * (CSP_NUM_PHASES + 1)];
    for (int p = 0; p < CSP_NUM_PHASES; p++) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, ev[p], ev[p + 1]) == cudaSuccess) ms[p] += t;
    }
  }
  const double scale = (double)h->phase_call_steps / h->phase_sampled;
  for (int p = 0; p < CSP_NUM_PHASES; p++) h->phase_ms[p] += ms[p] * scale;
  h->phase_steps += h->phase_call_steps;
  h->phase_sampled = 0;
}

static int finish_advance(csp_handle* h, int32_t* stop_flags) {
  int err = 0;
  CUDA_TRY(h, cudaMemcpyAsync(&err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  std::vector<RealCtl> ctl(h->n);
  CUDA_TRY(h, cudaMemcpyAsync(ctl.data(), h->d_ctl, h->n * sizeof(RealCtl), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  for (int r = 0; r < h->n; r++) {
    h->real[r].info.step = ctl[r].step;
    h->real[r].info.stopped = ctl[r].stopped;
    if (stop_flags) stop_flags[r] = ctl[r].stopped;
  }
  add_phase_sample(h);
  if (err) return fail(h, CSP_EDEVICE, "device error word %d (%s)", err,
                       (err & ERR_TIMEOUT) ? "bounded wait timed out" : "index out of bounds");
  return CSP_OK;
}

extern "C" int csp_profile_advance(csp_handle* h, int64_t nsteps, float* voxel_ms, float* boundary_ms) {
  if (!h || nsteps < 0) return fail(h, CSP_EINVAL, "bad handle or nsteps");
  CSP_NOT_PENDING(h);
  std::vector<cudaEvent_t> ev(3 * (size_t)nsteps);
  for (auto& e : ev) CUDA_TRY(h, cudaEventCreate(&e));
  for (int64_t i = 0; i < nsteps; i++) {
    cudaEventRecord(ev[3 * i], h->stream);
    launch_voxels(h);
    cudaEventRecord(ev[3 * i + 1], h->stream);
    launch_boundaries(h);
    cudaEventRecord(ev[3 * i + 2], h->stream);
  }
  cudaError_t le = cudaGetLastError();
  int rc = finish_advance(h, nullptr);
  float tv = 0.f, tb = 0.f;
  for (int64_t i = 0; i < nsteps; i++) {
    float a = 0.f, b = 0.f;
    cudaEventElapsedTime(&a, ev[3 * i], ev[3 * i + 1]);
    cudaEventElapsedTime(&b, ev[3 * i + 1], ev[3 * i + 2]);
    tv += a;
    tb += b;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (le != cudaSuccess) return fail(h, CSP_ECUDA, "launch: %s", cudaGetErrorString(le));
  if (voxel_ms) *voxel_ms = tv;
  if (boundary_ms) *boundary_ms = tb;
  return rc;
}

static int launch_advance(csp_handle* h, int64_t nsteps) {
  if (!h->inject_wait) {
    int rc = ensure_graph(h);
    if (rc) return rc;
  }
  CUDA_TRY(h, cudaEventRecord(h->ev0, h->stream));
  int64_t left = nsteps;
  h->phase_sampled = 0;
  if (h->phase_timing && left > 0) {
    const int ns = (int)std::min<int64_t>(left, PHASE_SAMPLE);
    for (int i = 0; i < ns; i++) launch_step_timed(h, &h->phase_ev[i * (CSP_NUM_PHASES + 1)]);
    CUDA_TRY(h, cudaGetLastError());
    h->phase_sampled = ns;
    h->phase_call_steps = nsteps;
    left -= ns;
  }
  while (!h->inject_wait && left >= STEPS_PER_GRAPH) {
    CUDA_TRY(h, cudaGraphLaunch(h->graph, h->stream));
    left -= STEPS_PER_GRAPH;
  }
  while (left-- > 0) CUDA_TRY(h, launch_step(h));
  CUDA_TRY(h, cudaEventRecord(h->ev1, h->stream));
  return CSP_OK;
}

extern "C" int csp_advance(csp_handle* h, int64_t nsteps, int32_t* stop_flags) {
  if (!h || nsteps < 0) return fail(h, CSP_EINVAL, "bad handle or nsteps");
  if (h->advance_pending) return fail(h, CSP_EINVAL, "an asynchronous advance is pending (csp_advance_wait)");
  int rc = launch_advance(h, nsteps);
  if (rc) return rc;
  int rc2 = finish_advance(h, stop_flags);
  cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1);
  return rc2;
}

extern "C" int csp_advance_async(csp_handle* h, int64_t nsteps) {
  if (!h || nsteps < 0) return fail(h, CSP_EINVAL, "bad handle or nsteps");
  if (h->advance_pending) return fail(h, CSP_EINVAL, "an asynchronous advance is pending (csp_advance_wait)");
  int rc = launch_advance(h, nsteps);
  if (rc) return rc;
  h->advance_pending = true;
  return CSP_OK;
}

extern "C" int csp_advance_wait(csp_handle* h, int32_t* stop_flags) {
  if (!h) return CSP_EINVAL;
  if (!h->advance_pending) return fail(h, CSP_EINVAL, "no asynchronous advance is pending");
  h->advance_pending = false;
  int rc = finish_advance(h, stop_flags);
  cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1);
  return rc;
}

static int read_ctl(csp_handle* h, int r, RealCtl& c) {
  CUDA_TRY(h, cudaMemcpyAsync(&c, h->d_ctl + r, sizeof(RealCtl), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return CSP_OK;
}

extern "C" int csp_get_info(const csp_handle* h, int32_t r, csp_info* info) {
  if (!h || !info) return CSP_EINVAL;
  if (r < 0 || r >= h->n) return CSP_ERANGE;
  *info = h->real[r].info;
  return CSP_OK;
}

// Physical-order host state (FP64 or FP32) <-> device-order FP32 fields of one realisation:
// one thread per (species, physical voxel); the physical index is linear (coalesced
// host-side layout), the device index follows the realisation's axis order.  Which buffer
// of a species is current is read from the realisation's progress block when the kernel
// runs, so a conversion queued behind steps converts what those steps leave current.
struct StateMap {
  float* f[2][NS];                   // both buffers of each species
  const RealCtl* ctl;                // the realisation's progress block
  const unsigned char* dom;          // domain bytes (device order)
  double base[ND][NS];               // field bases: value = base[domain][s] + field
  unsigned fixq;                     // fixed-point species: value = base + q * qunit
  float qunit[ND][NS];
  int n[3];                          // physical voxels per axis
  long long stride[3];               // device index stride of each physical axis
  long long nvox;
  int ns;
};

__device__ __forceinline__ long long state_index(const StateMap& m, long long v) {
  const int z = (int)(v % m.n[2]);
  const long long xy = v / m.n[2];
  const int y = (int)(xy % m.n[1]), x = (int)(xy / m.n[1]);
  return x * m.stride[0] + y * m.stride[1] + z * m.stride[2];
}

__device__ __forceinline__ float* state_field(const StateMap& m, int s) {
  const unsigned cur = m.ctl->cur_mask[m.ctl->step & 1];
  return m.f[(cur >> s) & 1u][s];
}

// host value u -> stored deviation (float)(u - base), one rounding
template <class T>
__global__ void k_state_in(const T* __restrict__ src, StateMap m) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= m.nvox * m.ns) return;
  const int s = (int)(i / m.nvox);
  const long long di = state_index(m, i - (long long)s * m.nvox);
  const int d = m.dom[di] & DOMAIN_BITS;
  const double dev = (double)src[i] - m.base[d][s];
  if (m.fixq >> s & 1u) {   // round to the unit, saturated to the integer range
    const double q = fmin(fmax(rint(dev / m.qunit[d][s]), -2147483647.0), 2147483647.0);
    state_field(m, s)[di] = __int_as_float((int)q);
  } else {
    state_field(m, s)[di] = (float)dev;
  }
}

__device__ __forceinline__ double state_value(const StateMap& m, int s, long long di) {
  const int d = m.dom[di] & DOMAIN_BITS;
  const float f = state_field(m, s)[di];
  const double dev = (m.fixq >> s & 1u) ? (double)__float_as_int(f) * m.qunit[d][s] : (double)f;
  return dev + m.base[d][s];
}

// stored deviation -> host value (double)field + base (FP32 hosts: rounded once more)
template <class T>
__global__ void k_state_out(T* __restrict__ dst, StateMap m) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= m.nvox * m.ns) return;
  const int s = (int)(i / m.nvox);
  dst[i] = static_cast<T>(state_value(m, s, state_index(m, i - (long long)s * m.nvox)));
}

// One species of the physical-order FP64 state (the species slot of k_state_out's output).
__global__ void k_state_out_species(double* __restrict__ dst, StateMap m, int s) {
  const long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (v >= m.nvox) return;
  dst[v] = state_value(m, s, state_index(m, v));
}

static StateMap make_state_map(const csp_handle* h, int r) {
  StateMap m;
  memset(&m, 0, sizeof m);
  const HostReal& hr = h->real[r];
  const RealDesc& D = hr.desc;
  m.ns = D.ns;
  for (int s = 0; s < D.ns; s++) { m.f[0][s] = D.u[0][s]; m.f[1][s] = D.u[1][s]; }
  m.ctl = h->d_ctl + r;
  m.dom = D.dom;
  memcpy(m.base, D.base, sizeof m.base);
  m.fixq = D.fixq;
  memcpy(m.qunit, D.qunit, sizeof m.qunit);
  for (int a = 0; a < 3; a++) m.n[a] = hr.nphys[a];
  // device axis i holds physical axis perm[i]; device strides P, nz, 1
  const long long dstr[3] = {(long long)D.P, (long long)D.nz, 1};
  for (int i = 0; i < 3; i++) m.stride[hr.perm[i]] = dstr[i];
  m.nvox = (long long)m.n[0] * m.n[1] * m.n[2];
  return m;
}

static int ensure_stage(csp_handle* h, size_t bytes) {
  if (bytes <= h->stage_bytes) return CSP_OK;
  cudaFree(h->d_stage);
  h->d_stage = nullptr;
  h->stage_bytes = 0;
  if (cudaMalloc(&h->d_stage, bytes) != cudaSuccess)
    return fail(h, CSP_ENOMEM, "state staging buffer of %.1f MB", bytes / 1e6);
  h->stage_bytes = bytes;
  return CSP_OK;
}

static unsigned blocks_of(long long n) { return (unsigned)((n + 255) / 256); }

// Realisations [r0, r1) from host arrays u[r] (a staging buffer reused in stream order),
// one wait at the end.
template <class T>
static int upload_range(csp_handle* h, const T* const* u, int r0, int r1) {
  size_t need = 0;
  for (int r = r0; r < r1; r++) {
    if (!u[r - r0]) return fail(h, CSP_EINVAL, "NULL state of realisation %d", r);
    const StateMap m = make_state_map(h, r);
    need = std::max(need, (size_t)(m.nvox * m.ns) * sizeof(T));
  }
  int rc = ensure_stage(h, need);
  if (rc) return rc;
  for (int r = r0; r < r1; r++) {
    const StateMap m = make_state_map(h, r);
    const long long n = m.nvox * m.ns;
    CUDA_TRY(h, cudaMemcpyAsync(h->d_stage, u[r - r0], n * sizeof(T), cudaMemcpyHostToDevice, h->stream));
    k_state_in<T><<<blocks_of(n), 256, 0, h->stream>>>(static_cast<const T*>(h->d_stage), m);
    CUDA_TRY(h, cudaGetLastError());
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return CSP_OK;
}

template <class T>
static int download_range(csp_handle* h, T* const* u, int r0, int r1) {
  size_t need = 0;
  for (int r = r0; r < r1; r++) {
    if (!u[r - r0]) return fail(h, CSP_EINVAL, "NULL state of realisation %d", r);
    const StateMap m = make_state_map(h, r);
    need = std::max(need, (size_t)(m.nvox * m.ns) * sizeof(T));
  }
  int rc = ensure_stage(h, need);
  if (rc) return rc;
  for (int r = r0; r < r1; r++) {
    const StateMap m = make_state_map(h, r);
    const long long n = m.nvox * m.ns;
    k_state_out<T><<<blocks_of(n), 256, 0, h->stream>>>(static_cast<T*>(h->d_stage), m);
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaMemcpyAsync(u[r - r0], h->d_stage, n * sizeof(T), cudaMemcpyDeviceToHost, h->stream));
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return CSP_OK;
}

extern "C" int csp_upload_state(csp_handle* h, int32_t r, const double* u) {
  if (!h || !u) return fail(h, CSP_EINVAL, "NULL argument");
  CSP_NOT_PENDING(h);
  if (r < 0 || r >= h->n) return fail(h, CSP_ERANGE, "realisation %d out of range", r);
  return upload_range<double>(h, &u, r, r + 1);
}

extern "C" int csp_download_state(csp_handle* h, int32_t r, double* u) {
  if (!h || !u) return fail(h, CSP_EINVAL, "NULL argument");
  CSP_NOT_PENDING(h);
  if (r < 0 || r >= h->n) return fail(h, CSP_ERANGE, "realisation %d out of range", r);
  return download_range<double>(h, &u, r, r + 1);
}

extern "C" int csp_upload_states(csp_handle* h, const double* const* u) {
  if (!h || !u) return fail(h, CSP_EINVAL, "NULL argument");
  CSP_NOT_PENDING(h);
  return upload_range<double>(h, u, 0, h->n);
}

extern "C" int csp_download_states(csp_handle* h, double* const* u) {
  if (!h || !u) return fail(h, CSP_EINVAL, "NULL argument");
  CSP_NOT_PENDING(h);
  return download_range<double>(h, u, 0, h->n);
}

extern "C" int csp_upload_states_f32(csp_handle* h, const float* const* u) {
  if (!h || !u) return fail(h, CSP_EINVAL, "NULL argument");
  CSP_NOT_PENDING(h);
  return upload_range<float>(h, u, 0, h->n);
}

extern "C" int csp_download_states_f32(csp_handle* h, float* const* u) {
  if (!h || !u) return fail(h, CSP_EINVAL, "NULL argument");
  CSP_NOT_PENDING(h);
  return download_range<float>(h, u, 0, h->n);
}

// csp_run_states: groups of consecutive realisations with about equal voxel counts.
static std::vector<int> run_groups(const csp_handle* h) {
  const int G = std::min(h->n, 8);
  long long total = 0;
  for (int r = 0; r < h->n; r++) total += h->real[r].desc.nx * (long long)h->real[r].desc.plane;
  std::vector<int> b{0};
  long long acc = 0;
  for (int r = 0; r < h->n; r++) {
    acc += h->real[r].desc.nx * (long long)h->real[r].desc.plane;
    const int g = (int)b.size();
    if (g < G && r + 1 < h->n && acc * G >= total * g) b.push_back(r + 1);
  }
  b.push_back(h->n);
  return b;
}

// One ensemble job from host memory, pipelined by realisation groups on three streams:
// the input copies of group g+1 (in_stream) and the output copies of group g-1
// (snap_stream) overlap the steps of group g (the handle stream).  Each group has two
// staging slots per direction; events order the reuse of a slot after its previous group.
template <class T>
static int run_states(csp_handle* h, const T* const* uin, int64_t nsteps, T* const* uout, int32_t* stop_flags,
                      int32_t* step_flags) {
  for (int r = 0; r < h->n; r++)
    if (!uin[r] || !uout[r]) return fail(h, CSP_EINVAL, "NULL state of realisation %d", r);
  const std::vector<int> gb = run_groups(h);
  const int G = (int)gb.size() - 1;
  std::vector<long long> off(h->n + 1, 0);      // element offset of realisation r in its group's slot
  size_t slot = 0;
  for (int g = 0; g < G; g++) {
    long long o = 0;
    for (int r = gb[g]; r < gb[g + 1]; r++) {
      off[r] = o;
      const StateMap m = make_state_map(h, r);
      o += (m.nvox * m.ns + 63) / 64 * 64;       // 256-byte aligned starts
    }
    slot = std::max(slot, (size_t)o);
  }
  const size_t slot_bytes = slot * sizeof(T);
  if (4 * slot_bytes > h->pipe_bytes) {
    cudaFree(h->d_pipe);
    h->d_pipe = nullptr;
    h->pipe_bytes = 0;
    if (cudaMalloc(&h->d_pipe, 4 * slot_bytes) != cudaSuccess)
      return fail(h, CSP_ENOMEM, "pipeline staging of %.1f MB", 4.0 * slot_bytes / 1e6);
    h->pipe_bytes = 4 * slot_bytes;
  }
  if (step_flags && (size_t)nsteps * h->n > h->stepflags_elems) {
    cudaFree(h->d_stepflags);
    h->d_stepflags = nullptr;
    h->stepflags_elems = 0;
    if (cudaMalloc(&h->d_stepflags, (size_t)nsteps * h->n * sizeof(int)) != cudaSuccess)
      return fail(h, CSP_ENOMEM, "per-step flags of %lld steps", (long long)nsteps);
    h->stepflags_elems = (size_t)nsteps * h->n;
  }
  if (!h->in_stream) CUDA_TRY(h, cudaStreamCreateWithFlags(&h->in_stream, cudaStreamNonBlocking));
  if (!h->snap_stream) {
    CUDA_TRY(h, cudaStreamCreateWithFlags(&h->snap_stream, cudaStreamNonBlocking));
    CUDA_TRY(h, cudaEventCreateWithFlags(&h->ev_snap, cudaEventDisableTiming));
    CUDA_TRY(h, cudaEventCreateWithFlags(&h->ev_copy, cudaEventDisableTiming));
  }
  std::vector<cudaEvent_t> ev(2 * G + 4, nullptr);
  for (auto& e : ev) CUDA_TRY(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaEvent_t* in_ready = ev.data();
  cudaEvent_t* out_ready = ev.data() + G;
  cudaEvent_t* in_free = ev.data() + 2 * G;      // [2]
  cudaEvent_t* out_free = ev.data() + 2 * G + 2; // [2]
  T* pipe = static_cast<T*>(h->d_pipe);
  cudaStream_t cs = h->stream, is = h->in_stream, os = h->snap_stream;
  cudaError_t e = cudaEventRecord(h->ev0, cs);
  for (int g = 0; g < G && e == cudaSuccess; g++) {
    const int r0 = gb[g], r1 = gb[g + 1], k = g & 1;
    T* in_slot = pipe + (size_t)k * slot;
    T* out_slot = pipe + (size_t)(2 + k) * slot;
    if (g >= 2) e = cudaStreamWaitEvent(is, in_free[k], 0);
    for (int r = r0; r < r1 && e == cudaSuccess; r++) {
      const StateMap m = make_state_map(h, r);
      e = cudaMemcpyAsync(in_slot + off[r], uin[r], (size_t)(m.nvox * m.ns) * sizeof(T), cudaMemcpyHostToDevice, is);
    }
    if (e == cudaSuccess) e = cudaEventRecord(in_ready[g], is);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, in_ready[g], 0);
    for (int r = r0; r < r1 && e == cudaSuccess; r++) {
      const StateMap m = make_state_map(h, r);
      k_state_in<T><<<blocks_of(m.nvox * m.ns), 256, 0, cs>>>(in_slot + off[r], m);
    }
    if (e == cudaSuccess) e = cudaEventRecord(in_free[k], cs);
    for (int64_t st = 0; st < nsteps && e == cudaSuccess; st++)
      e = launch_step(h, r0, r1, step_flags ? h->d_stepflags + st * h->n + r0 : nullptr);
    if (e == cudaSuccess && g >= 2) e = cudaStreamWaitEvent(cs, out_free[k], 0);
    for (int r = r0; r < r1 && e == cudaSuccess; r++) {
      const StateMap m = make_state_map(h, r);
      k_state_out<T><<<blocks_of(m.nvox * m.ns), 256, 0, cs>>>(out_slot + off[r], m);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(out_ready[g], cs);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(os, out_ready[g], 0);
    for (int r = r0; r < r1 && e == cudaSuccess; r++) {
      const StateMap m = make_state_map(h, r);
      e = cudaMemcpyAsync(uout[r], out_slot + off[r], (size_t)(m.nvox * m.ns) * sizeof(T), cudaMemcpyDeviceToHost, os);
    }
    if (e == cudaSuccess) e = cudaEventRecord(out_free[k], os);
  }
  if (e == cudaSuccess) e = cudaEventRecord(h->ev1, cs);
  // every queued operation ends before the events go and before an error returns
  const cudaError_t e_in = cudaStreamSynchronize(is), e_out = cudaStreamSynchronize(os);
  const cudaError_t e_c = cudaStreamSynchronize(cs);
  for (auto& x : ev) cudaEventDestroy(x);
  if (e == cudaSuccess) e = e_in != cudaSuccess ? e_in : (e_out != cudaSuccess ? e_out : e_c);
  if (e != cudaSuccess) return fail(h, CSP_ECUDA, "csp_run_states: %s", cudaGetErrorString(e));
  if (step_flags && nsteps > 0)
    CUDA_TRY(h, cudaMemcpy(step_flags, h->d_stepflags, (size_t)nsteps * h->n * sizeof(int), cudaMemcpyDeviceToHost));
  const int rc = finish_advance(h, stop_flags);
  cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1);
  return rc;
}

extern "C" int csp_run_states(csp_handle* h, int32_t host_dtype, const void* const* u_in, int64_t nsteps,
                              void* const* u_out, int32_t* stop_flags, int32_t* step_flags) {
  if (!h || !u_in || !u_out || nsteps < 0) return fail(h, CSP_EINVAL, "bad argument");
  CSP_NOT_PENDING(h);
  if (h->snap_pending) return fail(h, CSP_EINVAL, "a snapshot is pending (csp_snapshot_wait)");
  if (h->inject_wait) return fail(h, CSP_EINVAL, "the wait-timeout test hook is armed");
  if (host_dtype == CSP_HOST_F32)
    return run_states<float>(h, reinterpret_cast<const float* const*>(u_in), nsteps,
                             reinterpret_cast<float* const*>(u_out), stop_flags, step_flags);
  if (host_dtype == CSP_HOST_F64)
    return run_states<double>(h, reinterpret_cast<const double* const*>(u_in), nsteps,
                              reinterpret_cast<double* const*>(u_out), stop_flags, step_flags);
  return fail(h, CSP_EINVAL, "host_dtype %d is neither CSP_HOST_F32 nor CSP_HOST_F64", host_dtype);
}

extern "C" int csp_snapshot_async(csp_handle* h, int32_t r, uint32_t species_mask) {
  if (!h) return CSP_EINVAL;
  if (r < 0 || r >= h->n) return fail(h, CSP_ERANGE, "realisation %d out of range", r);
  if (h->advance_pending) return fail(h, CSP_EINVAL, "an asynchronous advance is pending (csp_advance_wait)");
  if (h->snap_pending) return fail(h, CSP_EINVAL, "a snapshot is pending (csp_snapshot_wait)");
  const StateMap m = make_state_map(h, r);
  const size_t need = (size_t)m.nvox * m.ns;
  if (!h->snap_stream) {
    CUDA_TRY(h, cudaStreamCreateWithFlags(&h->snap_stream, cudaStreamNonBlocking));
    CUDA_TRY(h, cudaEventCreateWithFlags(&h->ev_snap, cudaEventDisableTiming));
    CUDA_TRY(h, cudaEventCreateWithFlags(&h->ev_copy, cudaEventDisableTiming));
  }
  if (need > h->snap_elems) {
    cudaFree(h->d_snap);
    cudaFreeHost(h->h_snap);
    h->d_snap = nullptr;
    h->h_snap = nullptr;
    h->snap_elems = 0;
    if (cudaMalloc(&h->d_snap, need * sizeof(double)) != cudaSuccess ||
        cudaHostAlloc(&h->h_snap, need * sizeof(double), cudaHostAllocDefault) != cudaSuccess)
      return fail(h, CSP_ENOMEM, "snapshot buffers of %.1f MB", need * 8.0 / 1e6);
    h->snap_elems = need;
  }
  // (the previous copy out of d_snap ended in csp_snapshot_wait)
  for (int sp = 0; sp < m.ns; sp++) {
    if (!(species_mask >> sp & 1u)) continue;
    k_state_out_species<<<(unsigned)((m.nvox + 255) / 256), 256, 0, h->stream>>>(h->d_snap + (size_t)sp * m.nvox, m, sp);
  }
  CUDA_TRY(h, cudaGetLastError());
  CUDA_TRY(h, cudaEventRecord(h->ev_snap, h->stream));
  CUDA_TRY(h, cudaStreamWaitEvent(h->snap_stream, h->ev_snap, 0));
  for (int sp = 0; sp < m.ns; sp++) {
    if (!(species_mask >> sp & 1u)) continue;
    const size_t off = (size_t)sp * m.nvox;
    CUDA_TRY(h, cudaMemcpyAsync(h->h_snap + off, h->d_snap + off, (size_t)m.nvox * sizeof(double),
                                cudaMemcpyDeviceToHost, h->snap_stream));
  }
  CUDA_TRY(h, cudaEventRecord(h->ev_copy, h->snap_stream));
  h->snap_pending = true;
  return CSP_OK;
}

extern "C" int csp_snapshot_wait(csp_handle* h, const double** u) {
  if (!h || !u) return CSP_EINVAL;
  if (!h->snap_pending) return fail(h, CSP_EINVAL, "no snapshot is pending");
  h->snap_pending = false;
  CUDA_TRY(h, cudaEventSynchronize(h->ev_copy));
  *u = h->h_snap;
  return CSP_OK;
}

extern "C" int csp_get_channel_states(const csp_handle* hc, int32_t r, int32_t boundary, int32_t* states) {
  csp_handle* h = const_cast<csp_handle*>(hc);
  if (!h || !states) return CSP_EINVAL;
  CSP_NOT_PENDING(h);
  if (r < 0 || r >= h->n) return fail(h, CSP_ERANGE, "realisation %d out of range", r);
  const HostReal& hr = h->real[r];
  if (boundary < 0 || boundary >= (int)hr.boundary_channel_base.size() || hr.boundary_channel_base[boundary] < 0)
    return fail(h, CSP_ERANGE, "boundary %d is not a discrete boundary", boundary);
  RealCtl c;
  int rc = read_ctl(h, r, c);
  if (rc) return rc;
  const int nchb = hr.boundary_nch[boundary];
  std::vector<unsigned char> tmp(nchb);
  CUDA_TRY(h, cudaMemcpyAsync(tmp.data(), h->d_states + (c.step & 1) * (size_t)std::max(h->nch, 1) + hr.boundary_channel_base[boundary],
                              nchb, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  for (int i = 0; i < nchb; i++) states[i] = tmp[i];
  return CSP_OK;
}

extern "C" int csp_set_channel_states(csp_handle* h, int32_t r, int32_t boundary, const int32_t* states) {
  if (!h || !states) return CSP_EINVAL;
  CSP_NOT_PENDING(h);
  if (r < 0 || r >= h->n) return fail(h, CSP_ERANGE, "realisation %d out of range", r);
  const HostReal& hr = h->real[r];
  if (boundary < 0 || boundary >= (int)hr.boundary_channel_base.size() || hr.boundary_channel_base[boundary] < 0)
    return fail(h, CSP_ERANGE, "boundary %d is not a discrete boundary", boundary);
  RealCtl c;
  int rc = read_ctl(h, r, c);
  if (rc) return rc;
  const int nchb = hr.boundary_nch[boundary];
  std::vector<unsigned char> tmp(nchb);
  for (int i = 0; i < nchb; i++) tmp[i] = (unsigned char)(states[i] ? 1 : 0);
  CUDA_TRY(h, cudaMemcpyAsync(h->d_states + (c.step & 1) * (size_t)std::max(h->nch, 1) + hr.boundary_channel_base[boundary],
                              tmp.data(), nchb, cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return CSP_OK;
}

// ---- linescan: convolution of one species with a 3-D Gaussian along one axis
// (Species_compute_convolution_with_gaussian_function_locally, species.c:1960-2037) ----
//
// The reference sums, for every position a of the scanned axis A,
//   u(x,y,z) * g(o_x - x h) * g(o_y - y h) * g(o_z - z h)   with o_A = a h
// over all species voxels (or over voxels whose domain id is below num_domains, the
// reference's domain test, species.c:2013-2024).  The weight factorises, so one pass
// over the field builds S[i] = sum over the other two axes of u * w_B * w_C for every
// index i of A (FP64 bins in shared memory, then one global add per bin and block), and
// the host finishes out[a] = sum_i S[i] g((a - i) h).
struct LinescanMap {
  const float* f;
  const unsigned char* dom;
  double base[ND];           // the species' field base per domain
  int fixq;                  // the species is stored in fixed point: value = base + q * qunit
  double qunit[ND];
  int nd[3];                 // device extents (n0, n1, n2)
  int P;
  int phys_of_dev[3];        // physical axis of each device axis
  int axis;                  // scanned physical axis
  int num_domains;           // > 0: only voxels with domain id < num_domains
  const double* w[3];        // per physical axis weights (the scanned axis: unused)
  int nbins;
};

__global__ void k_linescan_bins(LinescanMap m, double* __restrict__ bins) {
  extern __shared__ double sb[];
  for (int i = threadIdx.x; i < m.nbins; i += blockDim.x) sb[i] = 0.0;
  __syncthreads();
  const long long plane = (long long)m.nd[1] * m.nd[2];
  const long long total = (long long)m.nd[0] * plane;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < total;
       v += (long long)gridDim.x * blockDim.x) {
    const int c0 = (int)(v / plane);
    const long long rem = v - c0 * plane;
    const int c1 = (int)(rem / m.nd[2]), c2 = (int)(rem - (long long)c1 * m.nd[2]);
    const long long dv = (long long)c0 * m.P + rem;
    const int dom = m.dom[dv] & DOMAIN_BITS;
    if (m.num_domains > 0 && dom >= m.num_domains) continue;
    int pc[3];
    pc[m.phys_of_dev[0]] = c0; pc[m.phys_of_dev[1]] = c1; pc[m.phys_of_dev[2]] = c2;
    double w = (m.fixq ? (double)__float_as_int(m.f[dv]) * m.qunit[dom] : (double)m.f[dv]) + m.base[dom];
    for (int a = 0; a < 3; a++)
      if (a != m.axis) w *= m.w[a][pc[a]];
    atomicAdd(&sb[pc[m.axis]], w);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < m.nbins; i += blockDim.x)
    if (sb[i] != 0.0) atomicAdd(&bins[i], sb[i]);
}

static double gauss_weight(double x, double sigma) {   // utils.c:209-213
  return 1.0 / std::sqrt(2.0 * M_PI * sigma) * std::exp(-x * x / 2.0 / sigma);
}

extern "C" int csp_linescan(csp_handle* h, int32_t r, int32_t species, int32_t axis, const double* offsets_nm,
                            const double* conv, int32_t num_domains, double* out) {
  if (!h || !offsets_nm || !conv || !out) return fail(h, CSP_EINVAL, "NULL argument");
  CSP_NOT_PENDING(h);
  if (r < 0 || r >= h->n) return fail(h, CSP_ERANGE, "realisation %d out of range", r);
  const HostReal& hr = h->real[r];
  const RealDesc& D = hr.desc;
  if (species < 0 || species >= D.ns) return fail(h, CSP_ERANGE, "species %d out of range", species);
  if (axis < 0 || axis > 2) return fail(h, CSP_ERANGE, "axis %d out of range", axis);
  const int nA = hr.nphys[axis];
  if ((size_t)nA * sizeof(double) > 48 * 1024) return fail(h, CSP_ENOTSUP, "linescan axis of %d voxels", nA);
  RealCtl c;
  int rc = read_ctl(h, r, c);
  if (rc) return rc;
  const unsigned cur = c.cur_mask[c.step & 1];
  const double hs = hr.info.h;
  // weights of the two fixed axes, then one device buffer: [w0 | w1 | w2 | bins]
  std::vector<double> host;
  size_t woff[3];
  for (int a = 0; a < 3; a++) {
    woff[a] = host.size();
    for (int i = 0; i < hr.nphys[a]; i++)
      host.push_back(a == axis ? 0.0 : gauss_weight(offsets_nm[a] - i * hs, conv[a]));
  }
  const size_t boff = host.size();
  host.resize(boff + nA, 0.0);
  double* dbuf = nullptr;
  if (cudaMalloc(&dbuf, host.size() * sizeof(double)) != cudaSuccess)
    return fail(h, CSP_ENOMEM, "linescan buffer");
  LinescanMap m;
  m.f = D.u[(cur >> species) & 1u][species];
  m.dom = D.dom;
  for (int dd = 0; dd < ND; dd++) {
    m.base[dd] = D.base[dd][species];
    m.qunit[dd] = D.qunit[dd][species];
  }
  m.fixq = (D.fixq >> species) & 1u;
  m.nd[0] = D.nx; m.nd[1] = D.ny; m.nd[2] = D.nz;
  m.P = D.P;
  for (int i = 0; i < 3; i++) m.phys_of_dev[i] = hr.perm[i];
  m.axis = axis;
  m.num_domains = num_domains;
  for (int a = 0; a < 3; a++) m.w[a] = dbuf + woff[a];
  m.nbins = nA;
  cudaError_t e = cudaMemcpyAsync(dbuf, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    k_linescan_bins<<<592, 256, nA * sizeof(double), h->stream>>>(m, dbuf + boff);
    e = cudaGetLastError();
  }
  std::vector<double> bins(nA);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(bins.data(), dbuf + boff, nA * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(dbuf);
  if (e != cudaSuccess) return fail(h, CSP_ECUDA, "linescan: %s", cudaGetErrorString(e));
  for (int a = 0; a < nA; a++) {
    double acc = 0.0;
    for (int i = 0; i < nA; i++) acc += bins[i] * gauss_weight((a - i) * hs, conv[axis]);
    out[a] = acc;
  }
  return CSP_OK;
}

extern "C" int csp_reduce_outputs(csp_handle* h, int32_t r, double* min_values, double* max_values,
                                  double* total_values, int32_t* openness) {
  if (!h) return CSP_EINVAL;
  CSP_NOT_PENDING(h);
  if (r < 0 || r >= h->n) return fail(h, CSP_ERANGE, "realisation %d out of range", r);
  const HostReal& hr = h->real[r];
  const RealDesc& D = hr.desc;
  const int nblk = 296;
  double out[3 * ND];
  for (int s = 0; s < D.ns; s++) {
    k_reduce_partial<<<nblk, 256, 0, h->stream>>>(h->d_desc, h->d_ctl, r, s, h->d_red);
    k_reduce_final<<<1, 32, 0, h->stream>>>(h->d_red, nblk, hr.dV, h->d_red_out);
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaMemcpyAsync(out, h->d_red_out, sizeof out, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    for (int d = 0; d < hr.nd; d++) {
      if (min_values) min_values[d * D.ns + s] = out[0 * ND + d];
      if (max_values) max_values[d * D.ns + s] = out[1 * ND + d];
      if (total_values) total_values[d * D.ns + s] = out[2 * ND + d];
    }
  }
  if (openness) {
    int off = 0;
    for (size_t b = 0; b < hr.boundary_channel_base.size(); b++) {
      if (hr.boundary_channel_base[b] < 0) continue;
      int rc = csp_get_channel_states(h, r, (int)b, openness + off);
      if (rc) return rc;
      off += hr.boundary_nch[b];
    }
  }
  return CSP_OK;
}

extern "C" int csp_status(const csp_handle* h, char* msg, size_t n) {
  const char* m = h ? h->msg.c_str() : g_create_error;
  if (msg && n) snprintf(msg, n, "%s", m);
  return CSP_OK;
}

extern "C" int csp_get_stream(const csp_handle* h, void** stream) {
  if (!h || !stream) return CSP_EINVAL;
  *stream = (void*)h->stream;
  return CSP_OK;
}

extern "C" int csp_last_advance_ms(const csp_handle* h, float* ms) {
  if (!h || !ms) return CSP_EINVAL;
  *ms = h->last_ms;
  return CSP_OK;
}

extern "C" int csp_set_device(int32_t device) {
  const cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(nullptr, CSP_ECUDA, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
  return CSP_OK;
}

extern "C" int csp_set_phase_timing(csp_handle* h, int32_t on) {
  if (!h) return CSP_EINVAL;
  CSP_NOT_PENDING(h);
  if (on && !h->phase_ev[0])
    for (auto& e : h->phase_ev) CUDA_TRY(h, cudaEventCreate(&e));
  h->phase_timing = on ? 1 : 0;
  return CSP_OK;
}

extern "C" int csp_get_phase_times(const csp_handle* h, double* ms, int64_t* steps) {
  if (!h || !ms) return CSP_EINVAL;
  for (int p = 0; p < CSP_NUM_PHASES; p++) ms[p] = h->phase_ms[p];
  if (steps) *steps = h->phase_steps;
  return CSP_OK;
}

extern "C" int csp_test_wait_timeout(csp_handle* h, int32_t on) {
  if (!h) return CSP_EINVAL;
  if (on && (h->kernel != 0 || !h->plan.ok || !h->plan.launch_inject))
    return fail(h, CSP_EINVAL, "the staged voxel kernel with the test hook is not in use");
  // the hook's variant does not classify voxels for the surrogate
  if (on && h->surrogate) return fail(h, CSP_EINVAL, "the test hook does not run with the surrogate on");
  h->inject_wait = on ? 1 : 0;
  return CSP_OK;
}

extern "C" int csp_set_kernel(csp_handle* h, int32_t which) {
  if (!h || which < 0 || which > 1) return CSP_EINVAL;
  CSP_NOT_PENDING(h);
  if (which == 0 && !h->plan.ok) return fail(h, CSP_ENOTSUP, "staged kernel unavailable for this batch");
  h->kernel = which;
  return CSP_OK;
}

// ---- autotuner of the staged kernel's tile shape ----
// Candidates: threads per CTA (positions per chunk = 4 x threads) and x planes per work
// unit.  Each candidate's voxel kernel runs `repeats` times at the current step: the
// kernel reads the current buffers and writes the next ones, so repeating it is free of
// side effects (the real step writes the same values), and every tiling gives bitwise
// equal fields.  The fastest plan replaces the current one.
extern "C" int csp_autotune(csp_handle* h, int32_t repeats, csp_tune_report* rep) {
  if (!h) return CSP_EINVAL;
  CSP_NOT_PENDING(h);
  if (repeats < 1) repeats = 3;
  std::vector<RealDesc> descs(h->n);
  for (int r = 0; r < h->n; r++) descs[r] = h->real[r].desc;
  int cand[CSP_TUNE_MAX][2] = {{256, 0}, {256, 16}, {256, 32}, {256, 1 << 20}, {128, 0}, {128, 32}};
  int ncand = 6;
  // two more segment lengths for 256 threads from a cost model: rounds of work units over
  // the resident CTAs times the planes a unit stages (its segment and two halo planes)
  {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long ctas = 2ll * sms, L = 1024;
    double best[2] = {1e300, 1e300};
    int bseg[2] = {0, 0};
    for (int seg = 8; seg <= 64; seg++) {
      if (seg == 16 || seg == 32) continue;
      long long units = 0;
      for (const RealDesc& D : descs) units += (long long)((D.nx + seg - 1) / seg) * ((D.plane + L - 1) / L);
      const double cost = (double)((units + ctas - 1) / ctas) * (seg + 2);
      if (cost < best[0]) {
        best[1] = best[0]; bseg[1] = bseg[0];
        best[0] = cost; bseg[0] = seg;
      } else if (cost < best[1]) {
        best[1] = cost; bseg[1] = seg;
      }
    }
    for (int k = 0; k < 2 && ncand < CSP_TUNE_MAX; k++)
      if (bseg[k]) { cand[ncand][0] = 256; cand[ncand][1] = bseg[k]; ncand++; }
  }
  cudaEvent_t e0, e1;
  CUDA_TRY(h, cudaEventCreate(&e0));
  CUDA_TRY(h, cudaEventCreate(&e1));
  int best = -1;
  float best_ms = 0.f;
  StagedPlan best_plan;
  csp_tune_report local;
  memset(&local, 0, sizeof local);
  for (int i = 0; i < ncand && i < CSP_TUNE_MAX - 1; i++) {
    StagedPlan pl = staged_plan(descs, cand[i][0], cand[i][1]);
    local.threads[local.n] = cand[i][0];
    local.segment[local.n] = pl.g.seg;
    local.ms[local.n] = -1.f;
    if (staged_prepare(pl) != cudaSuccess) {
      staged_release(pl);
      local.n++;
      continue;
    }
    staged_launch(pl, h->d_desc, h->d_ctl, h->d_err, h->stream);      // warm-up
    cudaEventRecord(e0, h->stream);
    for (int k = 0; k < repeats; k++) staged_launch(pl, h->d_desc, h->d_ctl, h->d_err, h->stream);
    cudaEventRecord(e1, h->stream);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
      staged_release(pl);
      if (best >= 0) staged_release(best_plan);
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return fail(h, CSP_ECUDA, "autotune: %s", cudaGetErrorString(e));
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= repeats;
    local.ms[local.n] = ms;
    if (best < 0 || ms < best_ms) {
      if (best >= 0) staged_release(best_plan);
      best = local.n;
      best_ms = ms;
      best_plan = pl;
    } else {
      staged_release(pl);
    }
    local.n++;
  }
  // the direct kernel (recomputes the same step, like the staged candidates)
  bool direct = false;
  {
    const int i = local.n;
    local.threads[i] = 256;
    local.segment[i] = -1;
    dim3 grid((unsigned)((h->max_vox + 255) / 256), (unsigned)h->n);
    k_voxels_direct<<<grid, 256, 0, h->stream>>>(h->d_desc, h->d_ctl, h->d_err);
    cudaEventRecord(e0, h->stream);
    for (int k = 0; k < repeats; k++) k_voxels_direct<<<grid, 256, 0, h->stream>>>(h->d_desc, h->d_ctl, h->d_err);
    cudaEventRecord(e1, h->stream);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
      if (best >= 0) staged_release(best_plan);
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return fail(h, CSP_ECUDA, "autotune: %s", cudaGetErrorString(e));
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    local.ms[i] = ms / repeats;
    if (best < 0 || local.ms[i] < best_ms) direct = true;
    local.n++;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (best >= 0) {
    staged_release(h->plan);
    h->plan = best_plan;
  }
  h->plan_epoch++;
  h->kernel = direct ? 1 : 0;
  local.chosen = direct ? local.n - 1 : best;
  if (rep) *rep = local;
  return CSP_OK;
}

// ---- learned reaction surrogate (csp_mlp.cuh) ----

extern "C" void csp_mlp_init(uint64_t seed, float* params) {
  // He-uniform hidden layers, zero biases, zero output layer: an untrained network gives
  // the reference's single explicit reaction step.
  std::mt19937_64 g(seed);
  std::uniform_real_distribution<float> u(-1.f, 1.f);
  float* p = params;
  const float a1 = std::sqrt(6.f / MLP_IN), a2 = std::sqrt(6.f / MLP_H);
  for (int i = 0; i < MLP_IN * MLP_H; i++) *p++ = a1 * u(g);
  for (int i = 0; i < MLP_H; i++) *p++ = 0.f;
  for (int i = 0; i < MLP_H * MLP_H; i++) *p++ = a2 * u(g);
  for (int i = 0; i < MLP_H; i++) *p++ = 0.f;
  for (int i = 0; i < MLP_H * MLP_OUT + MLP_OUT; i++) *p++ = 0.f;
}

static int surrogate_supported(csp_handle* h) {
  for (int r = 0; r < h->n; r++) {
    const RealDesc& D = h->real[r].desc;
    if (D.nbuf == 0) continue;
    if (!D.react_fast) return fail(h, CSP_ENOTSUP, "realisation %d: the surrogate needs every buffer bound to species 0", r);
    int dca = -1;
    for (int i = 0; i < D.ndiff; i++)
      if (D.diff_species[i] == 0) dca = i;
    if (dca < 0 || D.reaction_substep % D.substeps[dca] != 0)
      return fail(h, CSP_ENOTSUP, "realisation %d: the surrogate needs species 0 to diffuse on every reaction step", r);
    for (int d = 0; d < D.nd; d++)
      for (int s = MLP_SLOTS + 1; s < NS; s++)
        if (D.rtab[d][s] >= 0) return fail(h, CSP_ENOTSUP, "realisation %d: buffer species %d beyond the 5 slots", r, s);
  }
  return CSP_OK;
}

extern "C" int csp_set_surrogate(csp_handle* h, const float* params, double tol) {
  if (!h) return CSP_EINVAL;
  CSP_NOT_PENDING(h);
  const int on = params != nullptr;
  if (on && h->inject_wait) return fail(h, CSP_EINVAL, "the surrogate does not run with the wait-timeout test hook on");
  if (on) {
    int rc = surrogate_supported(h);
    if (rc) return rc;
    if (!h->d_mlp) {
      const long long chunks = (h->max_field + MLP_DEPLOY_SPAN - 1) / MLP_DEPLOY_SPAN;
      if (cudaMalloc(&h->d_mlp, MLP_NPARAM * sizeof(float)) != cudaSuccess ||
          cudaMalloc(&h->d_mlp_cnt, 3 * sizeof(unsigned long long)) != cudaSuccess ||
          cudaMalloc(&h->d_sur_list, (size_t)chunks * h->n * MLP_DEPLOY_SPAN * sizeof(unsigned short)) != cudaSuccess ||
          cudaMalloc(&h->d_sur_counts, (size_t)chunks * h->n * 2 * sizeof(unsigned)) != cudaSuccess ||
          cudaMalloc(&h->d_sur_tiles, (size_t)chunks * h->n * (MLP_DEPLOY_SPAN / 32) * 2 * sizeof(unsigned)) != cudaSuccess ||
          cudaMalloc(&h->d_sur_queue, 4 * sizeof(unsigned)) != cudaSuccess)
        return fail(h, CSP_ENOMEM, "surrogate buffers");
      if ((unsigned long long)chunks * h->n >= (1ull << (32 - MLP_TILE_BITS)))
        return fail(h, CSP_ENOTSUP, "surrogate: more than 2^%d blocks of %lld voxels", 32 - MLP_TILE_BITS, MLP_DEPLOY_SPAN);
      CUDA_TRY(h, cudaMemsetAsync(h->d_mlp_cnt, 0, 3 * sizeof(unsigned long long), h->stream));
      CUDA_TRY(h, cudaMemsetAsync(h->d_sur_queue, 0, 4 * sizeof(unsigned), h->stream));
      h->sur_tile_cap = chunks * (long long)h->n * (MLP_DEPLOY_SPAN / 32);
      int dev = 0, sms = 0;
      CUDA_TRY(h, cudaGetDevice(&dev));
      CUDA_TRY(h, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      h->sur_network_ctas = 2 * std::max(sms, 1);
    }
    unsigned fq = 0;
    for (int r = 0; r < h->n; r++) fq |= h->real[r].desc.fixq & 0x3Eu;
    h->surrogate_fq = fq == 0u ? 0u : fq == 0x10u ? 0x10u : 0x3Eu;
    CUDA_TRY(h, cudaFuncSetAttribute(network_kernel(h->surrogate_fq), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)MLP_NETWORK_SMEM));
    {
      int dev = 0, sms = 0, per_sm = 0;
      CUDA_TRY(h, cudaGetDevice(&dev));
      CUDA_TRY(h, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      CUDA_TRY(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, plain_kernel(h->surrogate_fq), MLP_DEPLOY_T, 0));
      h->sur_plain_ctas = std::max(per_sm, 1) * std::max(sms, 1);
      CUDA_TRY(h, cudaFuncSetAttribute(network_kernel_umma(h->surrogate_fq), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       UM_NET_SMEM));
      CUDA_TRY(h, cudaFuncSetAttribute(network_kernel_umma(h->surrogate_fq),
                                       cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
      // resident CTAs per SM from the kernel's shared memory and registers (the occupancy
      // query reports one for this kernel, which holds nearly half of the SM's shared memory):
      // static + dynamic + the driver's reserve per CTA, and up to 1 KB of alignment
      cudaFuncAttributes fa;
      int smem_sm = 0, reserved = 0, regs_sm = 0;
      CUDA_TRY(h, cudaFuncGetAttributes(&fa, network_kernel_umma(h->surrogate_fq)));
      CUDA_TRY(h, cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
      CUDA_TRY(h, cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
      CUDA_TRY(h, cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev));
      const int per_block = (int)fa.sharedSizeBytes + UM_NET_SMEM + reserved + 1024;
      const int by_regs = regs_sm / std::max(1, fa.numRegs * UM_T * UM_NET_WGS);
      per_sm = std::max(1, std::min({smem_sm / per_block, by_regs, 512 / (UM_TMEM_COLS * UM_NET_WGS)}));
      h->sur_umma_ctas = per_sm * std::max(sms, 1);
    }
    CUDA_TRY(h, cudaMemcpyAsync(h->d_mlp, params, MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    h->surrogate_tol = (float)tol;
  }
  if (on && !h->d_rx_class) {
    size_t bytes = 0;
    for (int r = 0; r < h->n; r++) bytes += h->real[r].field_elems;
    if (cudaMalloc(&h->d_rx_class, bytes + 16) != cudaSuccess) return fail(h, CSP_ENOMEM, "surrogate class bytes");
    CUDA_TRY(h, cudaMemsetAsync(h->d_rx_class, 0, bytes + 16, h->stream));
  }
  h->surrogate = on;
  std::vector<RealDesc> descs(h->n);
  for (int r = 0; r < h->n; r++) {
    RealDesc& D = h->real[r].desc;
    D.sur = on;
    D.mlp_domains = mlp_eligible_domains(D);
    // the class bytes share the domain bytes' layout and offsets
    D.rx_class = on ? h->d_rx_class + (D.dom - h->d_dom) : nullptr;
    for (int d = 0; d < ND; d++) {
      bool any = false;
      for (int sp = 0; sp < NS; sp++) {
        D.sur_cs[d][sp] = 0.f;
        D.sur_thr2[d][sp] = 0.f;
        if (d >= D.nd || !(D.rmask[d] >> sp & 1u)) continue;
        const int t = D.rtab[d][sp] * D.nd + d;
        D.sur_cs[d][sp] = (float)((double)D.tot[t] - D.base[d][sp]);
        D.sur_thr2[d][sp] = (float)(2.0 * (double)MLP_SKIP * (double)D.tot[t]);
        any = true;
      }
      D.sur_kind[d] = (unsigned char)(!any ? RX_NONE : ((D.mlp_domains >> d) & 1u) ? RX_ELIGIBLE : RX_STIFF);
    }
    descs[r] = D;
  }
  CUDA_TRY(h, cudaMemcpyAsync(h->d_desc, descs.data(), h->n * sizeof(RealDesc), cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return CSP_OK;
}

extern "C" int csp_set_surrogate_tensor_cores(csp_handle* h, int32_t kind) {
  if (!h || (kind != 1 && kind != 2)) return CSP_EINVAL;
  CSP_NOT_PENDING(h);
  h->sur_tc = kind;
  return CSP_OK;
}

extern "C" int csp_surrogate_counts(const csp_handle* hc, int64_t* voxels, int64_t* network, int64_t* fallbacks) {
  csp_handle* h = const_cast<csp_handle*>(hc);
  if (!h || !voxels || !network || !fallbacks) return CSP_EINVAL;
  CSP_NOT_PENDING(h);
  unsigned long long c[3] = {0, 0, 0};
  if (h->d_mlp_cnt) {
    CUDA_TRY(h, cudaMemcpyAsync(c, h->d_mlp_cnt, sizeof c, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  }
  *voxels = (int64_t)c[0];
  *network = (int64_t)c[1];
  *fallbacks = (int64_t)c[2];
  return CSP_OK;
}

static cudaError_t mlp_grad_launch(const float* dp, const float* dx, const float* dt, long long n, float* dg,
                                   float* dl, cudaStream_t st) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MLP_GRAD_SMEM);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  const unsigned blocks = (unsigned)((n + MLP_TB - 1) / MLP_TB);
  k_mlp_grad<<<blocks, MLP_TB, MLP_GRAD_SMEM, st>>>(dp, dx, dt, n, 1.f / (float)(n * MLP_OUT), dg, dl);
  return cudaGetLastError();
}

extern "C" int csp_mlp_gradient(const float* params, const float* x, const float* t, int64_t n, float* grad,
                                float* loss) {
  if (!params || !x || !t || !grad || !loss || n <= 0) return fail(nullptr, CSP_EINVAL, "bad argument");
  float *dp = nullptr, *dx = nullptr, *dt = nullptr, *dg = nullptr;
  const size_t nb = (MLP_NPARAM + 1) * sizeof(float);
  cudaError_t e = cudaMalloc(&dp, nb);
  if (e == cudaSuccess) e = cudaMalloc(&dx, n * MLP_IN * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dt, n * MLP_OUT * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dg, nb);
  if (e == cudaSuccess) e = cudaMemcpy(dp, params, MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dx, x, n * MLP_IN * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dt, t, n * MLP_OUT * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(dg, 0, nb);
  if (e == cudaSuccess) e = mlp_grad_launch(dp, dx, dt, n, dg, dg + MLP_NPARAM, 0);
  if (e == cudaSuccess) e = cudaMemcpy(grad, dg, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(loss, dg + MLP_NPARAM, sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(dp); cudaFree(dx); cudaFree(dt); cudaFree(dg);
  if (e != cudaSuccess) return fail(nullptr, CSP_ECUDA, "mlp gradient: %s", cudaGetErrorString(e));
  return CSP_OK;
}

extern "C" int csp_mlp_forward(const float* params, const float* x, int64_t n, int32_t tensor_cores, float* y) {
  if (!params || !x || !y || n <= 0 || tensor_cores < 0 || tensor_cores > 2) return fail(nullptr, CSP_EINVAL, "bad argument");
  float *dp = nullptr, *dx = nullptr, *dy = nullptr;
  int* derr = nullptr;
  cudaError_t e = tensor_cores == 2
                      ? cudaFuncSetAttribute(k_mlp_forward_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, UM_SMEM)
                      : cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)MLP_FORWARD_SMEM);
  if (e == cudaSuccess) e = cudaMalloc(&dp, MLP_NPARAM * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dx, n * MLP_IN * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dy, n * MLP_OUT * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&derr, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(derr, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpy(dp, params, MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dx, x, n * MLP_IN * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    if (tensor_cores == 2) {
      const long long tiles = (n + UM_T - 1) / UM_T;
      k_mlp_forward_umma<<<(unsigned)std::min<long long>(tiles, 592), UM_T, UM_SMEM>>>(dp, dx, n, dy, derr);
    } else {
      k_mlp_forward<<<(unsigned)((n + MLP_DEPLOY_T - 1) / MLP_DEPLOY_T), MLP_DEPLOY_T, MLP_FORWARD_SMEM>>>(
          dp, dx, n, tensor_cores, dy);
    }
    e = cudaGetLastError();
  }
  int herr = 0;
  if (e == cudaSuccess) e = cudaMemcpy(y, dy, n * MLP_OUT * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(dp); cudaFree(dx); cudaFree(dy); cudaFree(derr);
  if (e != cudaSuccess) return fail(nullptr, CSP_ECUDA, "mlp forward: %s", cudaGetErrorString(e));
  if (herr) return fail(nullptr, CSP_EDEVICE, "mlp forward: bounded wait timed out");
  return CSP_OK;
}

extern "C" int csp_mlp_harvest(csp_handle* h, int64_t n, uint64_t seed, int64_t capacity, int64_t* taken,
                               int64_t* held) {
  if (!h || n < 0 || capacity < 1) return fail(h, CSP_EINVAL, "bad argument");
  CSP_NOT_PENDING(h);
  int rc = surrogate_supported(h);
  if (rc) return rc;
  if (!h->d_hx) {
    if (cudaMalloc(&h->d_hx, (size_t)capacity * MLP_IN * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&h->d_ht, (size_t)capacity * MLP_OUT * sizeof(float)) != cudaSuccess) {
      cudaFree(h->d_hx); cudaFree(h->d_ht);
      h->d_hx = h->d_ht = nullptr;
      return fail(h, CSP_ENOMEM, "harvest buffer of %lld pairs", (long long)capacity);
    }
    h->harvest_cap = capacity;
    h->harvest_n = 0;
  } else if (capacity > h->harvest_cap) {
    return fail(h, CSP_EINVAL, "capacity %lld above the first call's %lld", (long long)capacity, h->harvest_cap);
  }
  unsigned long long* dcnt = nullptr;      // [BINS] histogram, then the cursor
  float* dprob = nullptr;
  unsigned* delig = nullptr;               // per realisation: the domains the surrogate serves
  std::vector<unsigned> elig(h->n);
  for (int r = 0; r < h->n; r++) elig[r] = mlp_eligible_domains(h->real[r].desc);
  cudaError_t e = cudaMalloc(&dcnt, (MLP_HARVEST_BINS + 1) * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&dprob, MLP_HARVEST_BINS * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&delig, h->n * sizeof(unsigned));
  cudaStream_t st = h->stream;
  if (e == cudaSuccess) e = cudaMemcpyAsync(delig, elig.data(), h->n * sizeof(unsigned), cudaMemcpyHostToDevice, st);
  unsigned long long hist[MLP_HARVEST_BINS + 1] = {};
  dim3 grid((unsigned)std::min<long long>(1184, (h->max_vox + 255) / 256), (unsigned)h->n);
  if (e == cudaSuccess) e = cudaMemsetAsync(dcnt, 0, (MLP_HARVEST_BINS + 1) * sizeof(unsigned long long), st);
  if (e == cudaSuccess) {
    k_mlp_harvest<<<grid, 256, 0, st>>>(h->d_desc, h->d_ctl, delig, 0, dprob, seed, dcnt, nullptr, 0, nullptr, nullptr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(hist, dcnt, MLP_HARVEST_BINS * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  // water filling: every bin gives min(count, level) pairs, the level set so the bins give n
  const long long want = std::min<long long>(n, h->harvest_cap - h->harvest_n);
  double total = 0.0;
  for (int b = 0; b < MLP_HARVEST_BINS; b++) total += (double)hist[b];
  double lo = 0.0, hi = 0.0;
  for (int b = 0; b < MLP_HARVEST_BINS; b++) hi = std::max(hi, (double)hist[b]);
  for (int it = 0; it < 100 && total > want; it++) {
    const double mid = 0.5 * (lo + hi);
    double s = 0.0;
    for (int b = 0; b < MLP_HARVEST_BINS; b++) s += std::min((double)hist[b], mid);
    (s > want ? hi : lo) = mid;
  }
  float prob[MLP_HARVEST_BINS];
  for (int b = 0; b < MLP_HARVEST_BINS; b++)
    prob[b] = hist[b] == 0 ? 0.f : (total <= want ? 1.f : (float)(std::min((double)hist[b], lo) / (double)hist[b]));
  const unsigned long long start = (unsigned long long)h->harvest_n;
  if (e == cudaSuccess) e = cudaMemcpyAsync(dprob, prob, sizeof prob, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dcnt + MLP_HARVEST_BINS, &start, sizeof start, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && want > 0) {
    k_mlp_harvest<<<grid, 256, 0, st>>>(h->d_desc, h->d_ctl, delig, 1, dprob, seed, nullptr, dcnt + MLP_HARVEST_BINS,
                                        h->harvest_cap, h->d_hx, h->d_ht);
    e = cudaGetLastError();
  }
  unsigned long long end = start;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&end, dcnt + MLP_HARVEST_BINS, sizeof end, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(dcnt);
  cudaFree(dprob);
  cudaFree(delig);
  if (e != cudaSuccess) return fail(h, CSP_ECUDA, "harvest: %s", cudaGetErrorString(e));
  const long long now = std::min<long long>((long long)end, h->harvest_cap);
  if (taken) *taken = now - h->harvest_n;
  h->harvest_n = now;
  if (held) *held = now;
  return CSP_OK;
}

extern "C" int csp_mlp_harvested(const csp_handle* hc, int64_t first, int64_t n, float* x, float* t) {
  csp_handle* h = const_cast<csp_handle*>(hc);
  if (!h || !x || !t || first < 0 || n < 0) return CSP_EINVAL;
  if (first + n > h->harvest_n) return fail(h, CSP_ERANGE, "pairs [%lld, %lld) beyond the %lld held", (long long)first,
                                            (long long)(first + n), h->harvest_n);
  CUDA_TRY(h, cudaMemcpy(x, h->d_hx + first * MLP_IN, (size_t)n * MLP_IN * sizeof(float), cudaMemcpyDeviceToHost));
  CUDA_TRY(h, cudaMemcpy(t, h->d_ht + first * MLP_OUT, (size_t)n * MLP_OUT * sizeof(float), cudaMemcpyDeviceToHost));
  return CSP_OK;
}

extern "C" int csp_mlp_train(csp_handle* h, int32_t r, const csp_mlp_config* cfg, float* params,
                             csp_mlp_report* rep) {
  if (!h || !cfg || !params) return CSP_EINVAL;
  if (r < 0 || r >= h->n) return fail(h, CSP_ERANGE, "realisation %d out of range", r);
  int rc = surrogate_supported(h);
  if (rc) return rc;
  const RealDesc& D = h->real[r].desc;
  std::vector<int> doms;
  const unsigned elig = mlp_eligible_domains(D);
  for (int d = 0; d < D.nd; d++)
    if ((elig >> d) & 1u) doms.push_back(d);
  if (doms.empty()) return fail(h, CSP_EINVAL, "realisation %d has no domain the surrogate can serve", r);
  const bool harvested = cfg->source == CSP_MLP_SOURCE_HARVEST;
  if (harvested && h->harvest_n < 2) return fail(h, CSP_EINVAL, "no harvested pairs (csp_mlp_harvest)");
  long long nt = cfg->samples > 0 ? cfg->samples : 1000000, nv = cfg->val_samples > 0 ? cfg->val_samples : 65536;
  if (harvested) {   // every harvested pair; the held-out share at most a tenth
    nv = std::max<long long>(1, std::min<long long>(nv, h->harvest_n / 10));
    nt = h->harvest_n - nv;
  }
  const int batch = cfg->batch > 0 ? cfg->batch : 16384, epochs = cfg->epochs > 0 ? cfg->epochs : 10;
  const long long ntot = nt + nv;
  float *dx = nullptr, *dtg = nullptr, *dp = nullptr, *dg = nullptr, *dm = nullptr, *dv = nullptr;
  int* dd = nullptr;
  unsigned long long* dcnt = nullptr;
  RealDesc* ddesc = nullptr;
  const size_t pb = (MLP_NPARAM + 1) * sizeof(float);
  cudaError_t e = cudaMalloc(&dx, ntot * MLP_IN * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dtg, ntot * MLP_OUT * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&dp, pb);
  if (e == cudaSuccess) e = cudaMalloc(&dg, pb);
  if (e == cudaSuccess) e = cudaMalloc(&dm, pb);
  if (e == cudaSuccess) e = cudaMalloc(&dv, pb);
  if (e == cudaSuccess) e = cudaMalloc(&dd, doms.size() * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&dcnt, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&ddesc, sizeof(RealDesc));
  cudaStream_t st = h->stream;
  if (e == cudaSuccess) e = cudaMemcpyAsync(ddesc, &D, sizeof(RealDesc), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dd, doms.data(), doms.size() * sizeof(int), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dp, params, MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(dg, 0, pb, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(dm, 0, pb, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(dv, 0, pb, st);
  if (e == cudaSuccess && !harvested) {
    k_mlp_pairs<<<(unsigned)((ntot + 255) / 256), 256, 0, st>>>(ddesc, cfg->seed, ntot, dd, (int)doms.size(), dx, dtg);
    e = cudaGetLastError();
  } else if (e == cudaSuccess) {
    // harvested pairs, shuffled by an affine bijection (a coprime with ntot)
    auto gcd = [](unsigned long long p, unsigned long long q) {
      while (q) { const unsigned long long t = p % q; p = q; q = t; }
      return p;
    };
    const unsigned long long nn = (unsigned long long)ntot;
    unsigned long long a = 1;
    if (nn > 2) {
      a = 2654435761ull % nn;
      while (a < 2 || gcd(a, nn) != 1) a = a + 1 < nn ? a + 1 : 2;
    }
    k_mlp_permute<<<(unsigned)((ntot + 255) / 256), 256, 0, st>>>(h->d_hx, h->d_ht, ntot, a, cfg->seed % ntot, dx, dtg);
    e = cudaGetLastError();
  }
  float val_first = 0.f, val_last = 0.f;
  auto val_loss = [&](float& out) -> cudaError_t {
    cudaError_t ee = cudaMemsetAsync(dg, 0, pb, st);
    if (ee == cudaSuccess) ee = mlp_grad_launch(dp, dx + nt * MLP_IN, dtg + nt * MLP_OUT, nv, dg, dg + MLP_NPARAM, st);
    if (ee == cudaSuccess) ee = cudaMemcpyAsync(&out, dg + MLP_NPARAM, sizeof(float), cudaMemcpyDeviceToHost, st);
    if (ee == cudaSuccess) ee = cudaStreamSynchronize(st);
    if (ee == cudaSuccess) ee = cudaMemsetAsync(dg, 0, pb, st);
    return ee;
  };
  if (e == cudaSuccess) e = val_loss(val_first);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  int step = 0;
  const float lr0 = cfg->lr > 0 ? cfg->lr : 1e-3f;
  const long long nbatches = (nt + batch - 1) / batch;
  for (int ep = 0; ep < epochs && e == cudaSuccess; ep++) {
    // cosine learning-rate decay over the run
    for (long long bi = 0; bi < nbatches && e == cudaSuccess; bi++) {
      const long long s0 = bi * batch, nb = std::min<long long>(batch, nt - s0);
      const double prog = (double)step / (double)(epochs * nbatches);
      const float lr = (float)(lr0 * 0.5 * (1.0 + std::cos(M_PI * prog)));
      e = mlp_grad_launch(dp, dx + s0 * MLP_IN, dtg + s0 * MLP_OUT, nb, dg, dg + MLP_NPARAM, st);
      step++;
      if (e == cudaSuccess) {
        k_mlp_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, st>>>(dp, dg, dm, dv, MLP_NPARAM, lr, 0.9f, 0.999f, 1e-8f, step);
        e = cudaGetLastError();
      }
    }
  }
  cudaEventRecord(e1, st);
  if (e == cudaSuccess) e = val_loss(val_last);
  unsigned long long acc = 0;
  if (e == cudaSuccess) e = cudaMemsetAsync(dcnt, 0, sizeof acc, st);
  if (e == cudaSuccess) {
    k_mlp_accept<<<(unsigned)((nv + 255) / 256), 256, 0, st>>>(ddesc, dp, dx + nt * MLP_IN, nv,
                                                               cfg->tol > 0 ? (float)cfg->tol : 1e-4f, dcnt);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&acc, dcnt, sizeof acc, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(params, dp, MLP_NPARAM * sizeof(float), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(dx); cudaFree(dtg); cudaFree(dp); cudaFree(dg); cudaFree(dm); cudaFree(dv); cudaFree(dd);
  cudaFree(dcnt); cudaFree(ddesc);
  if (e != cudaSuccess) return fail(h, CSP_ECUDA, "mlp training: %s", cudaGetErrorString(e));
  if (rep) {
    rep->val_loss_first = val_first;
    rep->val_loss_last = val_last;
    rep->val_accept_rate = (double)acc / (double)nv;
    rep->train_ms = ms;
    rep->steps = step;
    rep->samples = nt;
  }
  return CSP_OK;
}

extern "C" void csp_destroy(csp_handle* h) {
  if (!h) return;
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->graph) cudaGraphExecDestroy(h->graph);
  staged_release(h->plan);
  cudaFree(h->d_fields); cudaFree(h->d_dom); cudaFree(h->d_cls); cudaFree(h->d_desc); cudaFree(h->d_ctl);
  cudaFree(h->d_rec); cudaFree(h->d_drows);
  cudaFree(h->d_rows); cudaFree(h->d_entries); cudaFree(h->d_pairs); cudaFree(h->d_params);
  cudaFree(h->d_states); cudaFree(h->d_err); cudaFree(h->d_red); cudaFree(h->d_red_out);
  cudaFree(h->d_stage);
  if (h->in_stream) { cudaStreamSynchronize(h->in_stream); cudaStreamDestroy(h->in_stream); }
  cudaFree(h->d_pipe); cudaFree(h->d_stepflags);
  if (h->snap_stream) cudaStreamSynchronize(h->snap_stream);
  cudaFree(h->d_snap);
  cudaFreeHost(h->h_snap);
  if (h->ev_snap) cudaEventDestroy(h->ev_snap);
  if (h->ev_copy) cudaEventDestroy(h->ev_copy);
  if (h->snap_stream) cudaStreamDestroy(h->snap_stream);
  cudaFree(h->d_mlp); cudaFree(h->d_mlp_cnt); cudaFree(h->d_sur_list); cudaFree(h->d_sur_counts);
  cudaFree(h->d_sur_tiles); cudaFree(h->d_sur_queue); cudaFree(h->d_rx_class);
  cudaFree(h->d_hx); cudaFree(h->d_ht);
  for (auto& e : h->phase_ev)
    if (e) cudaEventDestroy(e);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}
