// csp_device.cuh -- device-side data layout and per-voxel arithmetic shared by the
// voxel kernels (direct and TMA-staged) and the boundary kernel.
//
// HBM layout of one realisation: for every species two FP32 buffers (the reference's
// u1 / du pair, species.h:52-53, become a double buffer: a step reads the current
// buffer and writes the other one) and one uint8 domain-id field.  Every field is
// [nx][P] with P = ny*nz rounded up to a multiple of 128 elements, so each x-plane
// starts on a 512-byte boundary (float) / 128-byte boundary (uint8) and can be moved by
// 16-byte aligned bulk copies.  Within a plane the index is p = y*nz + z (z fastest,
// species.c:1513).
#pragma once
#include <cstdint>
#include <cstring>

#include "../../include/csparks.h"

namespace csp {

constexpr int ND = CSP_MAX_DOMAINS;
constexpr int NS = CSP_MAX_SPECIES;
constexpr int NB = CSP_MAX_BUFFERS;
constexpr int PLANE_ALIGN = 128;
constexpr int DOMAIN_BITS = 7;      // domain id = domain byte & DOMAIN_BITS
constexpr int CLASS_L = 1024;       // plane positions per chunk of the chunk class table
constexpr unsigned char CLASS_MIXED = 0xff;
// Surrogate domain kinds (RealDesc::sur_kind) and voxel classes (RealDesc::rx_class).
enum : unsigned { RX_NONE = 0, RX_ELIGIBLE = 1, RX_STIFF = 2 };
enum : unsigned { RX_CLASS_NONE = 0, RX_CLASS_EXPLICIT = 1, RX_CLASS_NETWORK = 2, RX_CLASS_PLAIN = 3 };

enum FluxKind : int { FLUX_NONE = 0, FLUX_RYR = 1, FLUX_P_RYR = 2, FLUX_SERCA = 3 };

// Constant description of one realisation (device resident, read-only in kernels).
struct RealDesc {
  int nx, ny, nz, P, plane;          // plane = ny*nz
  int ns, nd, ndiff, nbuf;
  int reaction_substep, stochastic_substep;
  int dirichlet;
  int substeps[NS];                  // per diffusive index
  int diff_species[NS];
  unsigned reaction_flag_mask;       // species flagged after a reaction step (species.c:1695-1699)
  float dt_r;                        // dt * reaction_substep (species.c:1666)
  float coef[NS][ND * ND];           // dt*substeps*sigma/h^2 tables (species.c:1545-1560)
  // buffer constants [bi*nd + di] (species.c:249-253); the rates are stored multiplied by
  // the reaction time step dt_r
  float kon_dt[NB * ND], koff_dt[NB * ND], tot[NB * ND];
  float cdiag[ND][NS];               // coef of species s between two voxels of domain d (0: not diffusive)
  // fast reactions: {-kon_dt, -koff_dt, a_dt, j0_dt} of the buffer bound to s in d (see
  // buffer_dj), present where rmask[d] has bit s
  float4 rk[ND][NS];
  unsigned char bsp0[NB * ND], bsp1[NB * ND];
  unsigned char fixed_mask[ND];      // bit s: species s is fixed in domain d
  signed char dsi_of[NS];            // diffusive index of species s, or -1
  signed char rtab[ND][NS];          // fast reaction table: buffer index bi with bsp0 = s in domain d, or -1
  int react_fast;                    // every buffer binds species 0 and bound species are distinct per domain
  unsigned mlp_domains;              // bit d: domain d's reactions are mild enough for the surrogate
  // Reaction surrogate (csp_mlp.cuh).  With sur set, the voxel kernels also classify every
  // voxel on a reaction step into rx_class (RX_CLASS_*) from the increments they apply:
  // near equilibrium (the explicit increment stands), network, or plain integrator; the
  // class scan then corrects the voxels of the last two classes.  For the buffer bound to
  // s in d: sur_cs = tot - base_s, sur_thr2 = 2 MLP_SKIP tot (the near-equilibrium bound
  // times dt_r^2); sur_kind[d] = RX_NONE / RX_ELIGIBLE / RX_STIFF.
  int sur;
  unsigned char* rx_class;           // [nx][P]; positions >= plane stay 0
  float sur_cs[ND][NS], sur_thr2[ND][NS];
  unsigned char sur_kind[ND];
  // Density-boundary fluxes evaluated inside the voxel kernels.  A voxel's domain byte
  // holds the domain id in bits 0-2 and a flux pattern index in bits 3-7 (0 = none).
  // fpat[pattern][k] for neighbour direction k: 0 = no flux, else (slot + 1), with bit 7
  // set when this voxel is the receiving ("to") side of the pair.
  unsigned char fpat[32][6];
  int fslot_species[4];
  int fslot_kind[4];
  double fslot_p[4][10];
  float init[ND][NS];                // initial values (Species_init_values, species.c:887-935)
  // Every field holds a value as its deviation from a base: u = base[d][s] + field, with d
  // the voxel's domain.  The base of a species that diffuses is one value for each set of
  // domains that species diffuses between (the initial value of the set's first domain),
  // so neighbouring deviations differ exactly as the values do and the stencil is the
  // same on both; other species take their domain's initial value.  In FP32 a value near
  // 1300 uM (SR Ca) or 20 mM (bound CSQN) keeps increments down to 1e-4 uM only when
  // stored as a deviation: the per-step SERCA uptake and buffer binding would otherwise
  // round away.  dinit = init - base (what fixed and Dirichlet values write).
  double base[ND][NS];
  float fbase[ND][NS];
  float dinit[ND][NS];
  // buffer reactions about the base: for buffer t = bi*nd + d with bound species s0 and
  // ligand s1, a_dt = dt_r k_on (tot - base_s0), j0_dt = dt_r J(base_s0, base_s1)
  float a_dt[NB * ND], j0_dt[NB * ND];
  unsigned char rmask[ND];           // bit s: a buffer binds species s in domain d (fast reactions)
  // Species that diffuse in no domain and only ever are the bound form of a buffer (TRPN
  // in the reference model) hold a 32-bit integer q instead: value = base + q qunit[d][s],
  // qunit a power of two with |q| < 2^30 over [0, 2 tot].  Such a buffer relaxes slowly;
  // in FP32 its per-step increments would round away once below half an ulp of the
  // deviation, stalling it short of equilibrium by about ulp / (2 rate dt) (0.02 uM for
  // TRPN at the channel mouth); the integer adds every increment at 2^-30 of the total.
  unsigned fixq;                     // bit s: species s is stored as q
  float qunit[ND][NS], qinv[ND][NS];
  float* u[2][NS];                   // the two buffers of every species
  const unsigned char* dom;          // [nx][P]
  // Chunk class table [nx][ncls]: for plane x and chunk c (positions c*CLASS_L ...
  // c*CLASS_L + CLASS_L - 1), the domain id when every voxel of planes x-1..x+1 within
  // nz positions of the chunk lies in that domain with no flux pattern, else CLASS_MIXED.
  const unsigned char* cls;
  int ncls;
  long long total_steps;
  double dt, h, tabort;
  unsigned long long seed;           // Philox key of the realisation's channel draws
  unsigned stream;                   // Philox stream: batch index + csp_options.stream_offset
  int has_channels;
};

// Mutable per-realisation progress (device).
struct RealCtl {
  long long step;                    // steps taken; the running step has time_ind = step+1
  unsigned cur_mask[2];              // [step&1]: bit s = index of the current buffer of species s
  int stopped;
  int open_count[2];                 // open channels after the step, by (step+1)&1
  double last_closed;                // abort rule bookkeeping
};

// What a realisation's running step does, for the density-row kernel: written at creation
// and by the step epilogue for the next step (one 16-byte load per row).
struct alignas(16) StepRec {
  unsigned active;                   // not stopped
  unsigned cur;                      // bit s: index of the current buffer of species s
  unsigned updated;                  // species written by the step
  unsigned sub;                      // bit dsi: diffusive index dsi takes its substep (and its fluxes)
};

// A density-boundary row in 32 bytes (two 16-byte loads): the receiving voxel, the other
// voxel of its first pair, the first pair's law with the SERCA scale inline, and the
// entries of any further pairs.  A pair row (DROW_PAIR) stands for the two rows of a pair
// whose voxels touch no other pair: v is the "to" voxel, vo the "from" voxel, and the one
// flux goes to both (DROW_APPLY: to v, DROW_APPLY_FROM: to vo).
enum : unsigned { DROW_APPLY = 1u, DROW_TO = 2u, DROW_SERCA = 4u, DROW_PAIR = 8u, DROW_APPLY_FROM = 16u };
struct alignas(16) DensityRow {
  int v, vo;                         // receiving voxel, other voxel of the first pair (field indices)
  int r;                             // realisation
  int more_begin;                    // further pairs: entries[more_begin .. more_begin + nmore)
  double scale;                      // first pair, kind SERCA: the flux scale (FluxParams::p[9])
  unsigned meta0;                    // first pair's parameter block (bits 0-15), species (16-23), dsi (24-31)
  unsigned meta1;                    // DROW_* flags (bits 0-7), nmore (8-15), domain ids of v (16-18), vo (19-21)
};
static_assert(sizeof(DensityRow) == 32, "density row");

// One boundary pair (species voxels), with the law applied across it.
struct FluxPair {
  int r;                  // realisation
  int species;            // flux species (species index)
  int dsi;                // diffusive index of the flux species
  int kind;               // FluxKind
  int channel;            // global channel index (discrete boundaries) or -1
  int boundary;           // boundary index within the realisation
  int inner;              // inner boundary: the "from" voxel loses J
  int param;              // index into the parameter blocks
  long long v0, v1;       // padded linear indices x*P + p of from / to voxels
  int local_channel;      // channel index within its boundary (RNG counter)
  int doms;               // domain ids of v0 (bits 0-2) and v1 (bits 3-5): the fields' bases
};

// One voxel receiving flux.  Its first pair is stored inline (most voxels touch one
// pair); further pairs are entries [more_begin, more_end) of the entry list, in pair order.
struct FluxRow {
  long long v;            // receiving voxel
  long long v0, v1;       // first pair: from / to voxel
  int r;                  // realisation
  int param;              // first pair: parameter block
  int channel;            // first pair: global channel index, -1 for density boundaries
  int local_channel;      // first pair: channel index within its boundary (RNG counter)
  float sign;             // first pair: +1 receiving side, -1 giving side
  int more_begin, more_end;
  unsigned char species, dsi, kind, owner, boundary, apply;
  unsigned char doms;     // first pair: domain ids of v0 (bits 0-2) and v1 (bits 3-5)
  unsigned char pad1;
};
static_assert(sizeof(FluxRow) == 64, "a flux row is one 64-byte line");

struct FluxEntry {
  int pair;
  float sign;             // +1 "to" side, -1 "from" side (inner boundaries)
  int owner;              // this entry writes the channel's new state
  int pad;
};

struct FluxParams {
  double p[10];           // RyR_model::params layout (boundaryfluxes.h:54) / SERCA params
  double t_close;
};

// Species updated at step time_ind, and the subset flagged before the reaction runs
// (diffusion and boundary fluxes flag their species, species.c:1542, 1746).
__host__ __device__ inline void step_masks(const RealDesc& D, long long time_ind, unsigned& pre,
                                           unsigned& updated, unsigned& diffusing_dsi) {
  pre = 0;
  diffusing_dsi = 0;
  for (int d = 0; d < NS; d++) {
    if (d >= D.ndiff) break;
    if (time_ind % D.substeps[d] == 0) {
      pre |= 1u << D.diff_species[d];
      diffusing_dsi |= 1u << d;
    }
  }
  updated = pre;
  if (D.nbuf > 0 && time_ind % D.reaction_substep == 0) updated |= D.reaction_flag_mask;
}

// Fixed-point fields (RealDesc::fixq): the stored bits are the integer q.
__host__ __device__ inline int q_bits(float stored) {
#ifdef __CUDA_ARCH__
  return __float_as_int(stored);
#else
  int q;
  memcpy(&q, &stored, sizeof q);
  return q;
#endif
}
__device__ __forceinline__ float q_value(float stored, float unit) {       // deviation q * unit
  return __fmul_rn(__int2float_rn(__float_as_int(stored)), unit);
}
__device__ __forceinline__ float q_add(float stored, float inc, float inv) {   // q + round(inc / unit)
  return __int_as_float(__float_as_int(stored) + __float2int_rn(__fmul_rn(inc, inv)));
}
__device__ __forceinline__ float q_set(float dev, float inv) {             // round(dev / unit)
  return __int_as_float(__float2int_rn(__fmul_rn(dev, inv)));
}

// Register-array access with a run-time index, as a chain of selects (no local memory).
template <int N>
__device__ __forceinline__ float sel(const float (&a)[N], int i) {
  float r = a[0];
#pragma unroll
  for (int s = 1; s < N; s++)
    if (i == s) r = a[s];
  return r;
}

template <int N>
__device__ __forceinline__ void put(float (&a)[N], int i, float v) {
#pragma unroll
  for (int s = 0; s < N; s++)
    if (i == s) a[s] = v;
}

template <int N>
__device__ __forceinline__ void addto(float (&a)[N], int i, float v) {
#pragma unroll
  for (int s = 0; s < N; s++)
    if (i == s) a[s] += v;
}

// ---------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) for the channel draws.
__host__ __device__ inline void philox4x32(const unsigned (&ctr)[4], unsigned k0, unsigned k1, unsigned (&out)[4]) {
  unsigned c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  for (int i = 0; i < 10; i++) {
    unsigned long long p0 = 0xD2511F53ull * c0;
    unsigned long long p1 = 0xCD9E8D57ull * c2;
    unsigned hi0 = (unsigned)(p0 >> 32), lo0 = (unsigned)p0;
    unsigned hi1 = (unsigned)(p1 >> 32), lo1 = (unsigned)p1;
    c0 = hi1 ^ c1 ^ k0; c1 = lo1; c2 = hi0 ^ c3 ^ k1; c3 = lo0;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Uniform in [0,1) with 53 bits for (seed, realisation; channel, boundary, step).
__host__ __device__ inline double channel_uniform(unsigned long long seed, unsigned realisation, unsigned channel,
                                                  unsigned boundary, long long step) {
  const unsigned ctr[4] = {channel, boundary, (unsigned)step, (unsigned)((unsigned long long)step >> 32)};
  unsigned r[4];
  philox4x32(ctr, (unsigned)seed, realisation ^ (unsigned)(seed >> 32), r);
  return ((double)(r[0] >> 5) * 67108864.0 + (double)(r[1] >> 6)) * (1.0 / 9007199254740992.0);
}

// Flux laws in FP64 (boundaryfluxes.c:12-141).
__host__ __device__ inline double serca_flux(double dt, double h, double u0, double u1, const double* params) {
  const double Ca_sr = u1 / 1000, Ca_i = u0 / 1000;
  const double k_p1 = 25900, k_p2 = 2540, k_p3 = 20.5, k_m1 = 16, k_m2 = 67200, k_m3 = 149;
  const double kdcai = 0.9, kdcasr = 2.24, kdh1 = 1.09e-5, kdhi = 3.54e-3, kdhsr = 1.05e-8, kdh = 7.24e-5,
               H_i = 1e-4, ATP = 5, ADP = 36.3e-3, P_i = 1;
  const double T_Cai = Ca_i / kdcai, T_Casr = Ca_sr / kdcasr;
  const double T_Cai2 = T_Cai * T_Cai, T_Casr2 = T_Casr * T_Casr;
  const double T_H1 = H_i / kdh1, T_Hi = (H_i * H_i) / kdhi, T_Hsr = (H_i * H_i) / kdhsr, T_H = H_i / kdh;
  const double a_p1 = k_p1 * ATP;
  const double den_i = T_Cai2 + T_Cai2 * T_Hi + T_Hi * (1 + T_H1);
  const double den_sr = T_Casr2 * T_H + T_H + T_Hsr * (1 + T_H);
  const double a_p2 = k_p2 * T_Cai2 / den_i;
  const double a_p3 = k_p3 * T_Hsr / den_sr;
  const double a_m1 = k_m1 * T_Hi / den_i;
  const double a_m2 = k_m2 * ADP * T_Casr2 * T_H / den_sr;
  const double a_m3 = k_m3 * P_i;
  const double s1 = a_p2 * a_p3 + a_m1 * a_p3 + a_m1 * a_m2;
  const double s2 = a_p1 * a_p3 + a_m2 * a_p1 + a_m2 * a_m3;
  const double s3 = a_p1 * a_p2 + a_m3 * a_m1 + a_m3 * a_p2;
  const double v_cycle = (a_p1 * a_p2 * a_p3 - a_m1 * a_m2 * a_m3) / (s1 + s2 + s3);
  const double Q = 1e-3 / 6e17;
  const double J = h * h * (params[1] * (v_cycle * Q));
  const double V = 1e-24 * h * h * h;
  return dt * (J / V);
}

// The same SERCA law with its two common denominators cleared, so one division remains
// (den_i = T_Cai^2(1+T_Hi) + T_Hi(1+T_H1), den_sr = T_H(T_Casr^2+1) + T_Hsr(1+T_H)):
//   v = (a_p1 P2 P3 - M1 M2 a_m3) /
//       (P2 P3 + M1 P3 + M1 M2 + den_i (a_p1 P3 + a_p1 M2 + M2 a_m3) + den_sr (a_p1 P2 + a_m3 M1 + a_m3 P2))
// with P2 = k_p2 T_Cai^2, M1 = k_m1 T_Hi, P3 = k_p3 T_Hsr, M2 = k_m2 ADP T_Casr^2 T_H, the
// numerators of a_p2, a_m1, a_p3, a_m2 in serca_flux.  Equal to serca_flux up to FP64
// rounding; `scale` = dt*density*Q/(1e-24 h) folds the unit conversion of the flux.
__host__ __device__ inline double serca_flux_fast(double u0, double u1, double scale) {
  const double k_p1 = 25900, k_p2 = 2540, k_p3 = 20.5, k_m1 = 16, k_m2 = 67200, k_m3 = 149;
  const double inv_kdcai = 1.0 / 0.9, inv_kdcasr = 1.0 / 2.24;
  const double H_i = 1e-4, ATP = 5, ADP = 36.3e-3, P_i = 1;
  const double T_H1 = H_i / 1.09e-5, T_Hi = (H_i * H_i) / 3.54e-3, T_Hsr = (H_i * H_i) / 1.05e-8, T_H = H_i / 7.24e-5;
  const double T_Cai = u0 * 1e-3 * inv_kdcai, T_Casr = u1 * 1e-3 * inv_kdcasr;
  const double T_Cai2 = T_Cai * T_Cai, T_Casr2 = T_Casr * T_Casr;
  const double a_p1 = k_p1 * ATP, a_m3 = k_m3 * P_i;
  const double den_i = T_Cai2 * (1 + T_Hi) + T_Hi * (1 + T_H1);
  const double den_sr = T_H * (T_Casr2 + 1) + T_Hsr * (1 + T_H);
  const double P2 = k_p2 * T_Cai2, M1 = k_m1 * T_Hi, P3 = k_p3 * T_Hsr, M2 = k_m2 * ADP * T_Casr2 * T_H;
  const double num = a_p1 * P2 * P3 - M1 * M2 * a_m3;
  const double den = P2 * P3 + M1 * P3 + M1 * M2 + den_i * (a_p1 * P3 + a_p1 * M2 + M2 * a_m3) +
                     den_sr * (a_p1 * P2 + a_m3 * M1 + a_m3 * P2);
  return scale * (num / den);
}

__host__ __device__ inline double ryr_flux(double dt, double h, double u0, double u1, const double* params) {
  const double K_0 = exp(-2 * dt * 1e15 / (2 * 96485.) * params[6] / (1300. - 0.1) / (h * h * h));
  return (u0 - u1) * (1 - K_0) / 2;
}

}  // namespace csp
