// csp_mlp.cuh -- learned surrogate of the buffer-binding substep.
//
// With dt_update_react = n*dt the reference advances the buffer reactions once every n
// steps by one explicit step of dt_r = n*dt from the voxel's old state
// (Species_step_reaction, species.c:1653-1702: du += dt_r * J(u)).  The surrogate
// replaces that increment by a learned one.  For one voxel of domain d with Ca = c and
// bound buffer concentrations b_s (s = species 1..5, the slots of the buffers bound to
// Ca in d):
//   plain integrator (training target and fallback): n explicit steps of h = dt_r/n of
//     db_s/dt = g_s = k_on,s (tot_s - b_s) c - k_off,s b_s,  dc/dt = -sum_s g_s
//     (the reference's own reaction update applied at its native step dt, FP64);
//   network: x = [log10(c)/3, b_1/tot_1 .. b_5/tot_5, log10(dt_r)/4, d/4] (8 inputs),
//     two ReLU layers of 64, 5 outputs t_s; the increment is
//     df_s = dt_r g_s / tot_s + S_s t_s,
//     S_s = dt_r^2 / 2 (lambda_s |g_s| + k_on,s (tot_s - b_s) |G|) / tot_s,
//     lambda_s = k_off,s + k_on,s c, G = sum_q g_q (S_s is the size of the second-order
//     term of the exact solution, so t_s stays within about +-1 and the correction
//     vanishes at equilibrium), db_s = tot_s df_s, dc = -sum_s db_s (total Ca conserved by
//     construction): the network learns the correction of the single explicit step
//     towards the plain integrator; an untrained (zero) output layer is the reference's
//     own update;
//   eligible domains: dt_r (sum_s k_on,s tot_s + max_s (k_off,s + 500 k_on,s)) <= 0.25, i.e.
//     the reaction is far from stiff at dt_r over the network's Ca range; voxels of other
//     domains (SR with millimolar CSQN) always take the plain integrator and the network
//     is neither trained nor evaluated there;
//   near equilibrium: where max_s S_s <= MLP_SKIP (1e-8) the correction cannot exceed
//     ~2e-8 of the buffer totals (|t_s| <= 2 on the training data), below FP32
//     resolution, so the network is not evaluated and the increment is the explicit one;
//   acceptance: the increment must satisfy the trapezoidal rule of the ODE,
//     max_s |db_s - dt_r/2 (g_s(y0) + g_s(y0 + dy))| / tot_s <= tol (1e-4 by default);
//     otherwise the voxel takes the plain integrator.
// All FP32 except the plain integrator (FP64).
#pragma once
#include <cuda_runtime.h>

#include "csp_device.cuh"

namespace csp {

constexpr int MLP_IN = 8, MLP_H = 64, MLP_OUT = 5, MLP_SLOTS = 5;
constexpr int MLP_NPARAM = MLP_IN * MLP_H + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H * MLP_OUT + MLP_OUT;

// parameter layout (row-major, input index first): w1[8][64] b1[64] w2[64][64] b2[64] w3[64][5] b3[5]
struct MlpW {
  float w1[MLP_IN * MLP_H];
  float b1[MLP_H];
  float w2[MLP_H * MLP_H];
  float b2[MLP_H];
  float w3[MLP_H * MLP_OUT];
  float b3[MLP_OUT];
};
static_assert(sizeof(MlpW) == MLP_NPARAM * sizeof(float), "MLP parameter layout");

// buffer constants of one domain by slot (species 1..5), zero for absent slots
struct RxConst {
  float kon[MLP_SLOTS], koff[MLP_SLOTS], tot[MLP_SLOTS];
};

constexpr double MLP_STIFF_LIMIT = 0.25, MLP_CA_MAX = 500.0;
constexpr float MLP_SKIP = 1e-8f;

// Domains whose buffer reactions the network serves (see the header comment).
inline unsigned mlp_eligible_domains(const RealDesc& D);

__host__ __device__ inline RxConst rx_const(const RealDesc& D, int d) {
  RxConst k;
  for (int q = 0; q < MLP_SLOTS; q++) {
    const int s = q + 1;
    const bool on = s < NS && D.rtab[d][s] >= 0;
    const int t = on ? D.rtab[d][s] * D.nd + d : 0;
    const double dtr = D.dt_r;
    // the device tables hold the rates times dt_r
    k.kon[q] = on ? (float)(D.kon_dt[t] / dtr) : 0.f;
    k.koff[q] = on ? (float)(D.koff_dt[t] / dtr) : 0.f;
    k.tot[q] = on ? D.tot[t] : 0.f;
  }
  return k;
}

inline unsigned mlp_eligible_domains(const RealDesc& D) {
  unsigned mask = 0;
  const double dtr = D.dt * D.reaction_substep;
  for (int d = 0; d < D.nd; d++) {
    const RxConst k = rx_const(D, d);
    double sum = 0.0, lam = 0.0;
    bool any = false;
    for (int q = 0; q < MLP_SLOTS; q++) {
      if (k.tot[q] <= 0.f) continue;
      any = true;
      sum += (double)k.kon[q] * k.tot[q];
      lam = fmax(lam, (double)k.koff[q] + MLP_CA_MAX * k.kon[q]);
    }
    if (any && dtr * (sum + lam) <= MLP_STIFF_LIMIT) mask |= 1u << d;
  }
  return mask;
}

template <class T>
__host__ __device__ inline T rx_g(const RxConst& k, int q, T c, T b) {
  return (T)k.kon[q] * ((T)k.tot[q] - b) * c - (T)k.koff[q] * b;
}

// Scale S_s of the network's correction (see the header comment).
template <class T>
__host__ __device__ inline void rx_scale(const RxConst& k, T dtr, T c, const T* b, T* S) {
  T G = 0;
  for (int q = 0; q < MLP_SLOTS; q++)
    if (k.tot[q] > 0.f) G += rx_g<T>(k, q, c, b[q]);
  const T aG = G < 0 ? -G : G;
  for (int q = 0; q < MLP_SLOTS; q++) {
    if (k.tot[q] <= 0.f) { S[q] = 0; continue; }
    const T g = rx_g<T>(k, q, c, b[q]);
    const T lam = (T)k.koff[q] + (T)k.kon[q] * c;
    S[q] = (T)0.5 * dtr * dtr * (lam * (g < 0 ? -g : g) + (T)k.kon[q] * ((T)k.tot[q] - b[q]) * aG) / (T)k.tot[q];
  }
}

// The plain integrator: n explicit steps of h, FP64.  In: c, b[]; out: increments.
__host__ __device__ inline void rx_plain(const RxConst& k, int n, double h, double c, const double* b0, double& dc,
                                         double* db) {
  double b[MLP_SLOTS];
  for (int q = 0; q < MLP_SLOTS; q++) b[q] = b0[q];
  double cc = c;
  for (int i = 0; i < n; i++) {
    double g[MLP_SLOTS], sg = 0.0;
    for (int q = 0; q < MLP_SLOTS; q++) {
      g[q] = k.tot[q] > 0.f ? rx_g<double>(k, q, cc, b[q]) : 0.0;
      sg += g[q];
    }
    for (int q = 0; q < MLP_SLOTS; q++) b[q] += h * g[q];
    cc -= h * sg;
  }
  for (int q = 0; q < MLP_SLOTS; q++) db[q] = b[q] - b0[q];
  dc = cc - c;
}

__host__ __device__ inline void rx_features(const RxConst& k, int d, float dtr, float c, const float* b,
                                            float* x) {
  x[0] = log10f(fmaxf(c, 1e-3f)) * (1.f / 3.f);
  for (int q = 0; q < MLP_SLOTS; q++) x[1 + q] = k.tot[q] > 0.f ? b[q] / k.tot[q] : 0.f;
  x[6] = log10f(dtr) * 0.25f;
  x[7] = 0.25f * (float)d;
}

// Training target of one sample: the correction t_s that turns the single explicit step
// into the plain integrator's increment (0 for absent slots or S_s = 0), clipped to +-20.
__host__ __device__ inline void rx_target(const RxConst& k, float dtr, float c, const float* b, const double* db_plain,
                                          float* t) {
  double bd[MLP_SLOTS], S[MLP_SLOTS];
  for (int q = 0; q < MLP_SLOTS; q++) bd[q] = b[q];
  rx_scale<double>(k, (double)dtr, (double)c, bd, S);
  for (int q = 0; q < MLP_SLOTS; q++) {
    if (k.tot[q] <= 0.f || !(S[q] > 1e-30)) { t[q] = 0.f; continue; }
    const double g = rx_g<double>(k, q, (double)c, bd[q]);
    double v = (db_plain[q] / k.tot[q] - dtr * g / k.tot[q]) / S[q];
    v = v > 20.0 ? 20.0 : (v < -20.0 ? -20.0 : v);
    t[q] = (float)v;
  }
}

// Network forward pass of one sample; W in shared memory (broadcast reads).
__device__ __forceinline__ void mlp_forward(const MlpW& W, const float* x, float* y) {
  float h1[MLP_H];
#pragma unroll
  for (int j = 0; j < MLP_H; j++) {
    float a = W.b1[j];
#pragma unroll
    for (int i = 0; i < MLP_IN; i++) a = fmaf(x[i], W.w1[i * MLP_H + j], a);
    h1[j] = fmaxf(a, 0.f);
  }
  float o[MLP_OUT];
#pragma unroll
  for (int q = 0; q < MLP_OUT; q++) o[q] = W.b3[q];
  // second layer in chunks of 16 units, each folded into the outputs at once
#pragma unroll 1
  for (int j0 = 0; j0 < MLP_H; j0 += 16) {
    float a[16];
#pragma unroll
    for (int j = 0; j < 16; j++) a[j] = W.b2[j0 + j];
#pragma unroll
    for (int k = 0; k < MLP_H; k++) {
#pragma unroll
      for (int j = 0; j < 16; j++) a[j] = fmaf(h1[k], W.w2[k * MLP_H + j0 + j], a[j]);
    }
#pragma unroll
    for (int j = 0; j < 16; j++) {
      const float h2 = fmaxf(a[j], 0.f);
#pragma unroll
      for (int q = 0; q < MLP_OUT; q++) o[q] = fmaf(h2, W.w3[(j0 + j) * MLP_OUT + q], o[q]);
    }
  }
#pragma unroll
  for (int q = 0; q < MLP_OUT; q++) y[q] = o[q];
}

// ---- tensor-core forward pass: one warp, 32 samples (one per lane), two tiles of 16
// rows through mma.sync m16n8k8 (TF32 inputs, FP32 accumulation).  Fragment layouts of
// the PTX ISA for m16n8k8 .tf32 (g = lane / 4, q = lane % 4):
//   A (16x8, row): a0 (g, q), a1 (g+8, q), a2 (g, q+4), a3 (g+8, q+4)
//   B (8x8, col):  b0 (q, g), b1 (q+4, g)
//   C (16x8):      c0 (g, 2q), c1 (g, 2q+1), c2 (g+8, 2q), c3 (g+8, 2q+1)
// Weights sit in shared memory with padded rows (MLP_TC_LD) so that the fragment loads
// hit 32 different banks; activations are staged per warp in a [32][MLP_TC_LD] tile.
constexpr int MLP_TC_LD = MLP_H + 4;     // padded row length (floats)
constexpr int MLP_TC_N3 = 8;             // output layer padded to one n-tile
struct MlpTC {
  float w1[MLP_IN * MLP_TC_LD];
  float w2[MLP_H * MLP_TC_LD];
  float w3[MLP_H * MLP_TC_LD];           // [64][8 used of LD], columns 5..7 zero
  float b1[MLP_H], b2[MLP_H], b3[MLP_TC_N3];
};
constexpr int MLP_TC_STAGE = 32 * MLP_TC_LD;   // floats of one warp's activation tile

__device__ __forceinline__ void mlp_tc_load(MlpTC& T, const float* __restrict__ p) {
  const MlpW& W = *reinterpret_cast<const MlpW*>(p);
  for (int i = threadIdx.x; i < MLP_IN * MLP_H; i += blockDim.x) T.w1[(i / MLP_H) * MLP_TC_LD + i % MLP_H] = W.w1[i];
  for (int i = threadIdx.x; i < MLP_H * MLP_H; i += blockDim.x) T.w2[(i / MLP_H) * MLP_TC_LD + i % MLP_H] = W.w2[i];
  for (int i = threadIdx.x; i < MLP_H * MLP_TC_N3; i += blockDim.x) {
    const int k = i / MLP_TC_N3, n = i % MLP_TC_N3;
    T.w3[k * MLP_TC_LD + n] = n < MLP_OUT ? W.w3[k * MLP_OUT + n] : 0.f;
  }
  for (int i = threadIdx.x; i < MLP_H; i += blockDim.x) {
    T.b1[i] = W.b1[i];
    T.b2[i] = W.b2[i];
  }
  for (int i = threadIdx.x; i < MLP_TC_N3; i += blockDim.x) T.b3[i] = i < MLP_OUT ? W.b3[i] : 0.f;
}

__device__ __forceinline__ unsigned tf32_bits(float f) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
  return r;
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// out[32][NT*8] = act(in[32][K] W[K][NT*8] + bias), in / out: [32][MLP_TC_LD] warp tiles
// (out may be in: every read of a tile precedes its writes, and mma.sync converges the warp)
template <int K, int NT, bool RELU>
__device__ __forceinline__ void mlp_tc_layer(const float* in, const float* W, const float* bias, float* out,
                                             int lane) {
  const int g = lane >> 2, q = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 2; mt++) {
    float acc[NT][4];
#pragma unroll
    for (int nt = 0; nt < NT; nt++) {
      acc[nt][0] = acc[nt][2] = bias[nt * 8 + 2 * q];
      acc[nt][1] = acc[nt][3] = bias[nt * 8 + 2 * q + 1];
    }
    const float* r0 = in + (mt * 16 + g) * MLP_TC_LD;
    const float* r1 = r0 + 8 * MLP_TC_LD;
#pragma unroll
    for (int k0 = 0; k0 < K; k0 += 8) {
      const unsigned a[4] = {tf32_bits(r0[k0 + q]), tf32_bits(r1[k0 + q]), tf32_bits(r0[k0 + q + 4]),
                             tf32_bits(r1[k0 + q + 4])};
#pragma unroll
      for (int nt = 0; nt < NT; nt++) {
        const unsigned b[2] = {tf32_bits(W[(k0 + q) * MLP_TC_LD + nt * 8 + g]),
                               tf32_bits(W[(k0 + q + 4) * MLP_TC_LD + nt * 8 + g])};
        mma_tf32(acc[nt], a, b);
      }
    }
    __syncwarp();
    float* o0 = out + (mt * 16 + g) * MLP_TC_LD;
    float* o1 = o0 + 8 * MLP_TC_LD;
#pragma unroll
    for (int nt = 0; nt < NT; nt++) {
      float v[4] = {acc[nt][0], acc[nt][1], acc[nt][2], acc[nt][3]};
      if (RELU)
        for (int i = 0; i < 4; i++) v[i] = fmaxf(v[i], 0.f);
      o0[nt * 8 + 2 * q] = v[0];
      o0[nt * 8 + 2 * q + 1] = v[1];
      o1[nt * 8 + 2 * q] = v[2];
      o1[nt * 8 + 2 * q + 1] = v[3];
    }
    __syncwarp();
  }
}

// Forward pass of the 32 lanes' samples; every lane of the warp must call it.
__device__ __forceinline__ void mlp_forward_tc(const MlpTC& T, float* stage, const float* x, float* y) {
  const int lane = threadIdx.x & 31;
  float* row = stage + lane * MLP_TC_LD;
#pragma unroll
  for (int i = 0; i < MLP_IN; i++) row[i] = x[i];
  __syncwarp();
  mlp_tc_layer<MLP_IN, MLP_H / 8, true>(stage, T.w1, T.b1, stage, lane);
  mlp_tc_layer<MLP_H, MLP_H / 8, true>(stage, T.w2, T.b2, stage, lane);
  mlp_tc_layer<MLP_H, 1, false>(stage, T.w3, T.b3, stage, lane);
#pragma unroll
  for (int i = 0; i < MLP_OUT; i++) y[i] = row[i];
  __syncwarp();
}

// Increment of the network output t, with the acceptance test (see the header comment).
__device__ __forceinline__ bool rx_apply_output(const RxConst& k, float dtr, float c, const float* b, const float* t,
                                                float tol, float& dc, float* db) {
  float S[MLP_SLOTS];
  rx_scale<float>(k, dtr, c, b, S);
  float sdb = 0.f;
  for (int q = 0; q < MLP_SLOTS; q++) {
    if (k.tot[q] <= 0.f) { db[q] = 0.f; continue; }
    const float g = rx_g<float>(k, q, c, b[q]);
    db[q] = k.tot[q] * (dtr * g / k.tot[q] + S[q] * t[q]);
    sdb += db[q];
  }
  dc = -sdb;
  const float c1 = c + dc;
  float worst = 0.f;
  for (int q = 0; q < MLP_SLOTS; q++) {
    if (k.tot[q] <= 0.f) continue;
    const float g0 = rx_g<float>(k, q, c, b[q]), g1 = rx_g<float>(k, q, c1, b[q] + db[q]);
    worst = fmaxf(worst, fabsf(db[q] - 0.5f * dtr * (g0 + g1)) / k.tot[q]);
  }
  return worst <= tol && isfinite(worst);
}

// Surrogate increment of one voxel with acceptance test (FP32 forward pass); returns
// true when accepted.
__device__ __forceinline__ bool rx_surrogate(const MlpW& W, const RxConst& k, int d, float dtr, float c,
                                             const float* b, float tol, float& dc, float* db) {
  float x[MLP_IN], t[MLP_OUT];
  rx_features(k, d, dtr, c, b, x);
  mlp_forward(W, x, t);
  return rx_apply_output(k, dtr, c, b, t, tol, dc, db);
}

}  // namespace csp

namespace csp {

// ---- deployment: the reaction increments of a reaction step, after the voxel kernel
// (run with its reaction switched off) and the boundary kernels.  One thread per voxel;
// blockIdx.y = realisation.  Reads the old state, adds into the new one; species fixed
// in the voxel's domain and, with -f, species 0 on the outer faces keep the values the
// voxel kernel gave them.  The network runs on the tensor cores for a whole warp when
// any of its voxels needs it.  counters[0] += voxels, counters[1] += voxels the network
// ran for, counters[2] += voxels that took the plain integrator.
constexpr int MLP_DEPLOY_T = 256;
constexpr int MLP_DEPLOY_VPT = 128;      // voxels per thread (grid-stride within the realisation)
constexpr size_t MLP_DEPLOY_SMEM = sizeof(MlpTC) + sizeof(float) * (size_t)MLP_TC_STAGE * (MLP_DEPLOY_T / 32);

// One voxel's reaction inputs and the new values they are added to.
struct RxVoxel {
  int d;                       // domain
  bool mine;                   // in the grid and in a domain with buffers
  float c, b[MLP_SLOTS];       // old Ca and buffers
  float nc, nb[MLP_SLOTS];     // new Ca and buffers (after diffusion and boundary fluxes)
};

// p = v mod D.P (the position within the plane), tracked by the caller; uo / un = the
// old / new buffer of every species, dom = the domain bytes, base = the fields' bases
// (RealDesc::fbase; block-shared copies).  The old values are reconstructed (base plus
// stored deviation) for the network and the integrators; the new values stay deviations,
// which the increments are added to.
__device__ __forceinline__ void rx_fetch(const float* const* uo, const float* const* un,
                                         const unsigned char* __restrict__ dom, int plane, const RxConst* sk,
                                         const float (*base)[NS], unsigned fixq, const float (*qunit)[NS], long long v,
                                         int p, long long nvox, RxVoxel& X) {
  X.mine = false;
  X.d = 0;
  X.c = X.nc = 0.f;
#pragma unroll
  for (int q = 0; q < MLP_SLOTS; q++) X.b[q] = X.nb[q] = 0.f;
  if (v >= nvox || p >= plane) return;
  X.d = dom[v] & DOMAIN_BITS;
  const RxConst& kc = sk[X.d];
  bool any = false;
#pragma unroll
  for (int q = 0; q < MLP_SLOTS; q++) any = any || kc.tot[q] > 0.f;
  if (!any) return;
  X.mine = true;
  X.c = __fadd_rn(base[X.d][0], uo[0][v]);
  X.nc = un[0][v];
#pragma unroll
  for (int q = 0; q < MLP_SLOTS; q++) {
    if (kc.tot[q] > 0.f) {
      const float o = uo[q + 1][v];
      X.b[q] = __fadd_rn(base[X.d][q + 1], (fixq >> (q + 1) & 1u) ? q_value(o, qunit[X.d][q + 1]) : o);
      X.nb[q] = un[q + 1][v];     // stored form (an integer for fixed-point species)
    }
  }
}

// Near equilibrium (every S_s <= MLP_SKIP), with S_s <= MLP_SKIP tested as
// lam |g| + k_on (tot - b) |G| <= thr_s, thr_s = MLP_SKIP tot_s / (dt_r^2 / 2) (no division).
// g[] receives the reaction rates g_s (0 for absent buffers) for the explicit increment.
__device__ __forceinline__ bool rx_near_equilibrium(const RxConst& k, const float* thr, float c, const float* b,
                                                    float* g) {
  float G = 0.f;
#pragma unroll
  for (int q = 0; q < MLP_SLOTS; q++) {
    g[q] = k.tot[q] > 0.f ? rx_g<float>(k, q, c, b[q]) : 0.f;
    G += g[q];
  }
  const float aG = fabsf(G);
  bool near = true;
#pragma unroll
  for (int q = 0; q < MLP_SLOTS; q++) {
    if (k.tot[q] <= 0.f) continue;
    const float lam = k.koff[q] + k.kon[q] * c;
    near = near && lam * fabsf(g[q]) + k.kon[q] * (k.tot[q] - b[q]) * aG <= thr[q];
  }
  return near;
}

// The plain integrator's increments (the fallback), FP64, rounded to FP32.
__device__ __forceinline__ void rx_fallback(const RxConst& kc, int n, double dt, float c, const float* b, float& dc,
                                            float* db) {
  double bd[MLP_SLOTS], dbd[MLP_SLOTS], dcd;
  for (int q = 0; q < MLP_SLOTS; q++) bd[q] = b[q];
  rx_plain(kc, n, dt, (double)c, bd, dcd, dbd);
  for (int q = 0; q < MLP_SLOTS; q++) db[q] = (float)dbd[q];
  dc = (float)dcd;
}

// New values of one voxel: its buffers and Ca plus the increments, except fixed species
// and, with Dirichlet faces (-f), Ca on the outer faces.
// fm = the domain's fixed-species mask (RealDesc::fixed_mask).
__device__ __forceinline__ void rx_store(unsigned fm, const float* const* un, const RxConst& kc, long long v,
                                         bool face, float nc, const float* nb, float dc, const float* db,
                                         unsigned fixq, const float* qinv) {
#pragma unroll
  for (int q = 0; q < MLP_SLOTS; q++) {
    const int s = q + 1;
    if (kc.tot[q] <= 0.f || (fm >> s & 1u)) continue;
    const_cast<float*>(un[s])[v] = (fixq >> s & 1u) ? q_add(nb[q], db[q], qinv[s]) : __fadd_rn(nb[q], db[q]);
  }
  if (!(fm & 1u) && !face) const_cast<float*>(un[0])[v] = __fadd_rn(nc, dc);
}

__device__ __forceinline__ bool rx_on_face(const RealDesc& D, int x, int p) {
  const int c1 = p / D.nz, c2 = p - c1 * D.nz;
  return x == 0 || x == D.nx - 1 || c1 == 0 || c1 == D.ny - 1 || c2 == 0 || c2 == D.nz - 1;
}

// Each thread walks MLP_DEPLOY_VPT voxels, the next voxel's values loaded before the
// current one is worked on.  Voxels near equilibrium and voxels of stiff domains are
// finished at once; voxels that need the network are queued per warp (their indices in
// shared memory) and the network runs on full tiles of 32 queued voxels, which reload
// their state: the tensor-core passes carry no idle lanes but the last one.
__global__ void __launch_bounds__(MLP_DEPLOY_T) k_react_surrogate(const RealDesc* __restrict__ descs,
                                                                  const RealCtl* __restrict__ ctl,
                                                                  const float* __restrict__ params, float tol,
                                                                  unsigned long long* __restrict__ counters) {
  extern __shared__ __align__(16) float dsm[];
  MlpTC& T = *reinterpret_cast<MlpTC*>(dsm);
  float* stage = dsm + sizeof(MlpTC) / sizeof(float) + (threadIdx.x >> 5) * MLP_TC_STAGE;
  __shared__ RxConst sk[ND];
  __shared__ float s_thr[ND][MLP_SLOTS];
  __shared__ unsigned s_fm[ND];
  __shared__ float s_base[ND][NS];
  __shared__ float s_qunit[ND][NS], s_qinv[ND][NS];
  __shared__ const float* s_uo[NS];
  __shared__ const float* s_un[NS];
  __shared__ long long s_pend[MLP_DEPLOY_T / 32][64];   // per warp: queued voxels (up to two tiles)
  __shared__ unsigned s_vox, s_net, s_fall;
  const RealDesc& D = descs[blockIdx.y];
  const RealCtl& C = ctl[blockIdx.y];
  const long long k = C.step, ti = k + 1;
  const bool active = !C.stopped && D.react_external && D.nbuf > 0 && ti % D.reaction_substep == 0;
  if (!active) return;                              // uniform over the block
  const long long nvox = (long long)D.nx * D.P;
  const long long span = (long long)MLP_DEPLOY_T * MLP_DEPLOY_VPT;
  if ((long long)blockIdx.x * span >= nvox) return;  // uniform over the block
  const unsigned cur = C.cur_mask[k & 1];
  const float dtr = (float)(D.dt * D.reaction_substep);
  mlp_tc_load(T, params);
  if (threadIdx.x < ND) {
    const RxConst kc = rx_const(D, threadIdx.x < D.nd ? threadIdx.x : 0);
    sk[threadIdx.x] = kc;
    for (int q = 0; q < MLP_SLOTS; q++) s_thr[threadIdx.x][q] = MLP_SKIP * kc.tot[q] / (0.5f * dtr * dtr);
    s_fm[threadIdx.x] = D.fixed_mask[threadIdx.x < D.nd ? threadIdx.x : 0];
    for (int s = 0; s < NS; s++) {
      s_base[threadIdx.x][s] = D.fbase[threadIdx.x][s];
      s_qunit[threadIdx.x][s] = D.qunit[threadIdx.x][s];
      s_qinv[threadIdx.x][s] = D.qinv[threadIdx.x][s];
    }
  }
  if (threadIdx.x < NS) {
    const int t = threadIdx.x;
    s_uo[t] = D.u[(cur >> t) & 1u][t];
    s_un[t] = D.u[((cur >> t) & 1u) ^ 1u][t];
  }
  if (threadIdx.x == 0) { s_vox = 0; s_net = 0; s_fall = 0; }
  __syncthreads();
  const unsigned char* __restrict__ dom = D.dom;
  const int plane = D.plane;
  const unsigned elig_mask = D.mlp_domains;
  const bool dirichlet = D.dirichlet != 0;
  const unsigned fixq = D.fixq;
  unsigned n_vox = 0, n_net = 0, n_fall = 0;
  const long long v0 = (long long)blockIdx.x * span + threadIdx.x;
  // position within the plane and plane index of the voxel being fetched, advanced by
  // MLP_DEPLOY_T per iteration without divisions (one at the start)
  const int P = D.P;
  int pf = (int)(v0 % P), xf = (int)(v0 / P);
  int pc = pf, xc = xf;
  long long* pend = s_pend[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  int npend = 0;                                     // warp-uniform
  // the network on queued voxels pend[0 .. count) (lane i takes pend[i]), whole warp
  auto flush = [&](int count) {
    __syncwarp();
    const bool have = lane < count;
    const long long v = have ? pend[lane] : 0;
    RxVoxel Y;
    int pq = 0, xq = 0;
    if (have) {
      xq = (int)(v / P);
      pq = (int)(v - (long long)xq * P);
    }
    rx_fetch(s_uo, s_un, dom, plane, sk, s_base, fixq, s_qunit, have ? v : nvox, pq, nvox, Y);
    const RxConst& kc = sk[Y.d];
    float x[MLP_IN], t[MLP_OUT], db[MLP_SLOTS], dc = 0.f;
    if (have) rx_features(kc, Y.d, dtr, Y.c, Y.b, x);
    else
      for (int i = 0; i < MLP_IN; i++) x[i] = 0.f;
    mlp_forward_tc(T, stage, x, t);
    if (have) {
      n_vox++;
      n_net++;
      if (!rx_apply_output(kc, dtr, Y.c, Y.b, t, tol, dc, db)) {
        n_fall++;
        rx_fallback(kc, D.reaction_substep, D.dt, Y.c, Y.b, dc, db);
      }
      rx_store(s_fm[Y.d], s_un, kc, v, dirichlet && rx_on_face(D, xq, pq), Y.nc, Y.nb, dc, db, fixq, s_qinv[Y.d]);
    }
    __syncwarp();
  };
  RxVoxel X;
  rx_fetch(s_uo, s_un, dom, plane, sk, s_base, fixq, s_qunit, v0, pf, nvox, X);
  for (int it = 0; it < MLP_DEPLOY_VPT; it++) {
    const long long v = v0 + (long long)it * MLP_DEPLOY_T;
    const RxVoxel Y = X;
    pc = pf;
    xc = xf;
    pf += MLP_DEPLOY_T;
    while (pf >= P) { pf -= P; xf++; }
    if (it + 1 < MLP_DEPLOY_VPT) rx_fetch(s_uo, s_un, dom, plane, sk, s_base, fixq, s_qunit, v + MLP_DEPLOY_T, pf, nvox, X);
    const int d = Y.d;
    const RxConst& kc = sk[d];
    bool elig = false, skip = false;
    float g[MLP_SLOTS];
    if (Y.mine) {
      elig = (elig_mask >> d) & 1u;
      skip = elig && rx_near_equilibrium(kc, s_thr[d], Y.c, Y.b, g);
    }
    const bool net = Y.mine && elig && !skip;
    if (Y.mine && !net) {
      float db[MLP_SLOTS], dc;
      n_vox++;
      if (skip) {
        // near equilibrium: the explicit increment
        float sdb = 0.f;
        for (int q = 0; q < MLP_SLOTS; q++) {
          db[q] = kc.tot[q] > 0.f ? dtr * g[q] : 0.f;
          sdb += db[q];
        }
        dc = -sdb;
      } else {
        // a stiff domain: the plain integrator
        n_fall++;
        rx_fallback(kc, D.reaction_substep, D.dt, Y.c, Y.b, dc, db);
      }
      rx_store(s_fm[d], s_un, kc, v, dirichlet && rx_on_face(D, xc, pc), Y.nc, Y.nb, dc, db, fixq, s_qinv[d]);
    }
    const unsigned nm = __ballot_sync(0xffffffffu, net);
    if (net) pend[npend + __popc(nm & ((1u << lane) - 1u))] = v;
    npend += __popc(nm);
    // full tiles, and after the last voxel whatever is queued (one call site)
    while (npend >= 32 || (npend > 0 && it == MLP_DEPLOY_VPT - 1)) {
      const int cnt = min(npend, 32);
      flush(cnt);
      const int rest = npend - cnt;
      const long long mv = lane < rest ? pend[32 + lane] : 0;
      __syncwarp();
      if (lane < rest) pend[lane] = mv;
      __syncwarp();
      npend = rest;
    }
  }
  if (n_vox) atomicAdd(&s_vox, n_vox);
  if (n_net) atomicAdd(&s_net, n_net);
  if (n_fall) atomicAdd(&s_fall, n_fall);
  __syncthreads();
  if (threadIdx.x == 0 && s_vox) {
    atomicAdd(&counters[0], (unsigned long long)s_vox);
    atomicAdd(&counters[1], (unsigned long long)s_net);
    atomicAdd(&counters[2], (unsigned long long)s_fall);
  }
}

// Forward passes for checks: y[n][5] of x[n][8], FP32 (tc = 0) or tensor cores (tc = 1).
__global__ void __launch_bounds__(MLP_DEPLOY_T) k_mlp_forward(const float* __restrict__ params,
                                                              const float* __restrict__ x, long long n, int tc,
                                                              float* __restrict__ y) {
  extern __shared__ __align__(16) float dsm[];
  MlpTC& T = *reinterpret_cast<MlpTC*>(dsm);
  MlpW& W = *reinterpret_cast<MlpW*>(dsm + sizeof(MlpTC) / sizeof(float) + (size_t)MLP_TC_STAGE * (MLP_DEPLOY_T / 32));
  float* stage = dsm + sizeof(MlpTC) / sizeof(float) + (threadIdx.x >> 5) * MLP_TC_STAGE;
  mlp_tc_load(T, params);
  for (int i = threadIdx.x; i < MLP_NPARAM; i += blockDim.x) reinterpret_cast<float*>(&W)[i] = params[i];
  __syncthreads();
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  float xi[MLP_IN], yi[MLP_OUT];
  for (int j = 0; j < MLP_IN; j++) xi[j] = i < n ? x[i * MLP_IN + j] : 0.f;
  if (tc) mlp_forward_tc(T, stage, xi, yi);
  else mlp_forward(W, xi, yi);
  if (i < n)
    for (int j = 0; j < MLP_OUT; j++) y[i * MLP_OUT + j] = yi[j];
}
constexpr size_t MLP_FORWARD_SMEM = MLP_DEPLOY_SMEM + sizeof(MlpW);

// ---- training ----

// Voxel-state pairs for one realisation's buffer constants: Ca log-uniform over
// [0.1, 500] uM in cytosolic domains (initial Ca < 100 uM) and [10, 2000] uM in SR
// domains; bound fractions at equilibrium with a log-normally perturbed Ca (20 %:
// uniform in [0, 1]); dt_r = dt * reaction_substep.  x[n][8] features, t[n][5] targets.
__global__ void k_mlp_pairs(const RealDesc* __restrict__ desc, unsigned long long seed, long long n,
                            const int* __restrict__ doms, int ndoms, float* __restrict__ x, float* __restrict__ t) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RealDesc& D = *desc;
  unsigned ctr[4] = {(unsigned)i, (unsigned)(i >> 32), 0x6d6c70u, 0u}, r[4], r2[4];
  philox4x32(ctr, (unsigned)seed, (unsigned)(seed >> 32) ^ 0x5eedu, r);
  ctr[3] = 1u;
  philox4x32(ctr, (unsigned)seed, (unsigned)(seed >> 32) ^ 0x5eedu, r2);
  auto u01 = [](unsigned a) { return ((double)a + 0.5) * (1.0 / 4294967296.0); };
  const int d = doms[r[0] % (unsigned)ndoms];
  const bool sr = D.init[d][0] >= 100.f;
  const double lo = sr ? 10.0 : 0.1, hi = sr ? 2000.0 : 500.0;
  const double c = lo * exp(u01(r[1]) * log(hi / lo));
  // Box-Muller normal for the perturbation of the equilibrium Ca
  const double z = sqrt(-2.0 * log(u01(r[2]))) * cos(6.283185307179586 * u01(r[3]));
  const double ce = c * exp(z);
  const RxConst kc = rx_const(D, d);
  float b[MLP_SLOTS];
  for (int q = 0; q < MLP_SLOTS; q++) {
    if (kc.tot[q] <= 0.f) { b[q] = 0.f; continue; }
    double f = kc.kon[q] * ce / (kc.kon[q] * ce + kc.koff[q]);
    if (u01(r2[q & 3] ^ (unsigned)(q * 0x9E3779B9u)) < 0.2) f = u01(r2[(q + 1) & 3] * 2654435761u);
    b[q] = (float)(f * kc.tot[q]);
  }
  const float dtr = (float)(D.dt * D.reaction_substep);
  double bd[MLP_SLOTS], dbd[MLP_SLOTS], dcd;
  for (int q = 0; q < MLP_SLOTS; q++) bd[q] = b[q];
  rx_plain(kc, D.reaction_substep, D.dt, (double)(float)c, bd, dcd, dbd);
  float xf[MLP_IN], tf[MLP_OUT];
  rx_features(kc, d, dtr, (float)c, b, xf);
  rx_target(kc, dtr, (float)c, b, dbd, tf);
  for (int j = 0; j < MLP_IN; j++) x[i * MLP_IN + j] = xf[j];
  for (int j = 0; j < MLP_OUT; j++) t[i * MLP_OUT + j] = tf[j];
}

// ---- training pairs harvested from simulation states (csp_mlp_harvest) ----
// Candidates are the voxels of the surrogate's domains with Ca in [0.1, 500] uM; their
// log10 Ca falls in one of MLP_HARVEST_BINS bins.  Pass 0 counts the candidates per bin;
// pass 1 takes each with its bin's probability (prob[], chosen on the host so the taken
// pairs are as near log-uniform in Ca as the states allow) and writes its features and
// its target from the plain integrator, exactly as k_mlp_pairs does for drawn states.
constexpr int MLP_HARVEST_BINS = 32;
constexpr float MLP_HARVEST_LO = -1.f, MLP_HARVEST_HI = 2.69897f;   // log10(0.1), log10(500)

__global__ void k_mlp_harvest(const RealDesc* __restrict__ descs, const RealCtl* __restrict__ ctl,
                              const unsigned* __restrict__ elig, int pass, const float* __restrict__ prob,
                              unsigned long long seed,
                              unsigned long long* __restrict__ hist, unsigned long long* __restrict__ cursor,
                              long long cap, float* __restrict__ x, float* __restrict__ t) {
  __shared__ unsigned s_hist[MLP_HARVEST_BINS];
  if (threadIdx.x < MLP_HARVEST_BINS) s_hist[threadIdx.x] = 0;
  __syncthreads();
  const int r = blockIdx.y;
  const RealDesc& D = descs[r];
  const RealCtl& C = ctl[r];
  const unsigned cur = C.cur_mask[C.step & 1];
  const long long nvox = (long long)D.nx * D.P;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < nvox;
       v += (long long)gridDim.x * blockDim.x) {
    if ((int)(v % D.P) >= D.plane) continue;
    const int d = D.dom[v] & DOMAIN_BITS;
    if (!((elig[r] >> d) & 1u)) continue;
    const float c = __fadd_rn(D.fbase[d][0], D.u[cur & 1u][0][v]);
    if (!(c >= 0.1f && c <= 500.f)) continue;
    const int bin = min(MLP_HARVEST_BINS - 1,
                        (int)((log10f(c) - MLP_HARVEST_LO) * (MLP_HARVEST_BINS / (MLP_HARVEST_HI - MLP_HARVEST_LO))));
    if (pass == 0) {
      atomicAdd(&s_hist[max(bin, 0)], 1u);
      continue;
    }
    unsigned ctr[4] = {(unsigned)v, (unsigned)(v >> 32), (unsigned)r, 0x68727374u}, rr[4];
    philox4x32(ctr, (unsigned)seed, (unsigned)(seed >> 32), rr);
    if (((double)rr[0] + 0.5) * (1.0 / 4294967296.0) >= prob[max(bin, 0)]) continue;
    const unsigned long long slot = atomicAdd(cursor, 1ull);
    if ((long long)slot >= cap) continue;
    const RxConst kc = rx_const(D, d);
    float b[MLP_SLOTS];
    double bd[MLP_SLOTS], dbd[MLP_SLOTS], dcd;
    for (int q = 0; q < MLP_SLOTS; q++) {
      const float o = D.u[(cur >> (q + 1)) & 1u][q + 1][v];
      b[q] = kc.tot[q] > 0.f
                 ? __fadd_rn(D.fbase[d][q + 1], (D.fixq >> (q + 1) & 1u) ? q_value(o, D.qunit[d][q + 1]) : o)
                 : 0.f;
      bd[q] = b[q];
    }
    const float dtr = (float)(D.dt * D.reaction_substep);
    rx_plain(kc, D.reaction_substep, D.dt, (double)c, bd, dcd, dbd);
    float xf[MLP_IN], tf[MLP_OUT];
    rx_features(kc, d, dtr, c, b, xf);
    rx_target(kc, dtr, c, b, dbd, tf);
    for (int j = 0; j < MLP_IN; j++) x[slot * MLP_IN + j] = xf[j];
    for (int j = 0; j < MLP_OUT; j++) t[slot * MLP_OUT + j] = tf[j];
  }
  if (pass == 0) {
    __syncthreads();
    if (threadIdx.x < MLP_HARVEST_BINS && s_hist[threadIdx.x])
      atomicAdd(&hist[threadIdx.x], (unsigned long long)s_hist[threadIdx.x]);
  }
}

// Pairs [0, n) gathered in the order of the affine bijection j -> (a j + b) mod n (a odd
// and coprime with n), so training batches mix states from every part of the harvest.
__global__ void k_mlp_permute(const float* __restrict__ x, const float* __restrict__ t, long long n,
                              unsigned long long a, unsigned long long b, float* __restrict__ xo, float* __restrict__ to) {
  const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j >= n) return;
  const long long i = (long long)((a * (unsigned long long)j + b) % (unsigned long long)n);
  for (int q = 0; q < MLP_IN; q++) xo[j * MLP_IN + q] = x[i * MLP_IN + q];
  for (int q = 0; q < MLP_OUT; q++) to[j * MLP_OUT + q] = t[i * MLP_OUT + q];
}

constexpr int MLP_TB = 128;           // samples (threads) per CTA of the gradient kernel
constexpr int MLP_LD = MLP_H + 1;     // padded row length of the activation tiles

// Loss and gradient of the mean squared error over samples [0, n): every CTA takes
// MLP_TB samples, runs the forward and backward pass per sample (thread) into shared
// tiles, forms its weight gradients as small GEMMs over its samples and adds them (and
// its loss sum) to grad[MLP_NPARAM] / loss[0] with atomics.  scale = 1 / (n * MLP_OUT).
__global__ void __launch_bounds__(MLP_TB) k_mlp_grad(const float* __restrict__ params, const float* __restrict__ x,
                                                     const float* __restrict__ t, long long n, float scale,
                                                     float* __restrict__ grad, float* __restrict__ loss) {
  extern __shared__ float sm[];
  MlpW& W = *reinterpret_cast<MlpW*>(sm);
  float* X = sm + MLP_NPARAM;                  // [TB][8]
  float* H1 = X + MLP_TB * MLP_IN;             // [TB][LD] relu(layer 1)
  float* H2 = H1 + MLP_TB * MLP_LD;            // [TB][LD] relu(layer 2)
  float* D2 = H2 + MLP_TB * MLP_LD;            // [TB][LD] dL/d(pre-activation 2)
  float* D1 = D2 + MLP_TB * MLP_LD;            // [TB][LD] dL/d(pre-activation 1)
  float* DY = D1 + MLP_TB * MLP_LD;            // [TB][5]
  __shared__ float s_loss;
  const int tid = threadIdx.x;
  for (int i = tid; i < MLP_NPARAM; i += MLP_TB) sm[i] = params[i];
  if (tid == 0) s_loss = 0.f;
  const long long i0 = (long long)blockIdx.x * MLP_TB;
  const long long i = i0 + tid;
  const bool valid = i < n;
  for (int j = 0; j < MLP_IN; j++) X[tid * MLP_IN + j] = valid ? x[i * MLP_IN + j] : 0.f;
  __syncthreads();
  // forward
  float* h1 = H1 + tid * MLP_LD;
  float* h2 = H2 + tid * MLP_LD;
  for (int j = 0; j < MLP_H; j++) {
    float a = W.b1[j];
    for (int q = 0; q < MLP_IN; q++) a = fmaf(X[tid * MLP_IN + q], W.w1[q * MLP_H + j], a);
    h1[j] = fmaxf(a, 0.f);
  }
  for (int j = 0; j < MLP_H; j++) {
    float a = W.b2[j];
    for (int q = 0; q < MLP_H; q++) a = fmaf(h1[q], W.w2[q * MLP_H + j], a);
    h2[j] = fmaxf(a, 0.f);
  }
  float l = 0.f;
  for (int q = 0; q < MLP_OUT; q++) {
    float y = W.b3[q];
    for (int j = 0; j < MLP_H; j++) y = fmaf(h2[j], W.w3[j * MLP_OUT + q], y);
    const float e = valid ? y - t[i * MLP_OUT + q] : 0.f;
    l += e * e;
    DY[tid * MLP_OUT + q] = 2.f * e * scale;
  }
  atomicAdd(&s_loss, l * scale);
  // backward to the pre-activations
  float* d2 = D2 + tid * MLP_LD;
  float* d1 = D1 + tid * MLP_LD;
  for (int j = 0; j < MLP_H; j++) {
    float a = 0.f;
    for (int q = 0; q < MLP_OUT; q++) a = fmaf(W.w3[j * MLP_OUT + q], DY[tid * MLP_OUT + q], a);
    d2[j] = h2[j] > 0.f ? a : 0.f;
  }
  for (int k = 0; k < MLP_H; k++) {
    float a = 0.f;
    for (int j = 0; j < MLP_H; j++) a = fmaf(W.w2[k * MLP_H + j], d2[j], a);
    d1[k] = h1[k] > 0.f ? a : 0.f;
  }
  __syncthreads();
  // weight gradients: sums over the CTA's samples
  float* gw1 = grad;
  float* gb1 = gw1 + MLP_IN * MLP_H;
  float* gw2 = gb1 + MLP_H;
  float* gb2 = gw2 + MLP_H * MLP_H;
  float* gw3 = gb2 + MLP_H;
  float* gb3 = gw3 + MLP_H * MLP_OUT;
  {
    // w2[k][j] = sum_b H1[b][k] D2[b][j]: thread -> k = tid % 64, j in one half
    const int kk = tid % MLP_H, jh = (tid / MLP_H) * (MLP_H / 2);
    float acc[MLP_H / 2];
    for (int j = 0; j < MLP_H / 2; j++) acc[j] = 0.f;
    for (int b = 0; b < MLP_TB; b++) {
      const float hk = H1[b * MLP_LD + kk];
      for (int j = 0; j < MLP_H / 2; j++) acc[j] = fmaf(hk, D2[b * MLP_LD + jh + j], acc[j]);
    }
    for (int j = 0; j < MLP_H / 2; j++) atomicAdd(&gw2[kk * MLP_H + jh + j], acc[j]);
  }
  for (int e = tid; e < MLP_IN * MLP_H + 2 * MLP_H + MLP_H * MLP_OUT + MLP_OUT; e += MLP_TB) {
    float acc = 0.f;
    if (e < MLP_IN * MLP_H) {                                   // w1[q][k]
      const int q = e / MLP_H, kk = e % MLP_H;
      for (int b = 0; b < MLP_TB; b++) acc = fmaf(X[b * MLP_IN + q], D1[b * MLP_LD + kk], acc);
      atomicAdd(&gw1[e], acc);
    } else if (e < MLP_IN * MLP_H + MLP_H) {                    // b1[k]
      const int kk = e - MLP_IN * MLP_H;
      for (int b = 0; b < MLP_TB; b++) acc += D1[b * MLP_LD + kk];
      atomicAdd(&gb1[kk], acc);
    } else if (e < MLP_IN * MLP_H + 2 * MLP_H) {                // b2[j]
      const int j = e - MLP_IN * MLP_H - MLP_H;
      for (int b = 0; b < MLP_TB; b++) acc += D2[b * MLP_LD + j];
      atomicAdd(&gb2[j], acc);
    } else if (e < MLP_IN * MLP_H + 2 * MLP_H + MLP_H * MLP_OUT) {   // w3[j][q]
      const int f = e - MLP_IN * MLP_H - 2 * MLP_H;
      const int j = f / MLP_OUT, q = f % MLP_OUT;
      for (int b = 0; b < MLP_TB; b++) acc = fmaf(H2[b * MLP_LD + j], DY[b * MLP_OUT + q], acc);
      atomicAdd(&gw3[f], acc);
    } else {                                                    // b3[q]
      const int q = e - MLP_IN * MLP_H - 2 * MLP_H - MLP_H * MLP_OUT;
      for (int b = 0; b < MLP_TB; b++) acc += DY[b * MLP_OUT + q];
      atomicAdd(&gb3[q], acc);
    }
  }
  __syncthreads();
  if (tid == 0) atomicAdd(loss, s_loss);
}

constexpr size_t MLP_GRAD_SMEM =
    sizeof(float) * ((size_t)MLP_NPARAM + MLP_TB * MLP_IN + 4 * (size_t)MLP_TB * MLP_LD + MLP_TB * MLP_OUT);

// Adam step (Kingma & Ba, 2015) on every parameter; clears the gradient.
__global__ void k_mlp_adam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                           int n, float lr, float b1, float b2, float eps, int step) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / (1.f - powf(b1, (float)step)), vh = vi / (1.f - powf(b2, (float)step));
  p[i] -= lr * mh / (sqrtf(vh) + eps);
  g[i] = 0.f;
}

// Acceptance rate of the network on samples: rebuilds each voxel state from its features
// and applies the surrogate's acceptance test.  counts[0] += accepted.
__global__ void __launch_bounds__(256) k_mlp_accept(const RealDesc* __restrict__ desc, const float* __restrict__ params,
                                                    const float* __restrict__ x, long long n, float tol,
                                                    unsigned long long* __restrict__ counts) {
  __shared__ MlpW W;
  for (int i = threadIdx.x; i < MLP_NPARAM; i += blockDim.x) reinterpret_cast<float*>(&W)[i] = params[i];
  __syncthreads();
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RealDesc& D = *desc;
  const float* xi = x + i * MLP_IN;
  const int d = (int)lrintf(xi[7] * 4.f);
  const RxConst kc = rx_const(D, d);
  const float c = powf(10.f, 3.f * xi[0]);
  float b[MLP_SLOTS], db[MLP_SLOTS], dc;
  for (int q = 0; q < MLP_SLOTS; q++) b[q] = xi[1 + q] * kc.tot[q];
  const float dtr = (float)(D.dt * D.reaction_substep);
  if (rx_surrogate(W, kc, d, dtr, c, b, tol, dc, db)) atomicAdd(&counts[0], 1ull);
}

}  // namespace csp
