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
#include "csp_staged.cuh"   // mbarrier helpers and the bounded wait

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
  // absent slots (tot = 0) would add exact zeros: they are skipped
  bool on[MLP_SLOTS];
  for (int q = 0; q < MLP_SLOTS; q++) on[q] = k.tot[q] > 0.f;
  for (int i = 0; i < n; i++) {
    double g[MLP_SLOTS], sg = 0.0;
    for (int q = 0; q < MLP_SLOTS; q++) {
      g[q] = 0.0;
      if (!on[q]) continue;
      g[q] = rx_g<double>(k, q, cc, b[q]);
      sg += g[q];
    }
    for (int q = 0; q < MLP_SLOTS; q++)
      if (on[q]) b[q] += h * g[q];
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
// Weights sit in shared memory as TF32 bit patterns (converted once per CTA) in fragment
// order: for k-block kb and n-tile pair np, lane l's four words (b0, b1 of n-tile 2np, then
// of 2np + 1) are contiguous, so a lane fetches two B fragments with one 16-byte load
// (the output layer, a single n-tile: two words).  Activations are staged per warp in a
// [32][MLP_TC_LD] tile whose padded rows put the A-fragment loads in 32 different banks.
constexpr int MLP_TC_LD = MLP_H + 4;     // padded row length (floats)
constexpr int MLP_TC_N3 = 8;             // output layer padded to one n-tile
constexpr int MLP_F1 = (MLP_IN / 8) * (MLP_H / 16) * 32 * 4;
constexpr int MLP_F2 = (MLP_H / 8) * (MLP_H / 16) * 32 * 4;
constexpr int MLP_F3 = (MLP_H / 8) * 32 * 2;
struct MlpTC {
  unsigned f1[MLP_F1], f2[MLP_F2], f3[MLP_F3];
  float b1[MLP_H], b2[MLP_H], b3[MLP_TC_N3];
};
static_assert(sizeof(MlpTC) % 16 == 0, "activation tiles follow the weights");
constexpr int MLP_TC_STAGE = 32 * MLP_TC_LD;   // floats of one warp's activation tile

__device__ __forceinline__ unsigned tf32_bits(float f) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
  return r;
}

// Fragment-order word i of a layer with K inputs, NT n-tiles and W = [K][NV] (columns
// beyond NV read as 0).
template <int K, int NT, int NV>
__device__ __forceinline__ unsigned mlp_frag_word(const float* W, int i) {
  int kb, nt, lane, h;
  if constexpr (NT >= 2) {
    const int w = i & 3, rest = i >> 7;
    lane = (i >> 2) & 31;
    kb = rest / (NT / 2);
    nt = 2 * (rest % (NT / 2)) + (w >> 1);
    h = w & 1;
  } else {
    h = i & 1;
    lane = (i >> 1) & 31;
    kb = i >> 6;
    nt = 0;
  }
  const int k = kb * 8 + (lane & 3) + 4 * h, n = nt * 8 + (lane >> 2);
  return n < NV ? tf32_bits(W[k * NV + n]) : 0u;
}

__device__ __forceinline__ void mlp_tc_load(MlpTC& T, const float* __restrict__ p) {
  const MlpW& W = *reinterpret_cast<const MlpW*>(p);
  for (int i = threadIdx.x; i < MLP_F1; i += blockDim.x) T.f1[i] = mlp_frag_word<MLP_IN, MLP_H / 8, MLP_H>(W.w1, i);
  for (int i = threadIdx.x; i < MLP_F2; i += blockDim.x) T.f2[i] = mlp_frag_word<MLP_H, MLP_H / 8, MLP_H>(W.w2, i);
  for (int i = threadIdx.x; i < MLP_F3; i += blockDim.x) T.f3[i] = mlp_frag_word<MLP_H, 1, MLP_OUT>(W.w3, i);
  for (int i = threadIdx.x; i < MLP_H; i += blockDim.x) {
    T.b1[i] = W.b1[i];
    T.b2[i] = W.b2[i];
  }
  for (int i = threadIdx.x; i < MLP_TC_N3; i += blockDim.x) T.b3[i] = i < MLP_OUT ? W.b3[i] : 0.f;
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
__device__ __forceinline__ void mlp_tc_layer(const float* in, const unsigned* F, const float* bias, float* out,
                                             int lane) {
  const int g = lane >> 2, q = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 2; mt++) {
    float acc[NT][4];
#pragma unroll
    for (int nt = 0; nt < NT; nt++) {
      const float2 bb = *reinterpret_cast<const float2*>(bias + nt * 8 + 2 * q);
      acc[nt][0] = acc[nt][2] = bb.x;
      acc[nt][1] = acc[nt][3] = bb.y;
    }
    const float* r0 = in + (mt * 16 + g) * MLP_TC_LD;
    const float* r1 = r0 + 8 * MLP_TC_LD;
#pragma unroll
    for (int kb = 0; kb < K / 8; kb++) {
      const int k0 = kb * 8;
      const unsigned a[4] = {tf32_bits(r0[k0 + q]), tf32_bits(r1[k0 + q]), tf32_bits(r0[k0 + q + 4]),
                             tf32_bits(r1[k0 + q + 4])};
      if constexpr (NT >= 2) {
#pragma unroll
        for (int np = 0; np < NT / 2; np++) {
          const uint4 bb = *reinterpret_cast<const uint4*>(F + ((kb * (NT / 2) + np) * 32 + lane) * 4);
          const unsigned b0[2] = {bb.x, bb.y}, b1[2] = {bb.z, bb.w};
          mma_tf32(acc[2 * np], a, b0);
          mma_tf32(acc[2 * np + 1], a, b1);
        }
      } else {
        const uint2 bb = *reinterpret_cast<const uint2*>(F + (kb * 32 + lane) * 2);
        const unsigned b0[2] = {bb.x, bb.y};
        mma_tf32(acc[0], a, b0);
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
  mlp_tc_layer<MLP_IN, MLP_H / 8, true>(stage, T.f1, T.b1, stage, lane);
  mlp_tc_layer<MLP_H, MLP_H / 8, true>(stage, T.f2, T.b2, stage, lane);
  mlp_tc_layer<MLP_H, 1, false>(stage, T.f3, T.b3, stage, lane);
#pragma unroll
  for (int i = 0; i < MLP_OUT; i++) y[i] = row[i];
  __syncwarp();
}

// ---- tcgen05 forward pass: 128 samples per warpgroup (4 warps, one sample per thread).
// One thread of the warpgroup issues tcgen05.mma (kind::tf32, FP32 accumulation in the
// warpgroup's 64 columns of tensor memory) for a layer; the MMAs' completion arrives on
// the warpgroup's mbarrier (tcgen05.commit); each warp then reads its 32 TMEM lanes (rows:
// one sample per thread) with tcgen05.ld, adds the bias, applies the ReLU and writes the
// row back to shared memory as the next layer's A operand.  The warpgroups of a CTA share
// the weights and synchronise only among themselves (named barrier 1 + wg), so one
// warpgroup's MMAs overlap the other's epilogue.  Operands sit in shared memory in the
// canonical K-major layout without swizzle: element (row, k) of a matrix of R rows at byte
//   (k / 4) * 16 R + (row / 8) * 128 + (row % 8) * 16 + (k % 4) * 4,
// i.e. core matrices of 8 rows x 16 bytes, 128 bytes apart along the rows (the stride
// byte offset) and 16 R bytes apart along K (the leading byte offset); one MMA takes
// K = 8 (two core matrices along K).  Layers: [128 x 8] [8 x 64], [128 x 64] [64 x 64],
// [128 x 64] [64 x 16] (outputs 5..15 zero).
constexpr int UM_T = 128;                          // threads (and samples) per warpgroup
constexpr int UM_B1 = 0;                           // B of layer 1: 64 x 8 tf32, 2 KB
constexpr int UM_B2 = UM_B1 + 64 * 8 * 4;          // B of layer 2: 64 x 64, 16 KB
constexpr int UM_B3 = UM_B2 + 64 * 64 * 4;         // B of layer 3: 16 x 64, 4 KB
constexpr int UM_BIAS = UM_B3 + 16 * 64 * 4;       // b1[64], b2[64], b3[16] (FP32)
constexpr int UM_BAR = UM_BIAS + 1024;             // an mbarrier per warpgroup, then the TMEM base address
constexpr int UM_TMEM_SLOT = UM_BAR + 64;
constexpr int UM_ACT = UM_BAR + 1024;              // A: 128 x 64 activations per warpgroup, 32 KB each
constexpr int UM_ACT_BYTES = 128 * 64 * 4;
constexpr int UM_TMEM_COLS = 64;                   // per warpgroup
__host__ __device__ constexpr int um_smem(int wgs) { return UM_ACT + wgs * UM_ACT_BYTES; }
constexpr int UM_SMEM = um_smem(1);                // k_mlp_forward_umma: one warpgroup
constexpr int UM_NET_WGS = 2;                      // warpgroups per CTA of k_react_network_umma
constexpr int UM_NET_SMEM = um_smem(UM_NET_WGS);
static_assert(UM_ACT % 16 == 0 && UM_ACT_BYTES % 16 == 0, "matrix descriptors address 16-byte units");

__host__ __device__ constexpr unsigned um_off(int row, int k, int rows) {
  return (unsigned)((k >> 2) * (rows * 16) + (row >> 3) * 128 + (row & 7) * 16 + (k & 3) * 4);
}
// shared-memory matrix descriptor (sm100): start, leading / stride byte offsets (>> 4),
// version 1, no swizzle
__device__ __forceinline__ unsigned long long um_desc(unsigned saddr, unsigned lbo, unsigned sbo) {
  return (unsigned long long)((saddr >> 4) & 0x3FFFu) | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
         ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor, kind::tf32: D FP32, A and B TF32, both K-major, M x N
__host__ __device__ constexpr unsigned um_idesc(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(N >> 3) << 17) | ((unsigned)(M >> 4) << 24);
}
__device__ __forceinline__ void um_mma(unsigned tmem_d, unsigned long long da, unsigned long long db, unsigned idesc,
                                       unsigned accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate) : "memory");
}
// the mbarrier tracks the completion of the MMAs this thread issued before it
__device__ __forceinline__ void um_commit(unsigned bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void um_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void um_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
// barrier of warpgroup wg's 128 threads (named barrier 1 + wg, an immediate so that ptxas
// reserves only the barriers used; 0 is __syncthreads); wg is uniform over the warpgroup
static_assert(UM_NET_WGS <= 2, "named barriers 1 and 2");
__device__ __forceinline__ void um_wg_sync(int wg) {
  if (wg == 0) asm volatile("bar.sync 1, 128;" ::: "memory");
  else asm volatile("bar.sync 2, 128;" ::: "memory");
}
// the same, true when p holds on every thread of the warpgroup
__device__ __forceinline__ bool um_wg_and(int wg, bool p) {
  unsigned r;
  if (wg == 0)
    asm volatile("{\n .reg .pred a, b;\n setp.ne.b32 a, %1, 0;\n bar.red.and.pred b, 1, 128, a;\n selp.u32 %0, 1, 0, b;\n}\n"
                 : "=r"(r) : "r"((unsigned)p) : "memory");
  else
    asm volatile("{\n .reg .pred a, b;\n setp.ne.b32 a, %1, 0;\n bar.red.and.pred b, 2, 128, a;\n selp.u32 %0, 1, 0, b;\n}\n"
                 : "=r"(r) : "r"((unsigned)p) : "memory");
  return r != 0u;
}
// 16 consecutive columns of this thread's TMEM lane, waited for
__device__ __forceinline__ void um_ld16(unsigned taddr, float (&v)[16]) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr) : "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// The weights of params as the three B operands (TF32 bit patterns) and the biases;
// every thread of the CTA takes part.
__device__ __forceinline__ void um_load_weights(unsigned char* sm, const float* __restrict__ p) {
  const MlpW& W = *reinterpret_cast<const MlpW*>(p);
  for (int i = threadIdx.x; i < 64 * 8; i += blockDim.x) {       // B1 (n, k) = w1[k][n]
    const int n = i % 64, k = i / 64;
    *reinterpret_cast<unsigned*>(sm + UM_B1 + um_off(n, k, 64)) = tf32_bits(W.w1[k * MLP_H + n]);
  }
  for (int i = threadIdx.x; i < 64 * 64; i += blockDim.x) {
    const int n = i % 64, k = i / 64;
    *reinterpret_cast<unsigned*>(sm + UM_B2 + um_off(n, k, 64)) = tf32_bits(W.w2[k * MLP_H + n]);
  }
  for (int i = threadIdx.x; i < 16 * 64; i += blockDim.x) {
    const int n = i % 16, k = i / 16;
    *reinterpret_cast<unsigned*>(sm + UM_B3 + um_off(n, k, 16)) = n < MLP_OUT ? tf32_bits(W.w3[k * MLP_OUT + n]) : 0u;
  }
  float* bias = reinterpret_cast<float*>(sm + UM_BIAS);
  for (int i = threadIdx.x; i < 64; i += blockDim.x) {
    bias[i] = W.b1[i];
    bias[64 + i] = W.b2[i];
  }
  for (int i = threadIdx.x; i < 16; i += blockDim.x) bias[128 + i] = i < MLP_OUT ? W.b3[i] : 0.f;
}

// Warpgroup wg's part of a CTA: its activation tile, its mbarrier, its TMEM columns.
struct UmWg {
  int wg;
  unsigned act, bar, tmem;    // shared-memory addresses of the A tile and the mbarrier; TMEM column base
};
__device__ __forceinline__ UmWg um_wg(unsigned char* sm, int wg, unsigned tmem_base) {
  const unsigned base = smem_u32(sm);
  return UmWg{wg, base + UM_ACT + (unsigned)(wg * UM_ACT_BYTES), base + UM_BAR + 8u * (unsigned)wg,
              tmem_base + (unsigned)(wg * UM_TMEM_COLS)};
}

// One layer: D = A[:, :K] B^T over K / 8 MMAs, issued by the warpgroup's first thread;
// true once they completed (bounded wait: false after WAIT_NS, the caller gives up).
// phase: the mbarrier's parity.
template <int K, int N, int BROWS>
__device__ __forceinline__ bool um_layer(unsigned char* sm, const UmWg& g, unsigned& phase, int b_off) {
  if ((threadIdx.x & 127) == 0) {
    const unsigned base = smem_u32(sm);
    um_fence_after();
#pragma unroll
    for (int ks = 0; ks < K / 8; ks++) {
      const unsigned long long da = um_desc(g.act + (unsigned)(2 * ks) * (128 * 16), 128 * 16, 128);
      const unsigned long long db = um_desc(base + b_off + (unsigned)(2 * ks) * (BROWS * 16), BROWS * 16, 128);
      um_mma(g.tmem, da, db, um_idesc(128, N), ks > 0 ? 1u : 0u);
    }
    um_commit(g.bar);
  }
  const bool ok = mbar_wait_bounded(g.bar, phase, WAIT_NS);
  phase ^= 1u;
  um_fence_after();
  return ok;
}

// ReLU(D + bias) of this thread's row back into the A operand as TF32 (64 columns).
__device__ __forceinline__ void um_hidden(unsigned char* sm, const UmWg& g, const float* bias) {
  const int row = threadIdx.x & 127;
  const unsigned taddr = g.tmem + ((unsigned)(row & ~31) << 16);
  unsigned char* act = sm + (g.act - smem_u32(sm));
#pragma unroll
  for (int c0 = 0; c0 < 64; c0 += 16) {
    float v[16];
    um_ld16(taddr + c0, v);
#pragma unroll
    for (int c = 0; c < 16; c += 4) {
      uint4 q;
      q.x = tf32_bits(fmaxf(v[c] + bias[c0 + c], 0.f));
      q.y = tf32_bits(fmaxf(v[c + 1] + bias[c0 + c + 1], 0.f));
      q.z = tf32_bits(fmaxf(v[c + 2] + bias[c0 + c + 2], 0.f));
      q.w = tf32_bits(fmaxf(v[c + 3] + bias[c0 + c + 3], 0.f));
      *reinterpret_cast<uint4*>(act + um_off(row, c0 + c, 128)) = q;
    }
  }
}

// Forward pass of the warpgroup's 128 samples (its thread t: sample t, inputs x, outputs
// y); every thread of the warpgroup calls it.  false: an MMA did not complete within WAIT_NS.
__device__ __forceinline__ bool mlp_forward_umma(unsigned char* sm, const UmWg& g, unsigned& phase, const float* x,
                                                 float* y) {
  const int row = threadIdx.x & 127;
  const float* bias = reinterpret_cast<const float*>(sm + UM_BIAS);
  unsigned char* act = sm + (g.act - smem_u32(sm));
  {
    uint4 a, b;
    a.x = tf32_bits(x[0]); a.y = tf32_bits(x[1]); a.z = tf32_bits(x[2]); a.w = tf32_bits(x[3]);
    b.x = tf32_bits(x[4]); b.y = tf32_bits(x[5]); b.z = tf32_bits(x[6]); b.w = tf32_bits(x[7]);
    *reinterpret_cast<uint4*>(act + um_off(row, 0, 128)) = a;
    *reinterpret_cast<uint4*>(act + um_off(row, 4, 128)) = b;
  }
  bool ok = true;
  // before each layer: every thread's rows written (generic proxy -> async proxy) and its
  // TMEM reads of the previous layer done
  um_fence_before();
  fence_proxy_async();
  um_wg_sync(g.wg);
  ok = um_layer<MLP_IN, 64, 64>(sm, g, phase, UM_B1) && ok;
  if (ok) um_hidden(sm, g, bias);
  um_fence_before();
  fence_proxy_async();
  ok = um_wg_and(g.wg, ok);
  if (ok) ok = um_layer<MLP_H, 64, 64>(sm, g, phase, UM_B2);
  if (ok) um_hidden(sm, g, bias + 64);
  um_fence_before();
  fence_proxy_async();
  ok = um_wg_and(g.wg, ok);
  if (ok) ok = um_layer<MLP_H, 16, 16>(sm, g, phase, UM_B3);
  if (ok) {
    float v[16];
    um_ld16(g.tmem + ((unsigned)(row & ~31) << 16), v);
#pragma unroll
    for (int q = 0; q < MLP_OUT; q++) y[q] = v[q] + bias[128 + q];
  }
  return um_wg_and(g.wg, ok);
}

// TMEM for the CTA (warp 0 allocates and, at the end, frees cols columns: a power of two
// from 32 to 512).
__device__ __forceinline__ unsigned um_tmem_alloc(unsigned char* sm, unsigned cols) {
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(sm + UM_TMEM_SLOT)), "r"(cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  um_fence_before();
  __syncthreads();
  um_fence_after();
  return *reinterpret_cast<volatile unsigned*>(sm + UM_TMEM_SLOT);
}
__device__ __forceinline__ void um_tmem_free(unsigned tmem, unsigned cols) {
  um_fence_before();
  __syncthreads();
  um_fence_after();
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols) : "memory");
}

// Forward passes for checks on the tcgen05 path (one warpgroup per CTA): y[n][5] of
// x[n][8]; err[0] |= 1 when an MMA did not complete in time (the CTA then waits once more
// for it, frees its TMEM and stops).
__global__ void __launch_bounds__(UM_T) k_mlp_forward_umma(const float* __restrict__ params,
                                                           const float* __restrict__ x, long long n,
                                                           float* __restrict__ y, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char um_sm[];
  um_load_weights(um_sm, params);
  if (threadIdx.x == 0) {
    mbar_init(smem_u32(um_sm + UM_BAR), 1);
    fence_mbar_init();
  }
  fence_proxy_async();
  __syncthreads();
  const unsigned tmem = um_tmem_alloc(um_sm, UM_TMEM_COLS);
  const UmWg g = um_wg(um_sm, 0, tmem);
  unsigned phase = 0;
  for (long long t0 = (long long)blockIdx.x * UM_T; t0 < n; t0 += (long long)gridDim.x * UM_T) {
    const long long i = t0 + threadIdx.x;
    float xi[MLP_IN], yi[MLP_OUT];
#pragma unroll
    for (int j = 0; j < MLP_IN; j++) xi[j] = i < n ? x[i * MLP_IN + j] : 0.f;
    if (!mlp_forward_umma(um_sm, g, phase, xi, yi)) {
      // a late MMA may still write TMEM: wait for it once more (bounded) before freeing
      if (threadIdx.x == 0) {
        mbar_wait_bounded(g.bar, phase ^ 1u, WAIT_NS);
        atomicOr(err, 1);
      }
      break;
    }
    if (i < n)
#pragma unroll
      for (int j = 0; j < MLP_OUT; j++) y[i * MLP_OUT + j] = yi[j];
  }
  um_tmem_free(tmem, UM_TMEM_COLS);
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

// ---- deployment.  With the surrogate on (RealDesc::sur) the voxel kernel still applies
// the explicit increment dJ_s (buffer_dj) on a reaction step and also classifies every
// voxel (rx_classify): near equilibrium (the explicit increment stands), network (an
// eligible domain away from equilibrium) or plain integrator (a stiff domain).  After the
// boundary kernels, k_react_surrogate scans the class bytes; the voxels of the last two
// classes receive the correction (increment - dJ_s) for every bound species s and
// (sum dJ_s - sum increments) for Ca, from the old state: species fixed in the voxel's
// domain and, with -f, Ca on the outer faces keep the values the voxel kernel gave them.
//
// k_react_surrogate: a CTA takes MLP_DEPLOY_SPAN consecutive voxels of one realisation
// at a time; a thread reads the class bytes of MLP_SCAN_VPT consecutive voxels (a warp
// reads 256 contiguous bytes) and lists the voxels to correct (offsets within the CTA's
// span), network and plain-integrator voxels apart, queued as tiles of 32: network tiles
// for k_react_network (tensor cores), plain tiles for k_react_plain (FP64).  Both
// spread every list's tiles over all their warps: stiff domains are spatially clustered,
// and one CTA alone would run their integrations one after the other.  counters[0] +=
// voxels with buffers, counters[1] += voxels the network ran for, counters[2] += voxels
// that took the plain integrator.
constexpr int MLP_DEPLOY_T = 256;
constexpr int MLP_SCAN_VPT = 8;          // class bytes per thread and iteration
constexpr int MLP_DEPLOY_ITER = 8;
constexpr long long MLP_DEPLOY_SPAN = (long long)MLP_SCAN_VPT * MLP_DEPLOY_T * MLP_DEPLOY_ITER;   // voxels per CTA
static_assert(MLP_DEPLOY_SPAN <= 65536, "list entries are 16-bit offsets within a CTA's span");
constexpr int MLP_RX_NS = MLP_SLOTS + 1; // species the reaction touches: Ca and slots 1..5
constexpr size_t MLP_NETWORK_SMEM = sizeof(MlpTC) + sizeof(float) * (size_t)MLP_TC_STAGE * (MLP_DEPLOY_T / 32);

// The reaction constants of one domain (block- or warp-shared).
struct RxDom {
  RxConst k;
  float4 rk[MLP_RX_NS];                  // RealDesc::rk of the bound species (buffer_dj)
  float base[MLP_RX_NS], qunit[MLP_RX_NS], qinv[MLP_RX_NS];   // RealDesc::fbase / qunit / qinv
  unsigned store;                        // species corrected: Ca and the bound species, minus the fixed ones
};

__device__ __forceinline__ void rx_dom_fill(const RealDesc& D, int d, RxDom& S) {
  const int dd = d < D.nd ? d : 0;
  S.k = rx_const(D, dd);
  unsigned ld = 0;
  for (int q = 0; q < MLP_SLOTS; q++)
    if (S.k.tot[q] > 0.f) ld |= 2u << q;
  for (int s = 0; s < MLP_RX_NS; s++) {
    S.rk[s] = D.rk[dd][s];
    S.base[s] = D.fbase[dd][s];
    S.qunit[s] = D.qunit[dd][s];
    S.qinv[s] = D.qinv[dd][s];
  }
  S.store = (d < D.nd && ld) ? (ld | 1u) & ~(unsigned)D.fixed_mask[dd] : 0u;
}

// Deviation of species s from its stored form (fixed-point for the species in FQ & fqs).
template <unsigned FQ>
__device__ __forceinline__ float rx_dev(const RxDom& K, int s, float stored, unsigned fqs) {
  return ((FQ & fqs) >> s & 1u) ? q_value(stored, K.qunit[s]) : stored;
}

// Stored new value of species s plus an increment.
template <unsigned FQ>
__device__ __forceinline__ float rx_add(const RxDom& K, int s, float stored, float inc, unsigned fqs) {
  return ((FQ & fqs) >> s & 1u) ? q_add(stored, inc, K.qinv[s]) : __fadd_rn(stored, inc);
}

// The plain integrator's increments (the fallback), FP64, rounded to FP32.
// rx_plain for the slots of MASK only (known at compile time, so the slots a domain lacks
// issue no instructions); the same operations in the same order as rx_plain.
template <unsigned MASK>
__device__ __forceinline__ void rx_plain_mask(const RxConst& k, int n, double h, double c, const double* b0, double& dc,
                                              double* db) {
  double b[MLP_SLOTS];
#pragma unroll
  for (int q = 0; q < MLP_SLOTS; q++) b[q] = b0[q];
  double cc = c;
  for (int i = 0; i < n; i++) {
    double g[MLP_SLOTS], sg = 0.0;
#pragma unroll
    for (int q = 0; q < MLP_SLOTS; q++) {
      g[q] = 0.0;
      if (!(MASK >> q & 1u)) continue;
      g[q] = rx_g<double>(k, q, cc, b[q]);
      sg += g[q];
    }
#pragma unroll
    for (int q = 0; q < MLP_SLOTS; q++)
      if (MASK >> q & 1u) b[q] += h * g[q];
    cc -= h * sg;
  }
#pragma unroll
  for (int q = 0; q < MLP_SLOTS; q++) db[q] = b[q] - b0[q];
  dc = cc - c;
}

// The plain integrator's increments (the fallback), FP64, rounded to FP32: the slot sets of
// the reference model's domains (the jSR's two buffers, the cytosol's four, the nSR's one)
// take compiled forms, others the general loop.
__device__ __forceinline__ void rx_fallback(const RxConst& kc, int n, double dt, float c, const float* b, float& dc,
                                            float* db) {
  double bd[MLP_SLOTS], dbd[MLP_SLOTS], dcd;
  unsigned mask = 0;
#pragma unroll
  for (int q = 0; q < MLP_SLOTS; q++) {
    bd[q] = b[q];
    if (kc.tot[q] > 0.f) mask |= 1u << q;
  }
  switch (mask) {
    case 0x03u: rx_plain_mask<0x03u>(kc, n, dt, (double)c, bd, dcd, dbd); break;
    case 0x0Fu: rx_plain_mask<0x0Fu>(kc, n, dt, (double)c, bd, dcd, dbd); break;
    case 0x01u: rx_plain_mask<0x01u>(kc, n, dt, (double)c, bd, dcd, dbd); break;
    default: rx_plain(kc, n, dt, (double)c, bd, dcd, dbd);
  }
#pragma unroll
  for (int q = 0; q < MLP_SLOTS; q++) db[q] = (float)dbd[q];
  dc = (float)dcd;
}

__device__ __forceinline__ bool rx_on_face(const RealDesc& D, int x, int p) {
  const int c1 = p / D.nz, c2 = p - c1 * D.nz;
  return x == 0 || x == D.nx - 1 || c1 == 0 || c1 == D.ny - 1 || c2 == 0 || c2 == D.nz - 1;
}

// One voxel's old state: deviations dev[] (Ca and the slots' species) and the values
// c = Ca, b[q] (0 for absent slots).
template <unsigned FQ>
__device__ __forceinline__ void rx_load_old(const RxDom& K, const float* const* uo, long long v, unsigned fqs,
                                            float* dev, float& c, float* b) {
  dev[0] = __ldg(uo[0] + v);
  c = __fadd_rn(K.base[0], dev[0]);
#pragma unroll
  for (int q = 0; q < MLP_SLOTS; q++) {
    dev[q + 1] = 0.f;
    b[q] = 0.f;
    if (K.k.tot[q] > 0.f) {
      dev[q + 1] = rx_dev<FQ>(K, q + 1, __ldg(uo[q + 1] + v), fqs);
      b[q] = __fadd_rn(K.base[q + 1], dev[q + 1]);
    }
  }
}

// Replace the explicit increments the voxel kernel applied to voxel v by the surrogate's
// (db[], dc): the explicit ones are recomputed from the same deviations and constants,
// so they are the ones that were added.
template <unsigned FQ>
__device__ __forceinline__ void rx_correct(const RxDom& K, const RealDesc& D, float* const* un, long long v,
                                           unsigned fqs, const float* dev, float c, const float* db, float dc) {
  float sdj = 0.f;
#pragma unroll
  for (int q = 0; q < MLP_SLOTS; q++) {
    if (K.k.tot[q] <= 0.f) continue;
    const float4 k = K.rk[q + 1];
    const float dJ = buffer_dj(k.x, k.y, k.z, k.w, dev[q + 1], dev[0], c);
    sdj = __fadd_rn(sdj, dJ);
    if (K.store >> (q + 1) & 1u) un[q + 1][v] = rx_add<FQ>(K, q + 1, un[q + 1][v], __fsub_rn(db[q], dJ), fqs);
  }
  if (K.store & 1u) {
    const int vi = (int)v, xq = vi / D.P;
    if (!(D.dirichlet && rx_on_face(D, xq, vi - xq * D.P))) un[0][v] = __fadd_rn(un[0][v], __fadd_rn(sdj, dc));
  }
}

// Reaction step with the surrogate on, on the fast reactions (the steps the voxel kernel
// classifies).
__device__ __forceinline__ bool rx_active(const RealDesc& D, const RealCtl& C) {
  return !C.stopped && D.sur && step_info(D, C.step + 1).react_fast;
}

// list / counts: per segment (seg = r * chunks + chunk) MLP_DEPLOY_SPAN entries: the
// network voxels from the front, the plain-integrator voxels from the back;
// counts[2 seg] / counts[2 seg + 1] their numbers, written on reaction steps.  tiles /
// queue[0]: the network tiles of 32 listed voxels (seg << MLP_TILE_BITS | tile within
// the list) and their number; tiles + MLP_PLAIN_TILES / queue[2]: the same for the plain
// integrator.  k_epilogue empties the queues for the next step.
constexpr int MLP_TILE_BITS = 9;
static_assert(MLP_DEPLOY_SPAN / 32 <= (1 << MLP_TILE_BITS), "tile index field");

// Persistent: CTA b takes the segments seg = b, b + gridDim.x, ... (seg = r * chunks +
// chunk, chunk = the CTA-sized span of realisation r); on a step with no reaction step
// anywhere the CTAs return after one parallel check of the realisations.  tiles_plain =
// the plain-integrator half of the tile array.
__global__ void __launch_bounds__(MLP_DEPLOY_T) k_react_surrogate(const RealDesc* __restrict__ descs,
                                                                  const RealCtl* __restrict__ ctl, int chunks,
                                                                  int nreal, unsigned short* __restrict__ list,
                                                                  unsigned* __restrict__ counts,
                                                                  unsigned* __restrict__ tiles,
                                                                  unsigned* __restrict__ tiles_plain,
                                                                  unsigned* __restrict__ queue,
                                                                  unsigned long long* __restrict__ counters) {
  __shared__ unsigned s_vox, s_list[2], s_tile0[2];
  bool any = false;
  for (int r = threadIdx.x; r < nreal; r += MLP_DEPLOY_T) any = any || rx_active(descs[r], ctl[r]);
  if (!__syncthreads_or(any)) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long nseg = (long long)chunks * nreal;
  for (long long seg = blockIdx.x; seg < nseg; seg += gridDim.x) {
    const int r = (int)(seg / chunks);
    const RealDesc& D = descs[r];
    if (!rx_active(D, ctl[r])) continue;                // uniform over the block
    const long long nvox = (long long)D.nx * D.P;
    const long long vb0 = (seg - (long long)r * chunks) * MLP_DEPLOY_SPAN;
    if (vb0 >= nvox) {                                  // uniform over the block
      if (threadIdx.x == 0) counts[2 * seg] = counts[2 * seg + 1] = 0;
      continue;
    }
    if (threadIdx.x == 0) { s_vox = 0; s_list[0] = s_list[1] = 0; }
    __syncthreads();
    unsigned short* seg_list = list + seg * MLP_DEPLOY_SPAN;
    const unsigned char* __restrict__ cls = D.rx_class;
    unsigned n_vox = 0;
    for (int it = 0; it < MLP_DEPLOY_ITER; it++) {
      const long long w0 = vb0 + (long long)it * MLP_SCAN_VPT * MLP_DEPLOY_T + (long long)warp * MLP_SCAN_VPT * 32;
      if (w0 >= nvox) break;                             // warp-uniform
      const long long v = w0 + MLP_SCAN_VPT * lane;
      uint2 w = make_uint2(0u, 0u);
      if (v < nvox) w = __ldg(reinterpret_cast<const uint2*>(cls + v));
      unsigned m[2] = {0u, 0u};                          // network, plain integrator
#pragma unroll
      for (int j = 0; j < MLP_SCAN_VPT; j++) {
        const unsigned c = ((j < 4 ? w.x : w.y) >> (8 * (j & 3))) & 0xffu;
        if (c) n_vox++;
        if (c == RX_CLASS_NETWORK) m[0] |= 1u << j;
        if (c == RX_CLASS_PLAIN) m[1] |= 1u << j;
      }
      const unsigned off = (unsigned)(v - vb0);
#pragma unroll
      for (int k = 0; k < 2; k++) {
        if (!__any_sync(0xffffffffu, m[k] != 0u)) continue;
        // a warp-wide prefix sum of the counts, one shared atomic
        const unsigned cnt = __popc(m[k]);
        unsigned incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += t;
        }
        unsigned base = 0;
        if (lane == 31) base = atomicAdd(&s_list[k], incl);
        unsigned pos = __shfl_sync(0xffffffffu, base, 31) + incl - cnt;
#pragma unroll
        for (int j = 0; j < MLP_SCAN_VPT; j++) {
          if (!(m[k] >> j & 1u)) continue;
          seg_list[k == 0 ? pos : MLP_DEPLOY_SPAN - 1 - pos] = (unsigned short)(off + j);
          pos++;
        }
      }
    }
    if (n_vox) atomicAdd(&s_vox, n_vox);
    __syncthreads();
    const unsigned nt0 = (s_list[0] + 31u) / 32u, nt1 = (s_list[1] + 31u) / 32u;
    if (threadIdx.x == 0) {
      counts[2 * seg] = s_list[0];
      counts[2 * seg + 1] = s_list[1];
      if (nt0) s_tile0[0] = atomicAdd(&queue[0], nt0);
      if (nt1) s_tile0[1] = atomicAdd(&queue[2], nt1);
      if (s_vox) atomicAdd(&counters[0], (unsigned long long)s_vox);
    }
    __syncthreads();
    for (unsigned j = threadIdx.x; j < nt0 + nt1; j += MLP_DEPLOY_T) {
      if (j < nt0) tiles[s_tile0[0] + j] = (unsigned)seg << MLP_TILE_BITS | j;
      else tiles_plain[s_tile0[1] + (j - nt0)] = (unsigned)seg << MLP_TILE_BITS | (j - nt0);
    }
    __syncthreads();                                     // s_* are reused by the next segment
  }
}

// A warp's cache of one realisation (its domain constants and field pointers), filled by
// its lanes 0..7 and 8..13 when the realisation changes.
struct RxWarpCache {
  RxDom dom[8];
  const float* uo[MLP_RX_NS];
  float* un[MLP_RX_NS];
};
__device__ __forceinline__ void rx_cache_fill(const RealDesc& D, const RealCtl& C, RxWarpCache& W, int lane) {
  __syncwarp();
  if (lane < 8) {
    rx_dom_fill(D, lane, W.dom[lane]);
  } else if (lane < 8 + MLP_RX_NS) {
    const int t = lane - 8;
    const unsigned cur = C.cur_mask[C.step & 1];
    W.uo[t] = t < D.ns ? D.u[(cur >> t) & 1u][t] : nullptr;
    W.un[t] = t < D.ns ? D.u[((cur >> t) & 1u) ^ 1u][t] : nullptr;
  }
  __syncwarp();
}

// One tile's chain of dependent loads (tile, list entry, domain byte); back = the entry
// counts from the back of the list (plain-integrator voxels).
struct RxTile {
  long long v;
  int r, d;
  bool have;
};
__device__ __forceinline__ RxTile rx_fetch_tile(const RealDesc* __restrict__ descs,
                                                const unsigned short* __restrict__ list,
                                                const unsigned* __restrict__ counts, unsigned td, int chunks,
                                                int back, int lane) {
  RxTile f;
  const long long seg = td >> MLP_TILE_BITS;
  const unsigned i = (td & ((1u << MLP_TILE_BITS) - 1u)) * 32u + lane;
  f.r = (int)(seg / chunks);
  f.have = i < counts[2 * seg + back];
  const unsigned e = f.have ? list[seg * MLP_DEPLOY_SPAN + (back ? MLP_DEPLOY_SPAN - 1 - i : i)] : 0u;
  f.v = (seg - (long long)f.r * chunks) * MLP_DEPLOY_SPAN + e;
  f.d = f.have ? (descs[f.r].dom[f.v] & DOMAIN_BITS) : 0;
  return f;
}


// The network voxels that k_react_surrogate listed, in tiles of 32 on the tensor cores (a
// rejected output takes the plain integrator), each corrected from the old state
// (rx_correct).  Persistent CTAs: warp w of the grid takes a contiguous range of the
// queued tiles (tiles of one list are queued together, so a warp's realisation rarely
// changes); a CTA without a tile returns before it loads the weights.  The next tile's
// index chain is fetched while a tile runs.  chunks = the segments per realisation.
template <unsigned FQ>
__global__ void __launch_bounds__(MLP_DEPLOY_T, 2) k_react_network(const RealDesc* __restrict__ descs,
                                                                   const RealCtl* __restrict__ ctl,
                                                                   const float* __restrict__ params, float tol,
                                                                   const unsigned short* __restrict__ list,
                                                                   const unsigned* __restrict__ counts,
                                                                   const unsigned* __restrict__ tiles,
                                                                   unsigned* __restrict__ queue, int chunks,
                                                                   unsigned long long* __restrict__ counters) {
  extern __shared__ __align__(16) float dsm[];
  MlpTC& T = *reinterpret_cast<MlpTC*>(dsm);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* stage = dsm + sizeof(MlpTC) / sizeof(float) + warp * MLP_TC_STAGE;
  __shared__ RxWarpCache s_wc[MLP_DEPLOY_T / 32];
  __shared__ unsigned s_net, s_fall, s_total;
  if (threadIdx.x == 0) { s_total = queue[0]; s_net = 0; s_fall = 0; }
  __syncthreads();
  const unsigned total = s_total;
  const unsigned nw = gridDim.x * (MLP_DEPLOY_T / 32), per = (total + nw - 1) / nw;
  if (blockIdx.x * (MLP_DEPLOY_T / 32) * per < total) {  // uniform over the block
    mlp_tc_load(T, params);
    __syncthreads();
    RxWarpCache& W = s_wc[warp];
    const unsigned t_lo = (blockIdx.x * (MLP_DEPLOY_T / 32) + warp) * per, t_hi = min(total, t_lo + per);
    unsigned n_net = 0, n_fall = 0;
    int rc = -1;                                         // realisation whose constants are cached
    RxTile nx{};
    if (t_lo < t_hi) nx = rx_fetch_tile(descs, list, counts, tiles[t_lo], chunks, 0, lane);
    for (unsigned tw = t_lo; tw < t_hi; tw++) {
      const RxTile cu = nx;
      if (tw + 1 < t_hi) nx = rx_fetch_tile(descs, list, counts, tiles[tw + 1], chunks, 0, lane);
      const RealDesc& D = descs[cu.r];
      if (cu.r != rc) {                                  // warp-uniform
        rx_cache_fill(D, ctl[cu.r], W, lane);
        rc = cu.r;
      }
      const float dtr = (float)(D.dt * D.reaction_substep);
      const unsigned fqs = D.fixq;
      const RxDom& K = W.dom[cu.d];
      float dev[MLP_RX_NS], c = 0.f, b[MLP_SLOTS], x[MLP_IN], t[MLP_OUT];
#pragma unroll
      for (int i = 0; i < MLP_IN; i++) x[i] = 0.f;
#pragma unroll
      for (int q = 0; q < MLP_SLOTS; q++) b[q] = 0.f;
      if (cu.have) {
        rx_load_old<FQ>(K, W.uo, cu.v, fqs, dev, c, b);
        rx_features(K.k, cu.d, dtr, c, b, x);
      }
      mlp_forward_tc(T, stage, x, t);
      if (cu.have) {
        float dc, db[MLP_SLOTS];
        n_net++;
        if (!rx_apply_output(K.k, dtr, c, b, t, tol, dc, db)) {
          n_fall++;
          rx_fallback(K.k, D.reaction_substep, D.dt, c, b, dc, db);
        }
        rx_correct<FQ>(K, D, W.un, cu.v, fqs, dev, c, db, dc);
      }
    }
    if (n_net) atomicAdd(&s_net, n_net);
    if (n_fall) atomicAdd(&s_fall, n_fall);
    __syncthreads();
    if (threadIdx.x == 0) {
      if (s_net) atomicAdd(&counters[1], (unsigned long long)s_net);
      if (s_fall) atomicAdd(&counters[2], (unsigned long long)s_fall);
    }
  }
}

// k_react_network on the 5th-generation tensor cores: a CTA of UM_NET_WGS warpgroups
// (4 warps each) shares one copy of the weights; a warpgroup takes groups of four queued
// tiles, one per warp (each warp fetches its tile's voxels and caches its realisation's
// constants as in k_react_network), and runs the network for the group's 128 voxels as one
// tcgen05 MMA chain per layer (mlp_forward_umma, synchronised within the warpgroup only);
// rejected outputs take the plain integrator.  Persistent CTAs: CTA b takes a contiguous
// range of the groups, dealt to its warpgroups in turn.  An MMA that does not complete
// within WAIT_NS sets ERR_TIMEOUT in err and stops the warpgroup (after a second bounded
// wait for it); the CTA then frees its TMEM.
template <unsigned FQ>
__global__ void __launch_bounds__(UM_T * UM_NET_WGS, 2) k_react_network_umma(const RealDesc* __restrict__ descs,
                                                                          const RealCtl* __restrict__ ctl,
                                                                          const float* __restrict__ params, float tol,
                                                                          const unsigned short* __restrict__ list,
                                                                          const unsigned* __restrict__ counts,
                                                                          const unsigned* __restrict__ tiles,
                                                                          unsigned* __restrict__ queue, int chunks,
                                                                          unsigned long long* __restrict__ counters,
                                                                          int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char um_sm[];
  __shared__ RxWarpCache s_wc[UM_NET_WGS * UM_T / 32];
  __shared__ unsigned s_net, s_fall, s_total;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wi = warp & 3, wg = warp >> 2;
  if (threadIdx.x == 0) { s_total = queue[0]; s_net = 0; s_fall = 0; }
  __syncthreads();
  const unsigned total = s_total, groups = (total + 3u) / 4u;
  const unsigned per = (groups + gridDim.x - 1) / gridDim.x;
  const unsigned g_lo = blockIdx.x * per, g_hi = min(groups, g_lo + per);
  if (g_lo < g_hi) {                                     // uniform over the block
    um_load_weights(um_sm, params);
    if (threadIdx.x == 0) {
      for (int w = 0; w < UM_NET_WGS; w++) mbar_init(smem_u32(um_sm + UM_BAR + 8 * w), 1);
      fence_mbar_init();
    }
    fence_proxy_async();
    __syncthreads();
    const unsigned tmem = um_tmem_alloc(um_sm, UM_NET_WGS * UM_TMEM_COLS);
    const UmWg G = um_wg(um_sm, wg, tmem);
    unsigned phase = 0, n_net = 0, n_fall = 0;
    RxWarpCache& W = s_wc[warp];
    int rc = -1;                                         // realisation whose constants this warp caches
    RxTile nx{};
    const unsigned g0 = g_lo + (unsigned)wg;
    if (g0 < g_hi && 4 * g0 + wi < total) nx = rx_fetch_tile(descs, list, counts, tiles[4 * g0 + wi], chunks, 0, lane);
    for (unsigned g = g0; g < g_hi; g += UM_NET_WGS) {  // uniform over the warpgroup
      const bool tile = 4 * g + wi < total;              // warp-uniform
      RxTile cu = nx;
      if (!tile) cu.have = false;
      const unsigned gn = g + UM_NET_WGS;
      if (gn < g_hi && 4 * gn + wi < total)
        nx = rx_fetch_tile(descs, list, counts, tiles[4 * gn + wi], chunks, 0, lane);
      float dev[MLP_RX_NS], c = 0.f, b[MLP_SLOTS], x[MLP_IN], t[MLP_OUT];
#pragma unroll
      for (int i = 0; i < MLP_IN; i++) x[i] = 0.f;
#pragma unroll
      for (int q = 0; q < MLP_SLOTS; q++) b[q] = 0.f;
      const RealDesc& D = descs[tile ? cu.r : 0];
      if (tile && cu.r != rc) {                          // warp-uniform
        rx_cache_fill(D, ctl[cu.r], W, lane);
        rc = cu.r;
      }
      const float dtr = (float)(D.dt * D.reaction_substep);
      const unsigned fqs = D.fixq;
      const RxDom& K = W.dom[cu.d];
      if (cu.have) {
        rx_load_old<FQ>(K, W.uo, cu.v, fqs, dev, c, b);
        rx_features(K.k, cu.d, dtr, c, b, x);
      }
      if (!mlp_forward_umma(um_sm, G, phase, x, t)) {
        if ((threadIdx.x & 127) == 0) {
          mbar_wait_bounded(G.bar, phase ^ 1u, WAIT_NS);
          atomicOr(err, ERR_TIMEOUT);
        }
        break;
      }
      if (cu.have) {
        float dc, db[MLP_SLOTS];
        n_net++;
        if (!rx_apply_output(K.k, dtr, c, b, t, tol, dc, db)) {
          n_fall++;
          rx_fallback(K.k, D.reaction_substep, D.dt, c, b, dc, db);
        }
        rx_correct<FQ>(K, D, W.un, cu.v, fqs, dev, c, db, dc);
      }
    }
    um_tmem_free(tmem, UM_NET_WGS * UM_TMEM_COLS);
    if (n_net) atomicAdd(&s_net, n_net);
    if (n_fall) atomicAdd(&s_fall, n_fall);
    __syncthreads();
    if (threadIdx.x == 0) {
      if (s_net) atomicAdd(&counters[1], (unsigned long long)s_net);
      if (s_fall) atomicAdd(&counters[2], (unsigned long long)s_fall);
    }
  }
}

// The plain-integrator voxels that k_react_surrogate listed (stiff domains), one per lane
// (FP64), each corrected from the old state.  No weights and no activation tiles: the
// CTAs hold a few KB of shared memory, so many more warps per SM hide the latency of
// the voxels' dependent loads than the network kernel can.  Same tile distribution as
// k_react_network, over the queue q (q[0] tiles).
template <unsigned FQ>
__global__ void __launch_bounds__(MLP_DEPLOY_T, 4) k_react_plain(const RealDesc* __restrict__ descs,
                                                              const RealCtl* __restrict__ ctl,
                                                              const unsigned short* __restrict__ list,
                                                              const unsigned* __restrict__ counts,
                                                              const unsigned* __restrict__ tiles,
                                                              unsigned* __restrict__ q, int chunks,
                                                              unsigned long long* __restrict__ counters) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ RxWarpCache s_wc[MLP_DEPLOY_T / 32];
  __shared__ unsigned s_fall, s_total;
  if (threadIdx.x == 0) { s_total = q[0]; s_fall = 0; }
  __syncthreads();
  const unsigned total = s_total;
  const unsigned nw = gridDim.x * (MLP_DEPLOY_T / 32), per = (total + nw - 1) / nw;
  if (blockIdx.x * (MLP_DEPLOY_T / 32) * per < total) {  // uniform over the block
    RxWarpCache& W = s_wc[warp];
    const unsigned t_lo = (blockIdx.x * (MLP_DEPLOY_T / 32) + warp) * per, t_hi = min(total, t_lo + per);
    unsigned n_fall = 0;
    int rc = -1;
    RxTile nx{};
    if (t_lo < t_hi) nx = rx_fetch_tile(descs, list, counts, tiles[t_lo], chunks, 1, lane);
    for (unsigned tw = t_lo; tw < t_hi; tw++) {
      const RxTile cu = nx;
      if (tw + 1 < t_hi) nx = rx_fetch_tile(descs, list, counts, tiles[tw + 1], chunks, 1, lane);
      const RealDesc& D = descs[cu.r];
      if (cu.r != rc) {                                  // warp-uniform
        rx_cache_fill(D, ctl[cu.r], W, lane);
        rc = cu.r;
      }
      if (cu.have) {
        const RxDom& K = W.dom[cu.d];
        const unsigned fqs = D.fixq;
        float dev[MLP_RX_NS], c, b[MLP_SLOTS], dc, db[MLP_SLOTS];
        rx_load_old<FQ>(K, W.uo, cu.v, fqs, dev, c, b);
        n_fall++;
        rx_fallback(K.k, D.reaction_substep, D.dt, c, b, dc, db);
        rx_correct<FQ>(K, D, W.un, cu.v, fqs, dev, c, db, dc);
      }
    }
    if (n_fall) atomicAdd(&s_fall, n_fall);
    __syncthreads();
    if (threadIdx.x == 0 && s_fall) atomicAdd(&counters[2], (unsigned long long)s_fall);
  }
}

// Forward passes for checks: y[n][5] of x[n][8], FP32 (tc = 0) or tensor cores (tc = 1,
// the tiles of k_react_network).
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
constexpr size_t MLP_FORWARD_SMEM = MLP_NETWORK_SMEM + sizeof(MlpW);

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
