// csp_kernels.cuh -- the step kernels.
//
//   k_voxels_direct   one thread per voxel: diffusion of every species due this step,
//                     buffer reactions, fixed values (species.c:1501-1702, 1037-1121).
//   k_voxels_staged   (csp_staged.cuh) the same arithmetic over x-marching tiles staged
//                     in shared memory by bulk TMA copies.
//   k_boundaries      channel gating + boundary flux scatter + step epilogue
//                     (species.c:1704-1957, boundaryfluxes.c:295-359, species.c:3384-3488).
//   k_reduce_*        per (domain, species) min / max / FP64 sum (species.c:2785-2880).
#pragma once
#include <cfloat>

#include "csp_device.cuh"

namespace csp {

// Device error word bits.
enum : int { ERR_BOUNDS = 1, ERR_TIMEOUT = 2 };

// ---- per-voxel arithmetic, with explicit rounding (no contraction differences between
// the code paths that share it) ----

// Uniform neighbourhood (all six neighbours in the voxel's domain): the reference's fast
// path c*(sum_n u_n - 6u) + u (kernel_generic.cpp:529-533) in the form
// u + c*sum_axes((u_- + u_+) - 2u); out-of-box neighbours carry u_n = u and add nothing.
__device__ __forceinline__ float diffuse_uniform(float c, float u, const float (&un)[6]) {
  // per axis (u_- + u_+) - 2u: exact zero in a uniform field, one rounding per axis
  const float az = __fmaf_rn(-2.f, u, __fadd_rn(un[0], un[1]));
  const float ay = __fmaf_rn(-2.f, u, __fadd_rn(un[2], un[3]));
  const float ax = __fmaf_rn(-2.f, u, __fadd_rn(un[4], un[5]));
  return __fmaf_rn(c, __fadd_rn(__fadd_rn(az, ay), ax), u);
}

// General neighbourhood: u + sum_n c_n*(u_n - u) with c_n = c[d][d_n] (species.c:1572-1611,
// 1282-1498).
__device__ __forceinline__ float diffuse_coef6(const float (&c6)[6], float u, const float (&un)[6]) {
  float a = 0.f;
#pragma unroll
  for (int k = 0; k < 6; k++) a = __fmaf_rn(c6[k], __fsub_rn(un[k], u), a);
  return __fadd_rn(u, a);
}
__device__ __forceinline__ float diffuse_general(const float* c, const int (&dn)[6], float u, const float (&un)[6]) {
  const float c6[6] = {c[dn[0]], c[dn[1]], c[dn[2]], c[dn[3]], c[dn[4]], c[dn[5]]};
  return diffuse_coef6(c6, u, un);
}

// ---- two FP32 lanes per instruction (sm_100 add/sub/mul/fma .rn.f32x2): every lane is
// rounded exactly as the scalar __fadd_rn / __fsub_rn / __fmul_rn / __fmaf_rn ----
struct F2 {
  unsigned long long v;
};
__device__ __forceinline__ F2 f2(float lo, float hi) {
  F2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2_split(F2 a, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
}
__device__ __forceinline__ F2 f2_add(F2 a, F2 b) {
  F2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 f2_sub(F2 a, F2 b) {
  F2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 f2_mul(F2 a, F2 b) {
  F2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ F2 f2_fma(F2 a, F2 b, F2 c) {
  F2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return r;
}

__device__ __forceinline__ F2 f2_abs(F2 a) {
  F2 r;
  r.v = a.v & 0x7fffffff7fffffffull;
  return r;
}

// diffuse_uniform on two voxels: zs = z- + z+, ys, xs the other axis sums.
__device__ __forceinline__ F2 diffuse_uniform2(F2 c, F2 m2, F2 u, F2 zs, F2 ys, F2 xs) {
  const F2 az = f2_fma(m2, u, zs), ay = f2_fma(m2, u, ys), ax = f2_fma(m2, u, xs);
  return f2_fma(c, f2_add(f2_add(az, ay), ax), u);
}

// dt_r * J for one buffer, J = k_on (tot - B) Ca - k_off B (kernel_generic.cpp:495-507), from
// the deviations dB, dCa of the stored fields (B = base_B + dB, Ca = base_Ca + dCa, ca =
// the reconstructed Ca): J = J(base) + k_on (tot - base_B) dCa - dB (k_on Ca + k_off), so
// no term is the difference of two large near-equal products.  nkon = -dt_r k_on,
// nkoff = -dt_r k_off, a = dt_r k_on (tot - base_B), j0 = dt_r J(base).
__device__ __forceinline__ float buffer_dj(float nkon, float nkoff, float a, float j0, float db, float dca, float ca) {
  return __fmaf_rn(db, __fmaf_rn(nkon, ca, nkoff), __fmaf_rn(a, dca, j0));
}

// buffer_dj on two voxels.
__device__ __forceinline__ F2 buffer_dj2(F2 nkon, F2 nkoff, F2 a, F2 j0, F2 db, F2 dca, F2 ca) {
  return f2_fma(db, f2_fma(nkon, ca, nkoff), f2_fma(a, dca, j0));
}

// General buffer reactions: the reference's assign-or-accumulate rule, per buffer in
// buffer order (species.c:1653-1702, kernel_generic.cpp:397-509).
// fq: fixed-point species (RealDesc::fixq), whose out[] holds the increment (so the
// assign form writes dJ, not b0 + dJ).
template <int N>
__device__ __forceinline__ void react_general(const RealDesc& D, int d, const float (&val)[N], float (&out)[N],
                                              unsigned pre, unsigned fq) {
  for (int bi = 0; bi < NB; bi++) {
    if (bi >= D.nbuf) break;
    const int t = bi * D.nd + d;
    const int s0 = D.bsp0[t], s1 = D.bsp1[t];
    const float b0 = sel(val, s0), b1 = sel(val, s1);     // deviations from the bases
    const float dJ = buffer_dj(-D.kon_dt[t], -D.koff_dt[t], D.a_dt[t], D.j0_dt[t], b0, b1,
                               __fadd_rn(D.fbase[d][s1], b1));
    if (pre >> s0 & 1u) put(out, s0, __fadd_rn(sel(out, s0), dJ));
    else put(out, s0, (fq >> s0 & 1u) ? dJ : __fadd_rn(b0, dJ));
    if (pre >> s1 & 1u) put(out, s1, __fsub_rn(sel(out, s1), dJ)); else put(out, s1, __fsub_rn(b1, dJ));
  }
}

// What a step does for one realisation (computed once per CTA / unit).
struct StepInfo {
  unsigned pre;        // species flagged before the reaction (diffusing ones, species.c:1542, 1746)
  unsigned updated;    // species written this step (apply_du copies these, species.c:1080-1121)
  int react;           // reaction step (species.c:1657)
  int react_fast;      // the reaction can walk the per-species table rtab (see voxel_update)
};

__host__ __device__ inline StepInfo step_info(const RealDesc& D, long long time_ind) {
  StepInfo si;
  unsigned diffusing;
  step_masks(D, time_ind, si.pre, si.updated, diffusing);
  si.react = (D.nbuf > 0 && time_ind % D.reaction_substep == 0) ? 1 : 0;
  si.react_fast = (si.react && D.react_fast && (si.pre & 1u)) ? 1 : 0;
  return si;
}

// One voxel given its 7-point neighbourhood.  Loads go through the caller: ld(s, k) =
// species s at neighbour k (0..5 = z-, z+, y-, y+, x-, x+; 6 = the voxel; out-of-box
// neighbours may return anything: they are replaced by the voxel's own value), ldd(k) =
// the domain id there.  N = species slots the caller carries (>= D.ns).
//
//  diffusion (species.c:1501-1650): diffuse_uniform / diffuse_general above.
//  reactions (species.c:1653-1702): when every buffer binds species 0, the bound species
//  are distinct per domain and species 0 is already updated this step (react_fast), the
//  reference's assign-or-accumulate rule reduces to accumulation and the buffers are
//  walked per bound species (table rtab); otherwise react_general.
//  fixed values (species.c:1037-1077): fixed (domain, species) pairs and, with -f, the
//  outer faces of species 0 are reset to their initial values.
// Boundary flux of one pair, FP64 (boundaryfluxes.c:12-141), u0 on the "from" side.
// fslot_p[slot][9] holds the SERCA scale dt*density*Q/(1e-24 h) (serca_flux_fast).
__device__ __forceinline__ double pair_flux(const RealDesc& D, int slot, double u0, double u1) {
  return D.fslot_kind[slot] == FLUX_SERCA ? serca_flux_fast(u0, u1, D.fslot_p[slot][9])
                                          : ryr_flux(D.dt, D.h, u0, u1, D.fslot_p[slot]);
}

// Surrogate class of one voxel of domain d on a reaction step (RealDesc::sur) from the
// increments the fast reactions apply (dJ_s = dt_r J_s, buffer_dj; ca = the voxel's Ca,
// val = the stored deviations): the near-equilibrium test of the surrogate,
// lam |g_s| + k_on (tot - b_s) |sum g| <= MLP_SKIP tot / (dt_r^2 / 2) for every bound s,
// times dt_r^2, as the sign of the margin
// sur_thr2 - kon_dt (tot - b_s) |sum dJ| - (kon_dt ca + koff_dt) |dJ_s|
// = fma(in, |dJ_s|, fma(nkon (cs - db), |sum dJ|, sur_thr2)), in = nkon ca + nkoff (the
// voxel is near equilibrium when no margin is negative; a NaN margin counts as
// non-negative, which keeps the explicit increment).  The staged kernel's two-lane form
// rounds every step the same way.
template <int N>
__device__ __forceinline__ unsigned rx_classify(const RealDesc& D, int d, float ca, const float (&val)[N]) {
  const unsigned kind = D.sur_kind[d];
  if (kind != RX_ELIGIBLE) return kind == RX_STIFF ? RX_CLASS_PLAIN : RX_CLASS_NONE;
  const unsigned rm = D.rmask[d];
  const float dca = val[0];
  float G = 0.f;
#pragma unroll
  for (int s = 1; s < N; s++) {
    if (!(rm >> s & 1u)) continue;
    const float4 k = D.rk[d][s];
    G = __fadd_rn(G, buffer_dj(k.x, k.y, k.z, k.w, val[s], dca, ca));
  }
  const float aG = fabsf(G);
  unsigned neg = 0;   // sign bits of the margins
#pragma unroll
  for (int s = 1; s < N; s++) {
    if (!(rm >> s & 1u)) continue;
    const float4 k = D.rk[d][s];
    const float in = __fmaf_rn(k.x, ca, k.y);
    const float dJ = buffer_dj(k.x, k.y, k.z, k.w, val[s], dca, ca);
    const float margin = __fmaf_rn(in, fabsf(dJ), __fmaf_rn(__fmul_rn(k.x, __fsub_rn(D.sur_cs[d][s], val[s])), aG,
                                                            D.sur_thr2[d][s]));
    neg |= __float_as_uint(margin);
  }
  return (neg >> 31) ? RX_CLASS_NETWORK : RX_CLASS_EXPLICIT;
}

// SUR: on fast-reaction steps of a realisation with RealDesc::sur, cls receives the
// voxel's surrogate class (rx_classify); otherwise it is left alone.
template <int N, bool SUR = false, class LoadU, class LoadD>
__device__ __forceinline__ void voxel_update(const RealDesc& D, const StepInfo& si, unsigned valid, bool on_face,
                                             LoadU ld, LoadD ldd, float (&out)[N], unsigned* cls = nullptr) {
  const int braw = ldd(6);
  const int d = braw & DOMAIN_BITS;
  const int pat = braw >> 3;
  const unsigned fq = D.fixq & si.updated;        // fixed-point species: out[] holds the increment
  float val[N];
#pragma unroll
  for (int s = 0; s < N; s++) {
    const float v = (si.updated >> s & 1u) ? ld(s, 6) : 0.f;
    val[s] = (fq >> s & 1u) ? q_value(v, D.qunit[d][s]) : v;
    out[s] = (fq >> s & 1u) ? 0.f : v;
  }
  if (si.pre) {
    int dn[6];
    bool uniform = true;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const int dk = ldd(k) & DOMAIN_BITS;
      dn[k] = (valid >> k & 1u) ? dk : d;
      uniform = uniform && dn[k] == d;
    }
#pragma unroll
    for (int s = 0; s < N; s++) {
      if (!(si.pre >> s & 1u)) continue;
      const float u = val[s];
      float un[6];
#pragma unroll
      for (int k = 0; k < 6; k++) {
        const float v = ld(s, k);
        un[k] = (valid >> k & 1u) ? v : u;
      }
      const float* c = &D.coef[D.dsi_of[s]][d * ND];
      out[s] = uniform ? diffuse_uniform(c[d], u, un) : diffuse_general(c, dn, u, un);
      if (pat) {
        // density-boundary fluxes across this voxel's faces (Species_step_boundary_fluxes,
        // species.c:1751-1807: du[to] += J, du[from] -= J), after diffusion, before reactions
        double acc = 0.0;
        bool any = false;
#pragma unroll
        for (int k = 0; k < 6; k++) {
          const int code = D.fpat[pat][k];
          if (!code) continue;
          const int slot = (code & 0x7f) - 1;
          if (D.fslot_species[slot] != s) continue;
          const double self = (double)u + D.base[d][s], other = (double)un[k] + D.base[dn[k]][s];
          if (code & 0x80) acc += pair_flux(D, slot, other, self);
          else acc -= pair_flux(D, slot, self, other);
          any = true;
        }
        if (any) out[s] = (float)((double)out[s] + acc);
      }
    }
  }
  if (si.react) {
    if (si.react_fast) {
      const float dca = val[0], ca = __fadd_rn(D.fbase[d][0], dca);
      if (SUR && D.sur) *cls = rx_classify<N>(D, d, ca, val);
      const unsigned rm = D.rmask[d];
#pragma unroll
      for (int s = 1; s < N; s++) {
        if (!(rm >> s & 1u)) continue;
        const float4 k = D.rk[d][s];
        const float dJ = buffer_dj(k.x, k.y, k.z, k.w, val[s], dca, ca);
        out[s] = __fadd_rn(out[s], dJ);
        out[0] = __fsub_rn(out[0], dJ);
      }
    } else {
      react_general<N>(D, d, val, out, si.pre, fq);
    }
  }
  const unsigned fm = D.fixed_mask[d];
#pragma unroll
  for (int s = 0; s < N; s++) {
    if (fm >> s & 1u) out[s] = D.dinit[d][s];
    if (fq >> s & 1u)
      out[s] = (fm >> s & 1u) ? q_set(out[s], D.qinv[d][s]) : q_add(ld(s, 6), out[s], D.qinv[d][s]);
  }
  if (D.dirichlet && on_face) out[0] = D.dinit[d][0];
}

// One thread per voxel; blockIdx.y = realisation.
__global__ void __launch_bounds__(256) k_voxels_direct(const RealDesc* __restrict__ descs, RealCtl* __restrict__ ctl,
                                                        int* __restrict__ err) {
  __shared__ StepInfo s_si;
  __shared__ unsigned s_cur;
  const int r = blockIdx.y;
  const RealDesc& D = descs[r];
  RealCtl& C = ctl[r];
  if (C.stopped) return;
  if (threadIdx.x == 0) {
    const long long k = C.step;
    s_si = step_info(D, k + 1);
    s_cur = C.cur_mask[k & 1];
    if (blockIdx.x == 0) C.cur_mask[(k + 1) & 1] = s_cur ^ s_si.updated;
  }
  __syncthreads();
  const StepInfo si = s_si;
  const unsigned cur = s_cur;
  const int nz = D.nz, plane = D.plane;
  const int nvox = D.nx * plane;
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nvox || si.updated == 0) return;
  const int x = v / plane;
  const int p = v - x * plane;
  const int y = p / nz;
  const int z = p - y * nz;
  const long long idx = (long long)x * D.P + p;
  const unsigned valid = (z > 0 ? 1u : 0u) | (z < nz - 1 ? 2u : 0u) | (y > 0 ? 4u : 0u) |
                         (y < D.ny - 1 ? 8u : 0u) | (x > 0 ? 16u : 0u) | (x < D.nx - 1 ? 32u : 0u);
  // out-of-box neighbours read the voxel itself, so every address stays inside the field
  const long long off[6] = {(valid & 1u) ? -1ll : 0ll, (valid & 2u) ? 1ll : 0ll,
                            (valid & 4u) ? -(long long)nz : 0ll, (valid & 8u) ? (long long)nz : 0ll,
                            (valid & 16u) ? -(long long)D.P : 0ll, (valid & 32u) ? (long long)D.P : 0ll};
  const bool on_face = valid != 63u;
  auto ld = [&](int s, int kk) -> float {
    const float* __restrict__ u = D.u[(cur >> s) & 1u][s];
    return __ldg(u + idx + (kk < 6 ? off[kk] : 0));
  };
  auto ldd = [&](int kk) -> int { return __ldg(D.dom + idx + (kk < 6 ? off[kk] : 0)); };
  float out[NS];
  unsigned cls = RX_CLASS_NONE;
  voxel_update<NS, true>(D, si, valid, on_face, ld, ldd, out, &cls);
#pragma unroll
  for (int s = 0; s < NS; s++) {
    if (s < D.ns && (si.updated >> s & 1u)) D.u[((cur >> s) & 1u) ^ 1u][s][idx] = out[s];
  }
  if (D.sur && si.react_fast) D.rx_class[idx] = (unsigned char)cls;
}

// Channel gating of one channel at step time_ind (evaluate_RyR_stochastically,
// boundaryfluxes.c:295-359), with the Philox stream of the realisation.
__device__ __forceinline__ int gate(const FluxParams& fp, int state, double c0, double t, double dts,
                                    unsigned long long seed, unsigned r, unsigned ch, unsigned boundary,
                                    long long time_ind) {
  const double* p = fp.p;
  if (p[8] > 0) {
    if (p[8] <= t + dts) return 0;
    return state;
  }
  const double kc = fmax(fmin(pow(c0 / p[0], p[5]), p[1]), p[7]);
  const double ko = fmax(fmin(pow(c0 / p[9], p[2]), p[3]), p[4]);
  const double rv = channel_uniform(seed, r, ch, boundary, time_ind);
  if (state == 0) return rv <= dts * ko ? 1 : 0;
  if (state == 1) return rv <= dts * kc ? 0 : 1;
  return state;
}

// Flux of one pair at this step, with the channel gated first (a discrete pair flows
// only when its channel is open after this step's gating).  The owner side of a channel
// stores its new state.  Returns false when the pair carries no flux this step.  CH =
// false: the caller's rows hold density pairs only (no channel code is compiled).
template <bool CH>
__device__ __forceinline__ bool pair_step(const RealDesc& D, RealCtl* ctl_r, int species, int kind, int dsi,
                                          int channel, int local_channel, int boundary, int owner, long long v0,
                                          long long v1, int doms, const FluxParams& fp,
                                          const float* __restrict__ uold, const float* __restrict__ ca,
                                          unsigned char* __restrict__ states, int nch, long long k, bool stoch,
                                          double& J) {
  const long long ti = k + 1;
  const int d0 = doms & DOMAIN_BITS, d1 = (doms >> 3) & DOMAIN_BITS;
  if (CH && channel >= 0) {
    const int s_old = states[(k & 1) * (long long)nch + channel];
    int s_new = s_old;
    if (stoch && kind != FLUX_SERCA)
      s_new = gate(fp, s_old, (double)__ldg(ca + v1) + D.base[d1][0], (double)ti * D.dt, D.dt * D.stochastic_substep,
                   D.seed, D.stream, (unsigned)local_channel, (unsigned)boundary, ti);
    if (owner) {
      states[((k + 1) & 1) * (long long)nch + channel] = (unsigned char)s_new;
      if (s_new == 1) atomicAdd(&ctl_r->open_count[(k + 1) & 1], 1);
    }
    if (s_new != 1) return false;
  }
  if (ti % D.substeps[dsi] != 0) return false;
  const double u0 = (double)__ldg(uold + v0) + D.base[d0][species];
  const double u1 = (double)__ldg(uold + v1) + D.base[d1][species];
  J = kind == FLUX_SERCA ? serca_flux_fast(u0, u1, fp.p[9]) : ryr_flux(D.dt, D.h, u0, u1, fp.p);
  return true;
}

// One thread per flux row (a voxel receiving boundary flux): channel gating
// (evaluate_RyR_stochastically, boundaryfluxes.c:295-359) and the flux of every pair that
// touches the voxel, summed in pair order (Species_step_boundary_fluxes,
// species.c:1704-1907), added to the voxel's new value.  The rows are split by the host:
// CH = true for voxels touched by a discrete (channel) pair, CH = false for voxels touched
// by density pairs only (SERCA sheets: most rows), which run without the gating code and
// its registers, at higher occupancy.  Every voxel has one row, so the two launches write
// disjoint voxels.
template <bool CH>
__global__ void __launch_bounds__(256, CH ? 4 : 8) k_boundaries(const RealDesc* __restrict__ descs, RealCtl* __restrict__ ctl,
                                                     const FluxRow* __restrict__ rows, int nrows,
                                                     const FluxEntry* __restrict__ entries,
                                                     const FluxPair* __restrict__ pairs,
                                                     const FluxParams* __restrict__ params,
                                                     unsigned char* __restrict__ states,  // [2][nch]
                                                     int nch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nrows) return;
  const FluxRow row = rows[i];
  const RealDesc& D = descs[row.r];
  const RealCtl& C = ctl[row.r];
  if (C.stopped) return;
  const long long k = C.step;
  const long long ti = k + 1;
  unsigned pre, updated, diffusing;
  step_masks(D, ti, pre, updated, diffusing);
  const unsigned cur = C.cur_mask[k & 1];
  const bool stoch = (ti % D.stochastic_substep) == 0;
  const float* __restrict__ uold = D.u[(cur >> row.species) & 1u][row.species];
  const float* __restrict__ ca = D.u[cur & 1u][0];
  double acc = 0.0, J;
  bool any = false;
  if (pair_step<CH>(D, &ctl[row.r], row.species, row.kind, row.dsi, row.channel, row.local_channel, row.boundary,
                row.owner, row.v0, row.v1, row.doms, params[row.param], uold, ca, states, nch, k, stoch, J)) {
    acc += (double)row.sign * J;
    any = true;
  }
  for (int e = row.more_begin; e < row.more_end; e++) {
    const FluxEntry en = entries[e];
    const FluxPair pr = pairs[en.pair];
    if (pair_step<CH>(D, &ctl[row.r], row.species, pr.kind, pr.dsi, pr.channel, pr.local_channel, pr.boundary,
                  en.owner, pr.v0, pr.v1, pr.doms, params[pr.param], uold, ca, states, nch, k, stoch, J)) {
      acc += (double)en.sign * J;
      any = true;
    }
  }
  if (any && row.apply && (updated >> row.species & 1u)) {
    float* unew = D.u[((cur >> row.species) & 1u) ^ 1u][row.species];
    unew[row.v] = (float)((double)unew[row.v] + acc);
  }
}

// The step record of a realisation's running step (see StepRec).
__host__ __device__ inline void write_steprec(const RealDesc& D, const RealCtl& C, StepRec& R) {
  unsigned pre, updated, sub;
  step_masks(D, C.step + 1, pre, updated, sub);
  R.active = C.stopped ? 0u : 1u;
  R.cur = C.cur_mask[C.step & 1];
  R.updated = updated;
  R.sub = sub;
}

// Density-boundary rows (voxels touched by density pairs only: the SERCA sheets), one
// thread per row: what k_boundaries<false> computes -- the flux of every pair of the row
// in pair order, summed in FP64, added to the voxel's new value with one rounding -- from
// a 32-byte row, the realisation's step record and the voxel's new value loaded together
// with the pair's old values (three dependent loads instead of five).  A pair row gives
// both voxels of a pair their flux from one evaluation (each voxel still gets exactly the
// value its own row would give: 0 + J or 0 - J, then one rounding).
__global__ void __launch_bounds__(256, 8) k_density_rows(const RealDesc* __restrict__ descs,
                                                          const StepRec* __restrict__ rec,
                                                          const DensityRow* __restrict__ rows, int nrows,
                                                          const FluxEntry* __restrict__ entries,
                                                          const FluxPair* __restrict__ pairs,
                                                          const FluxParams* __restrict__ params) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nrows) return;
  const int4 a = __ldg(reinterpret_cast<const int4*>(rows + i));          // v, vo, r, more_begin
  const int4 b = __ldg(reinterpret_cast<const int4*>(rows + i) + 1);      // scale, meta0, meta1
  const uint4 R = __ldg(reinterpret_cast<const uint4*>(rec + a.z));       // active, cur, updated, sub
  if (!R.x) return;
  const RealDesc& D = descs[a.z];
  const unsigned meta0 = (unsigned)b.z, meta1 = (unsigned)b.w;
  const int sp = (int)((meta0 >> 16) & 0xffu), dsi = (int)(meta0 >> 24);
  const unsigned sel = (R.y >> sp) & 1u;
  const float* __restrict__ uold = D.u[sel][sp];
  float* __restrict__ unew = D.u[sel ^ 1u][sp];
  const bool upd = R.z >> sp & 1u;
  const bool write = (meta1 & DROW_APPLY) && upd;
  const bool write_from = (meta1 & DROW_APPLY_FROM) && upd;     // pair rows only
  const float nv = write ? unew[a.x] : 0.f;
  const float nvo = write_from ? unew[a.y] : 0.f;
  double acc = 0.0;
  bool any = false;
  if (R.w >> dsi & 1u) {
    const double us = (double)__ldg(uold + a.x) + D.base[(meta1 >> 16) & DOMAIN_BITS][sp];
    const double uo = (double)__ldg(uold + a.y) + D.base[(meta1 >> 19) & DOMAIN_BITS][sp];
    const bool to = meta1 & DROW_TO;
    const double u0 = to ? uo : us, u1 = to ? us : uo;
    const double J = (meta1 & DROW_SERCA) ? serca_flux_fast(u0, u1, __hiloint2double(b.y, b.x))
                                          : ryr_flux(D.dt, D.h, u0, u1, params[meta0 & 0xffffu].p);
    acc += to ? J : -J;
    any = true;
    if (write_from) unew[a.y] = (float)((double)nvo + -J);       // the "from" voxel's own row
  }
  const int nmore = (int)((meta1 >> 8) & 0xffu);
  for (int e = a.w; e < a.w + nmore; e++) {
    const FluxEntry en = entries[e];
    const FluxPair pr = pairs[en.pair];
    if (!(R.w >> pr.dsi & 1u)) continue;
    const FluxParams& fp = params[pr.param];
    const double u0 = (double)__ldg(uold + pr.v0) + D.base[pr.doms & DOMAIN_BITS][sp];
    const double u1 = (double)__ldg(uold + pr.v1) + D.base[(pr.doms >> 3) & DOMAIN_BITS][sp];
    const double J = pr.kind == FLUX_SERCA ? serca_flux_fast(u0, u1, fp.p[9]) : ryr_flux(D.dt, D.h, u0, u1, fp.p);
    acc += (double)en.sign * J;
    any = true;
  }
  if (any && write) unew[a.x] = (float)((double)nv + acc);
}

// Step epilogue, one thread per realisation, after the boundary kernel: advance the
// step counter, apply the abort rule (species.c:3476-3486) on the openness counted by
// the boundary kernel, stop at the last step.  flags (nullable): the stop flag of every
// realisation after this step.
// sur_queue (with the surrogate on): its tile queues, emptied for the next step once this
// step's correction kernels have taken their tiles.
__global__ void k_epilogue(const RealDesc* __restrict__ descs, RealCtl* __restrict__ ctl, StepRec* __restrict__ rec,
                           int nreal, int* __restrict__ flags, unsigned* __restrict__ sur_queue) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (sur_queue && r == 0) sur_queue[0] = sur_queue[1] = sur_queue[2] = sur_queue[3] = 0u;
  if (r >= nreal) return;
  RealCtl& C = ctl[r];
  if (C.stopped) {
    if (flags) flags[r] = 1;
    return;
  }
  const RealDesc& D = descs[r];
  const long long k = C.step;
  const long long ti = k + 1;
  const int open = C.open_count[(k + 1) & 1];
  C.open_count[k & 1] = 0;
  C.step = ti;
  if (D.has_channels && D.tabort != 0) {
    const double tt = (double)ti * D.dt;
    if (open) {
      C.last_closed = -1.0;
    } else if (D.tabort >= 0) {
      if (C.last_closed < 0) C.last_closed = tt;
      if (tt - C.last_closed >= D.tabort) C.stopped = 1;
    }
  }
  if (C.step >= D.total_steps) C.stopped = 1;
  write_steprec(D, C, rec[r]);
  if (flags) flags[r] = C.stopped;
}

// Output reductions: partial min / max / sum over a block for one species of one
// realisation, then a fixed-order final pass (deterministic FP64 sums).
__global__ void __launch_bounds__(256) k_reduce_partial(const RealDesc* __restrict__ descs,
                                                         const RealCtl* __restrict__ ctl, int r, int s,
                                                         double* __restrict__ part /*[nblk][3][ND]*/) {
  const RealDesc& D = descs[r];
  const unsigned cur = ctl[r].cur_mask[ctl[r].step & 1];
  const float* __restrict__ u = D.u[(cur >> s) & 1u][s];
  double mn[ND], mx[ND], sm[ND];
#pragma unroll
  for (int d = 0; d < ND; d++) { mn[d] = FLT_MAX; mx[d] = FLT_MIN; sm[d] = 0.0; }
  const long long nvox = (long long)D.nx * D.plane;
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(v / D.plane);
    const long long idx = (long long)x * D.P + (v - (long long)x * D.plane);
    const int d = D.dom[idx] & DOMAIN_BITS;
    const double val = ((D.fixq >> s & 1u) ? (double)q_bits(u[idx]) * D.qunit[d][s] : (double)u[idx]) + D.base[d][s];
#pragma unroll
    for (int dd = 0; dd < ND; dd++) {
      if (dd == d) {
        mn[dd] = val < mn[dd] ? val : mn[dd];
        mx[dd] = val > mx[dd] ? val : mx[dd];
        sm[dd] += val;
      }
    }
  }
  __shared__ double red[3][ND][256];
#pragma unroll
  for (int d = 0; d < ND; d++) { red[0][d][threadIdx.x] = mn[d]; red[1][d][threadIdx.x] = mx[d]; red[2][d][threadIdx.x] = sm[d]; }
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
#pragma unroll
      for (int d = 0; d < ND; d++) {
        double a = red[0][d][threadIdx.x + w];
        if (a < red[0][d][threadIdx.x]) red[0][d][threadIdx.x] = a;
        a = red[1][d][threadIdx.x + w];
        if (a > red[1][d][threadIdx.x]) red[1][d][threadIdx.x] = a;
        red[2][d][threadIdx.x] += red[2][d][threadIdx.x + w];
      }
    }
    __syncthreads();
  }
  if (threadIdx.x < ND) {
    const int d = threadIdx.x;
    part[(blockIdx.x * 3 + 0) * ND + d] = red[0][d][0];
    part[(blockIdx.x * 3 + 1) * ND + d] = red[1][d][0];
    part[(blockIdx.x * 3 + 2) * ND + d] = red[2][d][0];
  }
}

__global__ void k_reduce_final(const double* __restrict__ part, int nblk, double dV,
                               double* __restrict__ out /*[3][ND]*/) {
  const int d = threadIdx.x;
  if (d >= ND) return;
  double mn = FLT_MAX, mx = FLT_MIN, sm = 0.0;
  for (int b = 0; b < nblk; b++) {
    const double a = part[(b * 3 + 0) * ND + d], c = part[(b * 3 + 1) * ND + d];
    mn = a < mn ? a : mn;
    mx = c > mx ? c : mx;
    sm += part[(b * 3 + 2) * ND + d];
  }
  out[0 * ND + d] = mn;
  out[1 * ND + d] = mx;
  out[2 * ND + d] = sm * dV;
}

}  // namespace csp
