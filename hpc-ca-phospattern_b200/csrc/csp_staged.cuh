// csp_staged.cuh -- the TMA-staged voxel kernel.
//
// Work unit = (realisation r, plane chunk c, x segment [x0, x1)).  A CTA of T threads
// owns L = 4*T consecutive positions p = c*L .. c*L+L-1 of the (y,z) plane (each thread
// 4 consecutive positions along z) and marches along x.  Every x-plane of the chunk,
// widened by nz on both sides (the y-neighbours) and rounded out to 16 bytes, is moved
// HBM -> shared memory by 1D bulk TMA copies (cp.async.bulk, no multicast) into a ring of
// NST stages guarded by mbarriers: planes x-1, x, x+1 are resident while plane x is
// computed and two more are in flight.  A thread reads its own 4 positions of the three
// planes with 128-bit shared loads; z-neighbours inside those 4 positions come from
// registers, the y-neighbours and the two outer z-neighbours from the centre plane.  Outputs go straight to HBM with 128-bit
// stores.  The per-voxel arithmetic is voxel_update (csp_kernels.cuh), shared with the
// direct kernel, so both kernels give bitwise equal fields.
//
// Every mbarrier wait is bounded in time (WAIT_NS).  A thread that gives up sets its own
// flag; the CTA takes one decision from all flags at the end-of-plane barrier
// (__syncthreads_or), so every thread leaves the x loop together.  Before the CTA exits,
// its issuing thread waits (bounded again) for every stage whose bulk copies it has not
// seen land, so no copy still writes this CTA's shared memory; then ERR_TIMEOUT is set in
// the device error word and the kernel returns.  The fields of a launch that timed out
// are undefined (the host reports CSP_EDEVICE).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "csp_kernels.cuh"

namespace csp {

constexpr int NST = 4;                    // ring stages: planes x-1, x, x+1 resident, 1 in flight
constexpr unsigned long long WAIT_NS = 1000000000ull;       // 1 s per mbarrier wait
constexpr unsigned long long INJECT_WAIT_NS = 1000000ull;   // 1 ms for the test hook's wait

struct StagedGeom {
  int L;            // positions per chunk (4*T)
  int slot;         // floats per species slot per stage (>= L + 2*nz_max + 8, multiple of 4)
  int domcap;       // bytes of domain ids per stage (multiple of 16)
  int stage_bytes;  // bytes per stage
  int ms;           // species slots per stage
  int desc_off;     // smem offset of the descriptor copy
  int ring_off;     // smem offset of stage 0
  int smem;         // total dynamic smem
  int nunits;
  int seg;          // x planes per unit
};

struct StagedPlan;
using StagedLaunchFn = cudaError_t (*)(const StagedPlan&, int, int, const RealDesc*, RealCtl*, int*, cudaStream_t);

struct StagedPlan {
  bool ok = false;
  int T = 256;
  int slots = 0;                // resident CTAs of the whole GPU (persistent grid size)
  StagedGeom g{};
  int4* d_units = nullptr;      // (r, c, x0, x1), realisation-major
  int nunits = 0;
  std::vector<int> unit_first;  // [n+1]: the units of realisation r are [unit_first[r], unit_first[r+1])
  StagedLaunchFn launch = nullptr;
  StagedLaunchFn launch_sur = nullptr;      // the variant that also classifies voxels for the surrogate
  StagedLaunchFn launch_inject = nullptr;   // null: no test-hook variant for this plan
  unsigned fixq = 0;                        // union of the realisations' fixed-point species
};

// ---- PTX helpers (sm_90+ bulk copy / mbarrier) ----
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// true once phase `parity` of the barrier has completed; false after limit_ns
__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity, unsigned long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > limit_ns) return false;
  return true;
}
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(dst), "l"(src), "r"(bytes), "r"(bar) : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ int floor4(int a) { return a & ~3; }
__device__ __forceinline__ int ceil4(int a) { return (a + 3) & ~3; }
__device__ __forceinline__ int floor16(int a) { return a & ~15; }
__device__ __forceinline__ int ceil16(int a) { return (a + 15) & ~15; }

template <int MS>
__device__ __forceinline__ float pick(const float (&a)[MS][4], int s, int j) {
  float r = a[0][j];
#pragma unroll
  for (int q = 1; q < MS; q++)
    if (s == q) r = a[q][j];
  return r;
}

// Issue the bulk copies of plane q into stage st (one elected thread).
__device__ __forceinline__ void issue_plane(const RealDesc& D, unsigned cur, unsigned lmask, int q, int st,
                                            unsigned char* ring, const StagedGeom& g, unsigned bar, int lo,
                                            int hi, int lob, int hib) {
  const unsigned fbytes = (unsigned)(hi - lo) * 4u;
  const unsigned dbytes = (unsigned)(hib - lob);
  const unsigned nl = __popc(lmask);
  unsigned char* stage = ring + (size_t)st * g.stage_bytes;
  mbar_expect_tx(bar, nl * fbytes + dbytes);
  int slot = 0;
  for (int s = 0; s < NS; s++) {
    if (!(lmask >> s & 1u)) continue;
    const float* src = D.u[(cur >> s) & 1u][s] + (long long)q * D.P + lo;
    bulk_g2s(smem_u32(stage + (size_t)slot * g.slot * 4), src, fbytes, bar);
    slot++;
  }
  bulk_g2s(smem_u32(stage + (size_t)g.ms * g.slot * 4), D.dom + (long long)q * D.P + lob, dbytes, bar);
}

// 4 bytes starting at any byte address (two aligned 32-bit shared loads + funnel shift).
__device__ __forceinline__ unsigned ld_u32_any(const unsigned char* p) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const unsigned* w = reinterpret_cast<const unsigned*>(a & ~(uintptr_t)3);
  return __funnelshift_r(w[0], w[1], 8u * (unsigned)(a & 3));
}

// rx_classify on the four voxels of a group in one domain d, in two-lane FP32 with the
// same rounding (ca0 / ca1: Ca of voxels 0,1 / 2,3; G0 / G1: their sums of the increments
// dJ_s in slot order, accumulated by the reaction loop that applies them): the class of
// voxel j in byte j.
template <int MS>
__device__ __forceinline__ unsigned rx_classify4(const RealDesc& D, int d, F2 ca0, F2 ca1, const float (&val)[MS][4],
                                                 F2 G0, F2 G1) {
  const unsigned kind = D.sur_kind[d];
  if (kind != RX_ELIGIBLE) return kind == RX_STIFF ? RX_CLASS_PLAIN * 0x01010101u : 0u;
  const unsigned rm = D.rmask[d];
  const F2 dca0 = f2(val[0][0], val[0][1]), dca1 = f2(val[0][2], val[0][3]);
  const F2 aG0 = f2_abs(G0), aG1 = f2_abs(G1);
  unsigned long long neg0 = 0, neg1 = 0;   // sign bits of the margins, OR-ed over the slots
#pragma unroll
  for (int s = 1; s < MS; s++) {
    if (!(rm >> s & 1u)) continue;
    const float4 kk = D.rk[d][s];
    const F2 nkon = f2(kk.x, kk.x), nkoff = f2(kk.y, kk.y), a = f2(kk.z, kk.z), j0 = f2(kk.w, kk.w);
    const F2 cs = f2(D.sur_cs[d][s], D.sur_cs[d][s]), thr = f2(D.sur_thr2[d][s], D.sur_thr2[d][s]);
    const F2 db0 = f2(val[s][0], val[s][1]), db1 = f2(val[s][2], val[s][3]);
    const F2 in0 = f2_fma(nkon, ca0, nkoff), in1 = f2_fma(nkon, ca1, nkoff);
    const F2 dj0 = f2_fma(db0, in0, f2_fma(a, dca0, j0)), dj1 = f2_fma(db1, in1, f2_fma(a, dca1, j0));
    neg0 |= f2_fma(in0, f2_abs(dj0), f2_fma(f2_mul(nkon, f2_sub(cs, db0)), aG0, thr)).v;
    neg1 |= f2_fma(in1, f2_abs(dj1), f2_fma(f2_mul(nkon, f2_sub(cs, db1)), aG1, thr)).v;
  }
  const unsigned e = RX_CLASS_EXPLICIT, nt = RX_CLASS_NETWORK;
  return ((neg0 >> 31 & 1u) ? nt : e) | ((neg0 >> 63) ? nt : e) << 8 | ((neg1 >> 31 & 1u) ? nt : e) << 16 |
         ((neg1 >> 63) ? nt : e) << 24;
}

// INJ = true builds the test hook's variant (csp_test_wait_timeout); the kernel in use is
// INJ = false, which has none of that code.  FQ: the species that may be stored in fixed
// point (RealDesc::fixq is a subset), known at compile time so that the code for every
// other species has no fixed-point branch (a run-time mask over all species cost 18 %).
template <int MS, int T, bool INJ, unsigned FQ, bool SUR>
__global__ void __launch_bounds__(T, 2) k_voxels_staged(const RealDesc* __restrict__ descs, RealCtl* __restrict__ ctl,
                                                        const int4* __restrict__ units, StagedGeom g,
                                                        int* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem);
  RealDesc& D = *reinterpret_cast<RealDesc*>(smem + g.desc_off);
  unsigned char* ring = smem + g.ring_off;
  const int tid = threadIdx.x;
  int last_r = -1;
  unsigned phase = 0;    // bit st = parity of the next completion of stage st (CTA-uniform)

  if (tid == 0) {
    // bars[NST] is the test hook's barrier: initialised, never arrived on
    for (int i = 0; i <= NST; i++) mbar_init(smem_u32(&bars[i]), 1);
    fence_mbar_init();
  }
  __syncthreads();

  for (int u = blockIdx.x; u < g.nunits; u += gridDim.x) {
    const int4 un = units[u];
    const int r = un.x, c = un.y, x0 = un.z, x1 = un.w;
    if (r != last_r) {
      __syncthreads();
      const int* src = reinterpret_cast<const int*>(&descs[r]);
      int* dst = reinterpret_cast<int*>(&D);
      for (int i = tid; i < (int)(sizeof(RealDesc) / 4); i += T) dst[i] = src[i];
      __syncthreads();
      last_r = r;
    }
    if (ctl[r].stopped) continue;
    const long long k = ctl[r].step;
    const StepInfo si = step_info(D, k + 1);
    const unsigned cur = ctl[r].cur_mask[k & 1];
    if (tid == 0 && c == 0 && x0 == 0) ctl[r].cur_mask[(k + 1) & 1] = cur ^ si.updated;
    if (si.updated == 0) continue;
    const unsigned lmask = si.updated & ((1u << D.ns) - 1u);

    const int nz = D.nz, plane = D.plane, nx = D.nx;
    const int cL = c * g.L;
    const int lo = floor4(max(0, cL - nz));
    const int hi = ceil4(min(plane, cL + g.L + nz));
    const int lob = floor16(max(0, cL - nz));
    const int hib = ceil16(min(plane, cL + g.L + nz));
    const int ql = max(0, x0 - 1), qh = min(nx - 1, x1);
    const int p0 = cL + 4 * tid;
    unsigned vzy[4];
    bool all_in = true;
    unsigned ymask_m = 0, ymask_p = 0;     // bytes of the y-/y+ words that are in-box neighbours
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int p = p0 + j;
      all_in = all_in && p < plane;
      const int y = p / nz, z = p - y * nz;
      vzy[j] = (z > 0 ? 1u : 0u) | (z < nz - 1 ? 2u : 0u) | (y > 0 ? 4u : 0u) | (y < D.ny - 1 ? 8u : 0u);
      if (vzy[j] & 4u) ymask_m |= 0xffu << (8 * j);
      if (vzy[j] & 8u) ymask_p |= 0xffu << (8 * j);
    }
    // the y- word would start before the staged range only in the first chunk's first row
    const bool group_ok = all_in && (ymask_m == 0 || p0 - nz >= lob);
    // rows of a multiple of 4 voxels: every group lies in one row and its y-neighbour
    // rows are 16-byte aligned in the stage
    const bool yvec = (nz & 3) == 0;
    // class bytes of this chunk (one per plane), when the chunk matches the class table's
    const unsigned char* cls_row = (g.L == CLASS_L && D.cls) ? D.cls + c : nullptr;

    unsigned pending = 0;  // issuing thread: stages whose copies it has not yet seen land
    if (tid == 0) {
      fence_proxy_async();
      for (int q = ql; q <= min(qh, ql + NST - 1); q++) {
        const int st = (q - ql) % NST;
        issue_plane(D, cur, lmask, q, st, ring, g, smem_u32(&bars[st]), lo, hi, lob, hib);
        pending |= 1u << st;
      }
    }
    bool timeout = false;   // this thread gave up on a wait (the CTA decides at the next barrier)
    // test hook (INJ only): one thread that issues no copies waits on a barrier that nothing
    // completes, so the timeout path below runs with the threads of the CTA disagreeing
    if (INJ && blockIdx.x == 0 && u == (int)blockIdx.x && tid == 37)
      timeout = !mbar_wait_bounded(smem_u32(&bars[NST]), 0u, INJECT_WAIT_NS);
    auto wait_plane = [&](int q) {
      const int st = (q - ql) % NST;
      if (mbar_wait_bounded(smem_u32(&bars[st]), (phase >> st) & 1u, WAIT_NS)) {
        phase ^= 1u << st;
        pending &= ~(1u << st);
      } else {
        timeout = true;     // phase kept: the drain below waits on the same completion
      }
    };
    bool cta_timeout = false;
    auto stage_of = [&](int q) -> const unsigned char* { return ring + (size_t)((q - ql) % NST) * g.stage_bytes; };
    const int so = g.slot;
    const size_t dom_off = (size_t)g.ms * g.slot * 4;

    if (x0 > 0) wait_plane(x0 - 1);
    wait_plane(x0);
    int pc_next = cls_row ? __ldg(cls_row + (size_t)x0 * D.ncls) : CLASS_MIXED;
    for (int x = x0; x < x1; x++) {
      const bool has_prev = x > 0, has_next = x + 1 < nx;
      if (has_next) wait_plane(x + 1);
      const unsigned char* sc = stage_of(x);
      const unsigned char* sp = has_prev ? stage_of(x - 1) : sc;
      const unsigned char* sn = has_next ? stage_of(x + 1) : sc;
      const float* fc = reinterpret_cast<const float*>(sc) - lo;
      const float* fp = reinterpret_cast<const float*>(sp) - lo;
      const float* fn = reinterpret_cast<const float*>(sn) - lo;
      const unsigned char* dc = sc + dom_off - lob;
      const unsigned char* dp = sp + dom_off - lob;
      const unsigned char* dnx = sn + dom_off - lob;
      const unsigned xval = (has_prev ? 16u : 0u) | (has_next ? 32u : 0u);
      float out[MS][4];

      // ---- chunk class: the whole chunk neighbourhood in one domain (CTA-uniform);
      // the next plane's byte is fetched one plane ahead ----
      const int pc = pc_next;
      if (cls_row && x + 1 < x1) pc_next = __ldg(cls_row + (size_t)(x + 1) * D.ncls);
      unsigned wc, wp, wn, wym, wyp, ezm, ezp;
      int d0;
      bool uni;
      if (pc != CLASS_MIXED) {
        d0 = pc;
        uni = all_in;
        wc = wp = wn = wym = wyp = ezm = ezp = 0u;
      } else {
        // ---- domain bytes of the group and of its neighbourhood (4 per word) ----
        wc = *reinterpret_cast<const unsigned*>(dc + p0);
        wp = wc; wn = wc; wym = wc; wyp = wc; ezm = wc & 0xffu; ezp = wc >> 24;
        if (group_ok) {
          if (has_prev) wp = *reinterpret_cast<const unsigned*>(dp + p0);
          if (has_next) wn = *reinterpret_cast<const unsigned*>(dnx + p0);
          if (vzy[0] & 1u) ezm = dc[p0 - 1];
          if (vzy[3] & 2u) ezp = dc[p0 + 4];
          if (ymask_m) wym = ld_u32_any(dc + p0 - nz);
          if (ymask_p) wyp = ld_u32_any(dc + p0 + nz);
        }
        // ---- is the whole 4-voxel group and its neighbourhood in one domain? ----
        d0 = wc & 0xff;
        const unsigned dw = (unsigned)d0 * 0x01010101u;
        uni = group_ok && wc == dw && d0 <= DOMAIN_BITS && wp == dw && wn == dw &&
              ezm == (unsigned)d0 && ezp == (unsigned)d0 && ((wym ^ dw) & ymask_m) == 0u &&
              ((wyp ^ dw) & ymask_p) == 0u;
      }

      // the uniform path only when every in-range group of the warp takes it: a warp with
      // a few mixed groups would otherwise run both paths one after the other; the mixed
      // path gives uniform groups the same rounded values
      const bool uni_w = __all_sync(__activemask(), uni || !all_in);
      if (__builtin_expect(uni && uni_w, 1)) {
        // ---- uniform group: constants once per group, one species at a time, voxel
        // pairs (0,1) and (2,3) in two-lane FP32 ----
        float val[MS][4];
        F2 o2[MS][2];
        const unsigned fq = FQ & D.fixq & lmask;   // fixed-point species: o2 holds the increment
        int slot = 0;
#pragma unroll
        for (int s = 0; s < MS; s++) {
          if (lmask >> s & 1u) {
            const float4 a = *reinterpret_cast<const float4*>(fc + slot * so + p0);
            val[s][0] = a.x; val[s][1] = a.y; val[s][2] = a.z; val[s][3] = a.w;
            slot++;
          } else {
            val[s][0] = val[s][1] = val[s][2] = val[s][3] = 0.f;
          }
          if (fq >> s & 1u) {
            const float qu = D.qunit[d0][s];
#pragma unroll
            for (int j = 0; j < 4; j++) val[s][j] = q_value(val[s][j], qu);
            o2[s][0] = o2[s][1] = f2(0.f, 0.f);
          } else {
            o2[s][0] = f2(val[s][0], val[s][1]);
            o2[s][1] = f2(val[s][2], val[s][3]);
          }
        }
        const F2 m2 = f2(-2.f, -2.f);
        slot = 0;
#pragma unroll
        for (int s = 0; s < MS; s++) {
          if (!(lmask >> s & 1u)) continue;
          const int so_s = slot * so;
          slot++;
          if (!(si.pre >> s & 1u)) continue;
          const float cdd = D.cdiag[d0][s];
          // an out-of-box neighbour is read at the voxel itself (fp / fn point at the
          // centre plane on the first / last plane; y and z addresses are clamped), so
          // the values need no selection afterwards
          const float4 vp = *reinterpret_cast<const float4*>(fp + so_s + p0);
          const float4 vn = *reinterpret_cast<const float4*>(fn + so_s + p0);
          const float zm = fc[so_s + ((vzy[0] & 1u) ? p0 - 1 : p0)];
          const float zp = fc[so_s + ((vzy[3] & 2u) ? p0 + 4 : p0 + 3)];
          const float* v = val[s];
          float4 ym, yp;
          F2 zs0, zs1;
          if (yvec) {
            // rows of a multiple of 4 voxels: the group lies in one row
            const int pym = (vzy[0] & 4u) ? p0 - nz : p0, pyp = (vzy[0] & 8u) ? p0 + nz : p0;
            ym = *reinterpret_cast<const float4*>(fc + so_s + pym);
            yp = *reinterpret_cast<const float4*>(fc + so_s + pyp);
            zs0 = f2(__fadd_rn(zm, v[1]), __fadd_rn(v[0], v[2]));
            zs1 = f2(__fadd_rn(v[1], v[3]), __fadd_rn(v[2], zp));
          } else {
            // the group may straddle a row end: y and z neighbours per voxel
            const float* r = fc + so_s + p0;
            ym = make_float4(r[(vzy[0] & 4u) ? -nz : 0], r[(vzy[1] & 4u) ? 1 - nz : 1], r[(vzy[2] & 4u) ? 2 - nz : 2],
                             r[(vzy[3] & 4u) ? 3 - nz : 3]);
            yp = make_float4(r[(vzy[0] & 8u) ? nz : 0], r[(vzy[1] & 8u) ? 1 + nz : 1], r[(vzy[2] & 8u) ? 2 + nz : 2],
                             r[(vzy[3] & 8u) ? 3 + nz : 3]);
            const float zm1 = (vzy[1] & 1u) ? v[0] : v[1], zm2 = (vzy[2] & 1u) ? v[1] : v[2];
            const float zm3 = (vzy[3] & 1u) ? v[2] : v[3];
            const float zp0 = (vzy[0] & 2u) ? v[1] : v[0], zp1 = (vzy[1] & 2u) ? v[2] : v[1];
            const float zp2 = (vzy[2] & 2u) ? v[3] : v[2];
            zs0 = f2(__fadd_rn(zm, zp0), __fadd_rn(zm1, zp1));
            zs1 = f2(__fadd_rn(zm2, zp2), __fadd_rn(zm3, zp));
          }
          const F2 c2 = f2(cdd, cdd);
          const F2 ys0 = f2_add(f2(ym.x, ym.y), f2(yp.x, yp.y)), ys1 = f2_add(f2(ym.z, ym.w), f2(yp.z, yp.w));
          const F2 xs0 = f2_add(f2(vp.x, vp.y), f2(vn.x, vn.y)), xs1 = f2_add(f2(vp.z, vp.w), f2(vn.z, vn.w));
          o2[s][0] = diffuse_uniform2(c2, m2, f2(v[0], v[1]), zs0, ys0, xs0);
          o2[s][1] = diffuse_uniform2(c2, m2, f2(v[2], v[3]), zs1, ys1, xs1);
        }
        float out[MS][4];
        if (si.react && si.react_fast) {
          // deviations of Ca, and Ca itself (its base plus the deviation)
          const F2 dca0 = f2(val[0][0], val[0][1]), dca1 = f2(val[0][2], val[0][3]);
          const float cb = D.fbase[d0][0];
          const F2 ca0 = f2_add(f2(cb, cb), dca0), ca1 = f2_add(f2(cb, cb), dca1);
          const unsigned rm = D.rmask[d0];
          F2 G0 = f2(0.f, 0.f), G1 = G0;    // SUR: sums of the increments
#pragma unroll
          for (int s = 1; s < MS; s++) {
            if (!(rm >> s & 1u)) continue;
            const float4 kk = D.rk[d0][s];
            const F2 nkon = f2(kk.x, kk.x), nkoff = f2(kk.y, kk.y), a = f2(kk.z, kk.z), j0 = f2(kk.w, kk.w);
            const F2 dj0 = buffer_dj2(nkon, nkoff, a, j0, f2(val[s][0], val[s][1]), dca0, ca0);
            const F2 dj1 = buffer_dj2(nkon, nkoff, a, j0, f2(val[s][2], val[s][3]), dca1, ca1);
            o2[s][0] = f2_add(o2[s][0], dj0);
            o2[s][1] = f2_add(o2[s][1], dj1);
            o2[0][0] = f2_sub(o2[0][0], dj0);
            o2[0][1] = f2_sub(o2[0][1], dj1);
            if (SUR) {
              G0 = f2_add(G0, dj0);
              G1 = f2_add(G1, dj1);
            }
          }
          if (SUR && D.sur)
            *reinterpret_cast<unsigned*>(D.rx_class + (long long)x * D.P + p0) =
                rx_classify4<MS>(D, d0, ca0, ca1, val, G0, G1);
        }
#pragma unroll
        for (int s = 0; s < MS; s++) {
          f2_split(o2[s][0], out[s][0], out[s][1]);
          f2_split(o2[s][1], out[s][2], out[s][3]);
        }
        if (si.react && !si.react_fast) {
          {
#pragma unroll
            for (int j = 0; j < 4; j++) {
              float vj[MS], oj[MS];
#pragma unroll
              for (int s = 0; s < MS; s++) { vj[s] = val[s][j]; oj[s] = out[s][j]; }
              react_general<MS>(D, d0, vj, oj, si.pre, fq);
#pragma unroll
              for (int s = 0; s < MS; s++) out[s][j] = oj[s];
            }
          }
        }
        const unsigned fm = D.fixed_mask[d0];
#pragma unroll
        for (int s = 0; s < MS; s++) {
          if (fm >> s & 1u) {
            const float iv = D.dinit[d0][s];
#pragma unroll
            for (int j = 0; j < 4; j++) out[s][j] = iv;
          }
          if (fq >> s & 1u) {
            // the stored integers plus the increments (or the fixed value)
            const float4 raw = *reinterpret_cast<const float4*>(fc + __popc(lmask & ((1u << s) - 1u)) * so + p0);
            const float qi = D.qinv[d0][s];
            const float rw[4] = {raw.x, raw.y, raw.z, raw.w};
#pragma unroll
            for (int j = 0; j < 4; j++) out[s][j] = (fm >> s & 1u) ? q_set(out[s][j], qi) : q_add(rw[j], out[s][j], qi);
          }
        }
        if (D.dirichlet) {
#pragma unroll
          for (int j = 0; j < 4; j++)
            if ((vzy[j] | xval) != 63u) out[0][j] = D.dinit[d0][0];
        }
        // ---- stores (128-bit) ----
#pragma unroll
        for (int s = 0; s < MS; s++) {
          if (!(lmask >> s & 1u)) continue;
          float4* dst = reinterpret_cast<float4*>(D.u[((cur >> s) & 1u) ^ 1u][s] + (long long)x * D.P + p0);
          *dst = make_float4(out[s][0], out[s][1], out[s][2], out[s][3]);
        }
#ifdef CSP_FUSE_DENSITY
      } else if (group_ok) {
#else
      } else if (group_ok && (wc & 0xf8f8f8f8u) == 0u) {
#endif
        // ---- mixed-domain group: the same loads as above, domains and constants per voxel ----
        float val[MS][4];
        int dj[4], dnb[4][6];
        bool unij[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const unsigned valid = vzy[j] | xval;
          dj[j] = (wc >> (8 * j)) & DOMAIN_BITS;
          const int zmb = j > 0 ? (int)(wc >> (8 * (j > 0 ? j - 1 : 0))) : (int)ezm;
          const int zpb = j < 3 ? (int)(wc >> (8 * (j < 3 ? j + 1 : 3))) : (int)ezp;
          const int raw[6] = {zmb, zpb, (int)(wym >> (8 * j)), (int)(wyp >> (8 * j)), (int)(wp >> (8 * j)),
                              (int)(wn >> (8 * j))};
          bool u = true;
#pragma unroll
          for (int k = 0; k < 6; k++) {
            dnb[j][k] = (valid >> k & 1u) ? (raw[k] & DOMAIN_BITS) : dj[j];
            u = u && dnb[j][k] == dj[j];
          }
          unij[j] = u;
        }
        const unsigned fq = FQ & D.fixq & lmask;   // fixed-point species: out holds the increment
        int slot = 0;
#pragma unroll
        for (int s = 0; s < MS; s++) {
          if (lmask >> s & 1u) {
            const float4 a = *reinterpret_cast<const float4*>(fc + slot * so + p0);
            val[s][0] = a.x; val[s][1] = a.y; val[s][2] = a.z; val[s][3] = a.w;
            slot++;
          } else {
            val[s][0] = val[s][1] = val[s][2] = val[s][3] = 0.f;
          }
#pragma unroll
          for (int j = 0; j < 4; j++) {
            if (fq >> s & 1u) val[s][j] = q_value(val[s][j], D.qunit[dj[j]][s]);
            out[s][j] = (fq >> s & 1u) ? 0.f : val[s][j];
          }
        }
        slot = 0;
#pragma unroll
        for (int s = 0; s < MS; s++) {
          if (!(lmask >> s & 1u)) continue;
          const int so_s = slot * so;
          slot++;
          if (!(si.pre >> s & 1u)) continue;
          const float* cs = D.coef[D.dsi_of[s]];
          // out-of-box neighbours are read at the voxel itself (as in the uniform path)
          const float4 vp = *reinterpret_cast<const float4*>(fp + so_s + p0);
          const float4 vn = *reinterpret_cast<const float4*>(fn + so_s + p0);
          const float pv[4] = {vp.x, vp.y, vp.z, vp.w};
          const float nv[4] = {vn.x, vn.y, vn.z, vn.w};
          const float zm = fc[so_s + ((vzy[0] & 1u) ? p0 - 1 : p0)];
          const float zp = fc[so_s + ((vzy[3] & 2u) ? p0 + 4 : p0 + 3)];
#ifndef CSP_FUSE_DENSITY
          // two voxels per instruction: the uniform form and the per-neighbour-coefficient
          // form (diffuse_coef6) on the pair, then per voxel the one its neighbourhood calls
          // for -- each lane rounds exactly as the scalar functions do
          float unbv[4][6];
#pragma unroll
          for (int j = 0; j < 4; j++) {
            const unsigned valid = vzy[j] | xval;
            const float u = val[s][j];
            unbv[j][0] = j > 0 ? val[s][j > 0 ? j - 1 : 0] : zm;
            unbv[j][1] = j < 3 ? val[s][j < 3 ? j + 1 : 3] : zp;
            if (!yvec) {
              unbv[j][0] = (valid & 1u) ? unbv[j][0] : u;
              unbv[j][1] = (valid & 2u) ? unbv[j][1] : u;
            }
            unbv[j][2] = fc[so_s + ((valid & 4u) ? p0 + j - nz : p0 + j)];
            unbv[j][3] = fc[so_s + ((valid & 8u) ? p0 + j + nz : p0 + j)];
            unbv[j][4] = pv[j];
            unbv[j][5] = nv[j];
          }
          const F2 m2 = f2(-2.f, -2.f), zero2 = f2(0.f, 0.f);
#pragma unroll
          for (int q = 0; q < 2; q++) {
            const int ja = 2 * q, jb = 2 * q + 1;
            const F2 u2 = f2(val[s][ja], val[s][jb]);
            const float* ca = cs + dj[ja] * ND;
            const float* cb = cs + dj[jb] * ND;
            const F2 cu = f2(ca[dj[ja]], cb[dj[jb]]);
            const F2 zs = f2(__fadd_rn(unbv[ja][0], unbv[ja][1]), __fadd_rn(unbv[jb][0], unbv[jb][1]));
            const F2 ys = f2_add(f2(unbv[ja][2], unbv[jb][2]), f2(unbv[ja][3], unbv[jb][3]));
            const F2 xs = f2_add(f2(unbv[ja][4], unbv[jb][4]), f2(unbv[ja][5], unbv[jb][5]));
            const F2 ru = diffuse_uniform2(cu, m2, u2, zs, ys, xs);
            F2 a = zero2;
#pragma unroll
            for (int kk = 0; kk < 6; kk++)
              a = f2_fma(f2(ca[dnb[ja][kk]], cb[dnb[jb][kk]]), f2_sub(f2(unbv[ja][kk], unbv[jb][kk]), u2), a);
            const F2 rg = f2_add(u2, a);
            float ua, ub, ga, gb;
            f2_split(ru, ua, ub);
            f2_split(rg, ga, gb);
            out[s][ja] = unij[ja] ? ua : ga;
            out[s][jb] = unij[jb] ? ub : gb;
          }
#else
#pragma unroll
          for (int j = 0; j < 4; j++) {
            const unsigned valid = vzy[j] | xval;
            const float u = val[s][j];
            const float ym = fc[so_s + ((valid & 4u) ? p0 + j - nz : p0 + j)];
            const float yp = fc[so_s + ((valid & 8u) ? p0 + j + nz : p0 + j)];
            float unb[6];
            unb[0] = j > 0 ? val[s][j > 0 ? j - 1 : 0] : zm;
            unb[1] = j < 3 ? val[s][j < 3 ? j + 1 : 3] : zp;
            if (!yvec) {   // the group may straddle a row end: in-group z neighbours per voxel
              unb[0] = (valid & 1u) ? unb[0] : u;
              unb[1] = (valid & 2u) ? unb[1] : u;
            }
            unb[2] = ym; unb[3] = yp; unb[4] = pv[j]; unb[5] = nv[j];
            const float* c = cs + dj[j] * ND;
            out[s][j] = unij[j] ? diffuse_uniform(c[dj[j]], u, unb) : diffuse_general(c, dnb[j], u, unb);
#ifdef CSP_FUSE_DENSITY
            const int pat = (int)((wc >> (8 * j + 3)) & 0x1fu);
            if (pat) {   // density-boundary fluxes, as in voxel_update
              double acc = 0.0;
              bool any = false;
#pragma unroll
              for (int k = 0; k < 6; k++) {
                const int code = D.fpat[pat][k];
                if (!code) continue;
                const int fs = (code & 0x7f) - 1;
                if (D.fslot_species[fs] != s) continue;
                const double self = (double)u + D.base[dj[j]][s], other = (double)unb[k] + D.base[dnb[j][k]][s];
                if (code & 0x80) acc += pair_flux(D, fs, other, self);
                else acc -= pair_flux(D, fs, self, other);
                any = true;
              }
              if (any) out[s][j] = (float)((double)out[s][j] + acc);
            }
#endif
          }
#endif
        }
        // the four voxels in one domain (usual next to a domain sheet): the group form of
        // the buffer reactions, as in the uniform path
        const bool one_dom = dj[0] == dj[1] && dj[1] == dj[2] && dj[2] == dj[3];
        if (si.react && si.react_fast && one_dom) {
          const int d = dj[0];
          F2 o2[MS][2];
#pragma unroll
          for (int s = 0; s < MS; s++) {
            o2[s][0] = f2(out[s][0], out[s][1]);
            o2[s][1] = f2(out[s][2], out[s][3]);
          }
          const F2 dca0 = f2(val[0][0], val[0][1]), dca1 = f2(val[0][2], val[0][3]);
          const float cb = D.fbase[d][0];
          const F2 ca0 = f2_add(f2(cb, cb), dca0), ca1 = f2_add(f2(cb, cb), dca1);
          const unsigned rm = D.rmask[d];
          F2 G0 = f2(0.f, 0.f), G1 = G0;    // SUR: sums of the increments
#pragma unroll
          for (int s = 1; s < MS; s++) {
            if (!(rm >> s & 1u)) continue;
            const float4 kk = D.rk[d][s];
            const F2 nkon = f2(kk.x, kk.x), nkoff = f2(kk.y, kk.y), a = f2(kk.z, kk.z), j0 = f2(kk.w, kk.w);
            const F2 dj0 = buffer_dj2(nkon, nkoff, a, j0, f2(val[s][0], val[s][1]), dca0, ca0);
            const F2 dj1 = buffer_dj2(nkon, nkoff, a, j0, f2(val[s][2], val[s][3]), dca1, ca1);
            o2[s][0] = f2_add(o2[s][0], dj0);
            o2[s][1] = f2_add(o2[s][1], dj1);
            o2[0][0] = f2_sub(o2[0][0], dj0);
            o2[0][1] = f2_sub(o2[0][1], dj1);
            if (SUR) {
              G0 = f2_add(G0, dj0);
              G1 = f2_add(G1, dj1);
            }
          }
#pragma unroll
          for (int s = 0; s < MS; s++) {
            f2_split(o2[s][0], out[s][0], out[s][1]);
            f2_split(o2[s][1], out[s][2], out[s][3]);
          }
          if (SUR && D.sur)
            *reinterpret_cast<unsigned*>(D.rx_class + (long long)x * D.P + p0) =
                rx_classify4<MS>(D, d, ca0, ca1, val, G0, G1);
        }
        unsigned cls4 = 0;   // SUR, per-voxel reactions: the group's class bytes
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int d = dj[j];
          if (si.react && !(si.react_fast && one_dom)) {
            if (si.react_fast) {
              const float ca = __fadd_rn(D.fbase[d][0], val[0][j]);
              if (SUR && D.sur) {
                float vj[MS];
#pragma unroll
                for (int s = 0; s < MS; s++) vj[s] = val[s][j];
                cls4 |= rx_classify<MS>(D, d, ca, vj) << (8 * j);
              }
              const unsigned rm = D.rmask[d];
#pragma unroll
              for (int s = 1; s < MS; s++) {
                if (!(rm >> s & 1u)) continue;
                const float4 kk = D.rk[d][s];
                const float dJ = buffer_dj(kk.x, kk.y, kk.z, kk.w, val[s][j], val[0][j], ca);
                out[s][j] = __fadd_rn(out[s][j], dJ);
                out[0][j] = __fsub_rn(out[0][j], dJ);
              }
            } else {
              float vj[MS], oj[MS];
#pragma unroll
              for (int s = 0; s < MS; s++) { vj[s] = val[s][j]; oj[s] = out[s][j]; }
              react_general<MS>(D, d, vj, oj, si.pre, fq);
#pragma unroll
              for (int s = 0; s < MS; s++) out[s][j] = oj[s];
            }
          }
          const unsigned fm = D.fixed_mask[d];
#pragma unroll
          for (int s = 0; s < MS; s++) {
            if (fm >> s & 1u) out[s][j] = D.dinit[d][s];
            if (fq >> s & 1u) {
              const float rw = fc[__popc(lmask & ((1u << s) - 1u)) * so + p0 + j];
              out[s][j] = (fm >> s & 1u) ? q_set(out[s][j], D.qinv[d][s]) : q_add(rw, out[s][j], D.qinv[d][s]);
            }
          }
          if (D.dirichlet && (vzy[j] | xval) != 63u) out[0][j] = D.dinit[d][0];
        }
        if (SUR && D.sur && si.react_fast && !one_dom)
          *reinterpret_cast<unsigned*>(D.rx_class + (long long)x * D.P + p0) = cls4;
#pragma unroll
        for (int s = 0; s < MS; s++) {
          if (!(lmask >> s & 1u)) continue;
          float4* dst = reinterpret_cast<float4*>(D.u[((cur >> s) & 1u) ^ 1u][s] + (long long)x * D.P + p0);
          *dst = make_float4(out[s][0], out[s][1], out[s][2], out[s][3]);
        }
      } else {
        // ---- general path: per voxel, straight from the staged planes (kept small:
        // the 4 positions are not unrolled) ----
#pragma unroll 1
        for (int j = 0; j < 4; j++) {
          const int pj = p0 + j;
          if (pj >= plane) break;
          const unsigned valid = vzy[j] | xval;
          // out-of-box neighbours read the voxel itself (addresses stay inside the stage)
          const int ia[4] = {(valid & 1u) ? pj - 1 : pj, (valid & 2u) ? pj + 1 : pj,
                             (valid & 4u) ? pj - nz : pj, (valid & 8u) ? pj + nz : pj};
          auto ld = [&](int s, int kk) -> float {
            const int so_s = __popc(lmask & ((1u << s) - 1u)) * so;
            if (kk == 6) return fc[so_s + pj];
            if (kk == 4) return fp[so_s + pj];
            if (kk == 5) return fn[so_s + pj];
            return fc[so_s + ia[kk]];
          };
          auto ldd = [&](int kk) -> int {
            if (kk == 6) return dc[pj];
            if (kk == 4) return dp[pj];
            if (kk == 5) return dnx[pj];
            return dc[ia[kk]];
          };
          float oj[MS];
          unsigned cls = RX_CLASS_NONE;
          voxel_update<MS, SUR>(D, si, valid, valid != 63u, ld, ldd, oj, &cls);
#pragma unroll
          for (int s = 0; s < MS; s++)
            if (lmask >> s & 1u) D.u[((cur >> s) & 1u) ^ 1u][s][(long long)x * D.P + pj] = oj[s];
          if (SUR && D.sur && si.react_fast) D.rx_class[(long long)x * D.P + pj] = (unsigned char)cls;
        }
      }
      // plane x-1 is no longer needed: refill its stage with plane x-1+NST.  The barrier
      // also takes the CTA's one decision on the waits of this plane: if any thread gave
      // up, every thread leaves the loop here (plane x's outputs are then undefined)
      if (__syncthreads_or(timeout ? 1 : 0)) { cta_timeout = true; break; }
      if (tid == 0 && has_prev && x - 1 >= ql) {
        const int qn = x - 1 + NST;
        if (qn <= qh) {
          fence_proxy_async();
          const int st = (x - 1 - ql) % NST;
          issue_plane(D, cur, lmask, qn, st, ring, g, smem_u32(&bars[st]), lo, hi, lob, hib);
          pending |= 1u << st;
        }
      }
    }
    if (cta_timeout) {
      if (tid == 0) {
        // no bulk copy may still be writing this CTA's shared memory when it exits
        for (int st = 0; st < NST; st++)
          if (pending >> st & 1u) mbar_wait_bounded(smem_u32(&bars[st]), (phase >> st) & 1u, WAIT_NS);
        atomicOr(err, ERR_TIMEOUT);
      }
      __syncthreads();
      return;
    }
    __syncthreads();
  }
}

// Launch over the work units [u0, u1) (all units: one step of every realisation; the units
// of a range of realisations: one step of those only).
template <int MS, int T, bool INJ, unsigned FQ, bool SUR>
cudaError_t staged_launch_t(const StagedPlan& pl, int u0, int u1, const RealDesc* d, RealCtl* c, int* e,
                            cudaStream_t s) {
  if (u1 <= u0) return cudaSuccess;
  StagedGeom g = pl.g;
  g.nunits = u1 - u0;
  k_voxels_staged<MS, T, INJ, FQ, SUR><<<std::min(g.nunits, pl.slots), T, g.smem, s>>>(d, c, pl.d_units + u0, g, e);
  return cudaGetLastError();
}

template <int MS, int T, unsigned FQ, bool WITH_INJ>
cudaError_t staged_configure(StagedPlan& pl) {
  cudaError_t e = cudaFuncSetAttribute(k_voxels_staged<MS, T, false, FQ, false>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, pl.g.smem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_voxels_staged<MS, T, false, FQ, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           pl.g.smem);
  if (e != cudaSuccess) return e;
  if (WITH_INJ) {
    e = cudaFuncSetAttribute(k_voxels_staged<MS, T, WITH_INJ, FQ, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             pl.g.smem);
    if (e != cudaSuccess) return e;
  }
  int per_sm = 0, per_sm_sur = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_voxels_staged<MS, T, false, FQ, false>, T, pl.g.smem);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_sur, k_voxels_staged<MS, T, false, FQ, true>, T,
                                                    pl.g.smem);
  if (e != cudaSuccess) return e;
  per_sm = std::min(per_sm, per_sm_sur);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  pl.slots = per_sm * sms;
  pl.launch = &staged_launch_t<MS, T, false, FQ, false>;
  pl.launch_sur = &staged_launch_t<MS, T, false, FQ, true>;
  pl.launch_inject = WITH_INJ ? &staged_launch_t<MS, T, WITH_INJ, FQ, false> : nullptr;
  return cudaSuccess;
}

// Host: tile geometry and work units for a batch.  seg = x planes per unit.
inline StagedPlan staged_plan(const std::vector<RealDesc>& descs, int T = 256, int seg = 0) {
  StagedPlan pl;
  pl.T = T;
  int nz_max = 0, ns_max = 0;
  for (const RealDesc& D : descs) {
    nz_max = std::max(nz_max, D.nz);
    ns_max = std::max(ns_max, D.ns);
    pl.fixq |= D.fixq;
  }
  StagedGeom& g = pl.g;
  g.L = 4 * T;
  g.slot = (g.L + 2 * nz_max + 8 + 3) & ~3;
  g.domcap = (g.L + 2 * nz_max + 32 + 15) & ~15;
  g.ms = ns_max <= 5 ? 5 : 8;
  g.stage_bytes = ((g.ms * g.slot * 4 + g.domcap) + 127) & ~127;
  g.desc_off = 128;
  g.ring_off = (g.desc_off + (int)sizeof(RealDesc) + 127) & ~127;
  g.smem = g.ring_off + NST * g.stage_bytes;
  if (g.smem > 227 * 1024) return pl;   // plane halo too large for the ring
  // units: (r, x segment, chunk) order keeps the chunks of one x range together
  long long total_planes = 0;
  for (const RealDesc& D : descs) total_planes += D.nx * (long long)((D.plane + g.L - 1) / g.L);
  if (seg <= 0) {
    // aim for >= 8 units per resident CTA slot (148 SMs x 2), segments of 12..64 planes
    const long long want = 148 * 2 * 8;
    seg = (int)std::max<long long>(12, std::min<long long>(64, total_planes / std::max<long long>(1, want)));
  }
  g.seg = seg;
  std::vector<int4> units;
  pl.unit_first.assign(descs.size() + 1, 0);
  for (int r = 0; r < (int)descs.size(); r++) {
    const RealDesc& D = descs[r];
    const int nch = (D.plane + g.L - 1) / g.L;
    pl.unit_first[r] = (int)units.size();
    for (int x0 = 0; x0 < D.nx; x0 += seg)
      for (int c = 0; c < nch; c++) units.push_back(make_int4(r, c, x0, std::min(D.nx, x0 + seg)));
  }
  pl.unit_first[descs.size()] = (int)units.size();
  pl.nunits = (int)units.size();
  g.nunits = pl.nunits;
  if (cudaMalloc(&pl.d_units, units.size() * sizeof(int4)) != cudaSuccess) return pl;
  if (cudaMemcpy(pl.d_units, units.data(), units.size() * sizeof(int4), cudaMemcpyHostToDevice) != cudaSuccess) return pl;
  pl.ok = true;
  return pl;
}

// The kernel variants built: five species with fixed point only for species 4 (the
// reference model: TRPN), at 256 and 128 threads (the first with the test hook); five
// species with any of species 1-4 fixed; eight species with any of 1-7 fixed.
inline cudaError_t staged_prepare(StagedPlan& pl) {
  if (!pl.ok) return cudaErrorNotSupported;
  cudaError_t e = cudaErrorNotSupported;
  const bool only4 = (pl.fixq & ~(1u << 4)) == 0;
  if (pl.g.ms == 5 && only4)
    e = pl.T == 128 ? staged_configure<5, 128, 1u << 4, false>(pl) : staged_configure<5, 256, 1u << 4, true>(pl);
  else if (pl.g.ms == 5 && pl.T == 256)
    e = staged_configure<5, 256, 0x1Eu, false>(pl);
  else if (pl.T == 256)
    e = staged_configure<8, 256, 0xFEu, false>(pl);
  if (e != cudaSuccess) pl.ok = false;
  return e;
}

// One step of the realisations [r0, r1) (default: all); sur: the variant that classifies
// voxels for the reaction surrogate.
inline void staged_launch(const StagedPlan& pl, const RealDesc* d, RealCtl* c, int* e, cudaStream_t s,
                          bool inject = false, int r0 = 0, int r1 = -1, bool sur = false) {
  if (r1 < 0) r1 = (int)pl.unit_first.size() - 1;
  (inject && pl.launch_inject ? pl.launch_inject : sur ? pl.launch_sur : pl.launch)(pl, pl.unit_first[r0],
                                                                                   pl.unit_first[r1], d, c, e, s);
}

inline void staged_release(StagedPlan& pl) {
  if (pl.d_units) cudaFree(pl.d_units);
  pl.d_units = nullptr;
  pl.ok = false;
}

}  // namespace csp
