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
// Every mbarrier wait is bounded: after WAIT_LIMIT polls the kernel sets ERR_TIMEOUT in
// the device error word and leaves the unit.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "csp_kernels.cuh"

namespace csp {

constexpr int NST = 5;                    // ring stages: planes x-1, x, x+1 resident, 2 in flight
constexpr long long WAIT_LIMIT = 1ll << 26;

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

struct StagedPlan {
  bool ok = false;
  int T = 256;
  int ctas = 0;
  StagedGeom g{};
  int4* d_units = nullptr;      // (r, c, x0, x1)
  int nunits = 0;
  cudaError_t (*launch)(const StagedPlan&, const RealDesc*, RealCtl*, int*, cudaStream_t) = nullptr;
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

template <int MS, int T>
__global__ void __launch_bounds__(T, 1) k_voxels_staged(const RealDesc* __restrict__ descs, RealCtl* __restrict__ ctl,
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
    for (int i = 0; i < NST; i++) mbar_init(smem_u32(&bars[i]), 1);
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
    bool inb[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int p = p0 + j;
      inb[j] = p < plane;
      const int y = p / nz, z = p - y * nz;
      vzy[j] = (z > 0 ? 1u : 0u) | (z < nz - 1 ? 2u : 0u) | (y > 0 ? 4u : 0u) | (y < D.ny - 1 ? 8u : 0u);
    }
    // smem slot of every loaded species (popcount rank in lmask)
    int slot_of[MS];
#pragma unroll
    for (int s = 0; s < MS; s++) slot_of[s] = __popc(lmask & ((1u << s) - 1u));

    if (tid == 0) {
      fence_proxy_async();
      for (int q = ql; q <= min(qh, ql + NST - 1); q++) {
        const int st = (q - ql) % NST;
        issue_plane(D, cur, lmask, q, st, ring, g, smem_u32(&bars[st]), lo, hi, lob, hib);
      }
    }
    bool timeout = false;
    auto wait_plane = [&](int q) {
      const int st = (q - ql) % NST;
      const unsigned par = (phase >> st) & 1u;
      long long n = 0;
      while (!mbar_try_wait(smem_u32(&bars[st]), par)) {
        if (++n > WAIT_LIMIT) { timeout = true; break; }
      }
      phase ^= 1u << st;
    };
    auto stage_of = [&](int q) -> const unsigned char* { return ring + (size_t)((q - ql) % NST) * g.stage_bytes; };

    if (x0 > 0) wait_plane(x0 - 1);
    wait_plane(x0);
    for (int x = x0; x < x1; x++) {
      const bool has_prev = x > 0, has_next = x + 1 < nx;
      if (has_next) wait_plane(x + 1);
      if (timeout) break;
      const unsigned char* sc = stage_of(x);
      const unsigned char* sp = has_prev ? stage_of(x - 1) : sc;
      const unsigned char* sn = has_next ? stage_of(x + 1) : sc;
      const float* fc = reinterpret_cast<const float*>(sc) - lo;
      const float* fp = reinterpret_cast<const float*>(sp) - lo;
      const float* fn = reinterpret_cast<const float*>(sn) - lo;
      const unsigned char* dc = sc + (size_t)g.ms * g.slot * 4 - lob;
      const unsigned char* dp = sp + (size_t)g.ms * g.slot * 4 - lob;
      const unsigned char* dnp = sn + (size_t)g.ms * g.slot * 4 - lob;
      const int so = g.slot;
      // own positions of planes x-1, x, x+1: 128-bit shared loads
      float vc[MS][4], vp[MS][4], vn[MS][4];
#pragma unroll
      for (int s = 0; s < MS; s++) {
        if (lmask >> s & 1u) {
          const int o = slot_of[s] * so + p0;
          const float4 a = *reinterpret_cast<const float4*>(fc + o);
          vc[s][0] = a.x; vc[s][1] = a.y; vc[s][2] = a.z; vc[s][3] = a.w;
          if (si.pre >> s & 1u) {
            const float4 b = *reinterpret_cast<const float4*>(fp + o);
            const float4 e = *reinterpret_cast<const float4*>(fn + o);
            vp[s][0] = b.x; vp[s][1] = b.y; vp[s][2] = b.z; vp[s][3] = b.w;
            vn[s][0] = e.x; vn[s][1] = e.y; vn[s][2] = e.z; vn[s][3] = e.w;
          } else {
#pragma unroll
            for (int j = 0; j < 4; j++) vp[s][j] = vn[s][j] = 0.f;
          }
        } else {
#pragma unroll
          for (int j = 0; j < 4; j++) vc[s][j] = vp[s][j] = vn[s][j] = 0.f;
        }
      }
      const unsigned wc = *reinterpret_cast<const unsigned*>(dc + p0);
      const unsigned wp = *reinterpret_cast<const unsigned*>(dp + p0);
      const unsigned wn = *reinterpret_cast<const unsigned*>(dnp + p0);
      const unsigned xval = (has_prev ? 16u : 0u) | (has_next ? 32u : 0u);
      float outv[4][MS];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const unsigned valid = vzy[j] | xval;
        const bool on_face = valid != 63u;
        const int pj = p0 + j;
        auto ld = [&](int s, int kk) -> float {
          switch (kk) {
            case 6: return vc[s][j];
            case 4: return vp[s][j];
            case 5: return vn[s][j];
            // out-of-box neighbours read the voxel itself (addresses stay inside the stage)
            case 0: return j > 0 ? vc[s][j > 0 ? j - 1 : 0] : fc[slot_of[s] * so + ((valid & 1u) ? pj - 1 : pj)];
            case 1: return j < 3 ? vc[s][j < 3 ? j + 1 : 3] : fc[slot_of[s] * so + ((valid & 2u) ? pj + 1 : pj)];
            case 2: return fc[slot_of[s] * so + ((valid & 4u) ? pj - nz : pj)];
            default: return fc[slot_of[s] * so + ((valid & 8u) ? pj + nz : pj)];
          }
        };
        auto ldd = [&](int kk) -> int {
          switch (kk) {
            case 6: return (wc >> (8 * j)) & 0xff;
            case 4: return (wp >> (8 * j)) & 0xff;
            case 5: return (wn >> (8 * j)) & 0xff;
            case 0: return j > 0 ? (wc >> (8 * (j > 0 ? j - 1 : 0))) & 0xff : dc[(valid & 1u) ? pj - 1 : pj];
            case 1: return j < 3 ? (wc >> (8 * (j < 3 ? j + 1 : 3))) & 0xff : dc[(valid & 2u) ? pj + 1 : pj];
            case 2: return dc[(valid & 4u) ? pj - nz : pj];
            default: return dc[(valid & 8u) ? pj + nz : pj];
          }
        };
        if (inb[j]) {
          voxel_update<MS>(D, si, valid, on_face, ld, ldd, outv[j]);
        } else {
#pragma unroll
          for (int s = 0; s < MS; s++) outv[j][s] = 0.f;
        }
      }
      const long long base = (long long)x * D.P + p0;
      const bool full = p0 + 3 < plane;
#pragma unroll
      for (int s = 0; s < MS; s++) {
        if (!(lmask >> s & 1u)) continue;
        float* dst = D.u[((cur >> s) & 1u) ^ 1u][s] + base;
        if (full) {
          *reinterpret_cast<float4*>(dst) = make_float4(outv[0][s], outv[1][s], outv[2][s], outv[3][s]);
        } else {
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (inb[j]) dst[j] = outv[j][s];
        }
      }
      // plane x-1 is no longer needed: refill its stage with plane x-1+NST
      __syncthreads();
      if (tid == 0 && has_prev && x - 1 >= ql) {
        const int qn = x - 1 + NST;
        if (qn <= qh) {
          fence_proxy_async();
          issue_plane(D, cur, lmask, qn, (x - 1 - ql) % NST, ring, g, smem_u32(&bars[(x - 1 - ql) % NST]), lo, hi,
                      lob, hib);
        }
      }
    }
    if (timeout) {
      if (tid == 0) atomicOr(err, ERR_TIMEOUT);
      __syncthreads();
      return;   // ring state is unknown: leave the kernel
    }
    __syncthreads();
  }
}

template <int MS, int T>
cudaError_t staged_launch_t(const StagedPlan& pl, const RealDesc* d, RealCtl* c, int* e, cudaStream_t s) {
  k_voxels_staged<MS, T><<<pl.ctas, T, pl.g.smem, s>>>(d, c, pl.d_units, pl.g, e);
  return cudaGetLastError();
}

template <int MS, int T>
cudaError_t staged_configure(StagedPlan& pl) {
  cudaError_t e = cudaFuncSetAttribute(k_voxels_staged<MS, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, pl.g.smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_voxels_staged<MS, T>, T, pl.g.smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  pl.ctas = std::min(pl.nunits, per_sm * sms);
  pl.launch = &staged_launch_t<MS, T>;
  return cudaSuccess;
}

// Host: tile geometry and work units for a batch.  seg = x planes per unit.
inline StagedPlan staged_plan(const std::vector<RealDesc>& descs, int T = 256, int seg = 0) {
  StagedPlan pl;
  pl.T = T;
  int nz_max = 0, ns_max = 0;
  for (const RealDesc& D : descs) { nz_max = std::max(nz_max, D.nz); ns_max = std::max(ns_max, D.ns); }
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
  for (int r = 0; r < (int)descs.size(); r++) {
    const RealDesc& D = descs[r];
    const int nch = (D.plane + g.L - 1) / g.L;
    for (int x0 = 0; x0 < D.nx; x0 += seg)
      for (int c = 0; c < nch; c++) units.push_back(make_int4(r, c, x0, std::min(D.nx, x0 + seg)));
  }
  pl.nunits = (int)units.size();
  g.nunits = pl.nunits;
  if (cudaMalloc(&pl.d_units, units.size() * sizeof(int4)) != cudaSuccess) return pl;
  if (cudaMemcpy(pl.d_units, units.data(), units.size() * sizeof(int4), cudaMemcpyHostToDevice) != cudaSuccess) return pl;
  pl.ok = true;
  return pl;
}

inline cudaError_t staged_prepare(StagedPlan& pl) {
  if (!pl.ok) return cudaErrorNotSupported;
  cudaError_t e;
  if (pl.g.ms == 5) e = pl.T == 128 ? staged_configure<5, 128>(pl) : staged_configure<5, 256>(pl);
  else e = pl.T == 128 ? staged_configure<8, 128>(pl) : staged_configure<8, 256>(pl);
  if (e != cudaSuccess) pl.ok = false;
  return e;
}

inline void staged_launch(const StagedPlan& pl, const RealDesc* d, RealCtl* c, int* e, cudaStream_t s) {
  pl.launch(pl, d, c, e, s);
}

inline void staged_release(StagedPlan& pl) {
  if (pl.d_units) cudaFree(pl.d_units);
  pl.d_units = nullptr;
  pl.ok = false;
}

}  // namespace csp
