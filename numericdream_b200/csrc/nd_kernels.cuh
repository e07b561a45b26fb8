// Sphere-tracing kernels for sm_100a: the plain per-ray launch and the persistent
// wavefront kernel with warp-ballot refill.  Included once per formula (or per
// formula group) by the translated sources, which instantiate the launchers.  The
// ray program itself (march_to, normals, orbit trap, shadow) is in nd_rayprog.h.
#pragma once

#include <cuda_runtime.h>

#include <string.h>

#include <algorithm>

#include "nd_rayprog.h"
#include "nd_adjoint.cuh"

namespace nd {

__device__ __forceinline__ int64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return int64_t(t);
}

__device__ __forceinline__ void flush_stats(Stats* s, unsigned long long rays, unsigned long long m,
                                            unsigned long long nn, unsigned long long sh, unsigned long long hits,
                                            unsigned long long refills) {
  // warp reduction then one atomic per warp
  for (int o = 16; o > 0; o >>= 1) {
    rays += __shfl_xor_sync(0xffffffffu, rays, o);
    m += __shfl_xor_sync(0xffffffffu, m, o);
    nn += __shfl_xor_sync(0xffffffffu, nn, o);
    sh += __shfl_xor_sync(0xffffffffu, sh, o);
    hits += __shfl_xor_sync(0xffffffffu, hits, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&s->rays, rays);
    atomicAdd(&s->march_evals, m);
    atomicAdd(&s->normal_evals, nn);
    atomicAdd(&s->shadow_evals, sh);
    atomicAdd(&s->de_evals, m + nn + sh);
    atomicAdd(&s->hits, hits);
    atomicAdd(&s->refills, refills);
  }
}

// Residency the kernels are compiled for: 7 blocks of 128 threads per SM with an
// FP32 DE (at most 72 registers per thread; measured 4 % faster than 8 x 64 on the
// batched benchmark, where 64 registers spill the ray state), 4 with an FP64 DE.
template <class T> struct MinBlocks {
  static constexpr int value = sizeof(T) == 4 ? 7 : 4;
};
// The batched FP32 march that defers its shading (the forward calls) carries no
// normal or shadow state and fits in fewer registers.
#ifndef ND_MARCH_MIN_BLOCKS_F32
#define ND_MARCH_MIN_BLOCKS_F32 8
#endif
#ifndef ND_MARCH_MIN_BLOCKS_F64
#define ND_MARCH_MIN_BLOCKS_F64 4
#endif
template <class T, bool kBatched, bool kDefer> struct MarchBlocks {
  static constexpr int value = (sizeof(T) == 4 && kBatched && kDefer) ? ND_MARCH_MIN_BLOCKS_F32
                               : (sizeof(T) == 8 && kDefer)            ? ND_MARCH_MIN_BLOCKS_F64
                                                                       : MinBlocks<T>::value;
};

// --------------------------------------------------------------- plain kernel
// The reference's per-pixel program as a plain per-view launch: one thread per
// ray, the march loop of march_to, then the normal taps of estimate_normal, then
// the shadow loop of visibility_march, each loop running until its slowest lane
// in the warp is done (fs_simple tpl:4522-4538 / simple_geometry tpl:4492-4507).
template <class Set, class T, bool kDir64>
__global__ void __launch_bounds__(128, MinBlocks<T>::value) plain_kernel(const __grid_constant__ LaunchArgs a,
                                                    const __grid_constant__ DevView v) {
  const int64_t local = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;  // ray index inside the view
  unsigned long long rays = 0, hits = 0, m = 0, nn = 0, sh = 0;
  if (local < v.rays) {
    Lane<T, kDir64> L;
    L.start(v, int32_t(v.ray_offset + local), 0);
    if (L.phase == PH_DONE) L.finish(v, a.out, a.t_hit, 1.0f);
    while (L.phase == PH_MARCH) {
      const DEOut<T> de = Set::template de<T>(v.code, to_t<T>(L.sample_pos(v)), v);
      L.advance(v, de, a.out, a.t_hit);
    }
    m = L.evals;
    while (L.phase == PH_NORMAL) {
      const DEOut<T> de = Set::template de<T>(v.code, to_t<T>(L.sample_pos(v)), v);
      L.advance(v, de, a.out, a.t_hit);
    }
    nn = L.evals - m;
    while (L.phase == PH_SHADOW) {
      const DEOut<T> de = Set::template de<T>(v.code, to_t<T>(L.sample_pos(v)), v);
      L.advance(v, de, a.out, a.t_hit);
    }
    sh = L.evals - m - nn;
    rays = 1;
    hits = L.hit ? 1 : 0;
  }
  flush_stats(a.stats, rays, m, nn, sh, hits, 0);
}

// --------------------------------------------------------------- persistent kernel
// One resident grid; every warp keeps 32 rays in flight.  After each DE
// evaluation the warp ballots its idle lanes; once at least refill_threshold
// lanes are idle (or all are) it hands them the next ray indices by popc-prefix
// rank.  The indices come from a warp-private run of `chunk` consecutive rays that
// the warp takes from the global work counter with ONE atomicAdd whenever the run
// is used up, so most refills touch no global atomic (the reference reserves
// queue slots with workgroup-aggregated atomics instead, wf_reserve
// tpl:5083-5105), and a warp keeps marching neighbouring pixels.  Whatever phase
// a lane is in, each pass of the loop is one DE evaluation for every busy lane.

// kBlock: threads per block (the autotuner's block-size axis); every block size is
// compiled for the same threads per SM, and so the same registers per thread.
// kDefer: hit rays end at their hit and go to the hit list for the surface pass (the
// forward calls); without it (the no-allocation entry point, which has no per-ray
// scratch) the normal and shadow phases run inside the march.
template <class Set, class T, bool kDir64, bool kBatched, bool kScenes = false, bool kAccel = false,
          int kBlock = 128, bool kDefer = true>
__global__ void __launch_bounds__(kBlock, MarchBlocks<T, kBatched, kDefer>::value * 128 / kBlock)
    persistent_kernel(const __grid_constant__ LaunchArgs a, const __grid_constant__ DevView single) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  Lane<T, kDir64> L;
  L.item = -1;
  L.view = 0;
  L.phase = PH_DONE;
  L.evals = 0;
  L.hit = false;
  L.lazy = true;
  L.pending = 0;
  uint32_t rays = 0, hits = 0, ev_m = 0, ev_n = 0, ev_s = 0, refills = 0;
  const int64_t deadline = __shfl_sync(full, globaltimer_ns(), 0) + a.deadline_ns;
  int tick = 0;
  const int32_t total = int32_t(a.total_rays);  // < 2^31 (checked by the host)
  WarpRuns runs;  // warp-uniform
  const int thr = a.refill_threshold;
  constexpr bool defer = kDefer;
  // Finished rays keep their lane until the next refill: their outputs are written
  // then, all together, instead of in the pass that ends each ray.
  auto retire = [&]() {
    int32_t hit_item = -1;
    uint32_t hit_evals = 0;
    double hit_t = 0.0;
    if (L.item >= 0 && L.phase == PH_DONE) {
      const DevView& v = kBatched ? a.views[L.view] : single;
      if constexpr (kDefer) {
        // the hit distance travels in the hit list: no per-ray distance array
        L.flush_deferred(v, a.out, nullptr);
        ev_m += L.evals;
        if (L.hit) {
          hit_item = L.item;
          hit_evals = L.evals;
          hit_t = L.t;
        }
      } else {
        L.flush(v, a.out, a.t_hit);
        const uint32_t taps = L.hit ? normal_taps(v) : 0u;
        ev_m += L.mev;
        ev_n += taps;
        ev_s += L.evals - L.mev - taps;
      }
      ++rays;
      hits += L.hit ? 1 : 0;
      L.item = -1;
    }
    if constexpr (defer) {
      // append the retired hits to the shade pass's list, one atomic per warp
      const unsigned hm = __ballot_sync(full, hit_item >= 0);
      if (hm) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(a.hit_count, unsigned(__popc(hm)));
        base = __shfl_sync(full, base, 0);
        if (hit_item >= 0) a.hit_list[base + __popc(hm & lt_mask)] = HitEntry{hit_item, hit_evals, hit_t};
      }
    }
  };
  while (true) {
    // an idle lane (item < 0) is always in PH_DONE, so phase alone tells busy lanes
    const unsigned free_lanes = __ballot_sync(full, L.phase == PH_DONE);
    const int nfree = __popc(free_lanes);
    const bool have_work = runs.have_work();
    if (!have_work && free_lanes == full) {
      retire();
      break;
    }
    if (have_work && nfree != 0 && (nfree >= thr || free_lanes == full)) {
      retire();
      const unsigned idle = __ballot_sync(full, L.item < 0);
      const WarpRuns::Claim c = runs.claim(__popc(idle), a.chunk, total, [&](int take) {
        unsigned long long got = 0;
        if (lane == 0) got = atomicAdd(a.counter, (unsigned long long)take);
        return uint64_t(__shfl_sync(full, got, 0));
      });
      refills += c.fetched ? 1u : 0u;
      if (L.item < 0) {
        const int r = __popc(idle & lt_mask);
        if (r < c.used) {
          const int32_t it = c.item(r);
          L.view = kBatched ? find_view_from(a.views, a.nviews, it, L.view) : 0;
          const DevView& v = kBatched ? a.views[L.view] : single;
          L.start(v, it, L.view, true);
          if (L.phase == PH_DONE) L.finish(v, a.out, a.t_hit, 1.0f);
        }
      }
      continue;  // lanes that finished at once go back through the bookkeeping
    }
    if (((++tick) & 63) == 0) {
      // lane 0's clock decides for the whole warp, so the exit stays warp-uniform
      const int64_t now = __shfl_sync(full, globaltimer_ns(), 0);
      if (now > deadline) {
        retire();
        if (lane == 0) atomicAdd(&a.stats->timeouts, 1u);
        break;
      }
    }
    if (L.phase != PH_DONE) {
      const DevView& v = kBatched ? a.views[L.view] : single;
      bool probe = true;
      if constexpr (kAccel) {
        // the accelerator's jumps come before the probe; a ray with more jumps to take
        // than the per-pass limit takes the rest in later passes
        if (L.phase == PH_MARCH && L.probing && v.accel_levels > 0)
          probe = L.accel_skips(v, a.out, a.t_hit, a.accel_chain);
      }
      if (probe && L.phase != PH_DONE) {
        const DEOut<T> de = view_de<Set, T, false, kScenes>(v, to_t<T>(L.sample_pos(v)), a.scenes);
        L.template advance<kDefer>(v, de, a.out, a.t_hit, kDefer);
      }
    }
  }
  flush_stats(a.stats, rays, ev_m, ev_n, ev_s, hits, refills);
}

// --------------------------------------------------------------- shade pass
// Work at the hit points, after the march (the wavefront surface pass, after
// cs_wf_surface tpl:5215-5236): with a hit list (deferred shading) the normal taps,
// the Lambert level and, when asked, the orbit trap of every listed hit.  A hit whose
// view casts a shadow ray either marches it here (no shadow queue) or is appended to
// the shadow queue for the shadow kernel, which finishes the ray.  Without a hit list
// (the plain kernel) the pass computes the orbit trap of every ray that hit.  It
// strides over its work with a resident grid, warp by warp (the queue appends are
// warp-aggregated).
#ifndef ND_SHADE_MIN_BLOCKS_F32
#define ND_SHADE_MIN_BLOCKS_F32 7
#endif
template <class T> struct ShadeBlocks {
  static constexpr int value = sizeof(T) == 4 ? ND_SHADE_MIN_BLOCKS_F32 : MinBlocks<T>::value;
};
template <class Set, class T, bool kDir64, bool kBatched, bool kScenes = false, bool kAccel = false>
__global__ void __launch_bounds__(128, ShadeBlocks<T>::value)
    shade_kernel(const __grid_constant__ LaunchArgs a, const __grid_constant__ DevView single, int do_trap) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const bool list = a.hit_list != nullptr;
  const bool queue = a.shadow_queue != nullptr;
  const int64_t count = list ? int64_t(*a.hit_count) : a.total_rays;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  unsigned long long taps = 0, shadow = 0;
  for (int64_t i0 = int64_t(blockIdx.x) * blockDim.x + (threadIdx.x & ~31); i0 < count; i0 += stride) {
    const int64_t i = i0 + lane;  // the loop bound is warp-uniform: every lane takes part in the ballot
    bool want = false;
    ShadowEntry e;
    if (i < count) {
      HitEntry h{int32_t(i), 0u, 0.0};
      if (list) h = a.hit_list[i];
      const int64_t it = h.item;
      const int vi = kBatched ? find_view(a.views, a.nviews, it) : 0;
      const DevView& v = kBatched ? a.views[vi] : single;
      const int64_t local = it - v.ray_offset;
      const int64_t r = v.out_offset + local;
      const double t = list ? h.t : a.t_hit[r];
      if (t >= 0.0) {  // (all-rays mode: a miss has t < 0 and the march wrote its outputs)
        // one call site per kind of DE evaluation (normal taps, shadow steps, trap), so
        // that the formula set's code appears three times in the kernel
        Dir<kDir64> dir;
        dir.set(ray_dir(v, local));
        if (list) {
          const Surface sf = surface_at_hit<Set, T, kDir64, kScenes>(v, dir, t, r, a.out, a.scenes);
          taps += uint32_t(sf.taps);
          float vis = 1.0f;
          int sev = 0;
          if (casts_shadow(v)) {
            const D3 so = shadow_origin(sf);
            if (queue) {
              e = ShadowEntry{h.item, h.march_evals + uint32_t(sf.taps), sf.gx, sf.gy, sf.gz, 0, so.x, so.y, so.z};
              want = true;
            } else {
              vis = shadow_visibility<Set, T, kScenes, kAccel>(v, so, a.scenes, &sev);
              shadow += uint32_t(sev);
            }
          }
          if (!want)
            finish_at_hit(v, dir.get(), sf.gx, sf.gy, sf.gz, vis, h.march_evals + uint32_t(sf.taps + sev), r, a.out);
        }
        if (do_trap)
          trap_at_point<Set, T, kScenes>(v, fmadd(d3(v.org[0], v.org[1], v.org[2]), dir.get(), t), r, a.out,
                                         a.scenes);
      }
    }
    if (queue) {
      const unsigned qm = __ballot_sync(full, want);
      if (qm) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(a.shadow_count, unsigned(__popc(qm)));
        base = __shfl_sync(full, base, 0);
        if (want) a.shadow_queue[base + __popc(qm & ((1u << lane) - 1u))] = e;
      }
    }
  }
  if (list) {
    for (int o = 16; o > 0; o >>= 1) {
      taps += __shfl_xor_sync(full, taps, o);
      shadow += __shfl_xor_sync(full, shadow, o);
    }
    if (lane == 0 && taps + shadow) {
      atomicAdd(&a.stats->normal_evals, taps);
      atomicAdd(&a.stats->shadow_evals, shadow);
      atomicAdd(&a.stats->de_evals, taps + shadow);
    }
  }
}

// --------------------------------------------------------------- shadow pass
// The queued shadow rays (cs_wf_shadow tpl:5333-5346, with visibility_march
// tpl:2294-2341 for an opaque scene): a persistent kernel in which every lane
// marches one shadow ray, one DE evaluation per pass, and the warp refills its
// finished lanes from the queue by ballot and popc rank (WarpRuns, as the primary
// march), so that shadow rays of very different lengths do not idle the warp.  The
// arithmetic is shadow_visibility's, step for step, so the inline and the queued
// pass give the same bits.  At the end of a ray: the visibility, the Lambert level
// and the ray's evaluation count.
template <class Set, class T, bool kScenes = false>
__global__ void __launch_bounds__(128, MinBlocks<T>::value) shadow_kernel(const __grid_constant__ LaunchArgs a) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  const int32_t total = int32_t(*a.shadow_count);
  WarpRuns runs;
  // this lane's shadow ray
  bool busy = false;
  int32_t qi = -1, view = 0, k = 0, sev = 0;
  double ox = 0.0, oy = 0.0, oz = 0.0, dist = 0.0, res = 1.0;
  uint32_t steps_sum = 0;
  const int64_t deadline = __shfl_sync(full, globaltimer_ns(), 0) + a.deadline_ns;
  int tick = 0;
  const int thr = a.refill_threshold;
  auto finish = [&](float vis) {
    const ShadowEntry& e = a.shadow_queue[qi];
    const DevView& v = a.views[view];
    const int64_t r = v.out_offset + (int64_t(e.item) - v.ray_offset);
    // a view that casts shadow rays uses its light for the Lambert term (no ray direction)
    finish_at_hit(v, D3{0.0, 0.0, 0.0}, e.nx, e.ny, e.nz, vis, e.evals + uint32_t(sev), r, a.out);
    steps_sum += uint32_t(sev);
    busy = false;
  };
  while (true) {
    const unsigned free_lanes = __ballot_sync(full, !busy);
    const int nfree = __popc(free_lanes);
    const bool have_work = runs.have_work();
    if (!have_work && free_lanes == full) break;
    if (have_work && nfree != 0 && (nfree >= thr || free_lanes == full)) {
      const WarpRuns::Claim c = runs.claim(nfree, a.chunk, total, [&](int take) {
        unsigned long long got = 0;
        if (lane == 0) got = atomicAdd(a.shadow_counter, (unsigned long long)take);
        return uint64_t(__shfl_sync(full, got, 0));
      });
      if (!busy) {
        const int rk = __popc(free_lanes & lt_mask);
        if (rk < c.used) {
          qi = c.item(rk);
          const ShadowEntry& e = a.shadow_queue[qi];
          view = find_view_from(a.views, a.nviews, e.item, view);
          ox = e.ox;
          oy = e.oy;
          oz = e.oz;
          dist = kShadowBias;
          res = 1.0;
          k = 0;
          sev = 0;
          busy = true;
        }
      }
      continue;
    }
    if (((++tick) & 63) == 0) {
      const int64_t now = __shfl_sync(full, globaltimer_ns(), 0);
      if (now > deadline) {
        if (lane == 0) atomicAdd(&a.stats->timeouts, 1u);
        break;
      }
    }
    if (busy) {
      const DevView& v = a.views[view];
      const D3 q = fmadd(d3(ox, oy, oz), d3(v.light[0], v.light[1], v.light[2]), dist);
      const DEOut<T> de = view_de<Set, T, false, kScenes>(v, to_t<T>(q), a.scenes);
      ++sev;
      const double d = double(de.d);
      if (d < kShadowHitEps) {
        finish(0.0f);
      } else {
        res = fmin(res, double(v.shadow_k) * d / dist);
        dist += fmax(d, kShadowMinStep);
        ++k;
        const int steps = v.max_steps < kShadowMaxSteps ? v.max_steps : kShadowMaxSteps;
        if (k >= steps || dist >= 2.0 * v.max_dist) finish(float(fmin(fmax(res, 0.0), 1.0)));
      }
    }
  }
  unsigned long long s = steps_sum;
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(full, s, o);
  if (lane == 0 && s) {
    atomicAdd(&a.stats->shadow_evals, s);
    atomicAdd(&a.stats->de_evals, s);
  }
}

// --------------------------------------------------------------- launchers
struct LaunchConfig {
  int kernel;           // ND_KERNEL_PLAIN / ND_KERNEL_PERSISTENT
  int block;
  int blocks_per_sm;
  int num_sms;
};

template <class Set, class T, bool kDir64>
cudaError_t launch_plain(const LaunchArgs& a, const DevView& single, const LaunchConfig& c, cudaStream_t s) {
  const int block = 128;
  const int64_t grid = (single.rays + block - 1) / block;
  if (grid <= 0) return cudaSuccess;
  plain_kernel<Set, T, kDir64><<<unsigned(grid), block, 0, s>>>(a, single);
  return cudaGetLastError();
}

// Blocks per SM of a resident grid: the most that fit (c.blocks_per_sm 0), that many
// less (c.blocks_per_sm < 0), or the requested count clamped to what fits, so that
// every block of the persistent grid is resident at once.
template <class K> cudaError_t resident_blocks(K kernel, int block, int want, int* per_sm) {
  int fit = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, kernel, block, 0);
  if (e != cudaSuccess) return e;
  fit = std::max(fit, 1);
  *per_sm = want > 0 ? std::min(want, fit) : std::max(1, fit + want);
  return cudaSuccess;
}

template <class Set, class T, bool kDir64, bool kBatched, bool kScenes = false, bool kAccel = false,
          int kBlock = 128, bool kDefer = true>
cudaError_t launch_persistent(const LaunchArgs& a, const DevView& single, const LaunchConfig& c, cudaStream_t s) {
  const int block = kBlock;
  // the deferred march needs the hit list, the inline one must not get one
  if ((a.hit_list != nullptr) != kDefer) return cudaErrorInvalidValue;
  int per_sm = 0;
  cudaError_t e = resident_blocks(persistent_kernel<Set, T, kDir64, kBatched, kScenes, kAccel, kBlock, kDefer>,
                                  block, c.blocks_per_sm, &per_sm);
  if (e != cudaSuccess) return e;
  int64_t grid = int64_t(per_sm) * c.num_sms;
  const int64_t needed = (a.total_rays + block - 1) / block;
  if (grid > needed) grid = needed;
  if (grid <= 0) return cudaSuccess;
  // runs of up to 64 rays per warp refill, but at least ~4 runs per warp so that
  // small launches still spread over every warp
  LaunchArgs b = a;
  const int64_t warps = grid * (block / 32);
  b.chunk = int32_t(std::max<int64_t>(1, std::min<int64_t>(64, a.total_rays / (warps * 4))));
  persistent_kernel<Set, T, kDir64, kBatched, kScenes, kAccel, kBlock, kDefer><<<unsigned(grid), block, 0, s>>>(b,
                                                                                                         single);
  return cudaGetLastError();
}

typedef cudaError_t (*LaunchFn)(const LaunchArgs&, const DevView&, const LaunchConfig&, cudaStream_t);

// Blocks per SM a persistent launch would use (the clamp above) for the FP32 batched
// march at a block size: what the autotuner reports.
template <class Set, int kBlock> int resident_f32_batched(int want) {
  int per_sm = 0;
  if (resident_blocks(persistent_kernel<Set, float, false, true, false, false, kBlock>, kBlock, want, &per_sm) !=
      cudaSuccess)
    return 0;
  return per_sm;
}
typedef int (*ResidentFn)(int);

template <class Set, class T, bool kDir64, bool kBatched, bool kScenes = false, bool kAccel = false>
cudaError_t launch_shade(const LaunchArgs& a, const DevView& single, const LaunchConfig& c, int do_trap,
                         cudaStream_t s) {
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, shade_kernel<Set, T, kDir64, kBatched, kScenes, kAccel>, 128, 0);
  if (e != cudaSuccess) return e;
  int64_t grid = int64_t(std::max(per_sm, 1)) * c.num_sms;
  const int64_t needed = (a.total_rays + 127) / 128;
  if (grid > needed) grid = needed;
  if (grid <= 0) return cudaSuccess;
  shade_kernel<Set, T, kDir64, kBatched, kScenes, kAccel><<<unsigned(grid), 128, 0, s>>>(a, single, do_trap);
  return cudaGetLastError();
}

typedef cudaError_t (*ShadeFn)(const LaunchArgs&, const DevView&, const LaunchConfig&, int, cudaStream_t);

// The shadow pass over a launch's shadow queue: a resident grid (its size cannot
// depend on the queue length, which the surface pass writes on the device), runs of
// up to 16 queue entries per warp claim.
template <class Set, class T, bool kScenes = false>
cudaError_t launch_shadow(const LaunchArgs& a, const LaunchConfig& c, cudaStream_t s) {
  int per_sm = 0;
  cudaError_t e = resident_blocks(shadow_kernel<Set, T, kScenes>, 128, c.blocks_per_sm, &per_sm);
  if (e != cudaSuccess) return e;
  int64_t grid = int64_t(per_sm) * c.num_sms;
  const int64_t needed = (a.total_rays + 127) / 128;  // at most one queue entry per ray
  if (grid > needed) grid = needed;
  if (grid <= 0) return cudaSuccess;
  LaunchArgs b = a;
  b.chunk = 16;
  shadow_kernel<Set, T, kScenes><<<unsigned(grid), 128, 0, s>>>(b);
  return cudaGetLastError();
}

typedef cudaError_t (*ShadowFn)(const LaunchArgs&, const LaunchConfig&, cudaStream_t);

// --------------------------------------------------------------- lite shading
// One thread per ray of the call (resident grid, strided): misses take the view's
// background, hits lite_at_hit from the forward's depth64 / normal / trap.
template <class Set, class T, bool kDir64, bool kScenes = false>
__global__ void __launch_bounds__(128, MinBlocks<T>::value)
    lite_kernel(const __grid_constant__ LaunchArgs a, const nd_lite_desc* __restrict__ lites,
                const nd_lite_desc* __restrict__ scene_colors, float4* __restrict__ rgba) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < a.total_rays; i += stride) {
    const int vi = find_view(a.views, a.nviews, i);
    const DevView& v = a.views[vi];
    const nd_lite_desc& L = lites[vi];
    const int64_t local = i - v.ray_offset;
    const int64_t r = v.out_offset + local;
    const float4 n = reinterpret_cast<const float4*>(a.out.normal)[r];
    if (!(n.w > 0.5f)) {
      rgba[r] = make_float4(L.background[0], L.background[1], L.background[2], 0.0f);
      continue;
    }
    float rgb[3];
    lite_at_hit<Set, T, kDir64, kScenes>(v, L, local, a.out.depth64[r], n.x, n.y, n.z, a.out.trap[r], rgb, a.scenes,
                                         scene_colors);
    rgba[r] = make_float4(rgb[0], rgb[1], rgb[2], 1.0f);
  }
}

template <class Set, class T, bool kDir64, bool kScenes = false>
cudaError_t launch_lite(const LaunchArgs& a, const nd_lite_desc* lites, const nd_lite_desc* scene_colors, float* rgba,
                        int num_sms, cudaStream_t s) {
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lite_kernel<Set, T, kDir64, kScenes>, 128, 0);
  if (e != cudaSuccess) return e;
  int64_t grid = int64_t(std::max(per_sm, 1)) * num_sms;
  const int64_t needed = (a.total_rays + 127) / 128;
  if (grid > needed) grid = needed;
  if (grid <= 0) return cudaSuccess;
  lite_kernel<Set, T, kDir64, kScenes><<<unsigned(grid), 128, 0, s>>>(a, lites, scene_colors,
                                                                      reinterpret_cast<float4*>(rgba));
  return cudaGetLastError();
}

typedef cudaError_t (*LiteFn)(const LaunchArgs&, const nd_lite_desc*, const nd_lite_desc*, float*, int, cudaStream_t);

// --------------------------------------------------------------- accelerator build
// cs_build_accel (tpl:5412-5431): one thread per voxel of every accelerated view of
// a launch; the DE the view's rays see at the voxel centre, less the half diagonal of
// the cell, times the safety factor, floored at 0.  jobs[j] = (view index, first
// voxel) in voxel order; a view's voxels are [level][z][y][x] of its grid.  The
// centre and the skip are rounded step by step (no contraction), like the CPU
// restatement.
struct AccelJob {
  int32_t view;
  int32_t pad;
  int64_t begin;
};

template <class Set, class T, bool kScenes>
__global__ void __launch_bounds__(128) accel_build_kernel(const DevView* __restrict__ views,
                                                          const AccelJob* __restrict__ jobs, int njobs, int64_t total,
                                                          const DevScene* scenes) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += stride) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (jobs[mid].begin <= i) lo = mid;
      else hi = mid - 1;
    }
    const DevView& v = views[jobs[lo].view];
    const uint32_t local = uint32_t(i - jobs[lo].begin);  // < 8 * 160^3
    const uint32_t r = uint32_t(v.accel_res);
    const uint32_t x = local % r, y = (local / r) % r, gz = local / (r * r);
    const uint32_t l = gz / r, z = gz % r;
    const float cell = v.accel_prm[l][3];
    const float cx = __fadd_rn(v.accel_prm[l][0], __fmul_rn(__fadd_rn(float(x), 0.5f), cell));
    const float cy = __fadd_rn(v.accel_prm[l][1], __fmul_rn(__fadd_rn(float(y), 0.5f), cell));
    const float cz = __fadd_rn(v.accel_prm[l][2], __fmul_rn(__fadd_rn(float(z), 0.5f), cell));
    const DEOut<T> de = view_de<Set, T, false, kScenes>(v, ndw::v3<T>(T(cx), T(cy), T(cz)), scenes);
    const float d = float(de.d);
    const float safe = fmaxf(__fsub_rn(d, __fmul_rn(0.8660254f, cell)), 0.0f);  // HALF_SQRT3 tpl:62
    v.accel_grid[local] = __fmul_rn(safe, v.accel_safety);
  }
}

template <class Set, class T, bool kScenes>
cudaError_t launch_accel_build(const DevView* views, const AccelJob* jobs, int njobs, int64_t total,
                               const DevScene* scenes, int num_sms, cudaStream_t s) {
  if (total <= 0 || njobs <= 0) return cudaSuccess;
  int64_t grid = (total + 127) / 128;
  grid = std::min<int64_t>(grid, int64_t(num_sms) * 16);
  accel_build_kernel<Set, T, kScenes><<<unsigned(grid), 128, 0, s>>>(views, jobs, njobs, total, scenes);
  return cudaGetLastError();
}

typedef cudaError_t (*AccelBuildFn)(const DevView*, const AccelJob*, int, int64_t, const DevScene*, int, cudaStream_t);

// DE of one formula at n points (the formula wrapper with its orbit trap), for
// parity tests against fixed point sets.
template <class Set, class T>
__global__ void __launch_bounds__(128) de_points_kernel(const __grid_constant__ DevView v, int64_t n,
                                                        const double* __restrict__ pts, double* __restrict__ de,
                                                        double* __restrict__ trap, uint32_t* __restrict__ iters) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const ndw::v3<T> p = ndw::v3<T>(T(pts[3 * i]), T(pts[3 * i + 1]), T(pts[3 * i + 2]));
  const DEOut<T> o = Set::template de<T, true>(v.code, p, v);
  de[i] = double(o.d);
  if (trap) trap[i] = double(o.trap);
  if (iters) iters[i] = uint32_t(o.iters);
}

template <class Set, class T>
cudaError_t launch_de_points(const DevView& v, int64_t n, const double* pts, double* de, double* trap,
                             uint32_t* iters, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int64_t grid = (n + 127) / 128;
  de_points_kernel<Set, T><<<unsigned(grid), 128, 0, s>>>(v, n, pts, de, trap, iters);
  return cudaGetLastError();
}

typedef cudaError_t (*DePointsFn)(const DevView&, int64_t, const double*, double*, double*, uint32_t*, cudaStream_t);

// Launchers of one formula set.  Plain launches take one view (kernel param);
// persistent ones take one view (single) or a view table (batched).  "dir64" is
// the deep-zoom variant with FP64 ray directions; FP64 DEs always use it.
struct KernelTable {
  LaunchFn plain_f32, plain_f32_dir64, plain_f64;
  LaunchFn persistent_f32, persistent_f32_batched, persistent_f32_dir64, persistent_f32_dir64_batched;
  // the FP32 march at 64 and 256 threads per block (the default is 128), single and
  // batched (formula groups only; null in single-formula tables)
  LaunchFn persistent_f32_b64, persistent_f32_b256, persistent_f32_batched_b64, persistent_f32_batched_b256;
  ResidentFn resident_b64, resident_b128, resident_b256;
  LaunchFn persistent_f64, persistent_f64_batched;
  // the march with its normal and shadow phases inline (no hit list): the
  // no-allocation entry point
  LaunchFn inline_f32, inline_f32_batched, inline_f32_dir64, inline_f32_dir64_batched, inline_f64, inline_f64_batched;
  ShadeFn shade_f32, shade_f32_batched, shade_f32_dir64, shade_f32_dir64_batched, shade_f64, shade_f64_batched;
  DePointsFn de_points_f32, de_points_f64;
  AdjointFn adjoint_f32, adjoint_f32_batched, adjoint_f64, adjoint_f64_batched;
  // multi-instance scenes (formula groups only; null in single-formula tables)
  LaunchFn scene_persistent_f32, scene_persistent_f32_dir64, scene_persistent_f64;
  ShadeFn scene_shade_f32, scene_shade_f32_dir64, scene_shade_f64;
  // empty-space accelerator: its grid build and the batched march / shade pass that
  // read it (FP32 directions or FP64 DE), without and with scenes
  AccelBuildFn accel_build_f32, accel_build_f64;
  LaunchFn persistent_f32_accel, persistent_f64_accel;
  ShadeFn shade_f32_accel, shade_f64_accel;
  AccelBuildFn scene_accel_build_f32, scene_accel_build_f64;
  LaunchFn scene_persistent_f32_accel, scene_persistent_f64_accel;
  ShadeFn scene_shade_f32_accel, scene_shade_f64_accel;
  // lite shading of a forward's hits (with scenes: formula groups only)
  LiteFn lite_f32, lite_f32_dir64, scene_lite_f32;
  // the wavefront shadow pass (FP32 or FP64 DE; with scenes: formula groups only)
  ShadowFn shadow_f32, shadow_f64, scene_shadow_f32, scene_shadow_f64;
};

// kForwardOnly: the table of a formula compiled at run time (nd_formula_register):
// the forward march, its surface and shadow passes and the DE at points, FP32 and
// FP64; no accelerator, lite shading or adjoint (their entries are null).
template <class Set, bool kWithScenes = false, bool kForwardOnly = false> KernelTable make_kernel_table() {
  KernelTable t;
  memset(&t, 0, sizeof(t));
  if constexpr (kWithScenes) {
    t.scene_persistent_f32 = &launch_persistent<Set, float, false, true, true>;
    t.scene_persistent_f32_dir64 = &launch_persistent<Set, float, true, true, true>;
    t.scene_persistent_f64 = &launch_persistent<Set, double, true, true, true>;
    t.scene_shade_f32 = &launch_shade<Set, float, false, true, true>;
    t.scene_shade_f32_dir64 = &launch_shade<Set, float, true, true, true>;
    t.scene_shade_f64 = &launch_shade<Set, double, true, true, true>;
    t.scene_accel_build_f32 = &launch_accel_build<Set, float, true>;
    t.scene_accel_build_f64 = &launch_accel_build<Set, double, true>;
    t.scene_persistent_f32_accel = &launch_persistent<Set, float, false, true, true, true>;
    t.scene_persistent_f64_accel = &launch_persistent<Set, double, true, true, true, true>;
    t.scene_shade_f32_accel = &launch_shade<Set, float, false, true, true, true>;
    t.scene_shade_f64_accel = &launch_shade<Set, double, true, true, true, true>;
    t.scene_lite_f32 = &launch_lite<Set, float, false, true>;
    t.scene_shadow_f32 = &launch_shadow<Set, float, true>;
    t.scene_shadow_f64 = &launch_shadow<Set, double, true>;
  } else {
    t.scene_shadow_f32 = t.scene_shadow_f64 = nullptr;
    t.scene_lite_f32 = nullptr;
    t.scene_persistent_f32 = t.scene_persistent_f32_dir64 = t.scene_persistent_f64 = nullptr;
    t.scene_shade_f32 = t.scene_shade_f32_dir64 = t.scene_shade_f64 = nullptr;
    t.scene_accel_build_f32 = t.scene_accel_build_f64 = nullptr;
    t.scene_persistent_f32_accel = t.scene_persistent_f64_accel = nullptr;
    t.scene_shade_f32_accel = t.scene_shade_f64_accel = nullptr;
  }
  t.shadow_f32 = &launch_shadow<Set, float>;
  t.shadow_f64 = &launch_shadow<Set, double>;
  if constexpr (!kForwardOnly) {
    t.lite_f32 = &launch_lite<Set, float, false>;
    t.lite_f32_dir64 = &launch_lite<Set, float, true>;
    t.accel_build_f32 = &launch_accel_build<Set, float, false>;
    t.accel_build_f64 = &launch_accel_build<Set, double, false>;
    t.persistent_f32_accel = &launch_persistent<Set, float, false, true, false, true>;
    t.persistent_f64_accel = &launch_persistent<Set, double, true, true, false, true>;
    t.shade_f32_accel = &launch_shade<Set, float, false, true, false, true>;
    t.shade_f64_accel = &launch_shade<Set, double, true, true, false, true>;
  }
  t.plain_f32 = &launch_plain<Set, float, false>;
  t.plain_f32_dir64 = &launch_plain<Set, float, true>;
  t.plain_f64 = &launch_plain<Set, double, true>;
  if constexpr (kWithScenes) {
    t.persistent_f32_b64 = &launch_persistent<Set, float, false, false, false, false, 64>;
    t.persistent_f32_b256 = &launch_persistent<Set, float, false, false, false, false, 256>;
    t.persistent_f32_batched_b64 = &launch_persistent<Set, float, false, true, false, false, 64>;
    t.persistent_f32_batched_b256 = &launch_persistent<Set, float, false, true, false, false, 256>;
    t.resident_b64 = &resident_f32_batched<Set, 64>;
    t.resident_b256 = &resident_f32_batched<Set, 256>;
  } else {
    t.persistent_f32_b64 = t.persistent_f32_b256 = t.persistent_f32_batched_b64 = t.persistent_f32_batched_b256 =
        nullptr;
    t.resident_b64 = t.resident_b256 = nullptr;
  }
  t.resident_b128 = &resident_f32_batched<Set, 128>;
  t.inline_f32 = &launch_persistent<Set, float, false, false, false, false, 128, false>;
  t.inline_f32_batched = &launch_persistent<Set, float, false, true, false, false, 128, false>;
  t.inline_f32_dir64 = &launch_persistent<Set, float, true, false, false, false, 128, false>;
  t.inline_f32_dir64_batched = &launch_persistent<Set, float, true, true, false, false, 128, false>;
  t.inline_f64 = &launch_persistent<Set, double, true, false, false, false, 128, false>;
  t.inline_f64_batched = &launch_persistent<Set, double, true, true, false, false, 128, false>;
  t.persistent_f32 = &launch_persistent<Set, float, false, false>;
  t.persistent_f32_batched = &launch_persistent<Set, float, false, true>;
  t.persistent_f32_dir64 = &launch_persistent<Set, float, true, false>;
  t.persistent_f32_dir64_batched = &launch_persistent<Set, float, true, true>;
  t.persistent_f64 = &launch_persistent<Set, double, true, false>;
  t.persistent_f64_batched = &launch_persistent<Set, double, true, true>;
  t.shade_f32 = &launch_shade<Set, float, false, false>;
  t.shade_f32_batched = &launch_shade<Set, float, false, true>;
  t.shade_f32_dir64 = &launch_shade<Set, float, true, false>;
  t.shade_f32_dir64_batched = &launch_shade<Set, float, true, true>;
  t.shade_f64 = &launch_shade<Set, double, true, false>;
  t.shade_f64_batched = &launch_shade<Set, double, true, true>;
  t.de_points_f32 = &launch_de_points<Set, float>;
  t.de_points_f64 = &launch_de_points<Set, double>;
  if constexpr (!kForwardOnly) {
    t.adjoint_f32 = &launch_adjoint<Set, float, false>;
    t.adjoint_f32_batched = &launch_adjoint<Set, float, true>;
    t.adjoint_f64 = &launch_adjoint<Set, double, false>;
    t.adjoint_f64_batched = &launch_adjoint<Set, double, true>;
  }
  return t;
}

}  // namespace nd
