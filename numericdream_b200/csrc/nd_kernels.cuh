// Sphere-tracing kernels for sm_100a: the plain per-ray launch and the persistent
// wavefront kernel with warp-ballot refill.  Included once per formula (or per
// formula group) by the translated sources, which instantiate the launchers.  The
// ray program itself (march_to, normals, orbit trap, shadow) is in nd_rayprog.h.
#pragma once

#include <cuda_runtime.h>

#include "nd_rayprog.h"

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

// --------------------------------------------------------------- plain kernel
// One thread per ray, the reference's fragment-shader structure (fs_simple):
// march to completion, then the normal taps, then the shadow ray.  No refill: a
// warp runs until its slowest ray is done.
template <class Set, class T, bool kBatched>
__global__ void __launch_bounds__(128) plain_kernel(const __grid_constant__ LaunchArgs a,
                                                    const __grid_constant__ DevView single) {
  const int64_t item = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool live = item < a.total_rays;
  unsigned long long rays = 0, hits = 0;
  Lane<T> L;
  L.ev_march = L.ev_normal = L.ev_shadow = 0;
  if (live) {
    const int vi = kBatched ? find_view(a.views, a.nviews, item) : 0;
    const DevView& v = kBatched ? a.views[vi] : single;
    L.start(v, item, vi);
    if (v.max_samples <= 0) L.finish(v, a.out, false, 1.0f, a.stats);
    while (L.phase != PH_DONE) {
      const DEOut<T> de = Set::template de<T>(v.code, to_t<T>(L.sample_pos(v)), v);
      L.advance(v, de, a.out, a.stats);
    }
    rays = 1;
    hits = L.was_hit ? 1 : 0;
  }
  flush_stats(a.stats, rays, L.ev_march, L.ev_normal, L.ev_shadow, hits, 0);
}

// --------------------------------------------------------------- persistent kernel
// One resident grid; every warp keeps 32 rays in flight.  After each DE
// evaluation the warp ballots its idle lanes; once at least refill_threshold
// lanes are idle (or all are), the first idle lane takes that many new ray
// indices with ONE atomicAdd on the work counter and hands them out by
// popc-prefix rank (the analogue of the reference's workgroup-aggregated queue
// reservation wf_reserve, tpl:5083-5105).
template <class Set, class T, bool kBatched>
__global__ void __launch_bounds__(128) persistent_kernel(const __grid_constant__ LaunchArgs a,
                                                         const __grid_constant__ DevView single) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  Lane<T> L;
  L.item = -1;
  L.phase = PH_DONE;
  L.ev_march = L.ev_normal = L.ev_shadow = 0;
  unsigned long long rays = 0, hits = 0, refills = 0;
  bool exhausted = false;
  int vi = 0;
  const int64_t t0 = __shfl_sync(full, globaltimer_ns(), 0);
  int tick = 0;
  while (true) {
    if (L.phase == PH_DONE && L.item >= 0) {
      ++rays;
      hits += L.was_hit ? 1 : 0;
      L.item = -1;
    }
    const unsigned idle = __ballot_sync(full, L.item < 0);
    if (!exhausted && idle != 0u && (__popc(idle) >= a.refill_threshold || idle == full)) {
      const int want = __popc(idle);
      const int leader = __ffs(idle) - 1;
      unsigned long long base = 0;
      if (lane == leader) base = atomicAdd(a.counter, (unsigned long long)want);
      base = __shfl_sync(full, base, leader);
      ++refills;
      if (base + want >= (unsigned long long)a.total_rays) exhausted = true;
      if (L.item < 0) {
        const int64_t it = int64_t(base) + __popc(idle & lt_mask);
        if (it < a.total_rays) {
          vi = kBatched ? find_view(a.views, a.nviews, it) : 0;
          const DevView& v = kBatched ? a.views[vi] : single;
          L.start(v, it, vi);
          if (v.max_samples <= 0) L.finish(v, a.out, false, 1.0f, a.stats);
        }
      }
      if (__ballot_sync(full, L.item >= 0) == 0u) break;
      continue;  // lanes finished at start re-enter the bookkeeping above
    }
    if (exhausted && idle == full) break;
    if (((++tick) & 63) == 0) {
      // lane 0's clock decides for the whole warp, so the exit stays warp-uniform
      const int64_t now = __shfl_sync(full, globaltimer_ns(), 0);
      if (now - t0 > a.deadline_ns) {
        if (lane == 0) atomicAdd(&a.stats->timeouts, 1u);
        break;
      }
    }
    if (L.item >= 0) {
      const DevView& v = kBatched ? a.views[vi] : single;
      const DEOut<T> de = Set::template de<T>(v.code, to_t<T>(L.sample_pos(v)), v);
      L.advance(v, de, a.out, a.stats);
    }
  }
  flush_stats(a.stats, rays, L.ev_march, L.ev_normal, L.ev_shadow, hits, refills);
}

// --------------------------------------------------------------- launchers
struct LaunchConfig {
  int kernel;           // ND_KERNEL_PLAIN / ND_KERNEL_PERSISTENT
  int block;
  int blocks_per_sm;
  int num_sms;
};

template <class Set, class T, bool kBatched>
cudaError_t launch_plain(const LaunchArgs& a, const DevView& single, const LaunchConfig& c, cudaStream_t s) {
  const int block = 128;
  const int64_t grid = (a.total_rays + block - 1) / block;
  if (grid <= 0) return cudaSuccess;
  plain_kernel<Set, T, kBatched><<<unsigned(grid), block, 0, s>>>(a, single);
  return cudaGetLastError();
}

template <class Set, class T, bool kBatched>
cudaError_t launch_persistent(const LaunchArgs& a, const DevView& single, const LaunchConfig& c, cudaStream_t s) {
  const int block = 128;
  int per_sm = c.blocks_per_sm;
  if (per_sm <= 0) {
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persistent_kernel<Set, T, kBatched>, block, 0);
    if (e != cudaSuccess) return e;
    if (per_sm <= 0) per_sm = 1;
  }
  int64_t grid = int64_t(per_sm) * c.num_sms;
  const int64_t needed = (a.total_rays + block - 1) / block;
  if (grid > needed) grid = needed;
  if (grid <= 0) return cudaSuccess;
  persistent_kernel<Set, T, kBatched><<<unsigned(grid), block, 0, s>>>(a, single);
  return cudaGetLastError();
}

typedef cudaError_t (*LaunchFn)(const LaunchArgs&, const DevView&, const LaunchConfig&, cudaStream_t);

// DE of one formula at n points (the formula wrapper with its orbit trap), for
// parity tests against fixed point sets.
template <class Set, class T>
__global__ void __launch_bounds__(128) de_points_kernel(const __grid_constant__ DevView v, int64_t n,
                                                        const double* __restrict__ pts, double* __restrict__ de,
                                                        double* __restrict__ trap, uint32_t* __restrict__ iters) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const ndw::v3<T> p = ndw::v3<T>(T(pts[3 * i]), T(pts[3 * i + 1]), T(pts[3 * i + 2]));
  const DEOut<T> o = Set::template de<T>(v.code, p, v);
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

// Launchers of one formula set: [kernel][precision][batched].
struct KernelTable {
  LaunchFn plain_f32, plain_f32_batched, persistent_f32, persistent_f32_batched;
  LaunchFn plain_f64, plain_f64_batched, persistent_f64, persistent_f64_batched;
  DePointsFn de_points_f32, de_points_f64;
};

template <class Set> KernelTable make_kernel_table() {
  KernelTable t;
  t.plain_f32 = &launch_plain<Set, float, false>;
  t.plain_f32_batched = &launch_plain<Set, float, true>;
  t.persistent_f32 = &launch_persistent<Set, float, false>;
  t.persistent_f32_batched = &launch_persistent<Set, float, true>;
  t.plain_f64 = &launch_plain<Set, double, false>;
  t.plain_f64_batched = &launch_plain<Set, double, true>;
  t.persistent_f64 = &launch_persistent<Set, double, false>;
  t.persistent_f64_batched = &launch_persistent<Set, double, true>;
  t.de_points_f32 = &launch_de_points<Set, float>;
  t.de_points_f64 = &launch_de_points<Set, double>;
  return t;
}

}  // namespace nd
