// Sphere-tracing kernels for sm_100a: the plain per-ray launch and the persistent
// wavefront kernel with warp-ballot refill.  Included once per formula (or per
// formula group) by the translated sources, which instantiate the launchers.  The
// ray program itself (march_to, normals, orbit trap, shadow) is in nd_rayprog.h.
#pragma once

#include <cuda_runtime.h>

#include "nd_rayprog.h"

namespace nd {

#ifndef ND_PERSISTENT_MIN_BLOCKS
#define ND_PERSISTENT_MIN_BLOCKS 1
#endif

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
// The reference's per-pixel program as a plain per-view launch: one thread per
// ray, the march loop of march_to, then the normal taps of estimate_normal, then
// the shadow loop of visibility_march, each loop running until its slowest lane
// in the warp is done (fs_simple tpl:4522-4538 / simple_geometry tpl:4492-4507).
template <class Set, class T, bool kDir64>
__global__ void __launch_bounds__(128) plain_kernel(const __grid_constant__ LaunchArgs a,
                                                    const __grid_constant__ DevView v) {
  const int64_t local = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;  // ray index inside the view
  unsigned long long rays = 0, hits = 0, m = 0, nn = 0, sh = 0;
  if (local < v.rays) {
    Lane<T, kDir64> L;
    L.start(v, int32_t(v.ray_offset + local), 0);
    if (L.phase == PH_DONE) L.finish(v, a.out, 1.0f);
    while (L.phase == PH_MARCH) {
      const DEOut<T> de = Set::template de<T>(v.code, to_t<T>(L.sample_pos(v)), v);
      L.advance(v, de, a.out);
    }
    m = L.evals;
    while (L.phase == PH_NORMAL) {
      const DEOut<T> de = Set::template de<T>(v.code, to_t<T>(L.sample_pos(v)), v);
      L.advance(v, de, a.out);
    }
    nn = L.evals - m;
    while (L.phase == PH_SHADOW) {
      const DEOut<T> de = Set::template de<T>(v.code, to_t<T>(L.sample_pos(v)), v);
      L.advance(v, de, a.out);
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
// lanes are idle (or all are), the first idle lane takes that many new ray
// indices with ONE atomicAdd on the work counter and hands them out by
// popc-prefix rank (the analogue of the reference's workgroup-aggregated queue
// reservation wf_reserve, tpl:5083-5105).  Whatever phase a lane is in, each pass
// of the loop is one DE evaluation for every busy lane.
template <class Set, class T, bool kDir64, bool kBatched>
__global__ void __launch_bounds__(128, ND_PERSISTENT_MIN_BLOCKS) persistent_kernel(const __grid_constant__ LaunchArgs a,
                                                         const __grid_constant__ DevView single) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  Lane<T, kDir64> L;
  L.item = -1;
  L.phase = PH_DONE;
  L.evals = 0;
  L.hit = false;
  uint32_t rays = 0, hits = 0, ev_m = 0, ev_n = 0, ev_s = 0, refills = 0;
  bool exhausted = false;
  const int64_t deadline = __shfl_sync(full, globaltimer_ns(), 0) + a.deadline_ns;
  int tick = 0;
  const int32_t total = int32_t(a.total_rays);
  while (true) {
    if (L.phase == PH_DONE && L.item >= 0) {
      ++rays;
      hits += L.hit ? 1 : 0;
      const uint32_t taps = L.hit ? normal_taps(kBatched ? a.views[L.view] : single) : 0u;
      ev_m += L.mev;
      ev_n += taps;
      ev_s += L.evals - L.mev - taps;
      L.item = -1;
    }
    const unsigned idle = __ballot_sync(full, L.item < 0);
    if (!exhausted && idle != 0u && (__popc(idle) >= a.refill_threshold || idle == full)) {
      const int want = __popc(idle);
      const int leader = __ffs(idle) - 1;
      int32_t base = 0;
      if (lane == leader) base = int32_t(atomicAdd(a.counter, (unsigned long long)want));
      base = __shfl_sync(full, base, leader);
      ++refills;
      if (int64_t(base) + want >= int64_t(total)) exhausted = true;
      if (L.item < 0) {
        const int32_t it = base + __popc(idle & lt_mask);
        if (it < total && it >= 0) {
          L.view = kBatched ? find_view(a.views, a.nviews, it) : 0;
          const DevView& v = kBatched ? a.views[L.view] : single;
          L.start(v, it, L.view);
          if (L.phase == PH_DONE) L.finish(v, a.out, 1.0f);
        }
      }
      continue;  // lanes that finished at once go back through the bookkeeping
    }
    if (exhausted && idle == full) break;
    if (((++tick) & 63) == 0) {
      // lane 0's clock decides for the whole warp, so the exit stays warp-uniform
      const int64_t now = __shfl_sync(full, globaltimer_ns(), 0);
      if (now > deadline) {
        if (lane == 0) atomicAdd(&a.stats->timeouts, 1u);
        break;
      }
    }
    if (L.item >= 0) {
      const DevView& v = kBatched ? a.views[L.view] : single;
      const DEOut<T> de = Set::template de<T>(v.code, to_t<T>(L.sample_pos(v)), v);
      L.advance(v, de, a.out);
    }
  }
  flush_stats(a.stats, rays, ev_m, ev_n, ev_s, hits, refills);
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

template <class Set, class T, bool kDir64, bool kBatched>
cudaError_t launch_persistent(const LaunchArgs& a, const DevView& single, const LaunchConfig& c, cudaStream_t s) {
  const int block = 128;
  int per_sm = c.blocks_per_sm;
  if (per_sm <= 0) {
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, persistent_kernel<Set, T, kDir64, kBatched>, block, 0);
    if (e != cudaSuccess) return e;
    if (per_sm <= 0) per_sm = 1;
  }
  int64_t grid = int64_t(per_sm) * c.num_sms;
  const int64_t needed = (a.total_rays + block - 1) / block;
  if (grid > needed) grid = needed;
  if (grid <= 0) return cudaSuccess;
  persistent_kernel<Set, T, kDir64, kBatched><<<unsigned(grid), block, 0, s>>>(a, single);
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

// Launchers of one formula set.  Plain launches take one view (kernel param);
// persistent ones take one view (single) or a view table (batched).  "dir64" is
// the deep-zoom variant with FP64 ray directions; FP64 DEs always use it.
struct KernelTable {
  LaunchFn plain_f32, plain_f32_dir64, plain_f64;
  LaunchFn persistent_f32, persistent_f32_batched, persistent_f32_dir64, persistent_f32_dir64_batched;
  LaunchFn persistent_f64, persistent_f64_batched;
  DePointsFn de_points_f32, de_points_f64;
};

template <class Set> KernelTable make_kernel_table() {
  KernelTable t;
  t.plain_f32 = &launch_plain<Set, float, false>;
  t.plain_f32_dir64 = &launch_plain<Set, float, true>;
  t.plain_f64 = &launch_plain<Set, double, true>;
  t.persistent_f32 = &launch_persistent<Set, float, false, false>;
  t.persistent_f32_batched = &launch_persistent<Set, float, false, true>;
  t.persistent_f32_dir64 = &launch_persistent<Set, float, true, false>;
  t.persistent_f32_dir64_batched = &launch_persistent<Set, float, true, true>;
  t.persistent_f64 = &launch_persistent<Set, double, true, false>;
  t.persistent_f64_batched = &launch_persistent<Set, double, true, true>;
  t.de_points_f32 = &launch_de_points<Set, float>;
  t.de_points_f64 = &launch_de_points<Set, double>;
  return t;
}

}  // namespace nd
