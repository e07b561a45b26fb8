// C entry point of the op-counting library (libnd_opcount.so): algorithmic FP32
// operation counts of the ray program over a sample of a launch's rays.
#include <omp.h>
#include <string.h>

#include <vector>

#include "nd_opcount.h"
#include "nd_view.h"

typedef void (*NdOpFn)(const nd::DevView*, int64_t, ndw::OpCounts*, uint32_t*);
extern const NdOpFn nd_opcount_fns[];
extern const int nd_opcount_fn_count;

extern "C" {

// For each view, `rays_per_view` rays spread evenly over the view are traced on the
// host with counting arithmetic.  out[0..8] receives, summed over views and
// weighted by rays(view) / sampled rays(view): flops, sfu, other, de_evals, add,
// mul, div, fma, rays.  Returns 0, or -1 for an unknown formula id.
int nd_opcount(const nd_view_desc* views, int nviews, int64_t rays_per_view, double* out) {
  for (int k = 0; k < 9; ++k) out[k] = 0.0;
  for (int i = 0; i < nviews; ++i) {
    if (views[i].formula < 0 || views[i].formula >= nd_opcount_fn_count) return -1;
    const nd::DevView v = nd::make_dev_view(views[i], 0, 0, 0);
    const int64_t n = v.rays;
    if (n <= 0) continue;
    const int64_t m = rays_per_view < n ? rays_per_view : n;
    const NdOpFn fn = nd_opcount_fns[views[i].formula];
    std::vector<ndw::OpCounts> per(omp_get_max_threads());
    std::vector<uint64_t> ev(per.size(), 0);
#pragma omp parallel for schedule(dynamic, 8)
    for (int64_t j = 0; j < m; ++j) {
      // one ray per stride, at a scrambled offset inside the stride
      const int64_t stride = n / m;
      const int64_t ray = j * stride + (stride > 1 ? int64_t((uint64_t(j) * 2654435761ull) % uint64_t(stride)) : 0);
      uint32_t e = 0;
      fn(&v, ray, &per[omp_get_thread_num()], &e);
      ev[omp_get_thread_num()] += e;
    }
    ndw::OpCounts s;
    uint64_t evals = 0;
    for (size_t t = 0; t < per.size(); ++t) {
      s.add += per[t].add; s.mul += per[t].mul; s.div += per[t].div; s.fma += per[t].fma;
      s.sfu += per[t].sfu; s.other += per[t].other;
      evals += ev[t];
    }
    const double w = double(n) / double(m);
    out[0] += w * double(s.flops());
    out[1] += w * double(s.sfu);
    out[2] += w * double(s.other);
    out[3] += w * double(evals);
    out[4] += w * double(s.add);
    out[5] += w * double(s.mul);
    out[6] += w * double(s.div);
    out[7] += w * double(s.fma);
    out[8] += double(n);
  }
  return 0;
}

// Host run of the persistent kernel's work-list bookkeeping (WarpRuns, the same
// code the kernel runs) with a plain 64-bit counter standing in for the device
// atomic: `warps` warps claim rays for a pseudo-random number of idle lanes
// (1..32), round after round from a pseudo-random first warp, until every warp has
// run dry.  The counter starts at `start` (as if the rays before it were handed out
// already).  Each ray index handed out in [start, total) is counted in
// seen[index - start] (the caller zeroes seen); out[0] = rays handed out, out[1] = smallest index, out[2] = largest
// index, out[3] = final counter value, out[4] = claims.  Returns 0.
int nd_sim_work_runs(int32_t total, int32_t warps, int32_t chunk, int64_t start, uint64_t seed, uint8_t* seen,
                     int64_t* out) {
  std::vector<nd::WarpRuns> w(size_t(warps > 0 ? warps : 0));
  uint64_t counter = uint64_t(start), s = seed | 1u;
  int64_t handed = 0, lo = INT64_MAX, hi = INT64_MIN, claims = 0;
  auto rnd = [&s]() {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return s;
  };
  for (bool busy = true; busy;) {
    busy = false;
    const size_t off = size_t(rnd() % (w.size() ? w.size() : 1));
    for (size_t k = 0; k < w.size(); ++k) {
      nd::WarpRuns& r = w[(k + off) % w.size()];
      if (!r.have_work()) continue;
      busy = true;
      const int nidle = 1 + int(rnd() % 32);
      const nd::WarpRuns::Claim c = r.claim(nidle, chunk, total, [&](int take) {
        const uint64_t got = counter;
        counter += uint64_t(take);
        ++claims;
        return got;
      });
      for (int i = 0; i < c.used; ++i) {
        const int64_t it = c.item(i);
        ++handed;
        lo = it < lo ? it : lo;
        hi = it > hi ? it : hi;
        if (it >= start && it < total && seen) ++seen[it - start];
      }
    }
  }
  out[0] = handed;
  out[1] = lo;
  out[2] = hi;
  out[3] = int64_t(counter);
  out[4] = claims;
  return 0;
}

// floor(n[i] / d) by ray_uv's magic-number division (div_magic / div_by, the code the
// kernels run) into q[i]; n[i] < 2^31.
void nd_div_by(uint32_t d, int64_t count, const uint32_t* n, uint32_t* q) {
  uint32_t m, s;
  nd::div_magic(d, &m, &s);
  for (int64_t i = 0; i < count; ++i) q[i] = nd::div_by(n[i], m, s);
}

}  // extern "C"
