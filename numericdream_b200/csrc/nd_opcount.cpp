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

}  // extern "C"
