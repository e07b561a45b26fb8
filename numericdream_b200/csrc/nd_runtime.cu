// C-ABI implementation (include/nd_march.h): formula registry, contexts, view
// validation, launch planning, statistics, autotuning and CUDA-graph capture.
#include <cuda_runtime.h>
#include <dirent.h>
#include <dlfcn.h>
#include <stdarg.h>
#include <stdlib.h>
#include <stdio.h>
#include <string.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <complex>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "nd_json.h"
#include "nd_registry.h"
#include "nd_view.h"

using nd::DevView;
using nd::make_dev_view;
using nd::KernelTable;
using nd::LaunchArgs;
using nd::LaunchConfig;
using nd::LaunchFn;
using nd::Stats;

namespace {

constexpr int kMaxViews = 1 << 16;
constexpr int64_t kMaxRays = int64_t(1) << 40;
// Device counters per launch plan: the work counter, the hit count, the shadow-queue
// count and the shadow pass's work counter.
constexpr int kCountersPerPlan = 4;

const char* kStatusNames[] = {"ND_OK",          "ND_ERR_INVALID", "ND_ERR_COMPILE",     "ND_ERR_OOM",
                              "ND_ERR_TIMEOUT", "ND_ERR_CUDA",    "ND_ERR_UNSUPPORTED", "ND_ERR_NOT_FOUND"};

uint64_t fnv1a64(const char* s, size_t n) {
  uint64_t h = 0xCBF29CE484222325ull;
  for (size_t i = 0; i < n; ++i) {
    h ^= uint8_t(s[i]);
    h *= 0x100000001B3ull;
  }
  return h;
}

void copy_str(char* out, size_t out_len, const char* s, size_t len) {
  if (!out || out_len == 0) return;
  const size_t n = std::min(out_len - 1, len);
  memcpy(out, s, n);
  out[n] = 0;
}
void copy_str(char* out, size_t out_len, const std::string& s) { copy_str(out, out_len, s.data(), s.size()); }
void copy_str(char* out, size_t out_len, const char* s) { copy_str(out, out_len, s, strlen(s)); }

// Tuned launch parameters per (GPU, formula set), filled by nd_autotune and by
// nd_tune_cache_load.  blocks_per_sm: 0 = as many as fit, < 0 = that many fewer.
struct Tuned {
  int kernel = ND_KERNEL_PERSISTENT;
  int block = 128;
  int blocks_per_sm = 0;
  int refill_threshold = 6;
  double rays_per_s = 0.0;  // measured by the tuning run
  bool tuned = false;       // false: the defaults above, no tuning run or cache entry
};
std::mutex g_tune_mu;
std::map<std::string, Tuned> g_tuned;  // key: tune_key()

}  // namespace

struct nd_ctx {
  int device = 0;
  int num_sms = 0;
  std::string gpu_name;  // cudaDeviceProp::name (the tuning cache's key)
  std::string err;
  DevView* d_views = nullptr;
  int views_cap = 0;
  unsigned long long* d_counters = nullptr;
  int counters_cap = 0;
  Stats* d_stats = nullptr;
  double* d_thit = nullptr;    // FP64 hit distances for the shade pass
  nd::HitEntry* d_hits = nullptr;   // hit list of the deferred shade pass
  int64_t thit_cap = 0;
  nd::ShadowEntry* d_shadowq = nullptr;  // shadow queue of the wavefront shadow pass
  int64_t shadowq_cap = 0;
  nd::DevScene* d_scenes = nullptr;  // multi-instance scene table
  int scenes_cap = 0;
  float* d_accel = nullptr;          // accelerator grids of the views that have one
  int64_t accel_cap = 0;             // floats
  nd::AccelJob* d_accel_jobs = nullptr;
  int accel_jobs_cap = 0;
  uint64_t last_accel_voxels = 0;
  nd_lite_desc* d_lite = nullptr;    // lite-shading descriptors, in plan order
  int lite_cap = 0;
  bool last_trap = false;
  DevView* h_views = nullptr;  // pinned staging: two halves of h_views_cap records, forward calls alternate
  DevView* d_fviews = nullptr;  // the forward's device view table: two halves of fviews_half records, alternating
  int fviews_half = 0;          // like the staging
  cudaStream_t upload = nullptr;  // the view-table uploads of forward calls
  cudaEvent_t uploaded[2] = {nullptr, nullptr};  // after the upload into each half
  int h_views_cap = 0;
  cudaEvent_t staged[2] = {nullptr, nullptr};  // after the call that last used each half
  bool staged_valid[2] = {false, false};
  uint64_t calls = 0;
  cudaStream_t last_stream = nullptr;
  cudaEvent_t last_done = nullptr;
  std::vector<cudaEvent_t> tev;  // timing events per launch plan: accelerator build start, march start,
                                 // march end, shade end
  int tev_plans = 0;             // plans the last forward timed (0: none)
  bool have_last = false;
  int last_kernel = 0;
  int64_t last_rays = 0;
};

struct nd_graph {
  nd_ctx* ctx = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  DevView* d_views = nullptr;
  unsigned long long* d_counters = nullptr;
  double* d_thit = nullptr;
  nd::HitEntry* d_hits = nullptr;
  nd::ShadowEntry* d_shadowq = nullptr;
  float* d_accel = nullptr;
  nd::AccelJob* d_accel_jobs = nullptr;
  nd::DevScene* d_scenes = nullptr;
  bool trap = false;
};

namespace {

// The message of the last failure of a context-free call (nd_march_forward_noalloc),
// per host thread.
thread_local char g_noctx_err[256] = "";

nd_status fail(nd_ctx* ctx, nd_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(ctx ? buf : g_noctx_err, ctx ? sizeof(buf) : sizeof(g_noctx_err), fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  return s;
}

nd_status cuda_fail(nd_ctx* ctx, cudaError_t e, const char* what) {
  const nd_status s = (e == cudaErrorMemoryAllocation) ? ND_ERR_OOM : ND_ERR_CUDA;
  return fail(ctx, s, "%s: %s", what, cudaGetErrorString(e));
}

bool finite(double x) { return x == x && x < 1e300 && x > -1e300; }

nd_status validate_view(nd_ctx* ctx, const nd_view_desc& v, int idx) {
  if (v.formula < 0 || v.formula >= nd_formula_total())
    return fail(ctx, ND_ERR_NOT_FOUND, "view %d: unknown formula id %d", idx, v.formula);
  if (v.width <= 0 || v.height <= 0 || v.tile_w < 0 || v.tile_h < 0 || v.tile_x < 0 || v.tile_y < 0 ||
      int64_t(v.tile_x) + v.tile_w > v.width || int64_t(v.tile_y) + v.tile_h > v.height)
    return fail(ctx, ND_ERR_INVALID, "view %d: bad frame %dx%d / tile (%d,%d %dx%d)", idx, v.width, v.height,
                v.tile_x, v.tile_y, v.tile_w, v.tile_h);
  if (v.spp < 1 || v.spp > 4096) return fail(ctx, ND_ERR_INVALID, "view %d: spp %d out of [1, 4096]", idx, v.spp);
  if (v.max_steps < 0 || v.max_steps > (1 << 20))
    return fail(ctx, ND_ERR_INVALID, "view %d: max_steps %d out of range", idx, v.max_steps);
  if (v.refine_budget < 0 || v.refine_budget > 4096)
    return fail(ctx, ND_ERR_INVALID, "view %d: refine_budget %d out of range", idx, v.refine_budget);
  for (int i = 0; i < 3; ++i)
    if (!finite(v.cam_pos[i]) || !finite(v.fwd[i]) || !finite(v.right[i]) || !finite(v.up[i]))
      return fail(ctx, ND_ERR_INVALID, "view %d: non-finite camera", idx);
  for (int i = 0; i < ND_MAX_PARAMS; ++i)
    if (!finite(v.params[i])) return fail(ctx, ND_ERR_INVALID, "view %d: param %d is not finite", idx, i);
  if (!(v.max_dist > 0) || !finite(v.max_dist) || !finite(v.eps_coef) || !finite(v.eps_floor))
    return fail(ctx, ND_ERR_INVALID, "view %d: bad max_dist/epsilon", idx);
  if (v.normal_mode != ND_NORMAL_TETRA && v.normal_mode != ND_NORMAL_CENTRAL)
    return fail(ctx, ND_ERR_INVALID, "view %d: bad normal_mode %d", idx, v.normal_mode);
  if (v.accel_res < 0) return fail(ctx, ND_ERR_INVALID, "view %d: accel_res %d < 0", idx, v.accel_res);
  if (v.accel_res > 0 && !(v.accel_safety > 0.0f && v.accel_safety <= 1.0f))
    return fail(ctx, ND_ERR_INVALID, "view %d: accel_safety %g out of (0, 1]", idx, double(v.accel_safety));
  if (v.shadow) {
    const double l2 = double(v.light_dir[0]) * v.light_dir[0] + double(v.light_dir[1]) * v.light_dir[1] +
                      double(v.light_dir[2]) * v.light_dir[2];
    if (!(l2 > 0) || !finite(l2)) return fail(ctx, ND_ERR_INVALID, "view %d: shadow needs a light direction", idx);
  }
  return ND_OK;
}

template <class T> nd_status ensure_dev(nd_ctx* ctx, T** p, int* cap, int need, const char* what) {
  if (*cap >= need) return ND_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  const int n = std::max(need, 64);
  cudaError_t e = cudaMalloc((void**)p, sizeof(T) * size_t(n));
  if (e != cudaSuccess) return cuda_fail(ctx, e, what);
  *cap = n;
  return ND_OK;
}

// The pinned view staging (two halves, forward calls alternate).  Growing it waits for
// every call that may still read the old one.
nd_status ensure_staging(nd_ctx* ctx, int nviews) {
  if (ctx->h_views_cap >= nviews) return ND_OK;
  for (int k = 0; k < 2; ++k)
    if (ctx->staged_valid[k]) cudaEventSynchronize(ctx->staged[k]);
  if (ctx->have_last) cudaEventSynchronize(ctx->last_done);
  if (ctx->h_views) cudaFreeHost(ctx->h_views);
  ctx->h_views = nullptr;
  ctx->h_views_cap = 0;
  const int cap = std::max(nviews, 64);
  cudaError_t e = cudaMallocHost((void**)&ctx->h_views, 2 * sizeof(DevView) * size_t(cap));
  if (e != cudaSuccess) return cuda_fail(ctx, e, "pinned view staging");
  ctx->h_views_cap = cap;
  return ND_OK;
}

// The forward's device view table (two halves, used like the staging's), its upload
// stream and the events that order each half's upload before the march.
nd_status ensure_forward_views(nd_ctx* ctx, int nviews) {
  cudaError_t e = cudaSuccess;
  if (!ctx->upload && (e = cudaStreamCreateWithFlags(&ctx->upload, cudaStreamNonBlocking)) != cudaSuccess)
    return cuda_fail(ctx, e, "upload stream");
  for (int k = 0; k < 2; ++k)
    if (!ctx->uploaded[k] && (e = cudaEventCreateWithFlags(&ctx->uploaded[k], cudaEventDisableTiming)) != cudaSuccess)
      return cuda_fail(ctx, e, "upload event");
  if (ctx->fviews_half >= nviews) return ND_OK;
  if (ctx->have_last) cudaEventSynchronize(ctx->last_done);
  if (ctx->d_fviews) cudaFree(ctx->d_fviews);
  ctx->d_fviews = nullptr;
  ctx->fviews_half = 0;
  const int half = std::max(nviews, 64);
  e = cudaMalloc((void**)&ctx->d_fviews, 2 * sizeof(DevView) * size_t(half));
  if (e != cudaSuccess) return cuda_fail(ctx, e, "view table");
  ctx->fviews_half = half;
  return ND_OK;
}

// A launch plan: one or more launches, each over a subset of the views with one
// kernel table.
struct Launch {
  KernelTable table;
  std::vector<int> members; // formula ids of the table's set, in code order
  std::vector<int> views;  // indices into the caller's array
  std::vector<int> codes;  // formula code of each view inside the table's set
  int64_t rays = 0;
  std::string key;         // tuning key
};

std::string set_key(const std::vector<int>& formulas) {
  std::string k;
  for (int f : formulas) {
    k += nd_formula_at(f)->name;
    k += "+";
  }
  return k;
}

// The multi-instance scenes of a forward call (nd_march_forward_scenes).
struct SceneInput {
  const int32_t* view_scene = nullptr;  // per view: scene index or -1
  const nd_scene_desc* scenes = nullptr;
  int nscenes = 0;
  int scene_of(int view) const { return view_scene ? view_scene[view] : -1; }
};

// Every formula a view's rays evaluate: its own, or its scene's instances and mixins.
std::vector<int> view_formulas(const nd_view_desc& v, int scene, const SceneInput& sc) {
  if (scene < 0) return {v.formula};
  std::vector<int> f;
  const nd_scene_desc& S = sc.scenes[scene];
  for (int i = 0; i < S.instance_count; ++i) {
    const nd_instance_desc& in = S.instances[i];
    f.push_back(in.formula);
    for (int j = 0; j < in.mixin_count; ++j) f.push_back(in.mixins[j].formula);
  }
  return f;
}

// de_iterations() of a formula at a view's parameters, clamped like the kernels'.
double view_iterations(int formula, const float* params) {
  const nd::FormulaEntry& f = (*nd_formula_at(formula));
  if (!f.iterations) return 1.0;
  const int32_t n = f.iterations(params);
  return double(n < 1 ? 1 : (n > nd::kMaxIterations ? nd::kMaxIterations : n));
}

nd_status plan(nd_ctx* ctx, const nd_view_desc* views, int nviews, std::vector<Launch>* out,
               const SceneInput& sc = SceneInput()) {
  std::vector<int> distinct;
  const bool any_scene = sc.nscenes > 0;
  for (int i = 0; i < nviews; ++i)
    for (int f : view_formulas(views[i], sc.scene_of(i), sc))
      if (std::find(distinct.begin(), distinct.end(), f) == distinct.end()) distinct.push_back(f);
  out->clear();
  if (distinct.size() == 1 && !any_scene) {
    Launch L;
    L.table = nd_formula_at(distinct[0])->kernels();
    L.members = distinct;
    for (int i = 0; i < nviews; ++i) {
      L.views.push_back(i);
      L.codes.push_back(0);
    }
    L.key = set_key(distinct);
    out->push_back(L);
    return ND_OK;
  }
  // one launch when a compiled group covers every formula of the batch
  for (int g = 0; g < nd_group_entry_count; ++g) {
    const nd::GroupEntry& G = nd_group_entries[g];
    bool covers = true;
    for (int f : distinct) {
      bool in = false;
      for (int m = 0; m < G.count; ++m) in |= G.members[m] == f;
      covers &= in;
    }
    if (!covers) continue;
    Launch L;
    L.table = G.kernels();
    L.members.assign(G.members, G.members + G.count);
    // Views are grouped by formula code so that warps stay formula-uniform, and the
    // groups go in decreasing order of their views' mean formula iteration count (a
    // view's cost per DE evaluation): the persistent kernel hands out rays in table
    // order, so the rays still in flight when the work list runs out, which set how
    // long the last warps run with few lanes busy, are the cheapest ones.
    std::vector<int> order(nviews);
    for (int i = 0; i < nviews; ++i) order[i] = i;
    auto code_of = [&](int vi) {
      const int f = view_formulas(views[vi], sc.scene_of(vi), sc)[0];
      for (int m = 0; m < G.count; ++m)
        if (G.members[m] == f) return m;
      return 0;
    };
    std::vector<double> cost_sum(G.count, 0.0);
    std::vector<int> cost_n(G.count, 0);
    for (int i = 0; i < nviews; ++i) {
      double c = 0.0;
      const int k = sc.scene_of(i);
      if (k < 0) {
        c = view_iterations(views[i].formula, views[i].params);
      } else {
        const nd_scene_desc& S = sc.scenes[k];
        for (int j = 0; j < S.instance_count && j < ND_MAX_INSTANCES; ++j)
          c += view_iterations(S.instances[j].formula, S.instances[j].params);
      }
      cost_sum[code_of(i)] += c;
      ++cost_n[code_of(i)];
    }
    std::vector<int> rank(G.count);
    for (int m = 0; m < G.count; ++m) rank[m] = m;
    auto mean = [&](int m) { return cost_n[m] ? cost_sum[m] / cost_n[m] : 0.0; };
    std::stable_sort(rank.begin(), rank.end(), [&](int a, int b) { return mean(a) > mean(b); });
    std::vector<int> pos(G.count);
    for (int r = 0; r < G.count; ++r) pos[rank[r]] = r;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return pos[code_of(a)] < pos[code_of(b)]; });
    for (int vi : order) {
      L.views.push_back(vi);
      L.codes.push_back(code_of(vi));
    }
    L.key = std::string("group:") + G.name;
    out->push_back(L);
    return ND_OK;
  }
  if (any_scene) {
    std::string names;
    for (int f : distinct) names += std::string(names.empty() ? "" : ", ") + nd_formula_at(f)->name;
    return fail(ctx, ND_ERR_UNSUPPORTED, "the call's formulas (%s) are not in one compiled formula group "
                "(build with ND_GROUPS)", names.c_str());
  }
  // otherwise one launch per formula
  for (int f : distinct) {
    Launch L;
    L.table = nd_formula_at(f)->kernels();
    L.members = {f};
    for (int i = 0; i < nviews; ++i)
      if (views[i].formula == f) {
        L.views.push_back(i);
        L.codes.push_back(0);
      }
    L.key = set_key({f});
    out->push_back(L);
  }
  return ND_OK;
}

LaunchFn pick(const KernelTable& t, int kernel, int prec, bool batched, bool dir64, int block = 128) {
  if (kernel == ND_KERNEL_PLAIN) return prec == 64 ? t.plain_f64 : (dir64 ? t.plain_f32_dir64 : t.plain_f32);
  if (prec == 64) return batched ? t.persistent_f64_batched : t.persistent_f64;
  if (dir64) return batched ? t.persistent_f32_dir64_batched : t.persistent_f32_dir64;
  // block sizes other than 128 exist for the FP32 march (the autotuner's axis)
  if (block == 64 && (batched ? t.persistent_f32_batched_b64 : t.persistent_f32_b64))
    return batched ? t.persistent_f32_batched_b64 : t.persistent_f32_b64;
  if (block == 256 && (batched ? t.persistent_f32_batched_b256 : t.persistent_f32_b256))
    return batched ? t.persistent_f32_batched_b256 : t.persistent_f32_b256;
  return batched ? t.persistent_f32_batched : t.persistent_f32;
}

// The tuning key of a launch plan on a context's GPU: the GPU's name, the formula
// set, a hash of the set's formula sources (an edited formula is tuned anew) and the
// DE precision (the FP64 kernels fit fewer blocks per SM than the FP32 ones, so a
// residency tuned for one does not carry over to the other).
std::string tune_key(const nd_ctx* ctx, const Launch& L, int prec) {
  uint64_t h = 0xCBF29CE484222325ull;
  for (int f : L.members) {
    const uint64_t x = nd_formula_at(f)->source_hash;
    for (int b = 0; b < 8; ++b) {
      h ^= (x >> (8 * b)) & 0xffu;
      h *= 0x100000001B3ull;
    }
  }
  char hex[20];
  snprintf(hex, sizeof(hex), "%016llx", (unsigned long long)h);
  return ctx->gpu_name + "|" + L.key + "|" + hex + (prec == 64 ? "|fp64" : "|fp32");
}

Tuned tuned_for(const std::string& key) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tuned.find(key);
  return it == g_tuned.end() ? Tuned() : it->second;
}

// The kernels' table of a call's scenes; members: the formula group's formula ids in
// code order.
void scene_table(const SceneInput& sc, const std::vector<int>& members, std::vector<nd::DevScene>* out) {
  auto code_of = [&](int f) {
    for (size_t m = 0; m < members.size(); ++m)
      if (members[m] == f) return int(m);
    return -1;
  };
  out->assign(sc.nscenes, nd::DevScene());
  for (int k = 0; k < sc.nscenes; ++k) {
    const nd_scene_desc& S = sc.scenes[k];
    nd::DevScene& D = (*out)[k];
    memset(&D, 0, sizeof(D));
    D.count = S.instance_count;
    D.carve_count = S.carve_count;
    for (int i = 0; i < ND_MAX_INSTANCES && i < S.instance_count; ++i) {
      int mcode[ND_MAX_MIXINS] = {0, 0, 0};
      for (int j = 0; j < S.instances[i].mixin_count && j < ND_MAX_MIXINS; ++j)
        mcode[j] = code_of(S.instances[i].mixins[j].formula);
      D.inst[i] = nd::make_dev_instance(S.instances[i], code_of(S.instances[i].formula), mcode);
    }
    for (int c = 0; c < ND_MAX_CARVES; ++c)
      for (int q = 0; q < 4; ++q) D.carves[c][q] = S.carves[c][q];
  }
}

// Zeroes two word arrays (a statistics block and a call's counters).
__global__ void clear_words(unsigned long long* __restrict__ a, int na, unsigned long long* __restrict__ b, int nb) {
  for (int i = threadIdx.x; i < na; i += blockDim.x) a[i] = 0ull;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) b[i] = 0ull;
}

// Enqueue every launch of a forward call.  d_views / d_counters are device
// buffers with room for nviews views and kCountersPerPlan * plans.size() counters
// (work counters, hit counters, shadow-queue counts, shadow work counters);
// d_thit / d_hits / d_shadowq hold one entry per ray; h_views is host staging
// (pinned when owned by the context).  When views_ready is true the view
// table is already on the device (graph replay).
nd_status enqueue(nd_ctx* ctx, const nd_view_desc* views, int nviews, const nd_march_opts* opts,
                  const nd_gbuffer* out, cudaStream_t stream, const std::vector<Launch>& plans, DevView* d_views,
                  DevView* h_views, unsigned long long* d_counters, double* d_thit, nd::HitEntry* d_hits,
                  bool copy_views, int* kernel_used, cudaEvent_t* tev = nullptr,
                  const SceneInput& sc = SceneInput(), nd::DevScene* d_scenes = nullptr, float* d_accel = nullptr,
                  nd::AccelJob* d_jobs = nullptr, std::vector<nd::AccelJob>* jobs_out = nullptr,
                  nd::ShadowEntry* d_shadowq = nullptr, cudaStream_t upload = nullptr,
                  cudaEvent_t uploaded = nullptr) {
  const int prec = (opts && opts->de_precision == 64) ? 64 : 32;
  // global output offsets in call order
  std::vector<int64_t> out_off(nviews + 1, 0);
  for (int i = 0; i < nviews; ++i) out_off[i + 1] = out_off[i] + int64_t(views[i].spp) * views[i].tile_w * views[i].tile_h;
  // accelerator grids: one region of d_accel per view that has one, and per plan
  // the build jobs (plan-local view index, first voxel in the plan's voxel order)
  std::vector<nd::AccelJob> jobs;
  std::vector<int> job_begin(plans.size() + 1, 0);
  std::vector<int64_t> plan_voxels(plans.size(), 0);
  int64_t voxel_off = 0;
  int base = 0;
  for (size_t p = 0; p < plans.size(); ++p) {
    const Launch& L = plans[p];
    int64_t off = 0;
    job_begin[p] = int(jobs.size());
    for (size_t k = 0; k < L.views.size(); ++k) {
      const int vi = L.views[k];
      h_views[base + k] = make_dev_view(views[vi], off, out_off[vi], L.codes[k]);
      h_views[base + k].scene = sc.scene_of(vi);
      off += h_views[base + k].rays;
      const int64_t nvox = nd::accel_voxels_of(views[vi]);
      if (nvox > 0) {
        if (!d_accel || !d_jobs) return fail(ctx, ND_ERR_UNSUPPORTED, "view %d: no accelerator memory on this path", vi);
        nd::place_accel(h_views[base + k], views[vi], d_accel + voxel_off);
        nd::AccelJob j;
        j.view = int32_t(k);
        j.pad = 0;
        j.begin = plan_voxels[p];
        jobs.push_back(j);
        plan_voxels[p] += nvox;
        voxel_off += nvox;
      }
    }
    base += int(L.views.size());
  }
  job_begin[plans.size()] = int(jobs.size());
  if (jobs_out) *jobs_out = jobs;
  if (copy_views && !jobs.empty()) {
    // from pageable memory: returns once the jobs are staged
    cudaError_t e = cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(nd::AccelJob) * jobs.size(), cudaMemcpyHostToDevice,
                                    stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "copy accelerator jobs");
  }
  if (copy_views && sc.nscenes > 0 && d_scenes) {
    // scenes are only accepted when one formula group covers the call: one plan
    std::vector<nd::DevScene> hs;
    scene_table(sc, plans[0].members, &hs);
    // from pageable memory: returns once the table is staged, so hs may go
    cudaError_t e = cudaMemcpyAsync(d_scenes, hs.data(), sizeof(nd::DevScene) * hs.size(), cudaMemcpyHostToDevice,
                                    stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "copy scenes");
  }
  if (copy_views && base > 0) {
    // on the upload stream when there is one (the march waits for it there)
    cudaStream_t cs = upload && uploaded ? upload : stream;
    cudaError_t e = cudaMemcpyAsync(d_views, h_views, sizeof(DevView) * size_t(base), cudaMemcpyHostToDevice, cs);
    if (e == cudaSuccess && cs != stream) {
      e = cudaEventRecord(uploaded, cs);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, uploaded, 0);
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "copy view table");
  }
  // the statistics block and the counters: one small kernel instead of two memsets
  // (every command a forward enqueues is fetched over the bus, which a caller's
  // device-to-host read-back of an earlier frame may be keeping busy)
  static_assert(sizeof(Stats) % sizeof(unsigned long long) == 0, "the statistics block clears in 8-byte words");
  clear_words<<<1, 256, 0, stream>>>(reinterpret_cast<unsigned long long*>(ctx->d_stats),
                                     int(sizeof(Stats) / sizeof(unsigned long long)), d_counters,
                                     kCountersPerPlan * int(plans.size()));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "clear stats and work counters");
  base = 0;
  int used = 0;
  int64_t ray_base = 0;  // where this plan's rays start in d_hits
  const bool want_trap = out->trap || out->iters;
  for (size_t p = 0; p < plans.size(); ++p) {
    const Launch& L = plans[p];
    const int nv = int(L.views.size());
    int64_t rays = 0;
    for (int k = 0; k < nv; ++k) rays += h_views[base + k].rays;
    if (rays > 0) {
      const Tuned tu = tuned_for(tune_key(ctx, L, prec));
      int kernel = opts && opts->kernel ? opts->kernel : tu.kernel;
      const bool accel = plan_voxels[p] > 0;
      // Untuned, one view with no more rays than the persistent grid has lanes runs the
      // plain launch: with one ray per lane there is nothing to refill, and the plain
      // loop has no ballot per pass and no second pass for the normals (10 % faster on
      // a 256 x 256 Mandelbulb).
      if (!(opts && opts->kernel) && !tu.tuned && nv == 1 && !accel && sc.nscenes == 0 && L.table.resident_b128 &&
          rays <= int64_t(L.table.resident_b128(0)) * ctx->num_sms * 128)
        kernel = ND_KERNEL_PLAIN;
      if (accel && kernel == ND_KERNEL_PLAIN) {
        if (opts && opts->kernel == ND_KERNEL_PLAIN)
          return fail(ctx, ND_ERR_UNSUPPORTED, "the empty-space accelerator runs on the persistent kernel only");
        kernel = ND_KERNEL_PERSISTENT;
      }
      LaunchArgs a;
      memset(&a, 0, sizeof(a));
      a.views = d_views + base;
      a.nviews = nv;
      a.total_rays = rays;
      if (rays > int64_t(0x7fffffff)) return fail(ctx, ND_ERR_INVALID, "more than 2^31-1 rays in one launch");
      a.out = *out;
      a.t_hit = d_thit;
      a.counter = d_counters + p;
      a.scenes = d_scenes;
      a.stats = ctx->d_stats;
      // untuned, an FP64 DE (tens of FP64 iterations per evaluation) refills at 2 idle
      // lanes: on the 4096^2 deep-zoom frame 416 ms against 437 at 6 and 490 at 12
      const int thr_default = tu.tuned || prec != 64 ? tu.refill_threshold : 2;
      a.refill_threshold = std::max(1, std::min(32, opts && opts->refill_threshold ? opts->refill_threshold : thr_default));
      // 4 jumps per pass measured fastest on batched views (1, 2, 4 and no limit tried)
      const int chain = opts ? opts->accel_chain : 0;
      a.accel_chain = chain > 0 ? chain : (chain < 0 ? 0 : 4);
      const int wd = opts && opts->watchdog_ms > 0 ? opts->watchdog_ms : 10000;
      a.deadline_ns = int64_t(wd) * 1000000;
      LaunchConfig c;
      c.kernel = kernel;
      c.block = opts && opts->block ? opts->block : tu.block;
      c.blocks_per_sm = opts && opts->blocks_per_sm ? opts->blocks_per_sm : tu.blocks_per_sm;
      c.num_sms = ctx->num_sms;
      bool dir64 = false;
      for (int k = 0; k < nv; ++k) dir64 |= h_views[base + k].dir64 != 0;
      // the persistent march leaves the normal taps and shadow rays of its hits to
      // the shade pass
      const bool defer = kernel != ND_KERNEL_PLAIN && d_hits != nullptr && d_thit != nullptr;
      if (tev) cudaEventRecord(tev[4 * p], stream);
      if (sc.nscenes > 0 && kernel == ND_KERNEL_PLAIN)
        return fail(ctx, ND_ERR_UNSUPPORTED, "scenes run on the persistent kernel only");
      const nd::KernelTable& T = L.table;
      const bool scn = sc.nscenes > 0;
      if (accel) {
        if (prec == 32 && dir64)
          return fail(ctx, ND_ERR_UNSUPPORTED,
                      "the empty-space accelerator needs FP32 ray directions or an FP64 DE (deep-zoom view)");
        if (!defer) return fail(ctx, ND_ERR_UNSUPPORTED, "the empty-space accelerator needs the deferred shade pass");
        nd::AccelBuildFn bf = scn ? (prec == 64 ? T.scene_accel_build_f64 : T.scene_accel_build_f32)
                                  : (prec == 64 ? T.accel_build_f64 : T.accel_build_f32);
        if (!bf) return fail(ctx, ND_ERR_UNSUPPORTED, "no accelerator kernels in this formula set");
        e = bf(d_views + base, d_jobs + job_begin[p], job_begin[p + 1] - job_begin[p], plan_voxels[p],
               scn ? d_scenes : nullptr, ctx->num_sms, stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "accelerator build launch");
      }
      if (tev) cudaEventRecord(tev[4 * p + 1], stream);
      if (kernel == ND_KERNEL_PLAIN) {
        // the plain baseline: one launch per view, one thread per ray
        for (int k = 0; k < nv; ++k) {
          LaunchFn fn = pick(L.table, kernel, prec, false, h_views[base + k].dir64 != 0);
          if (!fn) return fail(ctx, ND_ERR_UNSUPPORTED, "no plain kernel for this formula set");
          e = fn(a, h_views[base + k], c, stream);
          if (e != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
        }
      } else {
        const bool batched = nv > 1;
        LaunchFn fn = pick(L.table, kernel, prec, batched, dir64, c.block);
        if (scn) {
          fn = prec == 64 ? T.scene_persistent_f64 : (dir64 ? T.scene_persistent_f32_dir64 : T.scene_persistent_f32);
          if (!fn) return fail(ctx, ND_ERR_UNSUPPORTED, "no scene kernels in this formula set");
        }
        if (accel) {
          fn = scn ? (prec == 64 ? T.scene_persistent_f64_accel : T.scene_persistent_f32_accel)
                   : (prec == 64 ? T.persistent_f64_accel : T.persistent_f32_accel);
          if (!fn) return fail(ctx, ND_ERR_UNSUPPORTED, "no accelerator kernels in this formula set");
        }
        if (defer) {
          a.hit_list = d_hits + ray_base;
          a.hit_count = reinterpret_cast<unsigned int*>(d_counters + plans.size() + p);
        }
        // the wavefront shadow pass: shadow rays queued by the surface pass and marched
        // by the persistent shadow kernel (the accelerator's shadow skips run inline)
        bool shadows = false;
        for (int k = 0; k < nv; ++k) shadows |= nd::casts_shadow(h_views[base + k]);
        if (defer && !accel && shadows && d_shadowq) {
          a.shadow_queue = d_shadowq + ray_base;
          a.shadow_count = reinterpret_cast<unsigned int*>(d_counters + 2 * plans.size() + p);
          a.shadow_counter = d_counters + 3 * plans.size() + p;
        }
        if (!fn) return fail(ctx, ND_ERR_UNSUPPORTED, "no persistent kernel for this formula set");
        e = fn(a, h_views[base], c, stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
      }
      if (tev) cudaEventRecord(tev[4 * p + 2], stream);
      if (defer || want_trap) {
        // normals of the deferred hits and/or the orbit trap at every hit point
        const bool batched = nv > 1;
        nd::ShadeFn sf = prec == 64 ? (batched ? T.shade_f64_batched : T.shade_f64)
                                    : dir64 ? (batched ? T.shade_f32_dir64_batched : T.shade_f32_dir64)
                                            : (batched ? T.shade_f32_batched : T.shade_f32);
        if (scn) sf = prec == 64 ? T.scene_shade_f64 : (dir64 ? T.scene_shade_f32_dir64 : T.scene_shade_f32);
        if (accel)
          sf = scn ? (prec == 64 ? T.scene_shade_f64_accel : T.scene_shade_f32_accel)
                   : (prec == 64 ? T.shade_f64_accel : T.shade_f32_accel);
        if (!sf) return fail(ctx, ND_ERR_UNSUPPORTED, "no shade kernel for this formula set");
        e = sf(a, h_views[base], c, want_trap ? 1 : 0, stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "shade pass launch");
        if (a.shadow_queue) {
          nd::ShadowFn hf = scn ? (prec == 64 ? T.scene_shadow_f64 : T.scene_shadow_f32)
                                : (prec == 64 ? T.shadow_f64 : T.shadow_f32);
          if (!hf) return fail(ctx, ND_ERR_UNSUPPORTED, "no shadow kernels in this formula set");
          LaunchConfig sc2 = c;
          sc2.blocks_per_sm = 0;
          e = hf(a, sc2, stream);
          if (e != cudaSuccess) return cuda_fail(ctx, e, "shadow pass launch");
        }
      }
      if (tev) cudaEventRecord(tev[4 * p + 3], stream);
      used = kernel;
    } else if (tev) {
      // a plan with no rays: its timing events mark an empty interval
      for (int k = 0; k < 4; ++k) cudaEventRecord(tev[4 * p + k], stream);
    }
    base += nv;
    ray_base += rays;
  }
  if (kernel_used) *kernel_used = used;
  return ND_OK;
}

nd_status prepare(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews, const nd_gbuffer* out,
                  std::vector<Launch>* plans, int64_t* total, const SceneInput& sc = SceneInput()) {
  if (!ctx) return ND_ERR_INVALID;
  if (!views || nviews <= 0 || nviews > kMaxViews) return fail(ctx, ND_ERR_INVALID, "nviews %d out of range", nviews);
  if (!out || !out->depth) return fail(ctx, ND_ERR_INVALID, "the G-buffer needs at least a depth pointer");
  if ((out->normal && (uintptr_t(out->normal) & 15)) || (out->depth64 && (uintptr_t(out->depth64) & 7)) ||
      (out->normal_half && (uintptr_t(out->normal_half) & 7)) || (uintptr_t(out->depth) & 3))
    return fail(ctx, ND_ERR_INVALID, "misaligned G-buffer pointer (normal needs 16 bytes, normal_half 8)");
  int64_t t = 0;
  for (int i = 0; i < nviews; ++i) {
    nd_status s = validate_view(ctx, views[i], i);
    if (s != ND_OK) return s;
    t += int64_t(views[i].spp) * views[i].tile_w * views[i].tile_h;
    if (t > kMaxRays) return fail(ctx, ND_ERR_INVALID, "too many rays in one call");
  }
  *total = t;
  for (int i = 0; i < nviews; ++i) {
    const int k = sc.scene_of(i);
    if (k < -1 || k >= sc.nscenes) return fail(ctx, ND_ERR_INVALID, "view %d: scene index %d out of range", i, k);
    if (k < 0) continue;
    const nd_scene_desc& S = sc.scenes[k];
    if (S.instance_count < 1 || S.instance_count > ND_MAX_INSTANCES || S.carve_count < 0 ||
        S.carve_count > ND_MAX_CARVES)
      return fail(ctx, ND_ERR_INVALID, "scene %d: instance_count 1..%d, carve_count 0..%d", k, ND_MAX_INSTANCES,
                  ND_MAX_CARVES);
    for (int j = 0; j < S.instance_count; ++j) {
      const nd_instance_desc& in = S.instances[j];
      if (in.formula < 0 || in.formula >= nd_formula_total() || in.mixin_count < 0 ||
          in.mixin_count > ND_MAX_MIXINS || in.combine_mode < ND_COMBINE_UNION || in.combine_mode > ND_COMBINE_SMOOTH_MIX)
        return fail(ctx, ND_ERR_INVALID, "scene %d instance %d: bad formula, mixin count or combine mode", k, j);
      for (int m = 0; m < in.mixin_count; ++m)
        if (in.mixins[m].formula < 0 || in.mixins[m].formula >= nd_formula_total())
          return fail(ctx, ND_ERR_INVALID, "scene %d instance %d mixin %d: bad formula", k, j, m);
    }
  }
  return plan(ctx, views, nviews, plans, sc);
}

}  // namespace

// ---------------------------------------------------------------- run-time formulas
// Formulas that nd_formula_register compiled at run time, after the build-time table.
// An entry is written completely before the count that publishes it, and entries are
// never removed (their libraries stay loaded), so readers need no lock.
namespace {
constexpr int kMaxRuntimeFormulas = 256;
nd::FormulaEntry g_rt_entries[kMaxRuntimeFormulas];
std::atomic<int> g_rt_count{0};
std::mutex g_rt_mu;  // one compile at a time

std::string shell_quote(const std::string& s) {
  std::string q = "'";
  for (char c : s) q += (c == '\'') ? std::string("'\\''") : std::string(1, c);
  return q + "'";
}

// Removes a compile directory and everything in it (files and the one level of
// subdirectories the compile worker makes).  A loaded library stays mapped after its
// file is gone.
void remove_tree(const std::string& path) {
  if (DIR* d = opendir(path.c_str())) {
    while (const dirent* ent = readdir(d)) {
      const std::string name = ent->d_name;
      if (name == "." || name == "..") continue;
      const std::string sub = path + "/" + name;
      if (unlink(sub.c_str()) != 0) remove_tree(sub);
    }
    closedir(d);
  }
  rmdir(path.c_str());
}

// The compile worker: the build's translator and nvcc, run as a child process
// (numericdream_b200/rtc.py beside this library) into a temporary directory, then the
// resulting library loaded and its entry published.  ND_PYTHON names the Python
// interpreter (default python3); ND_RTC_DIR the parent of the temporary directories
// (default /tmp).
nd_status runtime_compile(const char* src, size_t len, uint64_t hash, nd_formula_id* out, std::string* msg) {
  std::lock_guard<std::mutex> lk(g_rt_mu);
  const int have = g_rt_count.load(std::memory_order_acquire);
  for (int i = 0; i < have; ++i)  // compiled by another thread while this one waited
    if (g_rt_entries[i].source_hash == hash) {
      *out = nd_formula_entry_count + i;
      return ND_OK;
    }
  if (have >= kMaxRuntimeFormulas) {
    *msg = "too many formulas compiled at run time (at most 256)";
    return ND_ERR_COMPILE;
  }
  Dl_info info;
  if (!dladdr(reinterpret_cast<void*>(&runtime_compile), &info) || !info.dli_fname) {
    *msg = "cannot locate the library to find its formula compiler";
    return ND_ERR_COMPILE;
  }
  std::string pkg = info.dli_fname;
  pkg = pkg.substr(0, pkg.find_last_of('/'));
  const std::string root = pkg.substr(0, pkg.find_last_of('/'));
  const char* base = getenv("ND_RTC_DIR");
  std::string tmpl = std::string(base && *base ? base : "/tmp") + "/nd_rtc_XXXXXX";
  std::vector<char> dirbuf(tmpl.begin(), tmpl.end());
  dirbuf.push_back(0);
  if (!mkdtemp(dirbuf.data())) {
    *msg = "cannot create a directory under " + tmpl;
    return ND_ERR_COMPILE;
  }
  const std::string dir = dirbuf.data();
  FILE* f = fopen((dir + "/formula.wgsl").c_str(), "wb");
  if (!f || fwrite(src, 1, len, f) != len) {
    if (f) fclose(f);
    *msg = "cannot write the formula source to " + dir;
    remove_tree(dir);
    return ND_ERR_COMPILE;
  }
  fclose(f);
  const char* py = getenv("ND_PYTHON");
  const std::string cmd = "cd " + shell_quote(root) + " && " + shell_quote(py && *py ? py : "python3") +
                          " -m numericdream_b200.rtc " + shell_quote(dir + "/formula.wgsl") + " " + shell_quote(dir) +
                          " > " + shell_quote(dir + "/log.txt") + " 2>&1";
  const int rc = system(cmd.c_str());
  if (rc != 0) {
    std::string text;
    FILE* e = fopen((dir + "/error.txt").c_str(), "rb");
    if (!e) e = fopen((dir + "/log.txt").c_str(), "rb");
    if (e) {
      char buf[1024];
      size_t n;
      while ((n = fread(buf, 1, sizeof(buf), e)) > 0 && text.size() < 8192) text.append(buf, n);
      fclose(e);
    }
    *msg = text.empty() ? "the formula compiler failed (" + cmd + ")" : text;
    remove_tree(dir);
    return ND_ERR_COMPILE;
  }
  void* lib = dlopen((dir + "/formula.so").c_str(), RTLD_NOW | RTLD_LOCAL);
  remove_tree(dir);  // the loaded library stays mapped
  if (!lib) {
    const char* de = dlerror();
    *msg = std::string("cannot load the compiled formula: ") + (de ? de : "?");
    return ND_ERR_COMPILE;
  }
  typedef const nd::FormulaEntry* (*EntryFn)();
  EntryFn fn = reinterpret_cast<EntryFn>(dlsym(lib, "nd_rtc_entry"));
  const nd::FormulaEntry* e = fn ? fn() : nullptr;
  if (!e || e->source_hash != hash) {
    dlclose(lib);
    *msg = "the compiled formula library does not match the source";
    return ND_ERR_COMPILE;
  }
  g_rt_entries[have] = *e;
  g_rt_count.store(have + 1, std::memory_order_release);
  *out = nd_formula_entry_count + have;
  return ND_OK;
}
}  // namespace

const nd::FormulaEntry* nd_formula_at(int id) {
  if (id >= 0 && id < nd_formula_entry_count) return &nd_formula_entries[id];
  const int k = id - nd_formula_entry_count;
  if (k >= 0 && k < g_rt_count.load(std::memory_order_acquire)) return &g_rt_entries[k];
  return nullptr;
}

int nd_formula_total() { return nd_formula_entry_count + g_rt_count.load(std::memory_order_acquire); }

extern "C" {

int32_t nd_abi_version(void) { return ND_ABI_VERSION; }

const char* nd_status_string(nd_status s) {
  if (s < 0 || s > 7) return "ND_ERR_UNKNOWN";
  return kStatusNames[s];
}

nd_status nd_formula_count(int32_t* n) {
  if (!n) return ND_ERR_INVALID;
  *n = nd_formula_total();
  return ND_OK;
}

nd_status nd_formula_find(const char* name, nd_formula_id* out) {
  if (!name || !out) return ND_ERR_INVALID;
  for (int i = 0; i < nd_formula_total(); ++i)
    if (strcmp(nd_formula_at(i)->name, name) == 0) {
      *out = i;
      return ND_OK;
    }
  return ND_ERR_NOT_FOUND;
}

nd_status nd_formula_name(nd_formula_id id, char* out, size_t out_len) {
  if (id < 0 || id >= nd_formula_total()) return ND_ERR_NOT_FOUND;
  if (!out || out_len == 0) return ND_ERR_INVALID;
  copy_str(out, out_len, nd_formula_at(id)->name);
  return ND_OK;
}

// The reference compiles a formula source into the scene's shader module on a worker
// thread (rebuildAsync, fractal_renderer.zig:2951; compileWorker :1609) and reports
// errors into FormulaState.formula_error (formula.zig:73-77, 170-181).  Registering a
// source checks the contract functions like missingContractFn, then finds compiled
// code by the source hash (CodeTable.find, fractal_renderer.zig:585-590): the
// build-time formulas, then those compiled earlier at run time.  A new source is
// compiled now (runtime_compile) and gets the next id.
nd_status nd_formula_register(const char* src, size_t len, nd_formula_id* out, char* err, size_t err_len) {
  if (!src || !out) {
    copy_str(err, err_len, "null argument");
    return ND_ERR_INVALID;
  }
  const std::string s(src, len);
  const char* missing = nullptr;
  if (s.find("fn de_step(") == std::string::npos)
    missing = "fn de_step(carry: IterCarry, pos: vec3f, p: Params) -> IterCarry";
  else if (s.find("fn de_finalize(") == std::string::npos)
    missing = "fn de_finalize(carry: IterCarry) -> f32";
  else if (s.find("fn de_iterations(") == std::string::npos)
    missing = "fn de_iterations(p: Params) -> i32";
  if (missing) {
    copy_str(err, err_len, std::string("missing: ") + missing);
    return ND_ERR_COMPILE;
  }
  const uint64_t h = fnv1a64(src, len);
  for (int i = 0; i < nd_formula_total(); ++i)
    if (nd_formula_at(i)->source_hash == h) {
      *out = i;
      copy_str(err, err_len, "");
      return ND_OK;
    }
  std::string msg;
  const nd_status st = runtime_compile(src, len, h, out, &msg);
  copy_str(err, err_len, msg);
  return st;
}

nd_status nd_formula_params(nd_formula_id id, nd_param_info* out, int32_t* n) {
  if (id < 0 || id >= nd_formula_total()) return ND_ERR_NOT_FOUND;
  if (!n) return ND_ERR_INVALID;
  const nd::FormulaEntry& f = (*nd_formula_at(id));
  if (out) {
    for (int i = 0; i < f.nparams; ++i) {
      memset(&out[i], 0, sizeof(nd_param_info));
      copy_str(out[i].name, ND_PARAM_NAME_LEN, f.params[i].name);
      out[i].min_value = f.params[i].min_value;
      out[i].max_value = f.params[i].max_value;
      out[i].default_value = f.params[i].default_value;
      out[i].integral = f.params[i].integral;
    }
  }
  *n = f.nparams;
  return ND_OK;
}

// Defaults of the reference's render settings (render_precision.zig:3-30,
// scene_state.zig:192-210) with the formula's @param defaults packed in.
nd_status nd_view_defaults(nd_formula_id id, nd_view_desc* v) {
  if (id < 0 || id >= nd_formula_total()) return ND_ERR_NOT_FOUND;
  if (!v) return ND_ERR_INVALID;
  memset(v, 0, sizeof(*v));
  v->cam_pos[2] = -3.0;
  v->fwd[2] = 1.0;
  v->right[0] = 1.0;
  v->up[1] = 1.0;
  v->width = v->height = v->tile_w = v->tile_h = 256;
  v->formula = id;
  v->spp = 1;
  const nd::FormulaEntry& f = (*nd_formula_at(id));
  for (int i = 0; i < f.nparams; ++i) v->params[i] = f.params[i].default_value;
  v->trap.shape = ND_TRAP_POINT;
  v->trap.mode = ND_TRAP_MIN;
  v->trap.radius = 1.0f;
  v->trap.box[0] = v->trap.box[1] = v->trap.box[2] = 1.0f;
  v->trap.span = 1.5f;
  v->max_steps = 256;
  v->max_dist = 24.0f;
  v->eps_coef = 5e-4f;
  v->eps_floor = 5e-5f;
  v->refine_budget = 4;
  v->hq_footprint_px = 2.0f;
  v->normal_mode = ND_NORMAL_TETRA;
  v->shadow_k = 16.0f;
  v->step_safety = 1.0f;
  return ND_OK;
}

nd_status nd_ctx_create(int32_t device, nd_ctx** out) {
  if (!out) return ND_ERR_INVALID;
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) return ND_ERR_CUDA;
  if (device < 0 || device >= count) return ND_ERR_INVALID;
  nd_ctx* ctx = new nd_ctx();
  ctx->device = device;
  e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) {
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, device);
    if (e == cudaSuccess) ctx->gpu_name = prop.name;
  }
  if (e == cudaSuccess) e = cudaMalloc((void**)&ctx->d_stats, sizeof(Stats));
  if (e == cudaSuccess) e = cudaMemset(ctx->d_stats, 0, sizeof(Stats));
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->last_done, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    nd_ctx_destroy(ctx);
    return e == cudaErrorMemoryAllocation ? ND_ERR_OOM : ND_ERR_CUDA;
  }
  *out = ctx;
  return ND_OK;
}

nd_status nd_ctx_destroy(nd_ctx* ctx) {
  if (!ctx) return ND_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (ctx->have_last) cudaEventSynchronize(ctx->last_done);
  if (ctx->d_views) cudaFree(ctx->d_views);
  if (ctx->d_fviews) cudaFree(ctx->d_fviews);
  if (ctx->upload) cudaStreamDestroy(ctx->upload);
  for (int k = 0; k < 2; ++k)
    if (ctx->uploaded[k]) cudaEventDestroy(ctx->uploaded[k]);
  if (ctx->d_counters) cudaFree(ctx->d_counters);
  if (ctx->d_stats) cudaFree(ctx->d_stats);
  if (ctx->d_thit) cudaFree(ctx->d_thit);
  if (ctx->d_hits) cudaFree(ctx->d_hits);
  if (ctx->d_shadowq) cudaFree(ctx->d_shadowq);
  if (ctx->d_scenes) cudaFree(ctx->d_scenes);
  if (ctx->d_accel) cudaFree(ctx->d_accel);
  if (ctx->d_accel_jobs) cudaFree(ctx->d_accel_jobs);
  if (ctx->d_lite) cudaFree(ctx->d_lite);
  for (int k = 0; k < 2; ++k)
    if (ctx->staged[k]) {
      if (ctx->staged_valid[k]) cudaEventSynchronize(ctx->staged[k]);
      cudaEventDestroy(ctx->staged[k]);
    }
  if (ctx->h_views) cudaFreeHost(ctx->h_views);
  if (ctx->last_done) cudaEventDestroy(ctx->last_done);
  for (cudaEvent_t ev : ctx->tev) cudaEventDestroy(ev);
  delete ctx;
  return ND_OK;
}

nd_status nd_last_error(const nd_ctx* ctx, char* out, size_t out_len) {
  if (!ctx) return ND_ERR_INVALID;
  copy_str(out, out_len, ctx->err);
  return ND_OK;
}

nd_status nd_count_rays(const nd_view_desc* views, int32_t nviews, int64_t* total) {
  if (!views || !total || nviews < 0) return ND_ERR_INVALID;
  int64_t t = 0;
  for (int i = 0; i < nviews; ++i) {
    if (views[i].spp < 0 || views[i].tile_w < 0 || views[i].tile_h < 0) return ND_ERR_INVALID;
    t += int64_t(views[i].spp) * views[i].tile_w * views[i].tile_h;
  }
  *total = t;
  return ND_OK;
}

}  // extern "C"

namespace {
nd_status forward_impl(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews, const nd_march_opts* opts,
                       const nd_gbuffer* out, void* stream, const SceneInput& sc) {
  std::vector<Launch> plans;
  int64_t total = 0;
  nd_status s = prepare(ctx, views, nviews, out, &plans, &total, sc);
  if (s != ND_OK) return s;
  if (opts && opts->de_precision != 0 && opts->de_precision != 32 && opts->de_precision != 64)
    return fail(ctx, ND_ERR_INVALID, "de_precision must be 32 or 64");
  if (opts && opts->block != 0 && opts->block != 64 && opts->block != 128 && opts->block != 256)
    return fail(ctx, ND_ERR_INVALID, "block must be 0, 64, 128 or 256");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "set device");
  cudaStream_t st = (cudaStream_t)stream;
  // The device scratch (view table, counters, hit buffers) is reused by every call:
  // order this call after the previous one on the device (free on the same stream),
  // without blocking the host, so that a caller can enqueue the next frame while this
  // one runs.  The pinned staging alternates between two halves; a half is reused
  // once the call two back, which read it, is done.
  if (ctx->have_last && ctx->last_stream != st) cudaStreamWaitEvent(st, ctx->last_done, 0);
  const int half = int(ctx->calls & 1);
  for (int k = 0; k < 2; ++k)
    if (!ctx->staged[k] && (e = cudaEventCreateWithFlags(&ctx->staged[k], cudaEventDisableTiming)) != cudaSuccess)
      return cuda_fail(ctx, e, "staging event");
  if (ctx->staged_valid[half]) cudaEventSynchronize(ctx->staged[half]);
  if ((s = ensure_forward_views(ctx, nviews)) != ND_OK) return s;
  if ((s = ensure_dev(ctx, &ctx->d_counters, &ctx->counters_cap, kCountersPerPlan * int(plans.size()),
                      "work counters")) != ND_OK)
    return s;
  bool any_shadow = false;
  for (int i = 0; i < nviews; ++i) any_shadow |= views[i].shadow != 0;
  if (any_shadow && ctx->shadowq_cap < total) {
    if (ctx->d_shadowq) cudaFree(ctx->d_shadowq);
    ctx->d_shadowq = nullptr;
    ctx->shadowq_cap = 0;
    e = cudaMalloc((void**)&ctx->d_shadowq, sizeof(nd::ShadowEntry) * size_t(total));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "shadow queue");
    ctx->shadowq_cap = total;
  }
  const bool want_trap = out->trap || out->iters;
  if (ctx->thit_cap < total) {
    if (ctx->d_thit) cudaFree(ctx->d_thit);
    if (ctx->d_hits) cudaFree(ctx->d_hits);
    ctx->d_thit = nullptr;
    ctx->d_hits = nullptr;
    ctx->thit_cap = 0;
    e = cudaMalloc((void**)&ctx->d_thit, sizeof(double) * size_t(total));
    if (e == cudaSuccess) e = cudaMalloc((void**)&ctx->d_hits, sizeof(nd::HitEntry) * size_t(total));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "hit buffers");
    ctx->thit_cap = total;
  }
  if ((s = ensure_staging(ctx, nviews)) != ND_OK) return s;
  DevView* staging = ctx->h_views + size_t(half) * ctx->h_views_cap;
  int64_t voxels = 0;
  int accel_views = 0;
  for (int i = 0; i < nviews; ++i) {
    const int64_t nv = nd::accel_voxels_of(views[i]);
    voxels += nv;
    accel_views += nv > 0 ? 1 : 0;
  }
  if (voxels > 0 && ctx->accel_cap < voxels) {
    if (ctx->d_accel) cudaFree(ctx->d_accel);
    ctx->d_accel = nullptr;
    ctx->accel_cap = 0;
    e = cudaMalloc((void**)&ctx->d_accel, sizeof(float) * size_t(voxels));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "accelerator grids");
    ctx->accel_cap = voxels;
  }
  if (accel_views > 0 &&
      (s = ensure_dev(ctx, &ctx->d_accel_jobs, &ctx->accel_jobs_cap, accel_views, "accelerator jobs")) != ND_OK)
    return s;
  while (ctx->tev.size() < 4 * plans.size()) {
    cudaEvent_t ev;
    e = cudaEventCreate(&ev);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "timing event");
    ctx->tev.push_back(ev);
  }
  int kernel = 0;
  if (sc.nscenes > 0 && (s = ensure_dev(ctx, &ctx->d_scenes, &ctx->scenes_cap, sc.nscenes, "scene table")) != ND_OK)
    return s;
  // the view table goes up on the upload stream as soon as this call is made: it
  // then overlaps the previous call's march instead of waiting at the head of this
  // call for the bus, where a caller's device-to-host read-back of the previous frame
  // would slow it down
  // (a caller capturing its stream into a graph gets the copy on that stream)
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if ((e = cudaStreamIsCapturing(st, &cap)) != cudaSuccess) return cuda_fail(ctx, e, "stream capture status");
  const bool side = cap == cudaStreamCaptureStatusNone;
  s = enqueue(ctx, views, nviews, opts, out, st, plans, ctx->d_fviews + size_t(half) * ctx->fviews_half, staging,
              ctx->d_counters, ctx->d_thit, ctx->d_hits, true, &kernel, ctx->tev.data(), sc,
              sc.nscenes > 0 ? ctx->d_scenes : nullptr, ctx->d_accel, ctx->d_accel_jobs, nullptr,
              any_shadow ? ctx->d_shadowq : nullptr, side ? ctx->upload : nullptr,
              side ? ctx->uploaded[half] : nullptr);
  ctx->tev_plans = s == ND_OK ? int(plans.size()) : 0;
  if (s != ND_OK) return s;
  e = cudaEventRecord(ctx->last_done, st);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->staged[half], st);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "record event");
  ctx->staged_valid[half] = true;
  ++ctx->calls;
  ctx->have_last = true;
  ctx->last_stream = st;
  ctx->last_kernel = kernel;
  ctx->last_rays = total;
  ctx->last_trap = want_trap;
  ctx->last_accel_voxels = uint64_t(voxels);
  return ND_OK;
}
}  // namespace

extern "C" {

nd_status nd_march_forward(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews, const nd_march_opts* opts,
                           const nd_gbuffer* out, void* stream) {
  return forward_impl(ctx, views, nviews, opts, out, stream, SceneInput());
}

nd_status nd_march_forward_scenes(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews, const int32_t* view_scene,
                                  const nd_scene_desc* scenes, int32_t nscenes, const nd_march_opts* opts,
                                  const nd_gbuffer* out, void* stream) {
  if (!ctx) return ND_ERR_INVALID;
  if (nscenes < 0 || (nscenes > 0 && (!scenes || !view_scene)))
    return fail(ctx, ND_ERR_INVALID, "scenes need a view_scene array and a scene array");
  SceneInput sc;
  sc.view_scene = view_scene;
  sc.scenes = scenes;
  sc.nscenes = nscenes;
  return forward_impl(ctx, views, nviews, opts, out, stream, sc);
}

nd_status nd_last_stats(nd_ctx* ctx, nd_stats* out) {
  if (!ctx || !out) return ND_ERR_INVALID;
  memset(out, 0, sizeof(*out));
  cudaSetDevice(ctx->device);
  if (ctx->have_last) {
    cudaError_t e = cudaEventSynchronize(ctx->last_done);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "synchronise");
  }
  Stats h;
  cudaError_t e = cudaMemcpy(&h, ctx->d_stats, sizeof(Stats), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "read stats");
  out->rays = h.rays;
  out->de_evals = h.de_evals;
  out->march_evals = h.march_evals;
  out->normal_evals = h.normal_evals;
  out->shadow_evals = h.shadow_evals;
  out->trap_evals = ctx->last_trap ? h.hits : 0;
  out->de_evals += out->trap_evals;
  out->hits = h.hits;
  out->refills = h.refills;
  out->timeouts = h.timeouts;
  out->kernel = uint32_t(ctx->last_kernel);
  out->accel_voxels = ctx->last_accel_voxels;
  for (int p = 0; p < ctx->tev_plans; ++p) {
    float b = 0.0f, m = 0.0f, sh = 0.0f;
    if (cudaEventElapsedTime(&b, ctx->tev[4 * p], ctx->tev[4 * p + 1]) == cudaSuccess) out->accel_ms += b;
    if (cudaEventElapsedTime(&m, ctx->tev[4 * p + 1], ctx->tev[4 * p + 2]) == cudaSuccess) out->march_ms += m;
    if (cudaEventElapsedTime(&sh, ctx->tev[4 * p + 2], ctx->tev[4 * p + 3]) == cudaSuccess) out->shade_ms += sh;
  }
  if (h.timeouts) return fail(ctx, ND_ERR_TIMEOUT, "the device watchdog stopped %u warps", h.timeouts);
  return ND_OK;
}

// Times every candidate launch configuration on the given views (writing into
// scratch_out) and keeps the fastest for this call's formula sets.  Candidates: the
// plain per-view launch, and the persistent march at 64, 128 and 256 threads per
// block (FP32 DE; 128 otherwise) x as many blocks per SM as fit or two fewer x refill
// thresholds 3, 4, 6, 8 and 12.  Each candidate runs once to warm up, then three
// times with the L2 cache flushed before each run; its time is the median.
nd_status nd_autotune(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews, const nd_gbuffer* scratch_out,
                      nd_tune_result* result) {
  std::vector<Launch> plans;
  int64_t total = 0;
  nd_status s = prepare(ctx, views, nviews, scratch_out, &plans, &total);
  if (s != ND_OK) return s;
  cudaSetDevice(ctx->device);
  bool any_accel = false;
  bool block_axis = true;  // every plan has the FP32 block-size variants
  for (int i = 0; i < nviews; ++i) any_accel |= nd::accel_voxels_of(views[i]) > 0;
  for (const Launch& L : plans) block_axis &= L.table.persistent_f32_batched_b64 && L.table.persistent_f32_batched_b256;
  struct Cand {
    int kernel, block, per_sm, thr;
  };
  std::vector<Cand> cands;
  if (!any_accel) cands.push_back({ND_KERNEL_PLAIN, 128, 0, 1});  // the accelerator runs on the persistent kernel
  const int blocks[3] = {64, 128, 256};
  for (int b : blocks) {
    if (b != 128 && !block_axis) continue;
    for (int per_sm : {0, -2})
      for (int thr : {3, 4, 6, 8, 12}) cands.push_back({ND_KERNEL_PERSISTENT, b, per_sm, thr});
  }
  cudaStream_t st;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "stream");
  // a buffer larger than the L2 cache, written before every timed run
  const size_t flush_bytes = size_t(256) << 20;
  void* flush = nullptr;
  e = cudaMalloc(&flush, flush_bytes);
  if (e != cudaSuccess) {
    cudaStreamDestroy(st);
    return cuda_fail(ctx, e, "autotune L2 flush buffer");
  }
  cudaEvent_t ev[2];
  cudaEventCreate(&ev[0]);
  cudaEventCreate(&ev[1]);
  double best = 1e30;
  Cand bc = cands[any_accel ? 0 : 1];
  for (const Cand& c : cands) {
    nd_march_opts o;
    memset(&o, 0, sizeof(o));
    o.kernel = c.kernel;
    o.block = c.block;
    o.blocks_per_sm = c.per_sm;
    o.refill_threshold = c.thr;
    s = nd_march_forward(ctx, views, nviews, &o, scratch_out, st);  // warm-up
    if (s != ND_OK) break;
    float runs[3];
    for (int r = 0; r < 3 && s == ND_OK; ++r) {
      cudaMemsetAsync(flush, r, flush_bytes, st);
      cudaEventRecord(ev[0], st);
      s = nd_march_forward(ctx, views, nviews, &o, scratch_out, st);
      cudaEventRecord(ev[1], st);
      e = cudaEventSynchronize(ev[1]);
      if (s == ND_OK && e != cudaSuccess) s = cuda_fail(ctx, e, "autotune run");
      if (s == ND_OK) cudaEventElapsedTime(&runs[r], ev[0], ev[1]);
    }
    if (s != ND_OK) break;
    std::sort(runs, runs + 3);
    if (runs[1] < best) {
      best = runs[1];
      bc = c;
    }
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  cudaFree(flush);
  cudaStreamDestroy(st);
  if (s != ND_OK) return s;
  Tuned t;
  t.kernel = bc.kernel;
  t.block = bc.block;
  t.blocks_per_sm = bc.per_sm;
  t.refill_threshold = bc.thr;
  t.rays_per_s = best > 0 ? double(total) / (best * 1e-3) : 0.0;
  t.tuned = true;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (const Launch& L : plans) g_tuned[tune_key(ctx, L, 32)] = t;  // the candidates ran the FP32 DE
  }
  if (result) {
    result->kernel = t.kernel;
    result->block = t.block;
    // the blocks per SM the persistent march runs with (as many as fit, or fewer)
    int resident = 0;
    if (t.kernel == ND_KERNEL_PERSISTENT && !plans.empty()) {
      const KernelTable& T = plans[0].table;
      nd::ResidentFn rf = t.block == 64 ? T.resident_b64 : (t.block == 256 ? T.resident_b256 : T.resident_b128);
      if (rf) resident = rf(t.blocks_per_sm);
    }
    result->blocks_per_sm = resident;
    result->refill_threshold = t.refill_threshold;
    result->rays_per_s = t.rays_per_s;
  }
  return ND_OK;
}

// The tuning cache on disk: one JSON array of the tuned entries of every GPU and
// formula set (key: GPU name | formula set | hash of the formula sources | precision).
nd_status nd_tune_cache_save(const char* path) {
  if (!path) return ND_ERR_INVALID;
  std::string out = "[\n";
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    bool first = true;
    for (const auto& kv : g_tuned) {
      // the key as a JSON string (any length; quotes, backslashes and control
      // characters escaped)
      std::string key;
      for (char ch : kv.first) {
        if (ch == '"' || ch == '\\') {
          key += '\\';
          key += ch;
        } else if (static_cast<unsigned char>(ch) < 0x20) {
          char esc[8];
          snprintf(esc, sizeof(esc), "\\u%04x", unsigned(static_cast<unsigned char>(ch)));
          key += esc;
        } else {
          key += ch;
        }
      }
      char buf[256];
      snprintf(buf, sizeof(buf),
               "\", \"kernel\": %d, \"block\": %d, \"blocks_per_sm\": %d, \"refill_threshold\": %d, "
               "\"rays_per_s\": %.6g}",
               kv.second.kernel, kv.second.block, kv.second.blocks_per_sm, kv.second.refill_threshold,
               kv.second.rays_per_s);
      out += first ? " {\"key\": \"" : ",\n {\"key\": \"";
      out += key;
      out += buf;
      first = false;
    }
  }
  out += "\n]\n";
  FILE* f = fopen(path, "wb");
  if (!f) return ND_ERR_INVALID;
  const bool ok = fwrite(out.data(), 1, out.size(), f) == out.size();
  return (fclose(f) == 0 && ok) ? ND_OK : ND_ERR_INVALID;
}

nd_status nd_tune_cache_load(const char* path, int32_t* loaded) {
  if (loaded) *loaded = 0;
  if (!path) return ND_ERR_INVALID;
  FILE* f = fopen(path, "rb");
  if (!f) return ND_ERR_NOT_FOUND;
  std::string text;
  char buf[4096];
  size_t n;
  while ((n = fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, n);
  fclose(f);
  nd_json::JVal root;
  nd_json::JsonParser p(text.data(), text.size());
  if (!p.parse(&root) || root.kind != nd_json::JVal::ARR) return ND_ERR_INVALID;
  int count = 0;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (const nd_json::JVal& e : root.arr) {
    const nd_json::JVal* key = e.get("key");
    if (!key || key->kind != nd_json::JVal::STR) continue;
    auto num = [&](const char* k, double d) {
      const nd_json::JVal* v = e.get(k);
      return v && v->kind == nd_json::JVal::NUM ? v->num : d;
    };
    Tuned t;
    t.kernel = int(num("kernel", ND_KERNEL_PERSISTENT));
    t.block = int(num("block", 128));
    t.blocks_per_sm = int(num("blocks_per_sm", 0));
    t.refill_threshold = int(num("refill_threshold", 6));
    t.rays_per_s = num("rays_per_s", 0.0);
    t.tuned = true;
    if ((t.kernel != ND_KERNEL_PLAIN && t.kernel != ND_KERNEL_PERSISTENT) ||
        (t.block != 64 && t.block != 128 && t.block != 256) || t.refill_threshold < 1 || t.refill_threshold > 32)
      continue;
    g_tuned[key->str] = t;
    ++count;
  }
  if (loaded) *loaded = count;
  return ND_OK;
}

}  // extern "C"

namespace {
// Captures one forward call (work-counter and stats resets plus every launch)
// into a CUDA graph.  The graph owns device copies of the view table and of the
// scene table, so it can be replayed while the caller changes its own descriptors.
nd_status graph_capture_impl(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews, const nd_march_opts* opts,
                             const nd_gbuffer* out, void* stream, nd_graph** graph, const SceneInput& sc) {
  if (!graph) return ND_ERR_INVALID;
  *graph = nullptr;
  std::vector<Launch> plans;
  int64_t total = 0;
  nd_status s = prepare(ctx, views, nviews, out, &plans, &total, sc);
  if (s != ND_OK) return s;
  if (opts && opts->de_precision != 0 && opts->de_precision != 32 && opts->de_precision != 64)
    return fail(ctx, ND_ERR_INVALID, "de_precision must be 32 or 64");
  cudaSetDevice(ctx->device);
  nd_graph* g = new nd_graph();
  g->ctx = ctx;
  g->trap = out->trap || out->iters;
  cudaError_t e = cudaMalloc((void**)&g->d_views, sizeof(DevView) * size_t(nviews));
  if (e == cudaSuccess)
    e = cudaMalloc((void**)&g->d_counters, sizeof(unsigned long long) * kCountersPerPlan * plans.size());
  if (e == cudaSuccess) e = cudaMalloc((void**)&g->d_thit, sizeof(double) * size_t(std::max<int64_t>(total, 1)));
  if (e == cudaSuccess) e = cudaMalloc((void**)&g->d_hits, sizeof(nd::HitEntry) * size_t(std::max<int64_t>(total, 1)));
  bool any_shadow = false;
  for (int i = 0; i < nviews; ++i) any_shadow |= views[i].shadow != 0;
  if (e == cudaSuccess && any_shadow)
    e = cudaMalloc((void**)&g->d_shadowq, sizeof(nd::ShadowEntry) * size_t(std::max<int64_t>(total, 1)));
  int64_t voxels = 0;
  int accel_views = 0;
  for (int i = 0; i < nviews; ++i) {
    voxels += nd::accel_voxels_of(views[i]);
    accel_views += nd::accel_voxels_of(views[i]) > 0 ? 1 : 0;
  }
  if (e == cudaSuccess && voxels > 0) e = cudaMalloc((void**)&g->d_accel, sizeof(float) * size_t(voxels));
  if (e == cudaSuccess && accel_views > 0)
    e = cudaMalloc((void**)&g->d_accel_jobs, sizeof(nd::AccelJob) * size_t(accel_views));
  if (e == cudaSuccess && sc.nscenes > 0) e = cudaMalloc((void**)&g->d_scenes, sizeof(nd::DevScene) * size_t(sc.nscenes));
  if (e != cudaSuccess) {
    nd_graph_destroy(g);
    return cuda_fail(ctx, e, "graph buffers");
  }
  std::vector<nd::AccelJob> jobs;
  std::vector<DevView> hv(nviews);
  // fill the host table (enqueue builds it) without launching: capture does both
  cudaStream_t st = (cudaStream_t)stream;
  cudaStream_t cap;
  e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    nd_graph_destroy(g);
    return cuda_fail(ctx, e, "capture stream");
  }
  e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) {
    cudaStreamDestroy(cap);
    nd_graph_destroy(g);
    return cuda_fail(ctx, e, "begin capture");
  }
  s = enqueue(ctx, views, nviews, opts, out, cap, plans, g->d_views, hv.data(), g->d_counters, g->d_thit,
              g->d_hits, false, nullptr, nullptr, sc, g->d_scenes, g->d_accel, g->d_accel_jobs, &jobs, g->d_shadowq);
  cudaGraph_t gr = nullptr;
  e = cudaStreamEndCapture(cap, &gr);
  cudaStreamDestroy(cap);
  if (s != ND_OK || e != cudaSuccess) {
    if (gr) cudaGraphDestroy(gr);
    nd_graph_destroy(g);
    return s != ND_OK ? s : cuda_fail(ctx, e, "end capture");
  }
  g->graph = gr;
  e = cudaMemcpy(g->d_views, hv.data(), sizeof(DevView) * size_t(nviews), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !jobs.empty())
    e = cudaMemcpy(g->d_accel_jobs, jobs.data(), sizeof(nd::AccelJob) * jobs.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && sc.nscenes > 0) {
    std::vector<nd::DevScene> hs;
    scene_table(sc, plans[0].members, &hs);
    e = cudaMemcpy(g->d_scenes, hs.data(), sizeof(nd::DevScene) * hs.size(), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, gr, 0);
  if (e != cudaSuccess) {
    nd_graph_destroy(g);
    return cuda_fail(ctx, e, "instantiate graph");
  }
  (void)st;
  *graph = g;
  return ND_OK;
}
}  // namespace

extern "C" {

nd_status nd_graph_capture(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews, const nd_march_opts* opts,
                           const nd_gbuffer* out, void* stream, nd_graph** graph) {
  return graph_capture_impl(ctx, views, nviews, opts, out, stream, graph, SceneInput());
}

nd_status nd_graph_capture_scenes(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews, const int32_t* view_scene,
                                  const nd_scene_desc* scenes, int32_t nscenes, const nd_march_opts* opts,
                                  const nd_gbuffer* out, void* stream, nd_graph** graph) {
  if (graph) *graph = nullptr;
  if (!ctx) return ND_ERR_INVALID;
  if (nscenes < 0 || (nscenes > 0 && (!scenes || !view_scene)))
    return fail(ctx, ND_ERR_INVALID, "scenes need a view_scene array and a scene array");
  SceneInput sc;
  sc.view_scene = view_scene;
  sc.scenes = scenes;
  sc.nscenes = nscenes;
  return graph_capture_impl(ctx, views, nviews, opts, out, stream, graph, sc);
}

nd_status nd_graph_launch(nd_graph* g, void* stream) {
  if (!g || !g->exec) return ND_ERR_INVALID;
  cudaSetDevice(g->ctx->device);
  cudaError_t e = cudaGraphLaunch(g->exec, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(g->ctx, e, "graph launch");
  g->ctx->tev_plans = 0;
  e = cudaEventRecord(g->ctx->last_done, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(g->ctx, e, "record event");
  g->ctx->have_last = true;
  // a later forward on another stream waits for this replay (it shares the stats block)
  g->ctx->last_stream = (cudaStream_t)stream;
  g->ctx->last_trap = g->trap;
  return ND_OK;
}

nd_status nd_graph_destroy(nd_graph* g) {
  if (!g) return ND_ERR_INVALID;
  if (g->ctx) cudaSetDevice(g->ctx->device);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  if (g->d_views) cudaFree(g->d_views);
  if (g->d_counters) cudaFree(g->d_counters);
  if (g->d_thit) cudaFree(g->d_thit);
  if (g->d_hits) cudaFree(g->d_hits);
  if (g->d_shadowq) cudaFree(g->d_shadowq);
  if (g->d_accel) cudaFree(g->d_accel);
  if (g->d_accel_jobs) cudaFree(g->d_accel_jobs);
  if (g->d_scenes) cudaFree(g->d_scenes);
  delete g;
  return ND_OK;
}

nd_status nd_de_points(nd_ctx* ctx, const nd_view_desc* view, int64_t n, const double* pts, double* de,
                       double* trap, uint32_t* iters, int32_t de_precision, void* stream) {
  if (!ctx || !view || n < 0 || (n > 0 && (!pts || !de))) return fail(ctx, ND_ERR_INVALID, "bad nd_de_points arguments");
  if (view->formula < 0 || view->formula >= nd_formula_total())
    return fail(ctx, ND_ERR_NOT_FOUND, "unknown formula id %d", view->formula);
  cudaSetDevice(ctx->device);
  const DevView v = make_dev_view(*view, 0, 0, 0);
  const KernelTable t = nd_formula_at(view->formula)->kernels();
  const nd::DePointsFn fn = de_precision == 64 ? t.de_points_f64 : t.de_points_f32;
  if (!fn) return fail(ctx, ND_ERR_UNSUPPORTED, "no DE kernel for this formula");
  cudaError_t e = fn(v, n, pts, de, trap, iters, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "nd_de_points launch");
  return ND_OK;
}

}  // extern "C"

namespace {
// Sorts a descriptor's colour stops by position (stable, like sortedColorOrder).
nd_lite_desc sorted_stops(nd_lite_desc d) {
  for (int a = 1; a < d.color_count && a < ND_MAX_COLOR_STOPS; ++a)
    for (int b = a; b > 0 && d.colors[b - 1].position > d.colors[b].position; --b) std::swap(d.colors[b - 1], d.colors[b]);
  return d;
}

nd_status lite_check(nd_ctx* ctx, const nd_lite_desc& L, const char* what, int i) {
  if (L.color_count < 0 || L.color_count > ND_MAX_COLOR_STOPS || L.light_count < 0 || L.light_count > ND_MAX_LIGHTS)
    return fail(ctx, ND_ERR_INVALID, "%s %d: color_count 0..%d, light_count 0..%d", what, i, ND_MAX_COLOR_STOPS,
                ND_MAX_LIGHTS);
  for (int k = 0; k < L.light_count; ++k)
    if (L.lights[k].type != ND_LIGHT_POINT && L.lights[k].type != ND_LIGHT_GLOBAL)
      return fail(ctx, ND_ERR_UNSUPPORTED, "%s %d light %d: only point and global lights", what, i, k);
  return ND_OK;
}

nd_status shade_lite_impl(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews, const nd_lite_desc* lite,
                          const nd_lite_desc* instance_colors, const nd_gbuffer* in, float* rgba, void* stream,
                          const SceneInput& sc) {
  if (!ctx) return ND_ERR_INVALID;
  if (!lite || !rgba || (uintptr_t(rgba) & 15)) return fail(ctx, ND_ERR_INVALID, "lite descriptors and a 16-byte aligned rgba");
  if (!in || !in->depth64 || !in->normal || !in->trap)
    return fail(ctx, ND_ERR_INVALID, "lite shading reads the forward's depth64, normal and trap");
  std::vector<Launch> plans;
  int64_t total = 0;
  nd_status s = prepare(ctx, views, nviews, in, &plans, &total, sc);
  if (s != ND_OK) return s;
  for (int i = 0; i < nviews; ++i)
    if ((s = lite_check(ctx, lite[i], "view", i)) != ND_OK) return s;
  if (sc.nscenes > 0 && !instance_colors)
    return fail(ctx, ND_ERR_INVALID, "scenes need their instances' colour descriptors");
  for (int i = 0; i < sc.nscenes * ND_MAX_INSTANCES; ++i)
    if ((s = lite_check(ctx, instance_colors[i], "instance colour descriptor", i)) != ND_OK) return s;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "set device");
  cudaStream_t st = (cudaStream_t)stream;
  if (ctx->have_last) cudaEventSynchronize(ctx->last_done);  // the staging buffer may feed an earlier copy
  if ((s = ensure_dev(ctx, &ctx->d_views, &ctx->views_cap, nviews, "view table")) != ND_OK) return s;
  const int nlite = nviews + sc.nscenes * ND_MAX_INSTANCES;
  if ((s = ensure_dev(ctx, &ctx->d_lite, &ctx->lite_cap, nlite, "lite descriptors")) != ND_OK) return s;
  if (sc.nscenes > 0 && (s = ensure_dev(ctx, &ctx->d_scenes, &ctx->scenes_cap, sc.nscenes, "scene table")) != ND_OK)
    return s;
  if ((s = ensure_staging(ctx, nviews)) != ND_OK) return s;
  // views and descriptors in plan order; colour stops sorted by position
  std::vector<int64_t> out_off(nviews + 1, 0);
  for (int i = 0; i < nviews; ++i) out_off[i + 1] = out_off[i] + int64_t(views[i].spp) * views[i].tile_w * views[i].tile_h;
  // per view in plan order, then the scenes' instance colours (scene-major)
  std::vector<nd_lite_desc> hl(nlite);
  int base = 0;
  for (const Launch& L : plans) {
    int64_t off = 0;
    for (size_t k = 0; k < L.views.size(); ++k) {
      const int vi = L.views[k];
      ctx->h_views[base + k] = make_dev_view(views[vi], off, out_off[vi], L.codes[k]);
      ctx->h_views[base + k].scene = sc.scene_of(vi);
      off += ctx->h_views[base + k].rays;
      hl[base + k] = sorted_stops(lite[vi]);
    }
    base += int(L.views.size());
  }
  for (int i = 0; i < sc.nscenes * ND_MAX_INSTANCES; ++i) hl[nviews + i] = sorted_stops(instance_colors[i]);
  e = cudaMemcpyAsync(ctx->d_views, ctx->h_views, sizeof(DevView) * size_t(nviews), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ctx->d_lite, hl.data(), sizeof(nd_lite_desc) * size_t(nlite), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && sc.nscenes > 0) {
    std::vector<nd::DevScene> hs;
    scene_table(sc, plans[0].members, &hs);
    e = cudaMemcpyAsync(ctx->d_scenes, hs.data(), sizeof(nd::DevScene) * hs.size(), cudaMemcpyHostToDevice, st);
  }
  if (e != cudaSuccess) return cuda_fail(ctx, e, "copy lite tables");
  base = 0;
  for (const Launch& L : plans) {
    const int nv = int(L.views.size());
    int64_t rays = 0;
    bool dir64 = false;
    for (int k = 0; k < nv; ++k) {
      rays += ctx->h_views[base + k].rays;
      dir64 |= ctx->h_views[base + k].dir64 != 0;
    }
    LaunchArgs a;
    memset(&a, 0, sizeof(a));
    a.views = ctx->d_views + base;
    a.nviews = nv;
    a.total_rays = rays;
    a.out = *in;
    a.scenes = sc.nscenes > 0 ? ctx->d_scenes : nullptr;
    // the shading arithmetic is f32 like the reference's; so is the DE of its AO taps
    nd::LiteFn fn = dir64 ? L.table.lite_f32_dir64 : L.table.lite_f32;
    if (!fn) return fail(ctx, ND_ERR_UNSUPPORTED, "no lite shading kernels for this formula set");
    if (sc.nscenes > 0) {
      if (dir64) return fail(ctx, ND_ERR_UNSUPPORTED, "lite shading of scenes with FP64 ray directions");
      fn = L.table.scene_lite_f32;
      if (!fn) return fail(ctx, ND_ERR_UNSUPPORTED, "no scene kernels in this formula set");
    }
    e = fn(a, ctx->d_lite + base, ctx->d_lite + nviews, rgba, ctx->num_sms, st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "lite shading launch");
    base += nv;
  }
  e = cudaEventRecord(ctx->last_done, st);
  // the view table went up from the staging's first half: a forward call that reuses
  // that half waits for this copy as for its own
  if (e == cudaSuccess && !ctx->staged[0]) e = cudaEventCreateWithFlags(&ctx->staged[0], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->staged[0], st);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "record event");
  ctx->staged_valid[0] = true;
  ctx->have_last = true;
  return ND_OK;
}
}  // namespace

extern "C" {

nd_status nd_shade_lite(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews, const nd_lite_desc* lite,
                        const nd_gbuffer* in, float* rgba, void* stream) {
  return shade_lite_impl(ctx, views, nviews, lite, nullptr, in, rgba, stream, SceneInput());
}

nd_status nd_shade_lite_scenes(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews, const int32_t* view_scene,
                               const nd_scene_desc* scenes, int32_t nscenes, const nd_lite_desc* lite,
                               const nd_lite_desc* instance_colors, const nd_gbuffer* in, float* rgba, void* stream) {
  if (!ctx) return ND_ERR_INVALID;
  if (nscenes < 0 || (nscenes > 0 && (!scenes || !view_scene)))
    return fail(ctx, ND_ERR_INVALID, "scenes need a view_scene array and a scene array");
  SceneInput sc;
  sc.view_scene = view_scene;
  sc.scenes = scenes;
  sc.nscenes = nscenes;
  return shade_lite_impl(ctx, views, nviews, lite, instance_colors, in, rgba, stream, sc);
}

}  // extern "C"

namespace {
// 8 independent FMA chains per thread (enough to cover the FMA latency at full
// occupancy); the sum goes to out so that nothing is eliminated.
__global__ void __launch_bounds__(256) fp32_peak_kernel(int iters, float b, float c, float* out) {
  float a0 = threadIdx.x * 1e-7f, a1 = a0 + 1e-7f, a2 = a0 + 2e-7f, a3 = a0 + 3e-7f;
  float a4 = a0 + 4e-7f, a5 = a0 + 5e-7f, a6 = a0 + 6e-7f, a7 = a0 + 7e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      a0 = fmaf(a0, b, c); a1 = fmaf(a1, b, c); a2 = fmaf(a2, b, c); a3 = fmaf(a3, b, c);
      a4 = fmaf(a4, b, c); a5 = fmaf(a5, b, c); a6 = fmaf(a6, b, c); a7 = fmaf(a7, b, c);
    }
  }
  const float s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
  if (s == 1234.5f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // never true for these inputs
}
}  // namespace

extern "C" {

nd_status nd_measure_fp32_peak(nd_ctx* ctx, double ms, double* tflops) {
  if (!ctx || !tflops || !(ms > 0)) return fail(ctx, ND_ERR_INVALID, "bad nd_measure_fp32_peak arguments");
  cudaSetDevice(ctx->device);
  const int blocks = ctx->num_sms * 8, threads = 256;
  float* out = nullptr;
  cudaError_t e = cudaMalloc((void**)&out, sizeof(float) * size_t(blocks) * threads);
  cudaEvent_t a = nullptr, b = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  double best = 0.0;
  int iters = 256;
  for (int rep = 0; e == cudaSuccess && rep < 8; ++rep) {
    cudaEventRecord(a, nullptr);
    fp32_peak_kernel<<<blocks, threads>>>(iters, 0.999999f, 1e-7f, out);
    cudaEventRecord(b, nullptr);
    e = cudaEventSynchronize(b);
    if (e != cudaSuccess) break;
    float t = 0.0f;
    cudaEventElapsedTime(&t, a, b);
    const double flops = 2.0 * 8.0 * 16.0 * double(iters) * blocks * threads;
    if (t > 0.25 * ms) best = std::max(best, flops / (double(t) * 1e-3) / 1e12);
    // grow toward `ms` at most 100x per run, and never past 2^20 iterations (about 1 s)
    if (t < ms) iters = int(std::min<double>(double(iters) * std::min(100.0, std::max(2.0, ms / std::max(double(t), 1e-3))),
                                             double(1 << 20)));
  }
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  if (out) cudaFree(out);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "nd_measure_fp32_peak");
  *tflops = best;
  return ND_OK;
}

nd_status nd_accel_grid(nd_ctx* ctx, const nd_view_desc* view, int32_t de_precision, float* grid, int64_t capacity,
                        float* prm, int64_t* count) {
  if (!ctx || !view || !grid || !prm || !count) return fail(ctx, ND_ERR_INVALID, "bad nd_accel_grid arguments");
  nd_status s = validate_view(ctx, *view, 0);
  if (s != ND_OK) return s;
  const int64_t n = nd::accel_voxels_of(*view);
  if (n <= 0) return fail(ctx, ND_ERR_INVALID, "the view has no accelerator (accel_res 0)");
  if (n > capacity) return fail(ctx, ND_ERR_INVALID, "grid capacity %lld < %lld", (long long)capacity, (long long)n);
  cudaSetDevice(ctx->device);
  DevView v = make_dev_view(*view, 0, 0, 0);
  nd::place_accel(v, *view, grid);
  for (int l = 0; l < nd::kAccelMaxCascades; ++l)
    for (int a = 0; a < 4; ++a) prm[4 * l + a] = l < v.accel_levels ? v.accel_prm[l][a] : 0.0f;
  const KernelTable t = nd_formula_at(view->formula)->kernels();
  const nd::AccelBuildFn fn = de_precision == 64 ? t.accel_build_f64 : t.accel_build_f32;
  if (!fn) return fail(ctx, ND_ERR_UNSUPPORTED, "no accelerator kernels for this formula");
  DevView* dv = nullptr;
  nd::AccelJob* dj = nullptr;
  nd::AccelJob job;
  job.view = 0;
  job.pad = 0;
  job.begin = 0;
  cudaError_t e = cudaMalloc((void**)&dv, sizeof(DevView));
  if (e == cudaSuccess) e = cudaMalloc((void**)&dj, sizeof(job));
  if (e == cudaSuccess) e = cudaMemcpy(dv, &v, sizeof(DevView), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dj, &job, sizeof(job), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = fn(dv, dj, 1, n, nullptr, ctx->num_sms, nullptr);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (dv) cudaFree(dv);
  if (dj) cudaFree(dj);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "nd_accel_grid");
  *count = n;
  return ND_OK;
}

// Layout check for bindings: sizes of the public structs.
size_t nd_sizeof(const char* name) {
  if (!name) return 0;
  const std::string n(name);
  if (n == "nd_view_desc") return sizeof(nd_view_desc);
  if (n == "nd_trap_desc") return sizeof(nd_trap_desc);
  if (n == "nd_gbuffer") return sizeof(nd_gbuffer);
  if (n == "nd_march_opts") return sizeof(nd_march_opts);
  if (n == "nd_stats") return sizeof(nd_stats);
  if (n == "nd_param_info") return sizeof(nd_param_info);
  if (n == "nd_tune_result") return sizeof(nd_tune_result);
  if (n == "nd_orbit_camera") return sizeof(nd_orbit_camera);
  if (n == "nd_scene_desc") return sizeof(nd_scene_desc);
  if (n == "nd_instance_desc") return sizeof(nd_instance_desc);
  if (n == "nd_mixin_desc") return sizeof(nd_mixin_desc);
  if (n == "nd_lite_desc") return sizeof(nd_lite_desc);
  if (n == "nd_color_stop") return sizeof(nd_color_stop);
  if (n == "nd_light") return sizeof(nd_light);
  if (n == "DevView") return sizeof(DevView);  // the per-view record a forward call copies to the device
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Forward march without any allocation.
//
// Some callers cannot allocate device memory: code that runs inside a host
// framework whose allocator owns all device memory (a renderer plug-in, a game
// engine with a fixed budget), hosts that forbid cudaMalloc on their render thread
// because it may synchronise the device, and embedded or real-time loops that must
// not allocate after start-up.  nd_march_forward_noalloc serves them with the
// persistent kernel and no context: its only scratch (the view table, the work
// counters and the statistics block, about 28 KB) lives in the file-scope array
// below, which the library's module brings with it on every GPU that loads the
// library, until the process exits.
namespace {

constexpr int kNoAllocMaxViews = 64;  // views (and launches) per call

struct NoAllocScratch {
  DevView views[kNoAllocMaxViews];
  unsigned long long counters[kNoAllocMaxViews];
  Stats stats;
};

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
// Per device: the scratch array's device address and the SM count, and the id of
// the CUDA context they were looked up in.  A host that resets the device
// (cudaDeviceReset) or re-creates its primary context gets a new context in which
// the library's module, and with it the array, may sit elsewhere: a call in a
// context other than the recorded one repeats the set-up.
NoAllocScratch* g_noalloc_ptr[kNoAllocMaxDevices] = {};
int g_noalloc_sms[kNoAllocMaxDevices] = {};
unsigned long long g_noalloc_ctx[kNoAllocMaxDevices] = {};

// The id of the calling thread's current CUDA context (driver entry points looked up
// through the runtime, so the library needs no link to the driver library); 0 when
// the driver cannot tell.
unsigned long long current_context_id() {
  typedef int (*GetCurrent)(void**);
  typedef int (*GetId)(void*, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  });
  void* c = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&c) != 0 || !c || get_id(c, &id) != 0) return 0;
  return id;
}

}  // namespace

// The scratch array.  In host code this name is only a stand-in: its device
// address comes from cudaGetSymbolAddress, once per device (and context).
static __device__ __align__(256) unsigned char g_nd_noalloc_scratch[sizeof(NoAllocScratch)];

namespace {

// First call on a device (in its current context): look up the device address of
// the scratch array and the SM count, with that device current.
nd_status noalloc_setup(int dev, NoAllocScratch** ptr, int* sms) {
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    return fail(nullptr, ND_ERR_UNSUPPORTED, "device %d: at most %d devices", dev, kNoAllocMaxDevices);
  // 0 when no context is current yet on this thread: the set-up below makes the
  // device's primary context current (cudaGetSymbolAddress loads the module)
  const unsigned long long ctx = current_context_id();
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev] || ctx != g_noalloc_ctx[dev] || ctx == 0) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_nd_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(nullptr, ND_ERR_CUDA, "scratch address on device %d: %s", dev, cudaGetErrorString(e));
    int n = 0;
    e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || n <= 0) return fail(nullptr, ND_ERR_CUDA, "SM count of device %d", dev);
    g_noalloc_sms[dev] = n;
    g_noalloc_ptr[dev] = static_cast<NoAllocScratch*>(p);
    g_noalloc_ctx[dev] = current_context_id();
  }
  *ptr = g_noalloc_ptr[dev];
  *sms = g_noalloc_sms[dev];
  return ND_OK;
}

}  // namespace

extern "C" nd_status nd_march_forward_noalloc(const nd_view_desc* views, int32_t nviews, const nd_march_opts* opts,
                                              const nd_gbuffer* out, void* stream) {
  g_noctx_err[0] = 0;
  if (!views || nviews <= 0 || !out || !out->depth)
    return fail(nullptr, ND_ERR_INVALID, "needs views, nviews > 0 and a G-buffer with a depth pointer");
  if (nviews > kNoAllocMaxViews)
    return fail(nullptr, ND_ERR_INVALID, "%d views: this entry point takes at most %d per call", nviews,
                kNoAllocMaxViews);
  if (out->trap || out->iters)
    return fail(nullptr, ND_ERR_UNSUPPORTED, "trap and iters outputs need per-ray scratch: use nd_march_forward");
  if ((out->normal && (uintptr_t(out->normal) & 15)) || (out->depth64 && (uintptr_t(out->depth64) & 7)) ||
      (out->normal_half && (uintptr_t(out->normal_half) & 7)) || (uintptr_t(out->depth) & 3))
    return fail(nullptr, ND_ERR_INVALID, "misaligned G-buffer pointer (normal needs 16 bytes, normal_half 8)");
  if (opts && opts->de_precision != 0 && opts->de_precision != 32 && opts->de_precision != 64)
    return fail(nullptr, ND_ERR_INVALID, "de_precision must be 32 or 64");
  int64_t total = 0;
  for (int i = 0; i < nviews; ++i) {
    const nd_status s = validate_view(nullptr, views[i], i);
    if (s != ND_OK) return s;
    if (views[i].accel_res > 0)
      return fail(nullptr, ND_ERR_UNSUPPORTED, "view %d: the accelerator grid needs device memory", i);
    total += int64_t(views[i].spp) * views[i].tile_w * views[i].tile_h;
    if (total > int64_t(0x7fffffff))
      return fail(nullptr, ND_ERR_INVALID, "more than 2^31-1 rays: this entry point takes at most 2^31-1 per call");
  }
  // the view table is copied from this call's stack, which a captured graph would
  // read again at replay, after the frame is gone
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t ce = cudaStreamIsCapturing((cudaStream_t)stream, &cap);
  if (ce != cudaSuccess) return fail(nullptr, ND_ERR_CUDA, "stream capture status: %s", cudaGetErrorString(ce));
  if (cap != cudaStreamCaptureStatusNone)
    return fail(nullptr, ND_ERR_UNSUPPORTED, "this entry point cannot be captured into a CUDA graph");
  int dev = 0;
  cudaError_t ge = cudaGetDevice(&dev);
  if (ge != cudaSuccess) return fail(nullptr, ND_ERR_CUDA, "current device: %s", cudaGetErrorString(ge));
  NoAllocScratch* scratch = nullptr;
  int sms = 0;
  nd_status s = noalloc_setup(dev, &scratch, &sms);
  if (s != ND_OK) return s;

  // plan without heap allocation: one launch when one formula or one compiled
  // group covers the call, else one launch per formula; views grouped by launch
  int order[kNoAllocMaxViews], codes[kNoAllocMaxViews], launch_of[kNoAllocMaxViews];
  KernelTable tables[kNoAllocMaxViews];
  int nlaunch = 0;
  int distinct[kNoAllocMaxViews], ndistinct = 0;
  for (int i = 0; i < nviews; ++i) {
    bool seen = false;
    for (int k = 0; k < ndistinct; ++k) seen |= distinct[k] == views[i].formula;
    if (!seen) distinct[ndistinct++] = views[i].formula;
  }
  int group = -1;
  if (ndistinct > 1) {
    for (int g = 0; g < nd_group_entry_count && group < 0; ++g) {
      bool covers = true;
      for (int k = 0; k < ndistinct; ++k) {
        bool in = false;
        for (int m = 0; m < nd_group_entries[g].count; ++m) in |= nd_group_entries[g].members[m] == distinct[k];
        covers &= in;
      }
      if (covers) group = g;
    }
  }
  int nv = 0;
  if (ndistinct == 1 || group >= 0) {
    tables[0] = group >= 0 ? nd_group_entries[group].kernels() : nd_formula_at(distinct[0])->kernels();
    nlaunch = 1;
    const int gcount = group >= 0 ? nd_group_entries[group].count : 1;
    for (int m = 0; m < gcount; ++m)  // views ordered by formula code
      for (int i = 0; i < nviews; ++i) {
        const int code = group >= 0 ? m : 0;
        const bool match = group >= 0 ? nd_group_entries[group].members[m] == views[i].formula : true;
        if (!match) continue;
        order[nv] = i;
        codes[nv] = code;
        launch_of[nv] = 0;
        ++nv;
      }
  } else {
    for (int k = 0; k < ndistinct; ++k) {
      tables[nlaunch] = nd_formula_at(distinct[k])->kernels();
      for (int i = 0; i < nviews; ++i)
        if (views[i].formula == distinct[k]) {
          order[nv] = i;
          codes[nv] = 0;
          launch_of[nv] = nlaunch;
          ++nv;
        }
      ++nlaunch;
    }
  }
  if (nv != nviews) return fail(nullptr, ND_ERR_INVALID, "view planning failed");

  // view table: G-buffer offsets in call order, work-item offsets per launch
  int64_t out_off[kNoAllocMaxViews + 1];
  out_off[0] = 0;
  for (int i = 0; i < nviews; ++i) out_off[i + 1] = out_off[i] + int64_t(views[i].spp) * views[i].tile_w * views[i].tile_h;
  DevView host[kNoAllocMaxViews];
  int first[kNoAllocMaxViews + 1];
  int64_t rays[kNoAllocMaxViews];
  for (int l = 0, k = 0; l < nlaunch; ++l) {
    first[l] = k;
    int64_t off = 0;
    while (k < nv && launch_of[k] == l) {
      host[k] = make_dev_view(views[order[k]], off, out_off[order[k]], codes[k]);
      off += host[k].rays;
      ++k;
    }
    rays[l] = off;
  }
  first[nlaunch] = nv;

  cudaStream_t st = (cudaStream_t)stream;
  // the host table is pageable: the copy returns once it has been staged
  cudaError_t e = cudaMemcpyAsync(scratch->views, host, sizeof(DevView) * size_t(nv), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(scratch->counters, 0, sizeof(unsigned long long) * size_t(nlaunch), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(&scratch->stats, 0, sizeof(Stats), st);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "scratch set-up");
  const int prec = (opts && opts->de_precision == 64) ? 64 : 32;
  for (int l = 0; l < nlaunch; ++l) {
    if (rays[l] <= 0) continue;
    const int n = first[l + 1] - first[l];
    bool dir64 = false;
    for (int k = first[l]; k < first[l + 1]; ++k) dir64 |= host[k].dir64 != 0;
    LaunchArgs a;
    memset(&a, 0, sizeof(a));
    a.views = scratch->views + first[l];
    a.nviews = n;
    a.total_rays = rays[l];
    a.out = *out;
    a.t_hit = nullptr;
    a.counter = scratch->counters + l;
    a.stats = &scratch->stats;
    a.refill_threshold = std::max(1, std::min(32, opts && opts->refill_threshold ? opts->refill_threshold : 4));
    a.deadline_ns = int64_t(opts && opts->watchdog_ms > 0 ? opts->watchdog_ms : 10000) * 1000000;
    LaunchConfig c;
    c.kernel = ND_KERNEL_PERSISTENT;
    c.block = 128;
    c.blocks_per_sm = opts ? opts->blocks_per_sm : 0;
    c.num_sms = sms;
    // the inline march (normal and shadow phases in the march: no hit list here)
    const KernelTable& T = tables[l];
    const bool batched = n > 1;
    LaunchFn fn = prec == 64 ? (batched ? T.inline_f64_batched : T.inline_f64)
                             : dir64 ? (batched ? T.inline_f32_dir64_batched : T.inline_f32_dir64)
                                     : (batched ? T.inline_f32_batched : T.inline_f32);
    if (!fn) return fail(nullptr, ND_ERR_UNSUPPORTED, "no inline march kernel for this formula set");
    e = fn(a, host[first[l]], c, st);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "kernel launch");
  }
  return ND_OK;
}

// Statistics of the last nd_march_forward_noalloc call enqueued on the current
// device, read from the scratch array after the stream's work is done; the message
// of the calling thread's last failed call goes to err.
extern "C" nd_status nd_march_forward_noalloc_stats(void* stream, nd_stats* out, char* err, size_t err_len) {
  copy_str(err, err_len, g_noctx_err);
  if (!out) return ND_ERR_INVALID;
  memset(out, 0, sizeof(*out));
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return ND_ERR_CUDA;
  NoAllocScratch* scratch = nullptr;
  int sms = 0;
  nd_status s = noalloc_setup(dev, &scratch, &sms);
  if (s != ND_OK) return s;
  Stats h;
  cudaStream_t st = (cudaStream_t)stream;
  e = cudaMemcpyAsync(&h, &scratch->stats, sizeof(Stats), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "read scratch statistics");
  out->rays = h.rays;
  out->de_evals = h.de_evals;
  out->march_evals = h.march_evals;
  out->normal_evals = h.normal_evals;
  out->shadow_evals = h.shadow_evals;
  out->hits = h.hits;
  out->refills = h.refills;
  out->timeouts = h.timeouts;
  out->kernel = ND_KERNEL_PERSISTENT;
  if (h.timeouts) {
    fail(nullptr, ND_ERR_TIMEOUT, "the device watchdog stopped %u warps", h.timeouts);
    copy_str(err, err_len, g_noctx_err);
    return ND_ERR_TIMEOUT;
  }
  return ND_OK;
}

// ---------------------------------------------------------------------------
// Orbit camera and the adjoint pass.

namespace {

// The orbit pose's camera: origin, forward and the FOV-scaled right/up, with
// FreeCamera's basis (src/app/camera.zig:98-112).  S is double, or a complex number
// for the complex-step derivative of the basis.
template <class S>
void orbit_basis(const nd_orbit_camera& c, S yaw, S pitch, S dist, S org[3], S f[3], S r[3], S u[3]) {
  using std::cos;
  using std::sin;
  using std::sqrt;
  const S cp = cos(pitch);
  org[0] = S(c.target[0]) + dist * cp * sin(yaw);
  org[1] = S(c.target[1]) + dist * sin(pitch);
  org[2] = S(c.target[2]) - dist * cp * cos(yaw);
  for (int i = 0; i < 3; ++i) f[i] = S(c.target[i]) - org[i];
  // normalise without a modulus, so that the complex step stays analytic
  S fn = sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
  for (int i = 0; i < 3; ++i) f[i] = f[i] / fn;
  const double wu[3] = {c.world_up[0], c.world_up[1], c.world_up[2]};
  r[0] = f[1] * S(wu[2]) - f[2] * S(wu[1]);
  r[1] = f[2] * S(wu[0]) - f[0] * S(wu[2]);
  r[2] = f[0] * S(wu[1]) - f[1] * S(wu[0]);
  S rn = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  for (int i = 0; i < 3; ++i) r[i] = r[i] / rn;
  u[0] = r[1] * f[2] - r[2] * f[1];
  u[1] = r[2] * f[0] - r[0] * f[2];
  u[2] = r[0] * f[1] - r[1] * f[0];
  S un = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
  const S sc = S(std::tan(c.fov_y_deg * 0.5 * 3.14159265358979323846 / 180.0));
  for (int i = 0; i < 3; ++i) {
    r[i] = r[i] * sc;
    u[i] = u[i] / un * sc;
  }
}

// d(origin, forward, right, up)/d(yaw, pitch, dist) by complex steps (exact to
// rounding: no subtraction, step 1e-30).
nd::PoseTangents pose_tangents(const nd_orbit_camera& c) {
  typedef std::complex<double> Z;
  const double h = 1e-30;
  nd::PoseTangents T;
  for (int j = 0; j < 3; ++j) {
    const Z yaw(c.yaw, j == 0 ? h : 0.0), pitch(c.pitch, j == 1 ? h : 0.0), dist(c.dist, j == 2 ? h : 0.0);
    Z o[3], f[3], r[3], u[3];
    orbit_basis<Z>(c, yaw, pitch, dist, o, f, r, u);
    for (int i = 0; i < 3; ++i) {
      T.dorg[j][i] = o[i].imag() / h;
      T.dfwd[j][i] = f[i].imag() / h;
      T.dright[j][i] = r[i].imag() / h;
      T.dup[j][i] = u[i].imag() / h;
    }
  }
  return T;
}

}  // namespace

extern "C" nd_status nd_orbit_view(const nd_orbit_camera* cam, nd_view_desc* view) {
  if (!cam || !view) return ND_ERR_INVALID;
  const double wl = cam->world_up[0] * cam->world_up[0] + cam->world_up[1] * cam->world_up[1] +
                    cam->world_up[2] * cam->world_up[2];
  if (!(cam->dist > 0.0) || !(wl > 0.0) || !(cam->fov_y_deg > 0.0) || !(cam->fov_y_deg < 180.0))
    return ND_ERR_INVALID;
  double o[3], f[3], r[3], u[3];
  orbit_basis<double>(*cam, cam->yaw, cam->pitch, cam->dist, o, f, r, u);
  for (int i = 0; i < 3; ++i) {
    view->cam_pos[i] = o[i];
    view->fwd[i] = f[i];
    view->right[i] = r[i];
    view->up[i] = u[i];
  }
  return ND_OK;
}

extern "C" nd_status nd_march_backward(nd_ctx* ctx, const nd_view_desc* views, const nd_orbit_camera* cams,
                                       int32_t nviews, const int32_t* param_idx, int32_t nparams,
                                       const nd_gbuffer* fwd, const float* dL_dshade, double* dL_dtheta,
                                       double* dshade_dtheta, const nd_march_opts* opts, void* stream) {
  if (!ctx) return ND_ERR_INVALID;
  if (!cams || !fwd || !fwd->depth64 || !fwd->normal)
    return fail(ctx, ND_ERR_INVALID, "backward needs cameras and the forward's depth64 and normal");
  if (!dL_dtheta && !dshade_dtheta) return fail(ctx, ND_ERR_INVALID, "backward needs dL/dtheta or dshade/dtheta");
  if (dL_dtheta && !dL_dshade) return fail(ctx, ND_ERR_INVALID, "dL/dtheta needs dL/dshade");
  const int prec = opts ? opts->de_precision : 32;
  if (prec != 32 && prec != 64) return fail(ctx, ND_ERR_INVALID, "de_precision must be 32 or 64");
  if (nparams < 0 || nparams > nd::kMaxAdjParams || (nparams > 0 && !param_idx))
    return fail(ctx, ND_ERR_INVALID, "nparams must be in [0, %d]", nd::kMaxAdjParams);
  for (int k = 0; k < nparams; ++k)
    if (param_idx[k] < 0 || param_idx[k] >= ND_MAX_PARAMS) return fail(ctx, ND_ERR_INVALID, "bad param index");
  std::vector<Launch> plans;
  int64_t total = 0;
  nd_status s = prepare(ctx, views, nviews, fwd, &plans, &total);
  if (s != ND_OK) return s;
  for (int i = 0; i < nviews; ++i) {
    const nd_view_desc& v = views[i];
    const double l2 = double(v.light_dir[0]) * v.light_dir[0] + double(v.light_dir[1]) * v.light_dir[1] +
                      double(v.light_dir[2]) * v.light_dir[2];
    if (v.shadow || !(l2 > 0) || v.normal_mode != ND_NORMAL_CENTRAL)
      return fail(ctx, ND_ERR_UNSUPPORTED, "view %d: the adjoint needs a directional light, central-difference "
                  "normals and no shadow ray", i);
  }
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "set device");
  cudaStream_t st = (cudaStream_t)stream;
  // view table and pose tangents in launch order (temporary device buffers)
  std::vector<DevView> hv;
  std::vector<nd::PoseTangents> ht;
  std::vector<int64_t> out_off(nviews + 1, 0);
  for (int i = 0; i < nviews; ++i) out_off[i + 1] = out_off[i] + int64_t(views[i].spp) * views[i].tile_w * views[i].tile_h;
  std::vector<int> first;
  for (const Launch& L : plans) {
    first.push_back(int(hv.size()));
    int64_t off = 0;
    for (size_t k = 0; k < L.views.size(); ++k) {
      const int vi = L.views[k];
      DevView d = make_dev_view(views[vi], off, out_off[vi], L.codes[k]);
      d.user_index = vi;
      off += d.rays;
      hv.push_back(d);
      ht.push_back(pose_tangents(cams[vi]));
    }
  }
  DevView* dv = nullptr;
  nd::PoseTangents* dt = nullptr;
  e = cudaMallocAsync((void**)&dv, sizeof(DevView) * hv.size(), st);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&dt, sizeof(nd::PoseTangents) * ht.size(), st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dv, hv.data(), sizeof(DevView) * hv.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dt, ht.data(), sizeof(nd::PoseTangents) * ht.size(), cudaMemcpyHostToDevice, st);
  for (size_t p = 0; p < plans.size() && e == cudaSuccess; ++p) {
    const int nv = int(plans[p].views.size());
    nd::AdjointArgs a;
    memset(&a, 0, sizeof(a));
    a.views = dv + first[p];
    a.nviews = nv;
    a.total_rays = 0;
    for (int k = 0; k < nv; ++k) a.total_rays += hv[first[p] + k].rays;
    a.tangents = dt + first[p];
    a.depth64 = fwd->depth64;
    a.normal4 = fwd->normal;
    a.dL_dshade = dL_dtheta ? dL_dshade : nullptr;
    a.grad = dL_dtheta;
    a.dshade = dshade_dtheta;
    a.nparam = nparams;
    for (int k = 0; k < nparams; ++k) a.param_idx[k] = param_idx[k];
    const KernelTable& kt = plans[p].table;
    const nd::AdjointFn fn = prec == 64 ? (nv > 1 ? kt.adjoint_f64_batched : kt.adjoint_f64)
                                        : (nv > 1 ? kt.adjoint_f32_batched : kt.adjoint_f32);
    if (!fn) {
      e = cudaErrorNotSupported;
      break;
    }
    e = fn(a, hv[first[p]], st);
  }
  // the host staging vectors are pageable: wait for the copies before they go away
  cudaError_t e2 = cudaStreamSynchronize(st);
  if (dv) cudaFreeAsync(dv, st);
  if (dt) cudaFreeAsync(dt, st);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint launch");
  if (e2 != cudaSuccess) return cuda_fail(ctx, e2, "adjoint");
  return ND_OK;
}
