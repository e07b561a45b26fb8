// Adjoint of the Lambert image with respect to formula @params and an orbit camera
// pose, by implicit differentiation at the hit point.
//
// For every hit ray, with t the forward's hit distance, p = o + d t, g = grad DE(p):
//   the march stops where DE(p(t); theta) = eps(t) = coef t + floor, so
//     dt/dtheta = -(dDE/dtheta|_t fixed) / (g . d - coef)
//   dp/dtheta = do/dtheta + t dd/dtheta + d dt/dtheta
//   the normal is n = D / |D| with D_i = DE(p + h e_i) - DE(p - h e_i), h = hc t
//   (central differences), so dD_i/dtheta is the difference of the DE's total
//   derivatives at the two taps, the taps moving with dp/dtheta +- e_i dh/dtheta
//   dn = (dD - n (n . dD)) / |D|
//   I = a + (1 - a) max(n . L, 0)  =>  dI = (1 - a) [n . L > 0] (L . dn)
// and dLoss/dtheta = sum over rays of dLoss/dI * dI/dtheta.  Every DE total
// derivative is ONE evaluation of the formula code with T = Dual<S>, the position
// seeded with its tangent and the parameters with theirs.  Silhouette (visibility)
// changes are not differentiated: the gradient is that of the image's interior.
// Neither are hits where DE - eps(t) changes sign by a jump rather than through
// zero: a DE can be discontinuous (a Mandelbulb of non-integer power jumps where an
// iterate crosses atan2's branch cut, the half-plane y = 0, x < 0), and a hit on such
// a sheet moves with the sheet, not with the level set.  Such hits are recognised by
// their residual |DE(p) - eps(t)|, which a root reached by bisection does not have.
#pragma once

#include "nd_dual.h"
#include "nd_rayprog.h"

namespace nd {

constexpr int kMaxAdjParams = 4;  // formula @params per backward call
constexpr int kPoseParams = 3;    // yaw, pitch, distance of the orbit camera

// Derivatives of a view's camera with respect to yaw, pitch and distance.
struct PoseTangents {
  double dorg[kPoseParams][3];
  double dfwd[kPoseParams][3];
  double dright[kPoseParams][3];
  double dup[kPoseParams][3];
};

struct AdjointArgs {
  const DevView* views;
  int32_t nviews;
  int64_t total_rays;
  const PoseTangents* tangents;  // per view (launch order)
  const double* depth64;         // forward G-buffer (by G-buffer index)
  const float* normal4;
  const float* dL_dshade;        // nullable when grad is null
  double* grad;                  // nullable: [user view][nparam + 3], added to
  double* dshade;                // nullable: dI/dtheta per G-buffer slot [slot][nparam + 3]
  int32_t param_idx[kMaxAdjParams];
  int32_t nparam;
};

// Parameter accessor with one dual tangent: parameter `seed` gets tangent 1.
template <class S> struct DualParams {
  const float* v;
  int seed;
  ND_DEV_INLINE ndw::Dual<S> operator[](int i) const { return ndw::mkd(S(v[i]), i == seed ? S(1) : S(0)); }
};

// The DE of view v at p and its derivative along (position tangent tan, parameter seed).
template <class Set, class S>
ND_DEV_INLINE ndw::Dual<S> de_dir_full(const DevView& v, D3 p, D3 tan, int seed) {
  typedef ndw::Dual<S> DS;
  const ndw::v3<DS> q = ndw::v3<DS>(ndw::mkd(S(p.x), S(tan.x)), ndw::mkd(S(p.y), S(tan.y)), ndw::mkd(S(p.z), S(tan.z)));
  return Set::template de_with<DS, DualParams<S>>(v.code, q, DualParams<S>{v.params, seed}, v).d;
}
template <class Set, class S>
ND_DEV_INLINE S de_dir(const DevView& v, D3 p, D3 tan, int seed) {
  return de_dir_full<Set, S>(v, p, tan, seed).d;
}

// Largest |DE(p) - eps(t)| / eps(t) at a hit that is a root of the level set.  FP64
// bisection leaves ~1e-13.  An FP32 DE near the surface carries rounding of ~1e-3 of
// eps (12 iterations amplify each ulp by about dr), so FP32 tells only jumps above
// 1e-2 of eps from roots; the smaller jumps it misses are the FP32 adjoint's limit.
template <class S> struct RootTol;
template <> struct RootTol<double> { static constexpr double value = 1e-6; };
template <> struct RootTol<float> { static constexpr double value = 1e-2; };

ND_DEV_INLINE D3 axpy(D3 a, double s, D3 b) { return D3{a.x + s * b.x, a.y + s * b.y, a.z + s * b.z}; }
ND_DEV_INLINE double dot3(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
ND_DEV_INLINE D3 axis(int i, double s) { return D3{i == 0 ? s : 0.0, i == 1 ? s : 0.0, i == 2 ? s : 0.0}; }

// dI/dtheta_k of one hit ray (k < nparam: params[param_idx[k]]; then yaw, pitch,
// dist), written to dI[0 .. nparam + 3).  Returns false when the pixel contributes
// nothing (a back-lit normal, a degenerate gradient, a hit on a jump of the DE).
template <class Set, class S>
ND_DEV_INLINE bool adjoint_pixel(const DevView& v, const PoseTangents& T, const int32_t* param_idx, int nparam,
                                 int64_t local, double t, double* dI) {
  const int K = nparam + kPoseParams;
  double ux, uy;
  ray_uv(v, local, &ux, &uy);
  const D3 w = D3{v.fwd[0] + v.right[0] * ux + v.up[0] * uy, v.fwd[1] + v.right[1] * ux + v.up[1] * uy,
                  v.fwd[2] + v.right[2] * ux + v.up[2] * uy};
  const double wn = sqrt(dot3(w, w));
  const D3 d = ray_dir(v, local);  // w / |w| exactly as the forward computed it
  const D3 p = fmadd(D3{v.org[0], v.org[1], v.org[2]}, d, t);
  // value and gradient of the DE at the hit
  const ndw::Dual<S> gx = de_dir_full<Set, S>(v, p, axis(0, 1.0), -1);
  const D3 g = D3{double(gx.d), double(de_dir<Set, S>(v, p, axis(1, 1.0), -1)),
                  double(de_dir<Set, S>(v, p, axis(2, 1.0), -1))};
  const double eps_t = double(v.eps_coef) * t + double(v.eps_floor);
  if (eps_t > 0.0 && !(fabs(double(gx.v) - eps_t) <= RootTol<S>::value * eps_t)) return false;
  const double denom = dot3(g, d) - double(v.eps_coef);
  const bool central = v.normal_h_coef > 0.0f;
  const double hc = central ? double(v.normal_h_coef) : double(v.eps_coef);
  const double h = central ? hc * t : double(v.eps_coef) * t + double(v.eps_floor);
  // the normal's central-difference vector D
  double Dv[3];
  for (int i = 0; i < 3; ++i)
    Dv[i] = double(de_dir_full<Set, S>(v, axpy(p, h, axis(i, 1.0)), D3{0, 0, 0}, -1).v) -
            double(de_dir_full<Set, S>(v, axpy(p, -h, axis(i, 1.0)), D3{0, 0, 0}, -1).v);
  const D3 D = D3{Dv[0], Dv[1], Dv[2]};
  const double Dn = sqrt(dot3(D, D));
  if (!(Dn > 0.0) || denom == 0.0) return false;
  const D3 n = D3{D.x / Dn, D.y / Dn, D.z / Dn};
  const D3 L = D3{v.light[0], v.light[1], v.light[2]};
  if (!(dot3(n, L) > 0.0)) return false;
  for (int k = 0; k < K; ++k) {
    D3 dorg = D3{0, 0, 0}, dd = D3{0, 0, 0};
    int seed = -1;
    if (k < nparam) {
      seed = param_idx[k];
    } else {
      const int j = k - nparam;
      dorg = D3{T.dorg[j][0], T.dorg[j][1], T.dorg[j][2]};
      const D3 dw = D3{T.dfwd[j][0] + ux * T.dright[j][0] + uy * T.dup[j][0],
                       T.dfwd[j][1] + ux * T.dright[j][1] + uy * T.dup[j][1],
                       T.dfwd[j][2] + ux * T.dright[j][2] + uy * T.dup[j][2]};
      const double dd_par = dot3(d, dw);
      dd = D3{(dw.x - d.x * dd_par) / wn, (dw.y - d.y * dd_par) / wn, (dw.z - d.z * dd_par) / wn};
    }
    const D3 ptan0 = axpy(dorg, t, dd);  // dp/dtheta with t held fixed
    const double a_k = double(de_dir<Set, S>(v, p, ptan0, seed));
    const double dt = -a_k / denom;
    const D3 dp = axpy(ptan0, dt, d);
    const double dh = hc * dt;
    double dD[3];
    for (int i = 0; i < 3; ++i) {
      const D3 tp = axpy(dp, dh, axis(i, 1.0));
      const D3 tm = axpy(dp, -dh, axis(i, 1.0));
      dD[i] = double(de_dir<Set, S>(v, axpy(p, h, axis(i, 1.0)), tp, seed)) -
              double(de_dir<Set, S>(v, axpy(p, -h, axis(i, 1.0)), tm, seed));
    }
    const double nd = n.x * dD[0] + n.y * dD[1] + n.z * dD[2];
    const D3 dn = D3{(dD[0] - n.x * nd) / Dn, (dD[1] - n.y * nd) / Dn, (dD[2] - n.z * nd) / Dn};
    dI[k] = (1.0 - kSimpleAmbient) * dot3(L, dn);
  }
  return true;
}

#if defined(__CUDACC__)
// One thread per ray; S is the dual numbers' scalar (float: the FP32 DE of the
// forward; double: FP64 duals, for the central-difference normal's cancellation).
template <class Set, class S, bool kBatched>
__global__ void __launch_bounds__(128) adjoint_kernel(const __grid_constant__ AdjointArgs a,
                                                      const __grid_constant__ DevView single) {
  const int64_t it = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int K = a.nparam + kPoseParams;
  double acc[kMaxAdjParams + kPoseParams];
  for (int k = 0; k < kMaxAdjParams + kPoseParams; ++k) acc[k] = 0.0;
  int vi = -1;
  if (it < a.total_rays) {
    vi = kBatched ? find_view(a.views, a.nviews, it) : 0;
    const DevView& v = kBatched ? a.views[vi] : single;
    const int64_t local = it - v.ray_offset;
    const int64_t r = v.out_offset + local;
    const float w_loss = a.grad ? a.dL_dshade[r] : 0.0f;
    double dI[kMaxAdjParams + kPoseParams];
    for (int k = 0; k < kMaxAdjParams + kPoseParams; ++k) dI[k] = 0.0;
    if (a.normal4[4 * r + 3] > 0.5f && (w_loss != 0.0f || a.dshade)) {
      if (adjoint_pixel<Set, S>(v, a.tangents[kBatched ? vi : 0], a.param_idx, a.nparam, local, a.depth64[r], dI)) {
        for (int k = 0; k < kMaxAdjParams + kPoseParams; ++k)
          if (k < K) acc[k] = double(w_loss) * dI[k];
      } else {
        for (int k = 0; k < kMaxAdjParams + kPoseParams; ++k) dI[k] = 0.0;
      }
    }
    if (a.dshade)
      for (int k = 0; k < kMaxAdjParams + kPoseParams; ++k)
        if (k < K) a.dshade[r * K + k] = dI[k];
  }
  if (!a.grad) return;
  // reduce within the warp when every lane has the same view, else per lane
  const unsigned full = 0xffffffffu;
  const int uv = vi >= 0 ? (kBatched ? a.views[vi].user_index : single.user_index) : -1;
  const int uv0 = __shfl_sync(full, uv, 0);
  const bool uniform = __all_sync(full, uv == uv0);
  for (int k = 0; k < kMaxAdjParams + kPoseParams; ++k) {
    if (k >= K) break;
    double x = acc[k];
    if (uniform) {
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(full, x, o);
      if ((threadIdx.x & 31) == 0 && uv0 >= 0 && x != 0.0) atomicAdd(&a.grad[uv0 * K + k], x);
    } else if (uv >= 0 && x != 0.0) {
      atomicAdd(&a.grad[uv * K + k], x);
    }
  }
}

template <class Set, class S, bool kBatched>
cudaError_t launch_adjoint(const AdjointArgs& a, const DevView& single, cudaStream_t s) {
  const int64_t grid = (a.total_rays + 127) / 128;
  if (grid <= 0) return cudaSuccess;
  adjoint_kernel<Set, S, kBatched><<<unsigned(grid), 128, 0, s>>>(a, single);
  return cudaGetLastError();
}

typedef cudaError_t (*AdjointFn)(const AdjointArgs&, const DevView&, cudaStream_t);
#endif

}  // namespace nd
