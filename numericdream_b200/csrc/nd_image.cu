// Formula images (`// @image`): the host preparation of an image's texels, as the
// reference prepares a height map after decoding it (HeightMaps.decode,
// src/gpu/height_maps.zig:264-320).  Host code only; the sampler the formulas call is
// image_sample in nd_helpers.h.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/nd_march.h"

namespace {

constexpr int kMaxEdge = 2048;            // max_edge, height_maps.zig:9
constexpr int kSlopeRadiusNear = 8;       // slope_radius_near :10
constexpr int kSlopeRadiusFar = 64;       // slope_radius_far :11
constexpr int kDilateMargin = 2;          // dilate_margin :20
constexpr float kSlopeRoundUp = 1.001f;   // slope_round_up :21
constexpr float kStepsPerOctave = 16.0f;  // slope_steps_per_octave :16
constexpr float kCodeMax = 255.0f;        // slope_code_max :17
constexpr float kCodeMaxLog2 = 1.0f;      // slope_code_max_log2 :18

struct Rgba {
  float c[4];
};

// 16-bit quantisation of a channel value (quantize, :327-330)
float quantize(float v) { return roundf(std::min(std::max(v, 0.0f), 1.0f) * 65535.0f) / 65535.0f; }

// The u8 code of a slope bound: ceil(16 (log2(1.001 s) - 1) + 255) in 1..255, 0 for no
// change (slopeCode, :332-336); image_slope_decode turns it back into a bound >= s.
uint32_t slope_code(float s) {
  if (!(s > 0.0f)) return 0;
  const float steps = ceilf(kStepsPerOctave * (log2f(s * kSlopeRoundUp) - kCodeMaxLog2) + kCodeMax);
  return uint32_t(std::min(std::max(steps, 1.0f), kCodeMax));
}

uint32_t pack_slopes(const Rgba& s) {
  uint32_t out = 0;
  for (int ch = 0; ch < 4; ++ch) out |= slope_code(s.c[ch]) << (8 * ch);
  return out;
}

// The maximum over a window of 2 radius + 1 samples along one line (clamped at its ends),
// in O(len): running maxima forward within blocks of the window's length and backward
// within the same blocks, the window's maximum is the larger of the backward maximum
// at its start and the forward maximum at its end (dilateLine, :349-370).
void dilate_line(Rgba* data, size_t start, size_t stride, size_t len, size_t radius, std::vector<Rgba>& fwd,
                 std::vector<Rgba>& bwd, std::vector<Rgba>& out) {
  const size_t k = 2 * radius + 1;
  for (size_t i = 0; i < len; ++i) {
    const Rgba& v = data[start + i * stride];
    if (i % k == 0) {
      fwd[i] = v;
    } else {
      for (int ch = 0; ch < 4; ++ch) fwd[i].c[ch] = std::max(fwd[i - 1].c[ch], v.c[ch]);
    }
  }
  for (size_t i = len; i-- > 0;) {
    const Rgba& v = data[start + i * stride];
    if (i == len - 1 || (i + 1) % k == 0) {
      bwd[i] = v;
    } else {
      for (int ch = 0; ch < 4; ++ch) bwd[i].c[ch] = std::max(bwd[i + 1].c[ch], v.c[ch]);
    }
  }
  for (size_t j = 0; j < len; ++j) {
    const size_t lo = j > radius ? j - radius : 0;
    const size_t hi = std::min(j + radius, len - 1);
    for (int ch = 0; ch < 4; ++ch) out[j].c[ch] = std::max(bwd[lo].c[ch], fwd[hi].c[ch]);
  }
  for (size_t j = 0; j < len; ++j) data[start + j * stride] = out[j];
}

// dilate (:344-347): rows, then columns
void dilate(std::vector<Rgba>& data, size_t w, size_t h, size_t radius) {
  const size_t m = std::max(w, h);
  std::vector<Rgba> fwd(m), bwd(m), out(m);
  for (size_t y = 0; y < h; ++y) dilate_line(data.data(), y * w, 1, w, radius, fwd, bwd, out);
  for (size_t x = 0; x < w; ++x) dilate_line(data.data(), x, w, h, radius, fwd, bwd, out);
}

}  // namespace

extern "C" nd_status nd_image_prepare(const float* rgba, int32_t width, int32_t height, uint32_t* texels,
                                      float* slope) {
  if (!rgba || !texels || !slope || width <= 0 || height <= 0 || width > kMaxEdge || height > kMaxEdge)
    return ND_ERR_INVALID;
  const size_t w = size_t(width), h = size_t(height), n = w * h;
  std::vector<Rgba> values(n);
  for (size_t i = 0; i < n; ++i)
    for (int ch = 0; ch < 4; ++ch) values[i].c[ch] = quantize(rgba[4 * i + ch]);
  // per texel: the larger change to the right and down, over the 2 x 2 block
  std::vector<Rgba> slopes(n);
  Rgba global{{0, 0, 0, 0}};
  for (size_t y = 0; y < h; ++y) {
    for (size_t x = 0; x < w; ++x) {
      const size_t x1 = std::min(x + 1, w - 1), y1 = std::min(y + 1, h - 1);
      const Rgba &a = values[y * w + x], &b = values[y * w + x1], &c = values[y1 * w + x], &d = values[y1 * w + x1];
      Rgba g;
      for (int ch = 0; ch < 4; ++ch) {
        const float dx = std::max(fabsf(b.c[ch] - a.c[ch]), fabsf(d.c[ch] - c.c[ch]));
        const float dy = std::max(fabsf(c.c[ch] - a.c[ch]), fabsf(d.c[ch] - b.c[ch]));
        g.c[ch] = sqrtf(dx * dx + dy * dy);
        global.c[ch] = std::max(global.c[ch], g.c[ch]);
      }
      slopes[y * w + x] = g;
    }
  }
  std::vector<Rgba> near = slopes;
  dilate(near, w, h, kSlopeRadiusNear + kDilateMargin);
  dilate(slopes, w, h, kSlopeRadiusFar + kDilateMargin);
  for (size_t i = 0; i < n; ++i) {
    uint32_t q[4];
    for (int ch = 0; ch < 4; ++ch) q[ch] = uint32_t(roundf(values[i].c[ch] * 65535.0f));
    uint32_t* t = texels + 4 * i;
    t[0] = q[0] | (q[1] << 16);
    t[1] = q[2] | (q[3] << 16);
    t[2] = pack_slopes(near[i]);
    t[3] = pack_slopes(slopes[i]);
  }
  for (int ch = 0; ch < 4; ++ch) slope[ch] = global.c[ch] * kSlopeRoundUp;
  return ND_OK;
}
