// Counter-based Gaussian noise: Philox4x32-10 (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11) and a Box-Muller
// transform on 24-bit uniforms.  Counter = (draw mode index, pair index,
// step lo, step hi); key = (seed lo, seed hi).  Complex value v = field*ncomp
// + comp of a step uses pair v/2, words (0,1) for even v and (2,3) for odd v.
#pragma once
#include "pf_common.cuh"

namespace pf {

struct u4 { uint32_t x, y, z, w; };

PF_D u4 philox4x32_10(u4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
    u4 n;
    n.x = hi1 ^ c.y ^ k0; n.y = lo1; n.z = hi0 ^ c.w ^ k1; n.w = lo0;
    c = n;
  }
  return c;
}

template <typename R> PF_D void box_muller(uint32_t a, uint32_t b, R& z0, R& z1);

template <> PF_D void box_muller<float>(uint32_t a, uint32_t b, float& z0, float& z1) {
  const float u = (float(a >> 8) + 0.5f) * (1.0f / 16777216.0f);
  const float v = (float(b >> 8) + 0.5f) * (1.0f / 16777216.0f);
  const float r = sqrtf(-2.0f * logf(u));
  float s, c;
  sincospif(2.0f * v, &s, &c);
  z0 = r * c; z1 = r * s;
}

template <> PF_D void box_muller<double>(uint32_t a, uint32_t b, double& z0, double& z1) {
  const double u = (double(a >> 8) + 0.5) * (1.0 / 16777216.0);
  const double v = (double(b >> 8) + 0.5) * (1.0 / 16777216.0);
  const double r = sqrt(-2.0 * log(u));
  double s, c;
  sincospi(2.0 * v, &s, &c);
  z0 = r * c; z1 = r * s;
}

// Hermitian pairing of a half-spectrum mode on the self-conjugate planes
// (last-axis index 0 and n_last/2).  idx = (i0, i1[, i2]) of the mode;
// returns the linear index whose draw is used, and flags conj / real.
struct DrawSite { uint32_t index; bool conj; bool real; };

PF_D DrawSite draw_site(const Geo& g, int i0, int i1, int i2) {
  DrawSite d;
  d.conj = false; d.real = false;
  if (g.dim == 3) {
    d.index = (uint32_t)(((long long)i0 * g.s[1] + i1) * g.nh + i2);
    const bool plane = (i2 == 0) || ((g.n[2] % 2 == 0) && i2 == g.n[2] / 2);
    if (plane) {
      const int m0 = (g.n[0] - i0) % g.n[0], m1 = (g.n[1] - i1) % g.n[1];
      const bool less = (i0 < m0) || (i0 == m0 && i1 < m1);
      const bool eq = (i0 == m0) && (i1 == m1);
      if (eq) d.real = true;
      else if (!less) {
        d.conj = true;
        d.index = (uint32_t)(((long long)m0 * g.s[1] + m1) * g.nh + i2);
      }
    }
  } else {
    d.index = (uint32_t)((long long)i0 * g.nh + i1);
    const bool plane = (i1 == 0) || ((g.n[1] % 2 == 0) && i1 == g.n[1] / 2);
    if (plane) {
      const int m0 = (g.n[0] - i0) % g.n[0];
      if (m0 == i0) d.real = true;
      else if (m0 < i0) {
        d.conj = true;
        d.index = (uint32_t)((long long)m0 * g.nh + i1);
      }
    }
  }
  return d;
}

// Raw (unnormalised) complex draw number v of a step at a draw site.
template <typename R>
PF_D cx<R> draw_value(const DrawSite& s, int v, uint64_t seed, uint64_t step) {
  u4 c;
  c.x = s.index; c.y = (uint32_t)(v >> 1);
  c.z = (uint32_t)step; c.w = (uint32_t)(step >> 32);
  const u4 o = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  R zr, zi;
  if (v & 1) box_muller<R>(o.z, o.w, zr, zi);
  else box_muller<R>(o.x, o.y, zr, zi);
  if (s.real) return mk<R>(zr * R(1.41421356237309504880), R(0));
  return mk<R>(zr, s.conj ? -zi : zi);
}

}  // namespace pf
