// bn_fp64.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Deterministic FP64 reference for image error (RMSE) reporting.  It
// computes, by fixed-step ray marching in double precision, the expected
// value of the frame Barney's structured-volume estimator converges to when
// its free-flight distances are exact exponentials (-log instead of the
// fastLog series of Volume.h:154-164):
//
//   E[pixel] = T_cam * bg
//            + integral over t of sigma(t) T(0,t) * albedo(x(t)) * S(x(t)) dt
//
// where sigma is the transfer-function density (TransferFunction.h:68-87,
// w channel times baseDensity), albedo is the phase tint (0.7 * TF rgb for
// SimplePhase, Phase.h:119-142; scatteringAlbedo * TF rgb for HGPhase,
// Phase.h:43-48), and S is the estimator's expected light term from
// shadeRays.cu:294-402,684-744:
//   constant environment: 4 pi A * 4 pi * E_w[ misWeight(w) * phase(w) * T(x,w) ]
//     (light pdf 1/4pi, radiance 4 pi A, MIS weight pdf_l/(pdf_l+pdf_bsdf)),
//     integrated over a fixed spherical Fibonacci set of directions;
//   each directional light: phase(w_l) * radiance_l * T(x, w_l).
// Emission-absorption mode: S is replaced by the TF colour and albedo by 1.
// The pixel footprint is a G x G grid of sub-pixel positions (box filter),
// which is what the jittered per-wave samples of generateRays.cu:89-92
// average to.
//
// The field is the trilinear interpolation (in double) of the stored voxel
// values with the clamp rules of rtcore/cpu/Texture.cpp:324-336.

#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "bn_oracle.h"

namespace {

struct d3 { double x, y, z; };
inline d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline d3 operator*(double s, d3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline d3 cross(d3 a, d3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline d3 normalize(d3 v) { return (1.0 / std::sqrt(dot(v, v))) * v; }

float h2f(uint16_t h) {
  uint32_t sign = (uint32_t)(h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu, out;
  if (e == 0) {
    if (m == 0) out = sign;
    else { float f = (float)m * (1.f / 16777216.f); uint32_t b; memcpy(&b, &f, 4); out = sign | b; }
  } else if (e == 31) out = sign | 0x7f800000u | (m << 13);
  else out = sign | ((e + 112u) << 23) | (m << 13);
  float r; memcpy(&r, &out, 4); return r;
}

struct Field {
  const OrcScene &s;
  d3 org, spc, lo, hi;
  explicit Field(const OrcScene &s) : s(s) {
    org = {s.origin[0], s.origin[1], s.origin[2]};
    spc = {s.spacing[0], s.spacing[1], s.spacing[2]};
    lo = org;
    hi = {org.x + spc.x * (s.dims[0] - 1), org.y + spc.y * (s.dims[1] - 1), org.z + spc.z * (s.dims[2] - 1)};
  }
  double texel(int64_t i) const {
    switch (s.dtype) {
    case 0: return ((const float *)s.voxels)[i];
    case 1: return ((const uint8_t *)s.voxels)[i] / 255.0;
    case 2: return h2f(((const uint16_t *)s.voxels)[i]);
    case 3: { uint32_t u = (uint32_t)((const uint16_t *)s.voxels)[i] << 16; float f; memcpy(&f, &u, 4); return f; }
    default: return ((const uint16_t *)s.voxels)[i] / 65535.0;
    }
  }
  static void coord(double u, int N, int &i0, int &i1, double &f) {
    if (u <= 0) { i0 = i1 = 0; f = 0; return; }
    if (u >= N - 1) { i0 = i1 = N - 1; f = 0; return; }
    i0 = (int)u; i1 = i0 + 1; f = u - i0;
  }
  // returns false outside [0, numCells)
  bool sample(d3 P, double &v) const {
    double rx = (P.x - org.x) / spc.x, ry = (P.y - org.y) / spc.y, rz = (P.z - org.z) / spc.z;
    if (rx < 0 || ry < 0 || rz < 0 || rx >= s.dims[0] - 1 || ry >= s.dims[1] - 1 || rz >= s.dims[2] - 1) return false;
    int x0, x1, y0, y1, z0, z1; double fx, fy, fz;
    coord(rx, s.dims[0], x0, x1, fx); coord(ry, s.dims[1], y0, y1, fy); coord(rz, s.dims[2], z0, z1, fz);
    const int64_t NX = s.dims[0], NXY = (int64_t)s.dims[0] * s.dims[1];
    auto T = [&](int x, int y, int z) { return texel(x + NX * y + NXY * z); };
    double c00 = (1 - fx) * T(x0, y0, z0) + fx * T(x1, y0, z0);
    double c01 = (1 - fx) * T(x0, y1, z0) + fx * T(x1, y1, z0);
    double c10 = (1 - fx) * T(x0, y0, z1) + fx * T(x1, y0, z1);
    double c11 = (1 - fx) * T(x0, y1, z1) + fx * T(x1, y1, z1);
    double c0 = (1 - fy) * c00 + fy * c01, c1 = (1 - fy) * c10 + fy * c11;
    v = (1 - fz) * c0 + fz * c1;
    return true;
  }
  void tf(double v, double rgba[4]) const {
    double span = (double)s.domain[1] - s.domain[0];
    double f = (v - s.domain[0]) / span;
    f = std::min(1.0, std::max(0.0, f)) * (s.tfN - 1);
    int idx = std::min(s.tfN - 2, std::max(0, (int)f));
    f -= idx;
    for (int c = 0; c < 4; c++) rgba[c] = (1 - f) * s.tf[4 * idx + c] + f * s.tf[4 * (idx + 1) + c];
    rgba[3] *= s.baseDensity;
  }
  double sigma(d3 P) const {
    double v;
    if (!sample(P, v)) return 0;
    double rgba[4];
    tf(v, rgba);
    return rgba[3];
  }
  bool clip(d3 o, d3 d, double &t0, double &t1) const {
    t0 = 0; t1 = 1e300;
    double O[3] = {o.x, o.y, o.z}, D[3] = {d.x, d.y, d.z}, L[3] = {lo.x, lo.y, lo.z}, H[3] = {hi.x, hi.y, hi.z};
    for (int a = 0; a < 3; a++) {
      if (D[a] == 0) { if (O[a] < L[a] || O[a] > H[a]) return false; continue; }
      double ta = (L[a] - O[a]) / D[a], tb = (H[a] - O[a]) / D[a];
      if (ta > tb) std::swap(ta, tb);
      t0 = std::max(t0, ta); t1 = std::min(t1, tb);
    }
    return t0 < t1;
  }
  // transmittance along o + t d, t in [0, inf), midpoint rule with step h
  double transmittance(d3 o, d3 d, double h) const {
    double t0, t1;
    if (!clip(o, d, t0, t1)) return 1.0;
    double tau = 0;
    for (double t = t0 + 0.5 * h; t < t1; t += h) {
      tau += sigma(o + t * d) * h;
      if (tau > 40) return 0.0;
    }
    return std::exp(-tau);
  }
};

inline double hg(double g, double c) {
  if (std::fabs(g) < 1e-3) return 1.0 / (4 * M_PI);
  double g2 = g * g, den = 1 + g2 - 2 * g * c;
  return (1.0 / (4 * M_PI)) * (1 - g2) / (den * std::sqrt(den));
}

} // namespace

extern "C" {

// Writes width*height float4 for the rectangle [x0,x1) x [y0,y1) (other
// pixels untouched).  step: march step in world units; subpix: G; envDirs:
// number of quadrature directions for the environment term.
void orc64_render_expected(const OrcScene *sp, int x0, int y0, int x1, int y1, double step, int subpix,
                           int envDirs, int numThreads, double *out) {
  const OrcScene &s = *sp;
  Field F(s);
  d3 pos = {s.camPos[0], s.camPos[1], s.camPos[2]};
  d3 dir = normalize({s.camDir[0], s.camDir[1], s.camDir[2]});
  d3 up = {s.camUp[0], s.camUp[1], s.camUp[2]};
  d3 du = normalize(cross(dir, up)), dv = normalize(cross(du, dir));
  d3 d00 = (1.0 / (2.0 * std::tan(0.5 * s.fovy * M_PI / 180.0))) * dir;
  const double W = s.width, H = s.height, aspect = W / H;
  std::vector<d3> env(envDirs);
  for (int k = 0; k < envDirs; k++) {  // spherical Fibonacci directions
    double z = 1 - (2.0 * k + 1) / envDirs, r = std::sqrt(std::max(0.0, 1 - z * z));
    double phi = k * M_PI * (3 - std::sqrt(5.0));
    env[k] = {r * std::cos(phi), r * std::sin(phi), z};
  }
  struct DL { d3 toLight; double rad[3]; };
  std::vector<DL> dls;
  for (int l = 0; l < s.numDirLights; l++) {
    const float *L = s.dirLights + 7 * l;
    DL d;
    d.toLight = -1.0 * normalize({L[0], L[1], L[2]});
    for (int c = 0; c < 3; c++) d.rad[c] = (double)L[4 + c] * L[3];
    dls.push_back(d);
  }
  if (numThreads <= 0) numThreads = (int)std::thread::hardware_concurrency();
  std::atomic<int> nextRow{y0};
  auto worker = [&]() {
    while (true) {
      int iy = nextRow++;
      if (iy >= y1) break;
      for (int ix = x0; ix < x1; ix++) {
        double acc[4] = {0, 0, 0, 0};
        for (int sy = 0; sy < subpix; sy++)
          for (int sx = 0; sx < subpix; sx++) {
            double u = (ix + (sx + 0.5) / subpix) / W, v = (iy + (sy + 0.5) / subpix) / H;
            d3 rd = normalize(d00 + (aspect * (u - 0.5)) * du + (v - 0.5) * dv);
            double t0, t1, T = 1.0, rgb[3] = {0, 0, 0};
            if (F.clip(pos, rd, t0, t1)) {
              for (double t = t0 + 0.5 * step; t < t1 && T > 1e-7; t += step) {
                d3 P = pos + t * rd;
                double val;
                if (!F.sample(P, val)) continue;
                double tf[4];
                F.tf(val, tf);
                double sg = tf[3];
                if (sg <= 0) continue;
                double w = T * (1 - std::exp(-sg * step));  // probability of colliding in this step
                if (s.emissionAbsorption) {
                  for (int c = 0; c < 3; c++) rgb[c] += w * tf[c];
                } else {
                  double alb[3];
                  double a = s.phaseMode == 0 ? 0.7 : s.scatteringAlbedo;
                  for (int c = 0; c < 3; c++) alb[c] = a * tf[c];
                  double S = 0;
                  if (s.ambientRadiance != 0) {
                    double e = 0;
                    for (int k = 0; k < envDirs; k++) {
                      double ph = s.phaseMode == 0 ? 1.0 / (4 * M_PI) : hg(s.anisotropy, dot(rd, env[k]));
                      double mis = (1.0 / (4 * M_PI)) / (1.0 / (4 * M_PI) + ph + 1e-10);
                      e += mis * ph * F.transmittance(P, env[k], step);
                    }
                    S += 4 * M_PI * s.ambientRadiance * 4 * M_PI * e / envDirs;
                  }
                  double Sc[3] = {S, S, S};
                  for (auto &d : dls) {
                    double ph = s.phaseMode == 0 ? 1.0 / (4 * M_PI) : hg(s.anisotropy, dot(rd, d.toLight));
                    double Tl = F.transmittance(P, d.toLight, step);
                    for (int c = 0; c < 3; c++) Sc[c] += ph * d.rad[c] * Tl;
                  }
                  for (int c = 0; c < 3; c++) rgb[c] += w * alb[c] * Sc[c];
                }
                T *= std::exp(-sg * step);
              }
            }
            double bgw = s.bgColor[3];
            double bg[3] = {s.bgColor[0], s.bgColor[1], s.bgColor[2]};
            if (s.bgColor[3] < 0) {
              double tt = (iy + 0.5) / H;
              bg[0] = (1 - tt) * 0.9 + tt * 0.15; bg[1] = (1 - tt) * 0.9 + tt * 0.25; bg[2] = (1 - tt) * 0.9 + tt * 0.8;
              bgw = 1;
            }
            for (int c = 0; c < 3; c++) acc[c] += rgb[c] + T * bg[c];
            acc[3] += (1 - T) + T * bgw;
          }
        double norm = 1.0 / (subpix * subpix);
        double *o = out + 4 * ((int64_t)iy * s.width + ix);
        for (int c = 0; c < 4; c++) o[c] = acc[c] * norm;
      }
    }
  };
  std::vector<std::thread> th;
  for (int i = 0; i < numThreads; i++) th.emplace_back(worker);
  for (auto &t : th) t.join();
}

} // extern "C"
