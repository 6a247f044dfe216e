// Host-side scene compilation: the reference's `compileScene` (src/simulation/scene.ts:233-278) with
// its noise (src/shared/noise.ts), materials (src/simulation/material.ts) and the initial span
// coupling of the yarn damage field (src/simulation/yarnField.ts:422-499). This is input
// preparation, as in the reference (it runs on the CPU before the solver is constructed); the solve
// itself is the CUDA path. Arithmetic follows the reference's JavaScript operation order, so the
// compiled arrays (and sceneHash, scene.ts:134-150) reproduce the reference's bit for bit.

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "btd.h"
#include "jsmath.h"

namespace btd {
void setError(const std::string& msg);
}

namespace {

using btd::jsHypot2;
using btd::toInt32;

// ------------------------------------------------------------------------------------ noise.ts

// lowbias32 integer hash (noise.ts:4-12).
uint32_t hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// hash3(a, b, c) = hash32(a ^ hash32(b ^ hash32(c))) on ToInt32 operands (noise.ts:14-16).
uint32_t hash3(double a, double b, double c) {
  uint32_t hc = hash32(static_cast<uint32_t>(toInt32(c)));
  uint32_t hb = hash32(static_cast<uint32_t>(toInt32(b)) ^ hc);
  return hash32(static_cast<uint32_t>(toInt32(a)) ^ hb);
}

double rand01(double a, double b = 0, double c = 0) { return hash3(a, b, c) / 4294967296.0; }

double fade(double t) { return t * t * t * (t * (t * 6 - 15) + 10); }

double grad(double seed, double ix, double iy, double fx, double fy) {
  double h = hash3(seed, ix, iy);
  double ang = (h / 4294967296.0) * M_PI * 2;
  return std::cos(ang) * fx + std::sin(ang) * fy;
}

// 2D gradient noise (noise.ts:38-53).
double gradientNoise(double seed, double x, double y) {
  double ix = std::floor(x), iy = std::floor(y);
  double fx = x - ix, fy = y - iy;
  double u = fade(fx), v = fade(fy);
  double n00 = grad(seed, ix, iy, fx, fy);
  double n10 = grad(seed, ix + 1, iy, fx - 1, fy);
  double n01 = grad(seed, ix, iy + 1, fx, fy - 1);
  double n11 = grad(seed, ix + 1, iy + 1, fx - 1, fy - 1);
  double a = n00 + (n10 - n00) * u;
  double b = n01 + (n11 - n01) * u;
  return a + (b - a) * v;
}

// Fractal sum (noise.ts:56-70).
double fbm(double seed, double x, double y, int octaves, double lacunarity = 2.03, double gain = 0.5) {
  double sum = 0, amp = 1, norm = 0, fx = x, fy = y;
  for (int o = 0; o < octaves; ++o) {
    sum += amp * gradientNoise(seed + o * 1013, fx, fy);
    norm += amp;
    amp *= gain;
    fx *= lacunarity;
    fy *= lacunarity;
  }
  return (sum / norm) * 1.6;
}

double noise1(double seed, double x) { return gradientNoise(seed, x, 0.5 + std::fmod(seed, 7.0) * 0.13); }

double smoothstep(double e0, double e1, double x) {
  double t = std::min(1.0, std::max(0.0, (x - e0) / (e1 - e0)));
  return t * t * (3 - 2 * t);
}

// ------------------------------------------------------------------------------------ material.ts

btd_yarn yarn(double ld, double lo, double hi, double crimp, double comp, double av, double br, double bvisc,
              double strength, double soft, double width, double height, double crimpAmp) {
  btd_yarn y{};
  y.linear_density = ld;
  y.ea_low = lo;
  y.ea_high = hi;
  y.crimp_strain = crimp;
  y.ea_compress = comp;
  y.axial_viscosity = av;
  y.bend_rigidity = br;
  y.bend_viscosity = bvisc;
  y.strength = strength;
  y.softening_opening = soft;
  y.width = width;
  y.height = height;
  y.crimp_amplitude = crimpAmp;
  y.yarns_per_span = 0;
  return y;
}

// DENIM and BACKING (material.ts:88-187).
btd_material preset(int index) {
  btd_material m{};
  if (index == 0) {
    m.id = 0;
    std::snprintf(m.name, sizeof m.name, "%s", "denim-3x1");
    m.pitch_u = 0.38e-3;
    m.pitch_v = 0.58e-3;
    m.yarns[0] = yarn(60e-6, 6, 140, 0.03, 3, 2e-4, 4e-8, 2e-2, 8.5, 0.4e-3, 0.4e-3, 0.16e-3, 0.0);
    m.yarns[1] = yarn(84e-6, 10, 180, 0.025, 5, 2e-4, 4.5e-8, 2e-2, 11, 0.4e-3, 0.7e-3, 0.26e-3, 0.13e-3);
    m.twill_repeat = 4;
    m.twill_warp_over = 3;
    m.shear_stiffness = 60;
    m.crossing_friction = 0.35;
    m.crossing_normal0 = 0.25;
    m.crossing_wrap = 0.3;
    m.thickness = 0.7e-3;
    m.cloth_friction = 0.45;
    m.air_drag = 1.5;
  } else {
    m.id = 1;
    std::snprintf(m.name, sizeof m.name, "%s", "brushed-backing");
    m.pitch_u = 0.5e-3;
    m.pitch_v = 0.5e-3;
    m.yarns[0] = yarn(55e-6, 5, 90, 0.04, 0.3, 2e-4, 6e-9, 2e-2, 6, 0.25e-3, 0.52e-3, 0.34e-3, 0.08e-3);
    m.yarns[1] = m.yarns[0];
    m.twill_repeat = 3;
    m.twill_warp_over = 2;
    m.shear_stiffness = 45;
    m.crossing_friction = 0.45;
    m.crossing_normal0 = 0.2;
    m.crossing_wrap = 0.3;
    m.thickness = 1.0e-3;
    m.cloth_friction = 0.55;
    m.air_drag = 1.5;
  }
  return m;
}

// bundleWeave (material.ts:198-226).
btd_material bundleWeave(const btd_material& m, int bu, int bv) {
  if (bu == 1 && bv == 1) return m;
  btd_material o = m;
  std::string name = std::string(m.name) + "/b" + std::to_string(bu) + "x" + std::to_string(bv);
  std::snprintf(o.name, sizeof o.name, "%s", name.c_str());
  o.pitch_u = bu * m.pitch_u;
  o.pitch_v = bv * m.pitch_v;
  auto scale = [](btd_yarn y, int b) {
    y.linear_density = b * y.linear_density;
    y.ea_low = b * y.ea_low;
    y.ea_high = b * y.ea_high;
    y.ea_compress = b * y.ea_compress;
    y.axial_viscosity = b * y.axial_viscosity;
    y.bend_rigidity = b * y.bend_rigidity;
    y.strength = b * y.strength;
    y.yarns_per_span = b;
    return y;
  };
  o.yarns[0] = scale(m.yarns[0], bv);
  o.yarns[1] = scale(m.yarns[1], bu);
  auto shape = [](double a, double c) { return (a * a + c * c) / (a * c); };
  o.shear_stiffness = (m.shear_stiffness * shape(bu * m.pitch_u, bv * m.pitch_v)) / shape(m.pitch_u, m.pitch_v);
  o.crossing_normal0 = bu * bv * m.crossing_normal0;
  return o;
}

double crossingMass(const btd_material& m) {
  return m.yarns[0].linear_density * m.pitch_u + m.yarns[1].linear_density * m.pitch_v;
}

// JSON.stringify of a material (key order of the reference's object literals and spreads).
std::string materialJson(const btd_material& m) {
  using btd::jsNumber;
  auto yarnJson = [](const btd_yarn& y) {
    std::string s = "{";
    s += "\"linearDensity\":" + jsNumber(y.linear_density);
    s += ",\"eaLow\":" + jsNumber(y.ea_low);
    s += ",\"eaHigh\":" + jsNumber(y.ea_high);
    s += ",\"crimpStrain\":" + jsNumber(y.crimp_strain);
    s += ",\"eaCompress\":" + jsNumber(y.ea_compress);
    s += ",\"axialViscosity\":" + jsNumber(y.axial_viscosity);
    s += ",\"bendRigidity\":" + jsNumber(y.bend_rigidity);
    s += ",\"bendViscosity\":" + jsNumber(y.bend_viscosity);
    s += ",\"strength\":" + jsNumber(y.strength);
    s += ",\"softeningOpening\":" + jsNumber(y.softening_opening);
    s += ",\"width\":" + jsNumber(y.width);
    s += ",\"height\":" + jsNumber(y.height);
    s += ",\"crimpAmplitude\":" + jsNumber(y.crimp_amplitude);
    if (y.yarns_per_span > 0) s += ",\"yarnsPerSpan\":" + jsNumber(y.yarns_per_span);
    return s + "}";
  };
  std::string s = "{\"id\":" + jsNumber(m.id);
  s += ",\"name\":\"" + std::string(m.name) + "\"";
  s += ",\"pitchU\":" + jsNumber(m.pitch_u);
  s += ",\"pitchV\":" + jsNumber(m.pitch_v);
  s += ",\"yarns\":[" + yarnJson(m.yarns[0]) + "," + yarnJson(m.yarns[1]) + "]";
  s += ",\"twillRepeat\":" + jsNumber(m.twill_repeat);
  s += ",\"twillWarpOver\":" + jsNumber(m.twill_warp_over);
  s += ",\"shearStiffness\":" + jsNumber(m.shear_stiffness);
  s += ",\"crossingFriction\":" + jsNumber(m.crossing_friction);
  s += ",\"crossingNormal0\":" + jsNumber(m.crossing_normal0);
  s += ",\"crossingWrap\":" + jsNumber(m.crossing_wrap);
  s += ",\"thickness\":" + jsNumber(m.thickness);
  s += ",\"clothFriction\":" + jsNumber(m.cloth_friction);
  s += ",\"airDrag\":" + jsNumber(m.air_drag);
  return s + "}";
}

// ------------------------------------------------------------------------------------ yarnField.ts

constexpr int DAMAGE_CUT = 255;
constexpr int DAMAGE_SEPARATED = 254;
constexpr uint16_t SEG_EXISTS = 1, SEG_BROKEN = 2, SEG_INITIAL_DEFECT = 4, SEG_SLIPPED = 8;

int bundleOf(const btd_layer_info& L, int f) { return f == 1 ? L.bundle[0] : L.bundle[1]; }
int spanLength(const btd_layer_info& L, int f) { return f == 1 ? L.bundle[1] : L.bundle[0]; }
double areaOf(int code) { return std::max(0.02, code / 255.0); }
int areaCode(double a) { return std::max(1, std::min(255, static_cast<int>(std::round(a * 255)))); }

// spanCrossing (yarnField.ts:201-204).
int spanCrossing(const btd_layer_info& L, int i, int j, int f, int q, int p) {
  int bu = L.bundle[0], bv = L.bundle[1], K = L.field_k;
  if (f == 1) return L.field_offset + (j * bv + bv / 2 + p) * K + i * bu + q;
  return L.field_offset + (j * bv + q) * K + i * bu + bu / 2 + p;
}

// partSpanYarns (yarnField.ts:422-434).
void partSpanYarns(const btd_layer_info& L, uint8_t* damage, int i, int j, int f, int slipEnd) {
  int P = spanLength(L, f);
  int half = P - P / 2;
  for (int q = 0; q < bundleOf(L, f); ++q) {
    bool ofA = slipEnd != 0;
    for (int p = 0; p < P; ++p) {
      int e = 2 * spanCrossing(L, i, j, f, q, p) + f;
      if (damage[e] >= DAMAGE_SEPARATED) {
        if (slipEnd < 0) ofA = false;
      } else if (ofA != (p < half)) {
        damage[e] = 254;
      }
    }
  }
}

// coupleSpans (yarnField.ts:443-499) over the scene's own span arrays.
int coupleSpans(btd_scene* s) {
  int ruptures = 0;
  for (int l = 0; l < s->n_layers; ++l) {
    const btd_layer_info& L = s->layers[l];
    for (int j = 0; j < L.ny; ++j) {
      for (int i = 0; i < L.nx; ++i) {
        for (int f = 0; f < 2; ++f) {
          if ((f == 0 && i >= L.nx - 1) || (f == 1 && j >= L.ny - 1)) continue;
          int n = L.node_offset + j * L.nx + i;
          int sp = 2 * n + f;
          if (s->seg_flags[sp] & SEG_SLIPPED) {
            partSpanYarns(L, s->field_damage, i, j, f, s->fail_site[sp] < 0.5 ? 0 : 1);
            s->seg_flags[sp] &= static_cast<uint16_t>(~SEG_SLIPPED);
            continue;
          }
          if ((s->seg_flags[sp] & (SEG_EXISTS | SEG_BROKEN)) != SEG_EXISTS) continue;
          int B = bundleOf(L, f), P = spanLength(L, f);
          double sum = 0, site = 0;
          uint32_t mask = 0;
          for (int q = 0; q < B; ++q) {
            int dmax = 0, first = -1;
            double compliance = 0;
            for (int p = 0; p < P; ++p) {
              int c = spanCrossing(L, i, j, f, q, p);
              int d = s->field_damage[2 * c + f];
              if (d > dmax) dmax = d;
              if (d >= DAMAGE_SEPARATED && first < 0) first = p;
              compliance += 1 / areaOf(s->field_area[2 * c + f]);
            }
            sum += (dmax >= DAMAGE_SEPARATED ? 0 : 1 - static_cast<double>(dmax) / DAMAGE_CUT) * (P / compliance);
            if (dmax >= DAMAGE_SEPARATED) {
              mask |= 1u << q;
              site += (first + 0.5) / P;
            }
          }
          s->intact[sp] = sum / B;
          s->cut_mask[sp] = mask;
          uint32_t full = B >= 32 ? 0xffffffffu : ((1u << B) - 1u);
          if (mask == full) {
            double phi = site / B;
            double rest = s->rest_length[sp];
            int b = f == 0 ? n + 1 : n + L.nx;
            s->seg_flags[sp] |= SEG_BROKEN;
            s->fail_site[sp] = static_cast<float>(phi);
            s->tails[4 * n + 2 * f + 1] += rest * phi;
            s->tails[4 * b + 2 * f] += rest * (1 - phi);
            ruptures++;
            partSpanYarns(L, s->field_damage, i, j, f, -1);
          }
        }
      }
    }
  }
  return ruptures;
}

// ------------------------------------------------------------------------------------ scene.ts

constexpr double DRAPE_SEED = 101;
constexpr int MECHANICS_VERSION = 10;
constexpr double FIELD_GRID = 1.0e-3;

void worley(double seed, double x, double y, double* f1o, double* f2o) {
  double ix = std::floor(x), iy = std::floor(y);
  double f1 = 1e9, f2 = 1e9;
  for (int dy = -1; dy <= 1; ++dy) {
    for (int dx = -1; dx <= 1; ++dx) {
      double cx = ix + dx, cy = iy + dy;
      double px = cx + 0.15 + 0.7 * rand01(seed, cx, cy);
      double py = cy + 0.15 + 0.7 * rand01(seed + 17, cx, cy);
      double d = jsHypot2(px - x, py - y);
      if (d < f1) {
        f2 = f1;
        f1 = d;
      } else if (d < f2) {
        f2 = d;
      }
    }
  }
  *f1o = f1;
  *f2o = f2;
}

// wearAt (scene.ts:182-212): [structural, visible].
void wearAt(const btd_wear& w0, double seed, double x, double y, double* structural, double* visible) {
  if (w0.amount <= 0) {
    *structural = 0;
    *visible = 0;
    return;
  }
  double al = jsHypot2(w0.axis[0], w0.axis[1]);
  if (!(al != 0)) al = 1;
  double ax = w0.axis[0] / al, ay = w0.axis[1] / al;
  double dx = x - w0.center[0], dy = y - w0.center[1];
  double a = (dx * ax + dy * ay) / w0.radii[0];
  double b = (-dx * ay + dy * ax) / w0.radii[1];
  double S = w0.feature_scale;
  double warp = 0.32 * fbm(seed + 3, x / (1.4 * S), y / (1.4 * S), 4);
  double r = jsHypot2(a, b) + warp;
  double w = 1 - smoothstep(0.4, 1.1, r);
  double cells = 1;
  if (w0.cell_size > 0) {
    double jx = x + 0.4 * S * fbm(seed + 11, x / S, y / S, 3);
    double jy = y + 0.4 * S * fbm(seed + 12, x / S, y / S, 3);
    double f1, f2;
    worley(seed + 5, jx / w0.cell_size, jy / w0.cell_size, &f1, &f2);
    cells = std::pow(smoothstep(0.03, 0.3, f2 - f1), 0.7);
  }
  w *= (0.82 + 0.18 * fbm(seed + 7, x / (0.3 * S), y / (0.3 * S), 3)) * w0.amount;
  auto clamp = [](double v) { return std::min(1.0, std::max(0.0, v)); };
  *structural = clamp(w * (0.12 + 0.88 * cells));
  *visible = clamp(std::pow(w, 2.2) * (0.35 + 0.65 * cells));
}

void restPlanePoint(const btd_layer_spec& spec, const btd_layer_info& info, double u, double v, double* rx, double* ry) {
  double c = std::cos(spec.angle), s = std::sin(spec.angle);
  double du = u - info.rest_center[0], dv = v - info.rest_center[1];
  *rx = c * du - s * dv;
  *ry = s * du + c * dv;
}

// fillLayer (scene.ts:289-343).
void fillLayer(btd_scene* sc, const btd_layer_spec& spec, const btd_layer_info& info) {
  const btd_material& m = info.material;
  int nx = info.nx, ny = info.ny;
  double mass = crossingMass(m);
  int cr = spec.collar_rows;
  for (int j = 0; j < ny; ++j) {
    for (int i = 0; i < nx; ++i) {
      int n = info.node_offset + j * nx + i;
      double u = i * m.pitch_u, v = j * m.pitch_v;
      sc->rest_uv[2 * n] = u;
      sc->rest_uv[2 * n + 1] = v;
      double du = u - info.rest_center[0], dv = v - info.rest_center[1];
      double px = info.map_origin[0] + info.map_a[0] * du + info.map_a[1] * dv;
      double py = info.map_origin[1] + info.map_a[2] * du + info.map_a[3] * dv;
      bool pinned = i < cr || j < cr || i >= nx - cr || j >= ny - cr;
      double fadeIn = 1 - smoothstep(0.16, 0.24, jsHypot2(px, py));
      double pz = pinned ? 0 : spec.perturbation * fadeIn * fbm(DRAPE_SEED, px / 0.04, py / 0.04, 3);
      sc->position[3 * n] = px;
      sc->position[3 * n + 1] = py;
      sc->position[3 * n + 2] = info.map_origin[2] + pz;
      sc->mass[n] = mass;
      sc->pinned[n] = pinned ? 1 : 0;
      double rx, ry, w, wv;
      restPlanePoint(spec, info, u, v, &rx, &ry);
      wearAt(spec.wear, spec.seed, rx, ry, &w, &wv);
      sc->wear[n] = static_cast<float>(wv);
      sc->structural_wear[n] = static_cast<float>(w);
      sc->crossing_normal0[n] = m.crossing_normal0 * (1 - 0.7 * w);
      for (int f = 0; f < 2; ++f) {
        int s = 2 * n + f;
        bool exists = f == 0 ? i < nx - 1 : j < ny - 1;
        if (!exists) continue;
        sc->seg_flags[s] = SEG_EXISTS;
        sc->rest_length[s] = f == 0 ? m.pitch_u : m.pitch_v;
        sc->intact[s] = 1;
        sc->softening[s] = m.yarns[f].softening_opening;
        sc->fail_site[s] = 0.5f;
      }
    }
  }
}

// fillField (scene.ts:355-428).
void fillField(btd_scene* sc, const btd_layer_spec& spec, const btd_layer_info& info) {
  const btd_material& weave = info.weave;
  double seed = spec.seed;
  double pu = weave.pitch_u, pv = weave.pitch_v;
  int bu = info.bundle[0], bv = info.bundle[1], K = info.field_k, M = info.field_m;
  double u0 = -bu * pu, v0 = -bv * pv;
  int gw = static_cast<int>(std::ceil((K + 2 * bu) * pu / FIELD_GRID)) + 2;
  int gh = static_cast<int>(std::ceil((M + 2 * bv) * pv / FIELD_GRID)) + 2;
  std::vector<float> gWear(static_cast<size_t>(gw) * gh), gCorr(gWear.size()), gEdge(gWear.size());
  for (int y = 0; y < gh; ++y) {
    for (int x = 0; x < gw; ++x) {
      double rx, ry, w, wv;
      restPlanePoint(spec, info, u0 + x * FIELD_GRID, v0 + y * FIELD_GRID, &rx, &ry);
      wearAt(spec.wear, seed, rx, ry, &w, &wv);
      size_t g = static_cast<size_t>(y) * gw + x;
      gWear[g] = static_cast<float>(w);
      gCorr[g] = static_cast<float>(fbm(seed + 503, rx / 0.011, ry / 0.011, 3));
      gEdge[g] = static_cast<float>(fbm(seed + 991, rx / 0.004, ry / 0.004, 2));
    }
  }
  auto sample = [&](const std::vector<float>& g, double u, double v) {
    double fx = std::min(gw - 1.001, std::max(0.0, (u - u0) / FIELD_GRID));
    double fy = std::min(gh - 1.001, std::max(0.0, (v - v0) / FIELD_GRID));
    int x = static_cast<int>(std::floor(fx)), y = static_cast<int>(std::floor(fy));
    double tx = fx - x, ty = fy - y;
    double g00 = g[static_cast<size_t>(y) * gw + x], g10 = g[static_cast<size_t>(y) * gw + x + 1];
    double g01 = g[static_cast<size_t>(y + 1) * gw + x], g11 = g[static_cast<size_t>(y + 1) * gw + x + 1];
    double a = g00 + (g10 - g00) * tx;
    double b = g01 + (g11 - g01) * tx;
    return a + (b - a) * ty;
  };
  double thr = spec.wear.defect_threshold;
  int R = weave.twill_repeat;
  for (int mm = 0; mm < M; ++mm) {
    double v = (mm - (bv - 1) / 2.0) * pv;
    for (int k = 0; k < K; ++k) {
      double u = (k - (bu - 1) / 2.0) * pu;
      int c = info.field_offset + mm * K + k;
      double w = sample(gWear, u, v);
      double corr = sample(gCorr, u, v);
      for (int f = 0; f < 2; ++f) {
        double loss = spec.wear_strength_loss[f];
        double wf = f == 0 ? std::pow(w, 1.3) : std::pow(w, 1.25);
        int yarnIndex = f == 1 ? k : mm;
        double along = f == 1 ? v : u;
        double slub = 1 + 0.25 * noise1(seed + 4099 + 13 * yarnIndex + 7 * f, along / 0.0025);
        double z = (rand01(seed + 503, c, f) + rand01(seed + 617, c, f) - 1) * 2.45;
        double scatter = std::exp((0.2 + 0.12 * w) * corr + (0.06 + 0.22 * w) * z);
        double area = std::max(0.02, 1 - loss * wf);
        sc->field_area[2 * c + f] = static_cast<uint8_t>(areaCode(area));
        sc->field_strength[2 * c + f] = static_cast<float>(weave.yarns[f].strength * std::max(0.005, area * scatter * slub));
      }
      double edge = thr + 0.04 * sample(gEdge, u, v) + 0.012 * (rand01(seed + 990, k) - 0.5);
      if (w > edge && rand01(seed + 991, k, mm) < spec.wear.defect_density) sc->field_damage[2 * c + 1] = DAMAGE_CUT;
      double flt = std::floor((mm - (k % R) + 4.0 * R) / R);
      double pf = 0.02 * std::pow(smoothstep(spec.wear.sparse_from, thr, w), 2);
      bool onFace = (((mm - k) % R) + R) % R < weave.twill_warp_over;
      if (pf > 0 && onFace && rand01(seed + 997, k, flt) < pf) sc->field_damage[2 * c + 1] = DAMAGE_CUT;
    }
  }
}

template <class T>
T* alloc(size_t n) {
  T* p = static_cast<T*>(std::calloc(n ? n : 1, sizeof(T)));
  if (!p) throw std::bad_alloc();
  return p;
}

}  // namespace

extern "C" {

int btd_material_preset(int32_t index, btd_material* out) {
  if (!out || index < 0 || index > 1) {
    btd::setError("btd_material_preset: index must be 0 (DENIM) or 1 (BACKING)");
    return BTD_E_INVALID;
  }
  *out = preset(index);
  return BTD_OK;
}

int btd_bundle_weave(const btd_material* m, int32_t bu, int32_t bv, btd_material* out) {
  if (!m || !out || bu < 1 || bv < 1) {
    btd::setError("bundle factors must be positive integers");
    return BTD_E_INVALID;
  }
  *out = bundleWeave(*m, bu, bv);
  return BTD_OK;
}

int btd_default_scene_spec(btd_layer_spec* out) {
  if (!out) return BTD_E_INVALID;
  btd_layer_spec s{};
  s.material = preset(0);
  s.bundle[0] = 9;
  s.bundle[1] = 6;
  s.size_u = 0.62;
  s.size_v = 0.4;
  s.z = 0;
  s.angle = 0.06;
  s.compress_u = 0.025;
  s.compress_v = -0.002;
  s.shear = 0.06;
  s.collar_rows = 2;
  s.wear.center[0] = 0.01;
  s.wear.center[1] = -0.006;
  s.wear.axis[0] = 1;
  s.wear.axis[1] = -1.15;
  s.wear.radii[0] = 0.2;
  s.wear.radii[1] = 0.14;
  s.wear.amount = 1;
  s.wear.cell_size = 0.075;
  s.wear.feature_scale = 0.05;
  s.wear.defect_threshold = 0.89;
  s.wear.defect_density = 1;
  s.wear.sparse_from = 0.6;
  s.wear_strength_loss[0] = 0.45;
  s.wear_strength_loss[1] = 0.9;
  s.seed = 1001;
  s.perturbation = 2.5e-3;
  *out = s;
  return BTD_OK;
}

int btd_scene_compile(const btd_layer_spec* specs, int32_t n_specs, btd_scene** out) {
  if (!specs || n_specs < 1 || !out) {
    btd::setError("btd_scene_compile: need at least one layer spec");
    return BTD_E_INVALID;
  }
  btd_scene* sc = nullptr;
  try {
    sc = alloc<btd_scene>(1);
    sc->n_layers = n_specs;
    sc->layers = alloc<btd_layer_info>(n_specs);
    long long offset = 0, foffset = 0;
    for (int l = 0; l < n_specs; ++l) {
      const btd_layer_spec& spec = specs[l];
      int bu = spec.bundle[0] > 0 ? spec.bundle[0] : 1;
      int bv = spec.bundle[1] > 0 ? spec.bundle[1] : 1;
      if (bu > 32 || bv > 32) throw std::runtime_error("bundle too large for the cut masks");
      btd_layer_info& L = sc->layers[l];
      L.index = l;
      L.bundle[0] = bu;
      L.bundle[1] = bv;
      L.weave = spec.material;
      L.material = bundleWeave(spec.material, bu, bv);
      L.nx = static_cast<int>(std::floor(spec.size_u / L.material.pitch_u)) + 1;
      L.ny = static_cast<int>(std::floor(spec.size_v / L.material.pitch_v)) + 1;
      if (L.nx < 2 || L.ny < 2 || L.nx > 65535 || L.ny > 65535) throw std::runtime_error("lattice extent out of range");
      double c = std::cos(spec.angle), s = std::sin(spec.angle);
      double k00 = 1 - spec.compress_u, k01 = spec.shear, k11 = 1 - spec.compress_v;
      L.map_a[0] = c * k00;
      L.map_a[1] = c * k01 - s * k11;
      L.map_a[2] = s * k00;
      L.map_a[3] = s * k01 + c * k11;
      L.rest_center[0] = ((L.nx - 1) * L.material.pitch_u) / 2;
      L.rest_center[1] = ((L.ny - 1) * L.material.pitch_v) / 2;
      L.map_origin[0] = 0;
      L.map_origin[1] = 0;
      L.map_origin[2] = spec.z;
      L.node_offset = static_cast<int>(offset);
      L.node_count = L.nx * L.ny;
      L.field_offset = static_cast<int>(foffset);
      L.field_k = L.nx * bu;
      L.field_m = L.ny * bv;
      offset += L.node_count;
      foffset += static_cast<long long>(L.field_k) * L.field_m;
      if (offset > (1LL << 30) || foffset > (1LL << 30)) throw std::runtime_error("scene too large");
    }
    int N = static_cast<int>(offset);
    int C = static_cast<int>(foffset);
    sc->node_count = N;
    sc->crossing_count = C;
    sc->rest_uv = alloc<double>(2 * size_t(N));
    sc->position = alloc<double>(3 * size_t(N));
    sc->mass = alloc<double>(N);
    sc->pinned = alloc<uint8_t>(N);
    sc->wear = alloc<float>(N);
    sc->structural_wear = alloc<float>(N);
    sc->rest_length = alloc<double>(2 * size_t(N));
    sc->softening = alloc<double>(2 * size_t(N));
    sc->seg_flags = alloc<uint16_t>(2 * size_t(N));
    sc->intact = alloc<double>(2 * size_t(N));
    sc->cut_mask = alloc<uint32_t>(2 * size_t(N));
    sc->fail_site = alloc<float>(2 * size_t(N));
    sc->field_strength = alloc<float>(2 * size_t(C));
    sc->field_damage = alloc<uint8_t>(2 * size_t(C));
    sc->field_area = alloc<uint8_t>(2 * size_t(C));
    std::memset(sc->field_area, 255, 2 * size_t(C));
    sc->crossing_normal0 = alloc<double>(N);
    sc->tails = alloc<double>(4 * size_t(N));
    for (int l = 0; l < n_specs; ++l) {
      fillLayer(sc, specs[l], sc->layers[l]);
      fillField(sc, specs[l], sc->layers[l]);
    }
    std::vector<uint16_t> before(sc->seg_flags, sc->seg_flags + 2 * size_t(N));
    coupleSpans(sc);
    for (size_t q = 0; q < 2 * size_t(N); ++q)
      if ((sc->seg_flags[q] & SEG_BROKEN) && !(before[q] & SEG_BROKEN)) sc->seg_flags[q] |= SEG_INITIAL_DEFECT;
    *out = sc;
    return BTD_OK;
  } catch (const std::exception& e) {
    btd_scene_free(sc);
    btd::setError(std::string("btd_scene_compile: ") + e.what());
    return BTD_E_INVALID;
  }
}

int btd_scene_free(btd_scene* sc) {
  if (!sc) return BTD_OK;
  std::free(sc->layers);
  std::free(sc->rest_uv);
  std::free(sc->position);
  std::free(sc->mass);
  std::free(sc->pinned);
  std::free(sc->wear);
  std::free(sc->structural_wear);
  std::free(sc->rest_length);
  std::free(sc->softening);
  std::free(sc->seg_flags);
  std::free(sc->intact);
  std::free(sc->cut_mask);
  std::free(sc->fail_site);
  std::free(sc->field_strength);
  std::free(sc->field_damage);
  std::free(sc->field_area);
  std::free(sc->crossing_normal0);
  std::free(sc->tails);
  std::free(sc);
  return BTD_OK;
}

int btd_scene_hash(const btd_scene* s, uint32_t* out) {
  if (!s || !out) return BTD_E_INVALID;
  uint32_t h = 0x811c9dc5u;
  auto mix = [&](uint32_t v) { h = (h ^ v) * 0x01000193u; };
  mix(MECHANICS_VERSION);
  for (int l = 0; l < s->n_layers; ++l) {
    std::string json = materialJson(s->layers[l].material);
    for (unsigned char ch : json) mix(ch);
  }
  size_t nd = 2 * size_t(s->crossing_count);
  for (size_t i = 0; i < nd; i += 64)
    h = (h ^ s->field_damage[i] ^ (uint32_t(s->field_area[i]) << 16) ^ (uint32_t(i) << 8)) * 0x01000193u;
  for (size_t i = 0; i < 3 * size_t(s->node_count); ++i) {
    float f = static_cast<float>(s->position[i]);
    uint32_t u;
    std::memcpy(&u, &f, 4);
    h = (h ^ u) * 0x01000193u;
  }
  for (size_t i = 0; i < 2 * size_t(s->node_count); ++i) h = (h ^ s->seg_flags[i]) * 0x01000193u;
  *out = h;
  return BTD_OK;
}

}  // extern "C"
