// Oracle (test infrastructure only): collision primitives, CPU BVH broadphase
// and the ContactSystem, restated from src/collision/*.ts of the reference.
#include <algorithm>
#include <array>

#include "orc.hpp"
#include "jsmath.hpp"

namespace orc {

// src/collision/closest-point.ts:14-62 (Ericson 5.1.5, barycentric s on b, t on c).
Closest closest_vt(double px, double py, double pz, double ax, double ay, double az,
                   double bx, double by, double bz, double cx, double cy, double cz) {
  auto pack = [](double s, double t, double rx, double ry, double rz) {
    return Closest{s, t, js_hypot3(rx, ry, rz), rx, ry, rz};
  };
  const double abx = bx - ax, aby = by - ay, abz = bz - az;
  const double acx = cx - ax, acy = cy - ay, acz = cz - az;
  const double apx = px - ax, apy = py - ay, apz = pz - az;
  const double d1 = abx * apx + aby * apy + abz * apz;
  const double d2 = acx * apx + acy * apy + acz * apz;
  if (d1 <= 0 && d2 <= 0) return pack(0, 0, px - ax, py - ay, pz - az);
  const double bpx = px - bx, bpy = py - by, bpz = pz - bz;
  const double d3 = abx * bpx + aby * bpy + abz * bpz;
  const double d4 = acx * bpx + acy * bpy + acz * bpz;
  if (d3 >= 0 && d4 <= d3) return pack(1, 0, px - bx, py - by, pz - bz);
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0 && d1 >= 0 && d3 <= 0) {
    const double v = d1 / (d1 - d3);
    return pack(v, 0, px - (ax + v * abx), py - (ay + v * aby), pz - (az + v * abz));
  }
  const double cpx = px - cx, cpy = py - cy, cpz = pz - cz;
  const double d5 = abx * cpx + aby * cpy + abz * cpz;
  const double d6 = acx * cpx + acy * cpy + acz * cpz;
  if (d6 >= 0 && d5 <= d6) return pack(0, 1, px - cx, py - cy, pz - cz);
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) {
    const double w = d2 / (d2 - d6);
    return pack(0, w, px - (ax + w * acx), py - (ay + w * acy), pz - (az + w * acz));
  }
  const double va = d3 * d6 - d5 * d4;
  if (va <= 0 && d4 - d3 >= 0 && d5 - d6 >= 0) {
    const double w = (d4 - d3) / (d4 - d3 + (d5 - d6));
    const double qx = bx + w * (cx - bx), qy = by + w * (cy - by), qz = bz + w * (cz - bz);
    return pack(1 - w, w, px - qx, py - qy, pz - qz);
  }
  const double denom = 1 / (va + vb + vc);
  const double v = vb * denom;
  const double w = vc * denom;
  const double qx = ax + abx * v + acx * w;
  const double qy = ay + aby * v + acy * w;
  const double qz = az + abz * v + acz * w;
  return pack(v, w, px - qx, py - qy, pz - qz);
}

static inline double clamp01(double v, double lo, double hi) { return v < lo ? lo : v > hi ? hi : v; }

// src/collision/closest-point.ts:73-108 (Ericson 5.1.9 segment-segment).
Closest closest_ee(double ax, double ay, double az, double bx, double by, double bz,
                   double cx, double cy, double cz, double dx, double dy, double dz) {
  const double d1x = bx - ax, d1y = by - ay, d1z = bz - az;
  const double d2x = dx - cx, d2y = dy - cy, d2z = dz - cz;
  const double rx = ax - cx, ry = ay - cy, rz = az - cz;
  const double a = d1x * d1x + d1y * d1y + d1z * d1z;
  const double e = d2x * d2x + d2y * d2y + d2z * d2z;
  const double f = d2x * rx + d2y * ry + d2z * rz;
  double s, t;
  if (a <= 1e-30 && e <= 1e-30) {
    s = 0; t = 0;
  } else if (a <= 1e-30) {
    s = 0; t = clamp01(f / e, 0, 1);
  } else {
    const double c = d1x * rx + d1y * ry + d1z * rz;
    if (e <= 1e-30) {
      t = 0; s = clamp01(-c / a, 0, 1);
    } else {
      const double b = d1x * d2x + d1y * d2y + d1z * d2z;
      const double denom = a * e - b * b;
      s = denom > 1e-30 ? clamp01((b * f - c * e) / denom, 0, 1) : 0;
      t = (b * s + f) / e;
      if (t < 0) { t = 0; s = clamp01(-c / a, 0, 1); }
      else if (t > 1) { t = 1; s = clamp01((b - c) / a, 0, 1); }
    }
  }
  const double axp = ax + d1x * s, ayp = ay + d1y * s, azp = az + d1z * s;
  const double cxp = cx + d2x * t, cyp = cy + d2y * t, czp = cz + d2z * t;
  const double rx2 = axp - cxp, ry2 = ayp - cyp, rz2 = azp - czp;
  return Closest{s, t, js_hypot3(rx2, ry2, rz2), rx2, ry2, rz2};
}

// src/collision/cubic.ts:53-66 solveQuadratic01.
static std::vector<double> solve_quadratic01(double a2, double a1, double a0) {
  const double eps = 1e-12;
  std::vector<double> out;
  if (std::fabs(a2) < eps) {
    if (std::fabs(a1) < eps) return out;
    const double r = -a0 / a1;
    if (r >= 0 && r <= 1) out.push_back(r);
    return out;
  }
  const double disc = a1 * a1 - 4 * a2 * a0;
  if (disc < 0) return out;
  const double sd = std::sqrt(disc);
  const double rs[2] = {(-a1 - sd) / (2 * a2), (-a1 + sd) / (2 * a2)};
  for (double r : rs) if (r >= 0 && r <= 1) out.push_back(r);
  std::sort(out.begin(), out.end());
  return out;
}

// src/collision/cubic.ts:4-49 solveCubic01 (Cardano / trigonometric roots,
// 4 Newton polish steps, filtered to [0,1], sorted, deduplicated).
std::vector<double> solve_cubic01(double a3, double a2, double a1, double a0) {
  const double eps = 1e-12;
  if (std::fabs(a3) < eps) return solve_quadratic01(a2, a1, a0);
  const double A = a2 / a3, B = a1 / a3, C = a0 / a3;
  const double sqA = A * A;
  const double p = (3 * B - sqA) / 3;
  const double q = (2 * sqA * A - 9 * A * B + 27 * C) / 27;
  std::vector<double> roots;
  const double disc = (q * q) / 4 + (p * p * p) / 27;
  const double shift = A / 3;
  if (disc > eps) {
    const double sd = std::sqrt(disc);
    const double u = js_cbrt(-q / 2 + sd);
    const double v = js_cbrt(-q / 2 - sd);
    roots.push_back(u + v - shift);
  } else if (std::fabs(disc) <= eps) {
    const double u = js_cbrt(-q / 2);
    roots.push_back(2 * u - shift);
    roots.push_back(-u - shift);
  } else {
    const double r = std::sqrt(-(p * p * p) / 27);
    const double phi = js_acos(js_min(1, js_max(-1, -q / (2 * r))));
    const double s = 2 * js_cbrt(r);
    const double PI = 3.141592653589793;
    roots.push_back(s * std::cos(phi / 3) - shift);
    roots.push_back(s * std::cos((phi + 2 * PI) / 3) - shift);
    roots.push_back(s * std::cos((phi + 4 * PI) / 3) - shift);
  }
  std::vector<double> out;
  for (double r : roots) {
    if (!std::isfinite(r)) continue;
    for (int k = 0; k < 4; k++) {
      const double f = ((a3 * r + a2) * r + a1) * r + a0;
      const double df = (3 * a3 * r + 2 * a2) * r + a1;
      if (std::fabs(df) < 1e-18) break;
      r -= f / df;
    }
    if (r >= -1e-9 && r <= 1 + 1e-9) out.push_back(js_min(1, js_max(0, r)));
  }
  std::sort(out.begin(), out.end());
  std::vector<double> kept;
  for (size_t i = 0; i < out.size(); i++)
    if (i == 0 || out[i] - out[i - 1] > 1e-9) kept.push_back(out[i]);
  return kept;
}

static inline void cross3(double* o, const double* u, const double* v) {
  o[0] = u[1] * v[2] - u[2] * v[1];
  o[1] = u[2] * v[0] - u[0] * v[2];
  o[2] = u[0] * v[1] - u[1] * v[0];
}
static inline double dot3(const double* u, const double* v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; }

// Relative-motion early-out shared by both CCD tests (ccd-vt.ts:33-51).
static double stencil_dev(const double* P0, const double* P1) {
  double mx = 0, my = 0, mz = 0;
  for (int v = 0; v < 4; v++) {
    mx += P1[v * 3] - P0[v * 3];
    my += P1[v * 3 + 1] - P0[v * 3 + 1];
    mz += P1[v * 3 + 2] - P0[v * 3 + 2];
  }
  mx /= 4; my /= 4; mz /= 4;
  double dev = 0;
  for (int v = 0; v < 4; v++) {
    const double dx = P1[v * 3] - P0[v * 3] - mx;
    const double dy = P1[v * 3 + 1] - P0[v * 3 + 1] - my;
    const double dz = P1[v * 3 + 2] - P0[v * 3 + 2] - mz;
    const double m = js_max(js_max(std::fabs(dx), std::fabs(dy)), std::fabs(dz));
    if (m > dev) dev = m;
  }
  return dev;
}

// src/collision/ccd-vt.ts:20-115 vtCCD. Stencil order in P: p, a, b, c.
double vt_ccd(const double* P0, const double* P1, double thickness) {
  const double* p0 = P0; const double* a0 = P0 + 3; const double* b0 = P0 + 6; const double* c0 = P0 + 9;
  const double d0 = closest_vt(p0[0], p0[1], p0[2], a0[0], a0[1], a0[2], b0[0], b0[1], b0[2],
                               c0[0], c0[1], c0[2]).dist;
  if (d0 <= thickness) return 0;
  const double dev = stencil_dev(P0, P1);
  if (d0 - 4 * dev > thickness) return INF;
  double dp[3], da[3], db[3], dc[3];
  for (int i = 0; i < 3; i++) {
    dp[i] = P1[i] - P0[i]; da[i] = P1[3 + i] - P0[3 + i];
    db[i] = P1[6 + i] - P0[6 + i]; dc[i] = P1[9 + i] - P0[9 + i];
  }
  double u0[3], du[3], v0[3], dv[3], w0[3], dw[3];
  for (int i = 0; i < 3; i++) {
    u0[i] = p0[i] - a0[i]; du[i] = dp[i] - da[i];
    v0[i] = b0[i] - a0[i]; dv[i] = db[i] - da[i];
    w0[i] = c0[i] - a0[i]; dw[i] = dc[i] - da[i];
  }
  double n0[3], n1[3], n2[3], t1[3], t2[3];
  cross3(n0, v0, w0);
  cross3(t1, v0, dw); cross3(t2, dv, w0);
  for (int i = 0; i < 3; i++) n1[i] = t1[i] + t2[i];
  cross3(n2, dv, dw);
  const double c0c = dot3(u0, n0);
  const double c1c = dot3(u0, n1) + dot3(du, n0);
  const double c2c = dot3(u0, n2) + dot3(du, n1);
  const double c3c = dot3(du, n2);
  auto dist_at = [&](double t) {
    double pp[3], aa[3], bb[3], cc[3];
    for (int i = 0; i < 3; i++) {
      pp[i] = p0[i] + dp[i] * t; aa[i] = a0[i] + da[i] * t;
      bb[i] = b0[i] + db[i] * t; cc[i] = c0[i] + dc[i] * t;
    }
    return closest_vt(pp[0], pp[1], pp[2], aa[0], aa[1], aa[2], bb[0], bb[1], bb[2], cc[0], cc[1], cc[2]).dist;
  };
  for (double t : solve_cubic01(c3c, c2c, c1c, c0c))
    if (dist_at(t) <= thickness) return t;
  double minD = INF, minT = 0;
  const int N = 16;
  for (int k = 0; k <= N; k++) {
    const double t = (double)k / N;
    const double d = dist_at(t);
    if (d < minD) { minD = d; minT = t; }
  }
  if (minD <= thickness) return minT;
  return INF;
}

// src/collision/ccd-ee.ts:24-101 eeCCD. Stencil order in P: a, b, c, d.
double ee_ccd(const double* P0, const double* P1, double thickness) {
  const double* a0 = P0; const double* b0 = P0 + 3; const double* c0 = P0 + 6; const double* d0 = P0 + 9;
  double da[3], db[3], dc[3], dd[3];
  for (int i = 0; i < 3; i++) {
    da[i] = P1[i] - P0[i]; db[i] = P1[3 + i] - P0[3 + i];
    dc[i] = P1[6 + i] - P0[6 + i]; dd[i] = P1[9 + i] - P0[9 + i];
  }
  auto q = [&](double t) {
    double A[3], B[3], C[3], Dd[3];
    for (int i = 0; i < 3; i++) {
      A[i] = a0[i] + da[i] * t; B[i] = b0[i] + db[i] * t;
      C[i] = c0[i] + dc[i] * t; Dd[i] = d0[i] + dd[i] * t;
    }
    return closest_ee(A[0], A[1], A[2], B[0], B[1], B[2], C[0], C[1], C[2], Dd[0], Dd[1], Dd[2]);
  };
  const double q0 = q(0).dist;
  if (q0 <= thickness) return 0;
  const double dev = stencil_dev(P0, P1);
  if (q0 - 4 * dev > thickness) return INF;
  double e10[3], de1[3], e20[3], de2[3], r0[3], dr[3];
  for (int i = 0; i < 3; i++) {
    e10[i] = b0[i] - a0[i]; de1[i] = db[i] - da[i];
    e20[i] = d0[i] - c0[i]; de2[i] = dd[i] - dc[i];
    r0[i] = c0[i] - a0[i]; dr[i] = dc[i] - da[i];
  }
  double n0[3], n1[3], n2[3], t1[3], t2[3];
  cross3(n0, e10, e20);
  cross3(t1, e10, de2); cross3(t2, de1, e20);
  for (int i = 0; i < 3; i++) n1[i] = t1[i] + t2[i];
  cross3(n2, de1, de2);
  const double c0c = dot3(r0, n0);
  const double c1c = dot3(r0, n1) + dot3(dr, n0);
  const double c2c = dot3(r0, n2) + dot3(dr, n1);
  const double c3c = dot3(dr, n2);
  for (double t : solve_cubic01(c3c, c2c, c1c, c0c)) {
    const Closest cp = q(t);
    if (cp.dist <= thickness && cp.s >= -1e-6 && cp.s <= 1 + 1e-6 && cp.t >= -1e-6 && cp.t <= 1 + 1e-6)
      return t;
  }
  double minD = INF, minT = 0;
  const int N = 16;
  for (int k = 0; k <= N; k++) {
    const double t = (double)k / N;
    const double d = q(t).dist;
    if (d < minD) { minD = d; minT = t; }
  }
  if (minD <= thickness) return minT;
  return INF;
}

// src/collision/barrier.ts:4-24.
double barrier_value(double d, double dHat) {
  if (d >= dHat) return 0;
  const double dc = js_max(d, 1e-12);
  const double t = dc - dHat;
  return -t * t * js_log(dc / dHat);
}
double barrier_grad_scalar(double d, double dHat, double kappa, double w) {
  if (d >= dHat) return 0;
  const double dc = js_max(d, 1e-12);
  const double t = dc - dHat;
  const double db = -2 * t * js_log(dc / dHat) - (t * t) / dc;
  return kappa * w * db;
}
double barrier_normal_force(double d, double dHat, double kappa, double w) {
  return js_max(0, -barrier_grad_scalar(d, dHat, kappa, w));
}

// src/collision/friction.ts:14-23 coulombForce (lagged, regularized).
void coulomb_force(double ux, double uy, double uz, double nx, double ny, double nz,
                   double lambdaN, double mu, double eps, double f[3]) {
  const double vn = ux * nx + uy * ny + uz * nz;
  const double tx = ux - vn * nx, ty = uy - vn * ny, tz = uz - vn * nz;
  const double mag = std::sqrt(tx * tx + ty * ty + tz * tz + eps * eps);
  const double s = (mu * js_max(0, lambdaN)) / mag;
  f[0] = -s * tx; f[1] = -s * ty; f[2] = -s * tz;
}

// ---- CPU BVH (src/collision/bvh.ts, aabb.ts) --------------------------------

static Aabb swept_tri_aabb(const double* x0, const double* x1, int i0, int i1, int i2, double pad) {
  double minX = INF, minY = INF, minZ = INF, maxX = -INF, maxY = -INF, maxZ = -INF;
  const int ids[3] = {i0, i1, i2};
  for (int v : ids) {
    const double* xs[2] = {x0, x1};
    for (const double* x : xs) {
      const double px = x[v * 3], py = x[v * 3 + 1], pz = x[v * 3 + 2];
      if (px < minX) minX = px;
      if (py < minY) minY = py;
      if (pz < minZ) minZ = pz;
      if (px > maxX) maxX = px;
      if (py > maxY) maxY = py;
      if (pz > maxZ) maxZ = pz;
    }
  }
  return Aabb{minX - pad, minY - pad, minZ - pad, maxX + pad, maxY + pad, maxZ + pad};
}

void TriBvh::build(const double* x0, const double* x1, const uint32_t* idx, int triCount, double pad) {
  std::vector<Aabb> boxes(triCount);
  Vec cx(triCount), cy(triCount), cz(triCount);
  for (int t = 0; t < triCount; t++) {
    const int i0 = idx[t * 3], i1 = idx[t * 3 + 1], i2 = idx[t * 3 + 2];
    boxes[t] = swept_tri_aabb(x0, x1, i0, i1, i2, pad);
    cx[t] = (x0[i0 * 3] + x0[i1 * 3] + x0[i2 * 3] + x1[i0 * 3] + x1[i1 * 3] + x1[i2 * 3]) / 6;
    cy[t] = (x0[i0 * 3 + 1] + x0[i1 * 3 + 1] + x0[i2 * 3 + 1] + x1[i0 * 3 + 1] + x1[i1 * 3 + 1] + x1[i2 * 3 + 1]) / 6;
    cz[t] = (x0[i0 * 3 + 2] + x0[i1 * 3 + 2] + x0[i2 * 3 + 2] + x1[i0 * 3 + 2] + x1[i1 * 3 + 2] + x1[i2 * 3 + 2]) / 6;
  }
  nodes.clear();
  if (triCount == 0) { root = -1; return; }
  std::vector<int> order(triCount);
  for (int i = 0; i < triCount; i++) order[i] = i;
  root = build_rec(order, boxes, cx, cy, cz);
}

int TriBvh::build_rec(std::vector<int>& order, const std::vector<Aabb>& boxes, const Vec& cx,
                      const Vec& cy, const Vec& cz) {
  if (order.size() == 1) {
    const int id = (int)nodes.size();
    nodes.push_back({boxes[order[0]], -1, -1, order[0]});
    return id;
  }
  double minX = INF, maxX = -INF, minY = INF, maxY = -INF, minZ = INF, maxZ = -INF;
  for (int t : order) {
    if (cx[t] < minX) minX = cx[t];
    if (cx[t] > maxX) maxX = cx[t];
    if (cy[t] < minY) minY = cy[t];
    if (cy[t] > maxY) maxY = cy[t];
    if (cz[t] < minZ) minZ = cz[t];
    if (cz[t] > maxZ) maxZ = cz[t];
  }
  const double sx = maxX - minX, sy = maxY - minY, sz = maxZ - minZ;
  const int axis = sx >= sy && sx >= sz ? 0 : sy >= sz ? 1 : 2;
  const Vec& key = axis == 0 ? cx : axis == 1 ? cy : cz;
  std::sort(order.begin(), order.end(), [&](int p, int q) {
    return key[p] != key[q] ? key[p] < key[q] : p < q;
  });
  const size_t mid = std::max<size_t>(1, order.size() / 2);
  std::vector<int> lo(order.begin(), order.begin() + mid), hi(order.begin() + mid, order.end());
  const int left = build_rec(lo, boxes, cx, cy, cz);
  const int right = build_rec(hi, boxes, cx, cy, cz);
  const Aabb a = nodes[left].box, b = nodes[right].box;
  const int id = (int)nodes.size();
  nodes.push_back({Aabb{js_min(a.minX, b.minX), js_min(a.minY, b.minY), js_min(a.minZ, b.minZ),
                        js_max(a.maxX, b.maxX), js_max(a.maxY, b.maxY), js_max(a.maxZ, b.maxZ)},
                   left, right, -1});
  return id;
}

static inline int64_t tri_pair_key(int a, int b) {
  return (int64_t)std::min(a, b) * 1000003 + std::max(a, b);
}

std::vector<std::pair<int, int>> TriBvh::self_pairs(const std::vector<int64_t>& excl) const {
  std::vector<std::pair<int, int>> out;
  if (root < 0) return out;
  std::vector<std::pair<int, int>> stack{{root, root}};
  while (!stack.empty()) {
    auto [na, nb] = stack.back();
    stack.pop_back();
    const BvhNode& A = nodes[na];
    const BvhNode& B = nodes[nb];
    if (!overlaps(A.box, B.box)) continue;
    const bool leafA = A.tri >= 0, leafB = B.tri >= 0;
    if (leafA && leafB) {
      const int a = A.tri, b = B.tri;
      if (a == b) continue;
      const int tA = std::min(a, b), tB = std::max(a, b);
      if (std::binary_search(excl.begin(), excl.end(), tri_pair_key(tA, tB))) continue;
      out.push_back({tA, tB});
      continue;
    }
    if (na == nb) {
      stack.push_back({A.left, A.left});
      stack.push_back({A.left, A.right});
      stack.push_back({A.right, A.right});
    } else if (leafA) {
      stack.push_back({na, B.left});
      stack.push_back({na, B.right});
    } else if (leafB) {
      stack.push_back({A.left, nb});
      stack.push_back({A.right, nb});
    } else {
      stack.push_back({A.left, B.left});
      stack.push_back({A.left, B.right});
      stack.push_back({A.right, B.left});
      stack.push_back({A.right, B.right});
    }
  }
  std::sort(out.begin(), out.end());
  return out;
}

// src/collision/bvh.ts:133-151: pairs of triangles sharing a vertex, keyed
// min*1000003+max (sorted for binary search).
std::vector<int64_t> adjacency_exclusions(const uint32_t* idx, int triCount) {
  std::unordered_map<uint32_t, std::vector<int>> v2t;
  std::vector<uint32_t> order;
  for (int t = 0; t < triCount; t++)
    for (int k = 0; k < 3; k++) {
      uint32_t v = idx[t * 3 + k];
      auto it = v2t.find(v);
      if (it == v2t.end()) { order.push_back(v); v2t[v] = {t}; }
      else it->second.push_back(t);
    }
  std::vector<int64_t> ex;
  for (uint32_t v : order) {
    const auto& list = v2t[v];
    for (size_t i = 0; i < list.size(); i++)
      for (size_t j = i + 1; j < list.size(); j++) ex.push_back(tri_pair_key(list[i], list[j]));
  }
  std::sort(ex.begin(), ex.end());
  ex.erase(std::unique(ex.begin(), ex.end()), ex.end());
  return ex;
}

// ---- ContactSystem -------------------------------------------------------

// Lagged-map identity of a frozen contact (contact-assembly.ts:607-616): VT =
// vertex + sorted triangle ids; EE = unordered pair of unordered edges; floor = vertex.
Key4 contact_key(const Frozen& c) {
  Key4 k{};
  k.k[0] = c.kind;
  if (c.kind == 2) { k.k[1] = c.p; k.k[2] = k.k[3] = k.k[4] = 0; return k; }
  if (c.kind == 0) {
    int t[3] = {c.a, c.b, c.c};
    std::sort(t, t + 3);
    k.k[1] = c.p; k.k[2] = t[0]; k.k[3] = t[1]; k.k[4] = t[2];
    return k;
  }
  int e1a = std::min(c.a, c.b), e1b = std::max(c.a, c.b);
  int e2a = std::min(c.c, c.d), e2b = std::max(c.c, c.d);
  if (std::make_pair(e1a, e1b) > std::make_pair(e2a, e2b)) { std::swap(e1a, e2a); std::swap(e1b, e2b); }
  k.k[1] = e1a; k.k[2] = e1b; k.k[3] = e2a; k.k[4] = e2b;
  return k;
}

ContactSystem::ContactSystem(const ContactParams& p, const std::vector<uint32_t>& clothIndices)
    : params(p), clothIdx(clothIndices) {
  triCount = (int)clothIdx.size() / 3;
  exclusions = adjacency_exclusions(clothIdx.data(), triCount);
}

void ContactSystem::begin_step(const double* x0, int n3) {
  xStep.assign(x0, x0 + n3);
  lagged.clear();
  active.clear();
  candidates.clear();
  diag = ContactDiag();
}

void ContactSystem::pos_of(const double* x, int v, double out[3]) const {
  if (v >= 0) { out[0] = x[v * 3]; out[1] = x[v * 3 + 1]; out[2] = x[v * 3 + 2]; return; }
  const int i = -v - 2;
  out[0] = staticPos[i * 3]; out[1] = staticPos[i * 3 + 1]; out[2] = staticPos[i * 3 + 2];
}

std::vector<std::pair<int, int>> ContactSystem::query_bvh_all(const std::vector<Aabb>& sBoxes) const {
  std::vector<std::pair<int, int>> out;
  if (bvh.root < 0) return out;
  std::vector<int> stack;
  for (int s = 0; s < (int)sBoxes.size(); s++) {
    stack.assign(1, bvh.root);
    while (!stack.empty()) {
      const int nid = stack.back();
      stack.pop_back();
      const BvhNode& nd = bvh.nodes[nid];
      if (!overlaps(nd.box, sBoxes[s])) continue;
      if (nd.tri >= 0) { out.push_back({nd.tri, s}); continue; }
      stack.push_back(nd.left);
      stack.push_back(nd.right);
    }
  }
  std::sort(out.begin(), out.end());
  return out;
}

// contact-assembly.ts:87-121 buildCandidates.
std::vector<Cand> ContactSystem::build_candidates(const double* x, double pad) {
  bvh.build(xStep.data(), x, clothIdx.data(), triCount, pad);
  auto pairs = bvh.self_pairs(exclusions);
  std::vector<Cand> out;
  static const int TE[3][2] = {{0, 1}, {1, 2}, {2, 0}};
  for (auto [tA, tB] : pairs) {
    const int A[3] = {(int)clothIdx[tA * 3], (int)clothIdx[tA * 3 + 1], (int)clothIdx[tA * 3 + 2]};
    const int B[3] = {(int)clothIdx[tB * 3], (int)clothIdx[tB * 3 + 1], (int)clothIdx[tB * 3 + 2]};
    for (int p : A) out.push_back({0, p, B[0], B[1], B[2], -1});
    for (int p : B) out.push_back({0, p, A[0], A[1], A[2], -1});
    for (auto& ea : TE)
      for (auto& eb : TE) {
        const int a = A[ea[0]], b = A[ea[1]], c = B[eb[0]], d = B[eb[1]];
        if (a == c || a == d || b == c || b == d) continue;
        out.push_back({1, -1, a, b, c, d});
      }
  }
  if (!staticPos.empty() && !staticIdx.empty()) {
    const int sTri = (int)staticIdx.size() / 3;
    std::vector<Aabb> sBoxes(sTri);
    for (int t = 0; t < sTri; t++) {
      const uint32_t i0 = staticIdx[t * 3], i1 = staticIdx[t * 3 + 1], i2 = staticIdx[t * 3 + 2];
      double xs[3] = {staticPos[i0 * 3], staticPos[i1 * 3], staticPos[i2 * 3]};
      double ys[3] = {staticPos[i0 * 3 + 1], staticPos[i1 * 3 + 1], staticPos[i2 * 3 + 1]};
      double zs[3] = {staticPos[i0 * 3 + 2], staticPos[i1 * 3 + 2], staticPos[i2 * 3 + 2]};
      sBoxes[t] = Aabb{js_min(js_min(xs[0], xs[1]), xs[2]) - pad, js_min(js_min(ys[0], ys[1]), ys[2]) - pad,
                       js_min(js_min(zs[0], zs[1]), zs[2]) - pad, js_max(js_max(xs[0], xs[1]), xs[2]) + pad,
                       js_max(js_max(ys[0], ys[1]), ys[2]) + pad, js_max(js_max(zs[0], zs[1]), zs[2]) + pad};
    }
    for (auto [ct, st] : query_bvh_all(sBoxes)) {
      const int A[3] = {(int)clothIdx[ct * 3], (int)clothIdx[ct * 3 + 1], (int)clothIdx[ct * 3 + 2]};
      const int B[3] = {(int)staticIdx[st * 3], (int)staticIdx[st * 3 + 1], (int)staticIdx[st * 3 + 2]};
      for (int p : A) out.push_back({0, p, -(B[0] + 2), -(B[1] + 2), -(B[2] + 2), -2});
      const int be[3][2] = {{B[0], B[1]}, {B[1], B[2]}, {B[2], B[0]}};
      const int ae[3][2] = {{A[0], A[1]}, {A[1], A[2]}, {A[2], A[0]}};
      for (auto& e : ae)
        for (auto& f : be) out.push_back({1, -1, e[0], e[1], -(f[0] + 2), -(f[1] + 2)});
    }
  }
  std::sort(out.begin(), out.end(), [](const Cand& u, const Cand& v) {
    if (u.kind != v.kind) return u.kind < v.kind;
    if (u.p != v.p) return u.p < v.p;
    if (u.a != v.a) return u.a < v.a;
    if (u.b != v.b) return u.b < v.b;
    if (u.c != v.c) return u.c < v.c;
    return u.d < v.d;
  });
  diag.candidatePairs = (double)out.size();
  return out;
}

// contact-assembly.ts:164-220 updateActiveSet.
void ContactSystem::update_active_set(const double* x, int n3) {
  const double dHat = params.dHat;
  candidates = build_candidates(x, dHat);
  std::vector<Frozen> act;
  double minD = INF;
  for (const Cand& q : candidates) {
    if (q.kind == 0) {
      double P[3], A[3], B[3], C[3];
      pos_of(x, q.p, P); pos_of(x, q.a, A); pos_of(x, q.b, B); pos_of(x, q.c, C);
      const Closest cp = closest_vt(P[0], P[1], P[2], A[0], A[1], A[2], B[0], B[1], B[2], C[0], C[1], C[2]);
      if (cp.dist < minD) minD = cp.dist;
      if (cp.dist >= dHat || cp.dist < 1e-12) continue;
      const double nx = cp.rx / cp.dist, ny = cp.ry / cp.dist, nz = cp.rz / cp.dist;
      const double w1 = cp.s, w2 = cp.t, w0 = 1 - cp.s - cp.t;
      act.push_back({0, q.p, q.a, q.b, q.c, -1, w0, w1, w2, 0, nx, ny, nz});
    } else {
      double A[3], B[3], C[3], D[3];
      pos_of(x, q.a, A); pos_of(x, q.b, B); pos_of(x, q.c, C); pos_of(x, q.d, D);
      const Closest cp = closest_ee(A[0], A[1], A[2], B[0], B[1], B[2], C[0], C[1], C[2], D[0], D[1], D[2]);
      if (cp.dist < minD) minD = cp.dist;
      if (cp.dist >= dHat || cp.dist < 1e-12) continue;
      const double nx = cp.rx / cp.dist, ny = cp.ry / cp.dist, nz = cp.rz / cp.dist;
      act.push_back({1, -1, q.a, q.b, q.c, q.d, 1 - cp.s, cp.s, -(1 - cp.t), -cp.t, nx, ny, nz});
    }
  }
  if (hasFloor) {
    const int n = n3 / 3;
    for (int v = 0; v < n; v++) {
      const double d = x[v * 3 + 1] - floorY;
      if (d < minD) minD = d;
      if (d >= dHat) continue;
      act.push_back({2, v, -1, -1, -1, -1, 0, 0, 0, 0, 0, 1, 0});
    }
  }
  active = std::move(act);
  int vt = 0, ee = 0, fl = 0;
  for (const Frozen& c : active) (c.kind == 0 ? vt : c.kind == 1 ? ee : fl)++;
  diag.activePairs = (double)active.size();
  diag.vtPairs = vt; diag.eePairs = ee; diag.floorPairs = fl;
  if (minD < diag.minDistance) diag.minDistance = minD;
}

// contact-assembly.ts:222-258 frozenDist.
double ContactSystem::frozen_dist(const double* x, const Frozen& c) const {
  if (c.kind == 2) return x[c.p * 3 + 1] - floorY;
  if (c.kind == 0) {
    double ddx, ddy, ddz;
    if (c.a >= 0) {
      const double qx = c.w0 * x[c.a * 3] + c.w1 * x[c.b * 3] + c.w2 * x[c.c * 3];
      const double qy = c.w0 * x[c.a * 3 + 1] + c.w1 * x[c.b * 3 + 1] + c.w2 * x[c.c * 3 + 1];
      const double qz = c.w0 * x[c.a * 3 + 2] + c.w1 * x[c.b * 3 + 2] + c.w2 * x[c.c * 3 + 2];
      ddx = x[c.p * 3] - qx; ddy = x[c.p * 3 + 1] - qy; ddz = x[c.p * 3 + 2] - qz;
    } else {
      const float* s = staticPos.data();
      const int ia = -c.a - 2, ib = -c.b - 2, ic = -c.c - 2;
      const double sx = c.w0 * s[ia * 3] + c.w1 * s[ib * 3] + c.w2 * s[ic * 3];
      const double sy = c.w0 * s[ia * 3 + 1] + c.w1 * s[ib * 3 + 1] + c.w2 * s[ic * 3 + 1];
      const double sz = c.w0 * s[ia * 3 + 2] + c.w1 * s[ib * 3 + 2] + c.w2 * s[ic * 3 + 2];
      ddx = x[c.p * 3] - sx; ddy = x[c.p * 3 + 1] - sy; ddz = x[c.p * 3 + 2] - sz;
    }
    return c.nx * ddx + c.ny * ddy + c.nz * ddz;
  }
  double A[3], B[3], C[3], D[3];
  pos_of(x, c.a, A); pos_of(x, c.b, B); pos_of(x, c.c, C); pos_of(x, c.d, D);
  const double rx = c.w0 * A[0] + c.w1 * B[0] + c.w2 * C[0] + c.w3 * D[0];
  const double ry = c.w0 * A[1] + c.w1 * B[1] + c.w2 * C[1] + c.w3 * D[1];
  const double rz = c.w0 * A[2] + c.w1 * B[2] + c.w2 * C[2] + c.w3 * D[2];
  return c.nx * rx + c.ny * ry + c.nz * rz;
}

// contact-assembly.ts:288-315 addDistGrad.
void ContactSystem::add_dist_grad(double* grad, const Frozen& c, double g) const {
  if (c.kind == 2) { grad[c.p * 3 + 1] += g; return; }
  if (c.kind == 0) {
    grad[c.p * 3] += g * c.nx;
    grad[c.p * 3 + 1] += g * c.ny;
    grad[c.p * 3 + 2] += g * c.nz;
    const double ws[3] = {c.w0, c.w1, c.w2};
    const int vs[3] = {c.a, c.b, c.c};
    for (int k = 0; k < 3; k++) {
      if (vs[k] < 0) continue;
      grad[vs[k] * 3] += -g * ws[k] * c.nx;
      grad[vs[k] * 3 + 1] += -g * ws[k] * c.ny;
      grad[vs[k] * 3 + 2] += -g * ws[k] * c.nz;
    }
    return;
  }
  const double ws[4] = {c.w0, c.w1, c.w2, c.w3};
  const int vs[4] = {c.a, c.b, c.c, c.d};
  for (int k = 0; k < 4; k++) {
    if (vs[k] < 0) continue;
    grad[vs[k] * 3] += g * ws[k] * c.nx;
    grad[vs[k] * 3 + 1] += g * ws[k] * c.ny;
    grad[vs[k] * 3 + 2] += g * ws[k] * c.nz;
  }
}

// contact-assembly.ts:318-341 addFrictionForce.
void ContactSystem::add_friction_force(double* grad, const Frozen& c, double fx, double fy, double fz) const {
  if (c.kind == 2 || c.kind == 0) {
    grad[c.p * 3] += fx; grad[c.p * 3 + 1] += fy; grad[c.p * 3 + 2] += fz;
    if (c.kind == 2) return;
    const double ws[3] = {c.w0, c.w1, c.w2};
    const int vs[3] = {c.a, c.b, c.c};
    for (int k = 0; k < 3; k++) {
      if (vs[k] < 0) continue;
      grad[vs[k] * 3] += -fx * ws[k];
      grad[vs[k] * 3 + 1] += -fy * ws[k];
      grad[vs[k] * 3 + 2] += -fz * ws[k];
    }
    return;
  }
  const int vv[4] = {c.a, c.b, c.c, c.d};
  const double ww[4] = {c.w0, c.w1, -c.w2, -c.w3};
  for (int k = 0; k < 4; k++) {
    if (vv[k] < 0) continue;
    grad[vv[k] * 3] += fx * ww[k]; grad[vv[k] * 3 + 1] += fy * ww[k]; grad[vv[k] * 3 + 2] += fz * ww[k];
  }
}

// contact-assembly.ts:344-367 relativeSlip. For VT the third triangle vertex
// reads D(c.d) (always a negative id, so zero displacement): reference behaviour.
void ContactSystem::relative_slip(const double* x, const Frozen& c, double u[3]) const {
  auto D = [&](int v, double o[3]) {
    if (v < 0) { o[0] = o[1] = o[2] = 0; return; }
    o[0] = x[v * 3] - xStep[v * 3]; o[1] = x[v * 3 + 1] - xStep[v * 3 + 1]; o[2] = x[v * 3 + 2] - xStep[v * 3 + 2];
  };
  if (c.kind == 2) { D(c.p, u); return; }
  if (c.kind == 0) {
    double dp[3], da[3], db[3], dc[3];
    D(c.p, dp); D(c.a, da); D(c.b, db); D(c.d, dc);
    for (int i = 0; i < 3; i++) u[i] = dp[i] - (c.w0 * da[i] + c.w1 * db[i] + c.w2 * dc[i]);
    return;
  }
  double da[3], db[3], dc[3], dd[3];
  D(c.a, da); D(c.b, db); D(c.c, dc); D(c.d, dd);
  for (int i = 0; i < 3; i++) u[i] = c.w0 * da[i] + c.w1 * db[i] + c.w2 * dc[i] + c.w3 * dd[i];
}

// contact-assembly.ts:262-285 energyGrad (barrier + lagged friction residual).
double ContactSystem::energy_grad(const double* x, double* grad, int n3) {
  const double dHat = params.dHat, kappa = params.kappa, mu = params.mu, eps = params.eps;
  std::fill(grad, grad + n3, 0.0);
  double energy = 0, fwork = 0;
  for (const Frozen& c : active) {
    const double d = js_max(frozen_dist(x, c), 1e-12);
    if (d >= dHat) continue;
    energy += kappa * barrier_value(d, dHat);
    const double g = barrier_grad_scalar(d, dHat, kappa, 1);
    add_dist_grad(grad, c, g);
    auto it = lagged.find(contact_key(c));
    const bool has = it != lagged.end();
    const double nx = has ? it->second.nx : c.nx, ny = has ? it->second.ny : c.ny,
                 nz = has ? it->second.nz : c.nz;
    const double lambdaN = has ? it->second.lambdaN : barrier_normal_force(d, dHat, kappa, 1);
    double u[3], f[3];
    relative_slip(x, c, u);
    coulomb_force(u[0], u[1], u[2], nx, ny, nz, lambdaN, mu, eps, f);
    add_friction_force(grad, c, -f[0], -f[1], -f[2]);
    fwork += f[0] * u[0] + f[1] * u[1] + f[2] * u[2];
  }
  diag.barrierEnergy = energy;
  diag.frictionWork += fwork;
  return energy;
}

// contact-assembly.ts:394-414 distJvp.
double ContactSystem::dist_jvp(const Frozen& c, const double* v) const {
  if (c.kind == 2) return v[c.p * 3 + 1];
  if (c.kind == 0) {
    double j = c.nx * v[c.p * 3] + c.ny * v[c.p * 3 + 1] + c.nz * v[c.p * 3 + 2];
    const double ws[3] = {c.w0, c.w1, c.w2};
    const int vs[3] = {c.a, c.b, c.c};
    for (int k = 0; k < 3; k++) {
      if (vs[k] < 0) continue;
      j -= ws[k] * (c.nx * v[vs[k] * 3] + c.ny * v[vs[k] * 3 + 1] + c.nz * v[vs[k] * 3 + 2]);
    }
    return j;
  }
  const double ws[4] = {c.w0, c.w1, c.w2, c.w3};
  const int vs[4] = {c.a, c.b, c.c, c.d};
  double j = 0;
  for (int k = 0; k < 4; k++) {
    if (vs[k] < 0) continue;
    j += ws[k] * (c.nx * v[vs[k] * 3] + c.ny * v[vs[k] * 3 + 1] + c.nz * v[vs[k] * 3 + 2]);
  }
  return j;
}

// contact-assembly.ts:371-392 applyHvp (frozen barrier, coeff = kappa max(b'', 0)).
void ContactSystem::apply_hvp(const double* x, const double* v, double* out, int n3) {
  const double dHat = params.dHat, kappa = params.kappa;
  std::fill(out, out + n3, 0.0);
  Vec dd(active.size(), 0.0);
  for (size_t i = 0; i < active.size(); i++) {
    const Frozen& c = active[i];
    const double d = js_max(frozen_dist(x, c), 1e-12);
    if (d >= dHat) { dd[i] = 0; continue; }
    const double L = js_log(d / dHat);
    const double u = d - dHat;
    const double b2 = -(2 * L + (4 * u) / d - (u * u) / (d * d));
    const double coeff = kappa * js_max(b2, 0);
    dd[i] = coeff * dist_jvp(c, v);
  }
  for (size_t i = 0; i < active.size(); i++) {
    if (dd[i] == 0) continue;
    add_dist_grad(out, active[i], dd[i]);
  }
}

// contact-assembly.ts:419-428 meritEnergy.
double ContactSystem::merit_energy(const double* x) {
  const double dHat = params.dHat, kappa = params.kappa;
  double e = 0;
  for (const Frozen& c : active) {
    const double d = js_max(frozen_dist(x, c), 1e-12);
    if (d >= dHat) continue;
    e += kappa * barrier_value(d, dHat);
  }
  return e;
}

// contact-assembly.ts:436-471 addDiagEstimate (accumulates into diag).
void ContactSystem::add_diag_estimate(double* dg, const double* x) {
  const double dHat = params.dHat, kappa = params.kappa;
  for (const Frozen& c : active) {
    const double d = js_max(frozen_dist(x, c), 1e-12);
    if (d >= dHat) continue;
    const double L = js_log(d / dHat);
    const double u = d - dHat;
    const double b2 = js_max(-(2 * L + (4 * u) / d - (u * u) / (d * d)), 0);
    const double k = kappa * b2;
    if (c.kind == 2) { dg[c.p * 3 + 1] += k; continue; }
    const double n2[3] = {c.nx * c.nx, c.ny * c.ny, c.nz * c.nz};
    if (c.kind == 0) {
      for (int kk = 0; kk < 3; kk++) dg[c.p * 3 + kk] += k * n2[kk];
      const double ws[3] = {c.w0, c.w1, c.w2};
      const int vs[3] = {c.a, c.b, c.c};
      for (int j = 0; j < 3; j++) {
        if (vs[j] < 0) continue;
        for (int kk = 0; kk < 3; kk++) dg[vs[j] * 3 + kk] += k * ws[j] * ws[j] * n2[kk];
      }
      continue;
    }
    const double ws[4] = {c.w0, c.w1, c.w2, c.w3};
    const int vs[4] = {c.a, c.b, c.c, c.d};
    for (int j = 0; j < 4; j++) {
      if (vs[j] < 0) continue;
      for (int kk = 0; kk < 3; kk++) dg[vs[j] * 3 + kk] += k * ws[j] * ws[j] * n2[kk];
    }
  }
}

// contact-assembly.ts:475-485 commit.
void ContactSystem::commit(const double* x) {
  const double dHat = params.dHat, kappa = params.kappa;
  for (const Frozen& c : active) {
    const double d = js_max(frozen_dist(x, c), 1e-12);
    if (d >= dHat) continue;
    lagged[contact_key(c)] = Lagged{c.nx, c.ny, c.nz, barrier_normal_force(d, dHat, kappa, 1)};
  }
}

double ContactSystem::exact_dist(const double* x, const Cand& q) const {
  if (q.kind == 0) {
    double P[3], A[3], B[3], C[3];
    pos_of(x, q.p, P); pos_of(x, q.a, A); pos_of(x, q.b, B); pos_of(x, q.c, C);
    return closest_vt(P[0], P[1], P[2], A[0], A[1], A[2], B[0], B[1], B[2], C[0], C[1], C[2]).dist;
  }
  double A[3], B[3], C[3], D[3];
  pos_of(x, q.a, A); pos_of(x, q.b, B); pos_of(x, q.c, C); pos_of(x, q.d, D);
  return closest_ee(A[0], A[1], A[2], B[0], B[1], B[2], C[0], C[1], C[2], D[0], D[1], D[2]).dist;
}

// contact-assembly.ts:489-553 checkTrial: dMin-pad candidates, exact distance
// gate, VT/EE CCD against the Newton segment xStep -> xT, then floor CCD.
TrialResult ContactSystem::check_trial(const double* xT, int n3) {
  const double dMin = params.dMin;
  std::vector<Cand> cands = build_candidates(xT, dMin);
  double minDist = INF, minTOI = INF;
  for (const Cand& q : cands) {
    const double d = exact_dist(xT, q);
    if (d < minDist) minDist = d;
    if (!std::isfinite(d)) { diag.ccdFailures++; return {false, minDist, minTOI}; }
  }
  const int n = n3 / 3;
  if (hasFloor)
    for (int v = 0; v < n; v++) {
      const double d = xT[v * 3 + 1] - floorY;
      if (d < minDist) minDist = d;
    }
  if (minDist <= dMin) return {false, minDist, minTOI};
  double P0[12], P1[12];
  for (const Cand& q : cands) {
    double toi = INF;
    const int ids[4] = {q.kind == 0 ? q.p : q.a, q.kind == 0 ? q.a : q.b, q.kind == 0 ? q.b : q.c,
                        q.kind == 0 ? q.c : q.d};
    if (q.kind == 0) {
      if (q.p < 0 && q.a < 0) continue;
    } else {
      if (q.a < 0 && q.b < 0 && q.c < 0 && q.d < 0) continue;
    }
    for (int k = 0; k < 4; k++) {
      pos_of(xStep.data(), ids[k], P0 + k * 3);
      pos_of(xT, ids[k], P1 + k * 3);
    }
    toi = q.kind == 0 ? vt_ccd(P0, P1, dMin) : ee_ccd(P0, P1, dMin);
    if (std::isnan(toi)) { diag.ccdFailures++; return {false, minDist, minTOI}; }
    if (toi < minTOI) minTOI = toi;
    if (toi > 0 && toi < 1 - 1e-9) return {false, minDist, minTOI};
  }
  if (hasFloor)
    for (int v = 0; v < n; v++) {
      const double y0 = xStep[v * 3 + 1] - floorY;
      const double yT = xT[v * 3 + 1] - floorY;
      if (y0 - std::fabs(yT - y0) > dMin) continue;
      if (y0 > dMin && yT <= dMin && y0 > yT) {
        const double toi = (y0 - dMin) / (y0 - yT);
        if (toi < minTOI) minTOI = toi;
        if (toi < 1 - 1e-9) return {false, minDist, minTOI};
      }
    }
  if (minDist < diag.minDistance) diag.minDistance = minDist;
  if (minTOI < diag.minTOI) diag.minTOI = minTOI;
  return {true, minDist, minTOI};
}

}  // namespace orc
