// TEST INFRASTRUCTURE ONLY -- the CPU oracle for the paint-mixing MPM step.
//
// This file restates, on the CPU, the algorithm of the reference solver's time step
// (Natashaaak/pigment_mixing, matter/src/simulation/simulation.cpp:225-291, advanceStep and
// the kernels it calls).  It is the checker for the CUDA path and the timed CPU baseline:
// only tests/, __graft_entry__.smoke() and bench.py's CPU legs may load it.  Nothing in the
// product library calls it.
//
// Parity pinning: the reference itself cannot be built (Eigen3, OpenVDB, tinyply,
// tph_poisson and googletest are absent and there is no network), so this restatement is
// checked against the reference's own known-answer tests (matter/tests/tests.cpp: the curve
// slide, Coulomb friction on a plate and on the ground object, the bulk modulus, the rotation
// energy and the Drucker-Prager column collapse; restated in tests/reference_kats.py and run by
// tests/test_reference_kats.py) and against golden vectors produced by the reference's mixbox
// library compiled in place.
//
// Structure mirrors the reference on purpose so that its CPU cost is representative:
//   * AoS particle/grid storage, a 4x4x4 precomputed weight stencil per particle
//     (precompute_weight.cpp:3-43),
//   * per-thread full-grid copies merged under a critical section in P2G and MUSL
//     (p2g.cpp:12-91, musl.cpp:166-222),
//   * atomic force scatter with a fresh Hencky SVD per particle (explicit_euler_update.cpp:12-55),
//   * a second SVD in the return map (plasticity.cpp:18-26).
// Real is the arithmetic type: double gives the FP64 oracle, float the reference-faithful
// build (the reference compiles T=float with -O3 -ffast-math -fopenmp, matter/CMakeLists.txt:7).
//
// Deviations (all numerically below float rounding of the reference):
//   * grid node coordinates are low + i*dx instead of the float running sum of arange
//     (tools.hpp:325-330);
//   * the 3x3 SVD is a one-sided Jacobi (Hestenes) SVD with sigma >= 0 instead of Eigen's
//     two-sided JacobiSVD; U g(Sigma) V^T is the same for any SVD with sigma >= 0 and
//     det F != 0 (it is R g(S) of the polar decomposition F = R S);
//   * spatula velocities start at zero (the reference leaves them uninitialised,
//     object_spatula.hpp:266-270).

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

// Enum values follow matter/src/tools.hpp:55-59.
enum PlateType { PT_TOP = 0, PT_BOTTOM, PT_LEFT, PT_RIGHT, PT_FRONT, PT_BACK };
enum BCType { BC_NOSLIP = 0, BC_SLIPSTICK, BC_SLIPFREE };
enum PlasticModel { PM_NOPLASTICITY = 0, PM_VM, PM_DP, PM_DPSOFT, PM_MCC, PM_VMVISC, PM_DPVISC,
                    PM_MCCVISC, PM_DPMUI, PM_MCCMUI };

// Error bits (the reference's `exit` flag, simulation.hpp:30, split by cause).
enum ErrorBits {
  ERR_NEG_DGAMMA = 1u << 0,      // plasticity.cpp:186-192, 286-289
  ERR_NEWTON_NOCONV = 1u << 1,   // plasticity.cpp:200-203, 298-301
  ERR_NEWTON_FLAT = 1u << 2,     // plasticity.cpp:219-222, 314-317
  ERR_INVALID_BC = 1u << 3,      // boundary_collision.cpp:84-88
  ERR_NAN_PARTICLE = 1u << 4,    // position_update.cpp:311-327 (deactivations)
};

// ---------------------------------------------------------------------------------------
// Small fixed-size linear algebra
// ---------------------------------------------------------------------------------------
template <class R> struct V3 {
  R c[3];
  V3() : c{0, 0, 0} {}
  V3(R a, R b, R d) : c{a, b, d} {}
  R& operator[](int i) { return c[i]; }
  const R& operator[](int i) const { return c[i]; }
  V3 operator+(const V3& o) const { return V3(c[0] + o[0], c[1] + o[1], c[2] + o[2]); }
  V3 operator-(const V3& o) const { return V3(c[0] - o[0], c[1] - o[1], c[2] - o[2]); }
  V3 operator*(R s) const { return V3(c[0] * s, c[1] * s, c[2] * s); }
  V3& operator+=(const V3& o) { c[0] += o[0]; c[1] += o[1]; c[2] += o[2]; return *this; }
  R dot(const V3& o) const { return c[0] * o[0] + c[1] * o[1] + c[2] * o[2]; }
  R norm() const { return std::sqrt(dot(*this)); }
  R sq() const { return dot(*this); }
};
template <class R> V3<R> cross(const V3<R>& a, const V3<R>& b) {
  return V3<R>(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}

template <class R> struct M3 {
  R m[3][3];
  M3() { std::memset(m, 0, sizeof(m)); }
  static M3 I() { M3 r; r.m[0][0] = r.m[1][1] = r.m[2][2] = 1; return r; }
  R& operator()(int i, int j) { return m[i][j]; }
  const R& operator()(int i, int j) const { return m[i][j]; }
  M3 operator+(const M3& o) const { M3 r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.m[i][j] = m[i][j] + o.m[i][j]; return r; }
  M3 operator*(R s) const { M3 r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.m[i][j] = m[i][j] * s; return r; }
  M3 operator*(const M3& o) const {
    M3 r;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        R s = 0;
        for (int k = 0; k < 3; ++k) s += m[i][k] * o.m[k][j];
        r.m[i][j] = s;
      }
    return r;
  }
  V3<R> operator*(const V3<R>& v) const {
    return V3<R>(m[0][0] * v[0] + m[0][1] * v[1] + m[0][2] * v[2],
                 m[1][0] * v[0] + m[1][1] * v[1] + m[1][2] * v[2],
                 m[2][0] * v[0] + m[2][1] * v[1] + m[2][2] * v[2]);
  }
  M3 T() const { M3 r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.m[i][j] = m[j][i]; return r; }
  R det() const {
    return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
           m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
  }
  R frob() const { R s = 0; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) s += m[i][j] * m[i][j]; return std::sqrt(s); }
};

// One-sided Jacobi (Hestenes) SVD of a 3x3 matrix: A = U diag(s) V^T with s >= 0, sorted
// descending as Eigen's JacobiSVD returns them (plasticity.cpp:18, simulation.hpp:288).
template <class R> void svd3(const M3<R>& A, M3<R>& U, V3<R>& s, M3<R>& V) {
  M3<R> W = A;  // columns are rotated until mutually orthogonal
  V = M3<R>::I();
  const R eps = std::numeric_limits<R>::epsilon();
  for (int sweep = 0; sweep < 30; ++sweep) {
    bool rotated = false;
    for (int pq = 0; pq < 3; ++pq) {
      const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
      R alpha = 0, beta = 0, gamma = 0;
      for (int k = 0; k < 3; ++k) {
        alpha += W.m[k][p] * W.m[k][p];
        beta += W.m[k][q] * W.m[k][q];
        gamma += W.m[k][p] * W.m[k][q];
      }
      if (std::abs(gamma) <= eps * std::sqrt(alpha * beta) || gamma == 0) continue;
      rotated = true;
      const R zeta = (beta - alpha) / (2 * gamma);
      const R t = (zeta >= 0 ? R(1) : R(-1)) / (std::abs(zeta) + std::sqrt(R(1) + zeta * zeta));
      const R c = R(1) / std::sqrt(R(1) + t * t);
      const R sn = c * t;
      for (int k = 0; k < 3; ++k) {
        const R wp = W.m[k][p], wq = W.m[k][q];
        W.m[k][p] = c * wp - sn * wq;
        W.m[k][q] = sn * wp + c * wq;
        const R vp = V.m[k][p], vq = V.m[k][q];
        V.m[k][p] = c * vp - sn * vq;
        V.m[k][q] = sn * vp + c * vq;
      }
    }
    if (!rotated) break;
  }
  R nrm[3];
  for (int j = 0; j < 3; ++j) nrm[j] = std::sqrt(W.m[0][j] * W.m[0][j] + W.m[1][j] * W.m[1][j] + W.m[2][j] * W.m[2][j]);
  // sort descending
  int ord[3] = {0, 1, 2};
  std::sort(ord, ord + 3, [&](int a, int b) { return nrm[a] > nrm[b]; });
  M3<R> Vs, Us;
  for (int j = 0; j < 3; ++j) {
    const int o = ord[j];
    s[j] = nrm[o];
    for (int k = 0; k < 3; ++k) Vs.m[k][j] = V.m[k][o];
  }
  // left vectors; complete a null space with cross products
  const R tiny = std::numeric_limits<R>::min() * 16;
  int valid = 0;
  for (int j = 0; j < 3; ++j) {
    const int o = ord[j];
    if (s[j] > tiny) {
      for (int k = 0; k < 3; ++k) Us.m[k][j] = W.m[k][o] / s[j];
      ++valid;
    }
  }
  if (valid < 3) {
    if (valid == 0) { Us = M3<R>::I(); }
    else {
      V3<R> u0(Us.m[0][0], Us.m[1][0], Us.m[2][0]);
      if (valid == 1) {
        V3<R> a = std::abs(u0[0]) < R(0.9) ? V3<R>(1, 0, 0) : V3<R>(0, 1, 0);
        V3<R> u1 = cross(u0, a);
        u1 = u1 * (R(1) / u1.norm());
        for (int k = 0; k < 3; ++k) Us.m[k][1] = u1[k];
      }
      V3<R> u1(Us.m[0][1], Us.m[1][1], Us.m[2][1]);
      V3<R> u2 = cross(u0, u1);
      for (int k = 0; k < 3; ++k) Us.m[k][2] = u2[k];
    }
  }
  U = Us;
  V = Vs;
}

// ---------------------------------------------------------------------------------------
// Quadratic B-spline (matter/src/tools.hpp:153-177, 243-266)
// ---------------------------------------------------------------------------------------
template <class R> inline R bsN(R u) {
  R a = std::abs(u);
  if (a < R(0.5)) return R(0.75) - a * a;
  if (a < R(1.5)) return R(0.5) * (R(1.5) - a) * (R(1.5) - a);
  return 0;
}
template <class R> inline R bsdN(R u) {
  R a = std::abs(u);
  if (a < R(0.5)) return -2 * u;
  if (a < R(1.5)) return u - R(1.5) * R((R(0) < u) - (u < R(0)));
  return 0;
}

// ---------------------------------------------------------------------------------------
// Objects (matter/src/objects/object_plate.hpp, object_spatula.hpp, object_ground.hpp,
// object_curve.hpp) plus the box knife on a polyline path (the synthetic workloads' knife).
// ---------------------------------------------------------------------------------------
template <class R> struct Plate {
  R pos, lower, upper, vx, vy, vz, vx0, vy0, vz0, vmin_factor, load_factor, friction;
  int type, bc;
  bool inside(const V3<R>& X) const {  // object_plate.hpp:13-57
    switch (type) {
      case PT_LEFT: return X[1] < upper && X[1] > lower && (X[0] - pos) <= 0;
      case PT_RIGHT: return X[1] < upper && X[1] > lower && (pos - X[0]) <= 0;
      case PT_BOTTOM: return X[0] < upper && X[0] > lower && (X[1] - pos) <= 0;
      case PT_TOP: return X[0] < upper && X[0] > lower && (pos - X[1]) <= 0;
      case PT_BACK: return X[2] - pos <= 0;
      case PT_FRONT: return pos - X[2] <= 0;
    }
    return false;
  }
  void move(R dt, R frame_dt, R time) {  // object_plate.hpp:136-162
    R factor = (time < load_factor * frame_dt) ? (R(1) / vmin_factor) : R(1);
    vx = vx0 * factor; vy = vy0 * factor; vz = vz0 * factor;
    if (type == PT_LEFT || type == PT_RIGHT) { pos += dt * vx; upper += dt * vy; lower += dt * vy; }
    else if (type == PT_BOTTOM || type == PT_TOP) { pos += dt * vy; upper += dt * vx; lower += dt * vx; }
    else { pos += dt * vz; }
  }
};

enum ObjKind { OBJ_SPATULA = 0, OBJ_BOXKNIFE = 1, OBJ_GROUND = 2, OBJ_CURVE = 3 };

template <class R> struct Quat { R w, x, y, z; };
template <class R> Quat<R> qmul(const Quat<R>& a, const Quat<R>& b) {
  return {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z, a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
          a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x, a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}
// Spherical linear interpolation, shortest arc, with a linear blend for nearly parallel
// inputs (the standard published formula; object_spatula.hpp:202 calls Eigen's slerp).
template <class R> Quat<R> slerp(const Quat<R>& a, const Quat<R>& b, R t) {
  const R one = R(1) - std::numeric_limits<R>::epsilon();
  R d = a.w * b.w + a.x * b.x + a.y * b.y + a.z * b.z;
  R ad = std::abs(d);
  R s0, s1;
  if (ad >= one) { s0 = R(1) - t; s1 = t; }
  else {
    R th = std::acos(ad), sth = std::sin(th);
    s0 = std::sin((R(1) - t) * th) / sth;
    s1 = std::sin(t * th) / sth;
  }
  if (d < 0) s1 = -s1;
  return {s0 * a.w + s1 * b.w, s0 * a.x + s1 * b.x, s0 * a.y + s1 * b.y, s0 * a.z + s1 * b.z};
}
template <class R> M3<R> qrot(const Quat<R>& q) {  // normalised quaternion -> rotation
  M3<R> r;
  R n = std::sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
  R w = q.w / n, x = q.x / n, y = q.y / n, z = q.z / n;
  r.m[0][0] = 1 - 2 * (y * y + z * z); r.m[0][1] = 2 * (x * y - z * w); r.m[0][2] = 2 * (x * z + y * w);
  r.m[1][0] = 2 * (x * y + z * w); r.m[1][1] = 1 - 2 * (x * x + z * z); r.m[1][2] = 2 * (y * z - x * w);
  r.m[2][0] = 2 * (x * z - y * w); r.m[2][1] = 2 * (y * z + x * w); r.m[2][2] = 1 - 2 * (x * x + y * y);
  return r;
}

template <class R> struct GObject {
  int kind, bc;
  R friction;
  // pose: world = Rm * local + t ; inverse: local = Rinv * (world - t)
  M3<R> Rm, Rinv;
  V3<R> t;
  V3<R> vlin, omega;
  Quat<R> q;
  // spatula
  R halfWidth = R(0.368), halfLength = R(0.736), halfThickness = R(0.07), offset = R(0.05);
  std::vector<float> frames;  // n x 7 (pos xyz, quat xyzw), object_spatula.hpp:7-10
  R currentTime = 0;
  // box knife
  V3<R> half;
  std::vector<V3<R>> path;
  R speed = 0, s = 0;
  // ground
  R y0 = 0;

  void setPose(const V3<R>& p, const Quat<R>& qq) {
    q = qq; t = p; Rm = qrot(qq);
    // general inverse of the linear part (Eigen Affine inverse), then -Rinv t
    R d = Rm.det();
    M3<R> inv;
    inv.m[0][0] = (Rm.m[1][1] * Rm.m[2][2] - Rm.m[1][2] * Rm.m[2][1]) / d;
    inv.m[0][1] = (Rm.m[0][2] * Rm.m[2][1] - Rm.m[0][1] * Rm.m[2][2]) / d;
    inv.m[0][2] = (Rm.m[0][1] * Rm.m[1][2] - Rm.m[0][2] * Rm.m[1][1]) / d;
    inv.m[1][0] = (Rm.m[1][2] * Rm.m[2][0] - Rm.m[1][0] * Rm.m[2][2]) / d;
    inv.m[1][1] = (Rm.m[0][0] * Rm.m[2][2] - Rm.m[0][2] * Rm.m[2][0]) / d;
    inv.m[1][2] = (Rm.m[0][2] * Rm.m[1][0] - Rm.m[0][0] * Rm.m[1][2]) / d;
    inv.m[2][0] = (Rm.m[1][0] * Rm.m[2][1] - Rm.m[1][1] * Rm.m[2][0]) / d;
    inv.m[2][1] = (Rm.m[0][1] * Rm.m[2][0] - Rm.m[0][0] * Rm.m[2][1]) / d;
    inv.m[2][2] = (Rm.m[0][0] * Rm.m[1][1] - Rm.m[0][1] * Rm.m[1][0]) / d;
    Rinv = inv;
  }
  V3<R> toLocal(const V3<R>& X) const { return Rinv * (X - t); }

  // object_spatula.hpp:40-82
  R sdSpatula(const V3<R>& p) const {
    R px = std::abs(p[0]), py = p[2];
    R b1 = halfWidth + offset, b2 = (halfWidth + offset) * R(0.25), he = halfLength + offset;
    R bax = b2 - b1, bay = he - (-he);
    R pax = px - b1, pay = py - (-he);
    R h = std::max(R(0), std::min(R(1), (pax * bax + pay * bay) / (bax * bax + bay * bay)));
    R dxs = pax - bax * h, dys = pay - bay * h;
    R d_side = std::sqrt(dxs * dxs + dys * dys);
    R inside_x = b1 - (b1 - b2) * (py + he) / (R(2) * he);
    R d_inside = px - inside_x;
    R d2 = (px < inside_x) ? d_inside : d_side;
    if (py > he) {
      d2 = std::sqrt(px * px + (py - he) * (py - he)) - b2;
    } else if (py < -he) {
      R rx = halfWidth + offset, rz = R(1.5) * (halfWidth + offset);
      R qx = px, qz = py + he;
      R k0 = std::sqrt((qx / rx) * (qx / rx) + (qz / rz) * (qz / rz));
      R k1 = std::sqrt((qx / (rx * rx)) * (qx / (rx * rx)) + (qz / (rz * rz)) * (qz / (rz * rz)));
      d2 = k0 * (k0 - R(1)) / k1;
    }
    R dy = std::abs(p[1]) - halfThickness;
    R mx = std::max(d2, dy);
    R ex = std::max(d2, R(0)), ey = std::max(dy, R(0));
    return std::min(mx, R(0)) + std::sqrt(ex * ex + ey * ey);
  }
  R sdBox(const V3<R>& p) const {
    R qx = std::abs(p[0]) - half[0], qy = std::abs(p[1]) - half[1], qz = std::abs(p[2]) - half[2];
    R ox = std::max(qx, R(0)), oy = std::max(qy, R(0)), oz = std::max(qz, R(0));
    return std::sqrt(ox * ox + oy * oy + oz * oz) + std::min(std::max(qx, std::max(qy, qz)), R(0));
  }
  R sdLocal(const V3<R>& p) const { return kind == OBJ_SPATULA ? sdSpatula(p) : sdBox(p); }
  R sdWorld(const V3<R>& X) const { return sdLocal(toLocal(X)); }

  bool inside(const V3<R>& X) const {
    switch (kind) {
      case OBJ_SPATULA: case OBJ_BOXKNIFE: return sdWorld(X) < 0;  // object_spatula.hpp:84-97
      case OBJ_GROUND: return !(X[1] > y0);                        // object_ground.hpp:16-25
      case OBJ_CURVE: return !(X[1] > X[0] * X[0]);                // object_curve.hpp:15-25
    }
    return false;
  }
  V3<R> normal(const V3<R>& X) const {
    if (kind == OBJ_GROUND) return V3<R>(0, 1, 0);  // object_ground.hpp:27-36 (3D: z left 0)
    if (kind == OBJ_CURVE) {                           // object_curve.hpp:27-37
      V3<R> n(-2 * X[0], 1, 0);
      return n * (R(1) / n.norm());
    }
    // central differences in local space, e = 1e-4 (object_spatula.hpp:99-129)
    V3<R> p = toLocal(X);
    const R e = R(1e-4);
    V3<R> nl(sdLocal(p + V3<R>(e, 0, 0)) - sdLocal(p - V3<R>(e, 0, 0)),
             sdLocal(p + V3<R>(0, e, 0)) - sdLocal(p - V3<R>(0, e, 0)),
             sdLocal(p + V3<R>(0, 0, e)) - sdLocal(p - V3<R>(0, 0, e)));
    R nn = nl.norm();
    if (nn > 0) nl = nl * (R(1) / nn);
    // (linear^-1)^T n  == Rinv^T n
    V3<R> w = Rinv.T() * nl;
    R wn = w.norm();
    if (wn > 0) w = w * (R(1) / wn);
    return w;
  }
  V3<R> velocity(const V3<R>& X) const {  // object_spatula.hpp:136-162
    if (kind == OBJ_GROUND || kind == OBJ_CURVE) return V3<R>();
    return vlin + cross(omega, X - t);
  }
  V3<R> pathPoint(R arc) const {
    if (path.empty()) return V3<R>();
    R acc = 0;
    for (size_t i = 0; i + 1 < path.size(); ++i) {
      V3<R> d = path[i + 1] - path[i];
      R L = d.norm();
      if (arc <= acc + L && L > 0) return path[i] + d * ((arc - acc) / L);
      acc += L;
    }
    return path.back();
  }
  void move(R dt) {
    if (kind == OBJ_SPATULA) {  // object_spatula.hpp:164-233
      currentTime += dt;
      const int nf = int(frames.size() / 7);
      if (nf == 0) { vlin = V3<R>(); omega = V3<R>(); return; }
      R fi = currentTime * R(60);
      int i0u = int(std::floor(fi));
      int i0 = std::min(i0u, nf - 1), i1 = std::min(i0u + 1, nf - 1);
      i0 = std::max(i0, 0); i1 = std::max(i1, 0);
      R tt = fi - R(i0u);
      const float* f0 = &frames[7 * i0];
      const float* f1 = &frames[7 * i1];
      V3<R> p0(f0[0], f0[1], f0[2]), p1(f1[0], f1[1], f1[2]);
      V3<R> pi = p0 + (p1 - p0) * tt;
      Quat<R> q0{R(f0[6]), R(f0[3]), R(f0[4]), R(f0[5])}, q1{R(f1[6]), R(f1[3]), R(f1[4]), R(f1[5])};
      Quat<R> qi = slerp(q0, q1, tt);
      vlin = (pi - t) * (R(1) / dt);
      // relative rotation dq = q_new * conj(q_old) -> axis-angle with angle in [0, pi]
      Quat<R> qc{q.w, -q.x, -q.y, -q.z};
      Quat<R> dq = qmul(qi, qc);
      R n2 = dq.x * dq.x + dq.y * dq.y + dq.z * dq.z;
      if (n2 == 0) omega = V3<R>();
      else {
        R vn = std::sqrt(n2);
        R ang = 2 * std::atan2(vn, std::abs(dq.w));
        R sg = dq.w < 0 ? R(-1) : R(1);
        omega = V3<R>(dq.x, dq.y, dq.z) * (sg * ang / (vn * dt));
      }
      setPose(pi, qi);
    } else if (kind == OBJ_BOXKNIFE) {
      s += speed * dt;
      V3<R> pn = pathPoint(s);
      vlin = (pn - t) * (R(1) / dt);
      omega = V3<R>();
      setPose(pn, q);
    }
  }
};

// ---------------------------------------------------------------------------------------
// Simulation state and the step (matter/src/simulation/*.cpp)
// ---------------------------------------------------------------------------------------
struct NB { unsigned base[3]; };

template <class R> struct Sim {
  // public parameters (simulation.hpp:38-126)
  unsigned n_threads = 1, end_frame = 10, frame = 0;
  bool use_musl = false, use_particle_boundaries = false, use_pradhana = true;
  // use_musl as the caller set it: prepare() turns MUSL on like prepareSimulation
  // (simulation_units.cpp:185-186); simulate() keeps the field (false by default, simulation.hpp:49)
  bool use_musl_user = false;
  V3<R> grid_reference_point = V3<R>(R(2e10), R(2e10), R(2e10));
  V3<R> gravity;
  V3<R> particle_boundary_min = V3<R>(-5, -5, -5), particle_boundary_max = V3<R>(5, 5, 5);
  R min_dt = R(1e-14), fps = 1, cfl = R(0.5), cfl_elastic = 1, flip_ratio = R(-0.95), rho = 1000;
  R E = R(1e5), nu = R(0.3), xi = 0, q_max = 100, q_min = 100, p_min = R(-1e20), M = 1, q_cohesion = 0;
  R perzyna_exp = 1, perzyna_visc = 0, q_prefac = R(1.0 / std::sqrt(2.0));
  R D_max = R(10e-2), D_edge0 = R(0.5), D_edge1 = R(0.8), start_boost = 20, end_boost = 40, boost_factor = 2;
  int plastic_model = PM_NOPLASTICITY;
  R particle_mass = 0, particle_volume = 0, dx = 0;
  unsigned Np = 0;
  unsigned error_flags = 0;
  unsigned plastic_count = 0;

  // particles (data_structures.hpp:9-50), latent stored in Real
  std::vector<char> active;
  std::vector<V3<R>> x, v, pic, flip;
  std::vector<R> eps_pl_dev, eps_pl_vol, eps_pl_vol_pradhana, delta_gamma, diffusion;
  std::vector<M3<R>> F, Bmat;
  std::vector<std::array<R, 7>> lat;

  std::vector<Plate<R>> plates;
  std::vector<GObject<R>> objects;
  int spatula_index = -1;  // the knife (simulation.hpp:131, spatula_ptr)

  // private state (simulation.hpp:188-270)
  unsigned step_count = 0;
  R time = 0, final_time = 0, frame_dt = 1, dt = 0, dt_max = 0;
  R wave_speed = 0, mu = 0, lambda = 0, K = 0, d_prefac = 0, e_mu_prefac = 0, f_mu_prefac = 0;
  R one_over_dx = 0, apicDinverse = 0;
  unsigned Nx = 0, Ny = 0, Nz = 0, grid_nodes = 0;
  R low[3], high[3], min_init[3], max_init[3], low_init[3], high_init[3];
  std::vector<R> gx, gy, gz;
  std::vector<V3<R>> g_v, g_flip, g_v_update;
  std::vector<R> g_mass, g_shear;
  std::vector<std::array<R, 7>> g_lat;
  std::vector<std::array<unsigned, 3>> nb_base;
  std::vector<R> nb_w;          // 64 per particle
  std::vector<V3<R>> nb_g;      // 64 per particle

  inline unsigned ind(unsigned i, unsigned j, unsigned k) const { return (i * Ny + j) * Nz + k; }

  void resizeParticles(unsigned n) {
    Np = n;
    active.assign(n, 1);
    x.assign(n, V3<R>()); v.assign(n, V3<R>()); pic.assign(n, V3<R>()); flip.assign(n, V3<R>());
    eps_pl_dev.assign(n, 0); eps_pl_vol.assign(n, 0); eps_pl_vol_pradhana.assign(n, 0);
    delta_gamma.assign(n, 0); diffusion.assign(n, 0);
    F.assign(n, M3<R>::I()); Bmat.assign(n, M3<R>());
    lat.assign(n, std::array<R, 7>{});
  }

  // simulation_units.cpp:133-215 (prepareSimulation)
  void prepare() {
    apicDinverse = R(4) / (dx * dx);
    lambda = nu * E / ((R(1) + nu) * (R(1) - R(2) * nu));
    mu = E / (R(2) * (R(1) + nu));
    K = lambda + R(2) * mu / R(3);
    wave_speed = std::sqrt(E / rho);
    dt_max = cfl_elastic * dx / wave_speed;
    frame_dt = R(1) / fps;
    one_over_dx = R(1) / dx;
    d_prefac = R(1) / q_prefac;
    e_mu_prefac = R(2) * q_prefac * mu;
    f_mu_prefac = R(2) * q_prefac * q_prefac * mu;
    use_musl = true;
    if (step_count == 0) remeshInit(); else remeshCont();
    time = 0;
    frame = 0;
    final_time = R(end_frame) * frame_dt;
  }

  void aabb(R mn[3], R mx[3]) const {
    for (int d = 0; d < 3; ++d) { mn[d] = R(1e20); mx[d] = R(-1e20); }
    bool any = false;
    for (unsigned p = 0; p < Np; ++p) {
      if (!active[p]) continue;
      any = true;
      for (int d = 0; d < 3; ++d) { mn[d] = std::min(mn[d], x[p][d]); mx[d] = std::max(mx[d], x[p][d]); }
    }
    if (!any) for (int d = 0; d < 3; ++d) mn[d] = mx[d] = 0;
  }

  void buildCoords() {
    // node count as arange(low, high+dx, dx) produces it; coordinates low + i*dx
    unsigned n[3];
    for (int d = 0; d < 3; ++d) {
      R span = (high[d] + dx - low[d]) / dx;
      long c = (long)std::ceil(span - R(1e-6));
      n[d] = (unsigned)std::max(1L, c);
    }
    Nx = n[0]; Ny = n[1]; Nz = n[2];
    grid_nodes = Nx * Ny * Nz;
    gx.resize(Nx); gy.resize(Ny); gz.resize(Nz);
    for (unsigned i = 0; i < Nx; ++i) gx[i] = low[0] + R(i) * dx;
    for (unsigned i = 0; i < Ny; ++i) gy[i] = low[1] + R(i) * dx;
    for (unsigned i = 0; i < Nz; ++i) gz[i] = low[2] + R(i) * dx;
  }

  void remeshInit() {  // remesh.cpp:45-180 with safety factors (2,2,2)
    R mn[3], mx[3];
    aabb(mn, mx);
    if (grid_reference_point[0] < R(1e10)) {
      for (int d = 0; d < 3; ++d) {
        if (grid_reference_point[d] < mn[d]) mn[d] = grid_reference_point[d];
        else if (grid_reference_point[d] > mx[d]) mx[d] = grid_reference_point[d];
      }
    }
    for (int d = 0; d < 3; ++d) {
      max_init[d] = mx[d]; min_init[d] = mn[d];
      low_init[d] = mn[d] - dx * 2; high_init[d] = mx[d] + dx * 2;
      low[d] = low_init[d]; high[d] = high_init[d];
    }
    buildCoords();
  }

  void remeshCont() {  // remesh.cpp:182-297
    R mn[3], mx[3];
    aabb(mn, mx);
    for (int d = 0; d < 3; ++d) {
      if (mx[d] < max_init[d]) {
        unsigned r = (unsigned)std::floor(std::max(R(0), (max_init[d] - mx[d]) / dx - R(1e-8) * dx));
        high[d] = high_init[d] - R(r) * dx;
      } else {
        unsigned e = (unsigned)std::floor(std::max(R(0), (mx[d] - max_init[d]) / dx - R(1e-8) * dx));
        high[d] = high_init[d] + R(e) * dx;
      }
      if (mn[d] > min_init[d]) {
        unsigned r = (unsigned)std::floor(std::max(R(0), (mn[d] - min_init[d]) / dx - R(1e-8) * dx));
        low[d] = low_init[d] + R(r) * dx;
      } else {
        unsigned e = (unsigned)std::floor(std::max(R(0), (min_init[d] - mn[d]) / dx - R(1e-8) * dx));
        low[d] = low_init[d] - R(e) * dx;
      }
    }
    buildCoords();
  }

  void updateDt() {  // update_dt.cpp:5-41
    R m2 = 0;
#pragma omp parallel for reduction(max : m2) num_threads(n_threads)
    for (long p = 0; p < (long)Np; ++p) {
      if (!active[p]) continue;
      R s2 = v[p].sq();
      if (s2 > m2) m2 = s2;
    }
    R ms = std::sqrt(m2);
    if (std::abs(ms) > R(1e-10)) dt = std::min(cfl * dx / ms, dt_max);
    else dt = dt_max;
    dt = std::min(dt, frame_dt * R(frame + 1) - time);
    dt = std::max(dt, min_dt);
  }

  void resizeGrid() {  // remesh.cpp:5-13
    g_v.assign(grid_nodes, V3<R>());
    g_flip.assign(grid_nodes, V3<R>());
    g_mass.assign(grid_nodes, 0);
    g_lat.assign(grid_nodes, std::array<R, 7>{});
    g_shear.assign(grid_nodes, 0);
  }

  void precomputeWeights() {  // precompute_weight.cpp:3-43
    nb_base.resize(Np);
    nb_w.resize(size_t(Np) * 64);
    nb_g.resize(size_t(Np) * 64);
#pragma omp parallel for num_threads(n_threads)
    for (long p = 0; p < (long)Np; ++p) {
      if (!active[p]) continue;
      const V3<R>& xp = x[p];
      int b[3];
      for (int d = 0; d < 3; ++d) b[d] = std::max(0, (int)std::floor((xp[d] - low[d]) * one_over_dx) - 1);
      for (int d = 0; d < 3; ++d) nb_base[p][d] = (unsigned)b[d];
      int cnt = 0;
      for (int i = b[0]; i < b[0] + 4; ++i)
        for (int j = b[1]; j < b[1] + 4; ++j)
          for (int k = b[2]; k < b[2] + 4; ++k) {
            R xi = i < (int)Nx ? gx[i] : low[0] + R(i) * dx;
            R yi = j < (int)Ny ? gy[j] : low[1] + R(j) * dx;
            R zi = k < (int)Nz ? gz[k] : low[2] + R(k) * dx;
            R ux = (xp[0] - xi) * one_over_dx, uy = (xp[1] - yi) * one_over_dx, uz = (xp[2] - zi) * one_over_dx;
            R Nxv = bsN(ux), Nyv = bsN(uy), Nzv = bsN(uz);
            nb_w[size_t(p) * 64 + cnt] = Nxv * Nyv * Nzv;
            nb_g[size_t(p) * 64 + cnt] = V3<R>(bsdN(ux) * Nyv * Nzv * one_over_dx, Nxv * bsdN(uy) * Nzv * one_over_dx,
                                               Nxv * Nyv * bsdN(uz) * one_over_dx);
            ++cnt;
          }
    }
  }

  // True when node (i,j,k) exists; the 4x4x4 stencil's last layer carries zero weight and
  // may fall one node past the grid, which the reference reads out of range.
  inline bool inGrid(int i, int j, int k) const { return i < (int)Nx && j < (int)Ny && k < (int)Nz; }

  void P2G() {  // p2g.cpp:6-126
#pragma omp parallel num_threads(n_threads)
    {
      std::vector<V3<R>> lv(grid_nodes);
      std::vector<R> lm(grid_nodes, 0), ls(grid_nodes, 0);
      std::vector<std::array<R, 7>> ll(grid_nodes, std::array<R, 7>{});
#pragma omp for nowait
      for (long p = 0; p < (long)Np; ++p) {
        if (!active[p]) continue;
        const V3<R> xp = x[p];
        const unsigned* b = nb_base[p].data();
        int cnt = 0;
        for (unsigned i = b[0]; i < b[0] + 4; ++i)
          for (unsigned j = b[1]; j < b[1] + 4; ++j)
            for (unsigned k = b[2]; k < b[2] + 4; ++k) {
              R w = nb_w[size_t(p) * 64 + cnt];
              ++cnt;
              if (w > R(1e-25) && inGrid(i, j, k)) {
                unsigned id = ind(i, j, k);
                lm[id] += w;
                lv[id] += v[p] * w;
                for (int c = 0; c < 7; ++c) ll[id][c] += lat[p][c] * w;
                ls[id] += diffusion[p] * w;
                if (flip_ratio < 0) {
                  V3<R> pd(gx[i] - xp[0], gy[j] - xp[1], gz[k] - xp[2]);
                  lv[id] += (Bmat[p] * pd) * (apicDinverse * w);
                }
              }
            }
      }
#pragma omp critical
      {
        for (unsigned l = 0; l < grid_nodes; ++l) {
          g_mass[l] += lm[l];
          g_v[l] += lv[l];
          for (int c = 0; c < 7; ++c) g_lat[l][c] += ll[l][c];
          g_shear[l] += ls[l];
        }
      }
    }
#pragma omp parallel for num_threads(n_threads)
    for (long l = 0; l < (long)grid_nodes; ++l) {
      R mi = g_mass[l];
      if (mi > 0) {
        g_v[l] = g_v[l] * (R(1) / mi);
        for (int c = 0; c < 7; ++c) g_lat[l][c] /= mi;
        g_shear[l] /= mi;
        R s = g_lat[l][0] + g_lat[l][1] + g_lat[l][2] + g_lat[l][3];
        if (s > R(1e-6)) for (int c = 0; c < 4; ++c) g_lat[l][c] /= s;
      } else {
        g_v[l] = V3<R>();
        g_lat[l] = std::array<R, 7>{};
        g_shear[l] = 0;
      }
    }
    for (auto& m : g_mass) m *= particle_mass;
  }

  M3<R> henckyPiola(const M3<R>& Fe) const {  // simulation.hpp:287-294
    M3<R> U, V; V3<R> s;
    svd3(Fe, U, s, V);
    M3<R> D;
    R tr = 0;
    R lg[3];
    for (int i = 0; i < 3; ++i) { lg[i] = std::log(std::abs(s[i])); tr += lg[i]; }
    for (int i = 0; i < 3; ++i) D.m[i][i] = R(2) * mu * lg[i] / s[i] + lambda * tr / s[i];
    return U * D * V.T();
  }

  void boundaryCollision(V3<R> Xi, V3<R>& vi) {  // boundary_collision.cpp:5-316
    V3<R> vo = vi;
    Xi += vi * dt;
    bool infl = false;
    if (spatula_index >= 0) {
      if (objects[spatula_index].sdWorld(Xi) < R(2) * dx) infl = true;
    }
    for (size_t oi = 0; oi < objects.size(); ++oi) {
      GObject<R>& ob = objects[oi];
      if (!ob.inside(Xi)) continue;
      V3<R> vobj = ob.velocity(Xi);
      V3<R> vrel = vo - vobj;
      if (ob.bc == BC_NOSLIP) vrel = V3<R>();
      else if (ob.bc == BC_SLIPFREE) {
        V3<R> n = ob.normal(Xi);
        R dot = vrel.dot(n);
        if (dot < 0) {
          V3<R> vt = vrel - n * dot;
          if (ob.friction > 0) {
            R vtn = vt.norm();
            if (-dot * ob.friction < vtn) vrel = vt + vt * (dot * ob.friction / vtn);
            else vrel = V3<R>();
          } else vrel = vt;
        }
      } else if (ob.bc == BC_SLIPSTICK) {
        V3<R> n = ob.normal(Xi);
        R dot = vrel.dot(n);
        vrel = vrel - n * dot;
        if (dot < 0 && ob.friction > 0) {
          R vtn = vrel.norm();
          if (-dot * ob.friction < vtn) vrel = vrel + vrel * (dot * ob.friction / vtn);
          else vrel = V3<R>();
        }
      } else { error_flags |= ERR_INVALID_BC; return; }
      vi = vrel + vobj;
      if ((int)oi == spatula_index) {
        infl = true;
        if (Xi[1] < R(0.8) * dx) {
          V3<R> n = ob.normal(Xi);
          V3<R> up(0, 1, 0);
          V3<R> tv = up - n * up.dot(n);
          R tn = tv.norm();
          if (tn > R(1e-6)) tv = tv * (R(1) / tn); else tv = V3<R>();
          vi = vobj + tv * (R(0.2) * vobj.norm());
        }
      }
      vo = vi;
    }
    for (auto& pl : plates) {
      if (!pl.inside(Xi)) continue;
      if (infl && pl.type == PT_BOTTOM) {
        if (vi[1] < pl.vy) { vi[1] = pl.vy; vo = vi; }
        continue;
      }
      R vr[3] = {vo[0] - pl.vx, vo[1] - pl.vy, vo[2] - pl.vz};
      int nax = (pl.type == PT_TOP || pl.type == PT_BOTTOM) ? 1 : (pl.type == PT_LEFT || pl.type == PT_RIGHT) ? 0 : 2;
      int t0 = nax == 0 ? 1 : 0, t1 = nax == 2 ? 1 : 2;
      bool apply;
      if (pl.bc == BC_NOSLIP) { vr[0] = vr[1] = vr[2] = 0; apply = false; }
      else if (pl.bc == BC_SLIPSTICK) apply = true;
      else if (pl.bc == BC_SLIPFREE) {
        apply = (pl.type == PT_TOP && vr[1] > 0) || (pl.type == PT_BOTTOM && vr[1] < 0) ||
                (pl.type == PT_LEFT && vr[0] < 0) || (pl.type == PT_RIGHT && vr[0] > 0) ||
                (pl.type == PT_FRONT && vr[2] > 0) || (pl.type == PT_BACK && vr[2] < 0);
      } else { error_flags |= ERR_INVALID_BC; return; }
      if (apply) {
        R vel_t = std::sqrt(vr[t0] * vr[t0] + vr[t1] * vr[t1]);
        R fvn = pl.friction * std::abs(vr[nax]);
        if (pl.friction == 0) {
        } else if (vel_t <= fvn) { vr[t0] = 0; vr[t1] = 0; }
        else { R sc = (vel_t - fvn) / vel_t; vr[t0] *= sc; vr[t1] *= sc; }
        vr[nax] = 0;
      }
      vi = V3<R>(vr[0] + pl.vx, vr[1] + pl.vy, vr[2] + pl.vz);
      vo = vi;
    }
  }

  void explicitEulerUpdate() {  // explicit_euler_update.cpp:7-112
    std::vector<V3<R>> force(grid_nodes);
#pragma omp parallel for num_threads(n_threads)
    for (long p = 0; p < (long)Np; ++p) {
      if (!active[p]) continue;
      const unsigned* b = nb_base[p].data();
      M3<R> tau = henckyPiola(F[p]) * F[p].T();
      int cnt = 0;
      for (unsigned i = b[0]; i < b[0] + 4; ++i)
        for (unsigned j = b[1]; j < b[1] + 4; ++j)
          for (unsigned k = b[2]; k < b[2] + 4; ++k) {
            const V3<R>& g = nb_g[size_t(p) * 64 + cnt++];
            if (!inGrid(i, j, k)) continue;
            unsigned id = ind(i, j, k);
            if (g_mass[id] > 0) {
              V3<R> f = tau * g;
#pragma omp atomic
              force[id].c[0] += f[0];
#pragma omp atomic
              force[id].c[1] += f[1];
#pragma omp atomic
              force[id].c[2] += f[2];
            }
          }
    }
    R dtv = dt * particle_volume;
    V3<R> dtg = gravity * dt;
    g_v_update.assign(grid_nodes, V3<R>());
#pragma omp parallel for collapse(3) num_threads(n_threads)
    for (long i = 0; i < (long)Nx; ++i)
      for (long j = 0; j < (long)Ny; ++j)
        for (long k = 0; k < (long)Nz; ++k) {
          unsigned id = ind(i, j, k);
          R mi = g_mass[id];
          if (mi > 0) {
            V3<R> inc = force[id] * (-dtv / mi) + dtg;
            V3<R> old = g_v[id];
            V3<R> nv = old + inc;
            boundaryCollision(V3<R>(gx[i], gy[j], gz[k]), nv);
            g_v[id] = nv;
            g_flip[id] = nv - old;
          }
          g_v_update[id] = g_v[id];
        }
  }

  static R smoothStep(R e0, R e1, R xx) {  // g2p.cpp:7-10
    R t = std::max(R(0), std::min(R(1), (xx - e0) / (e1 - e0)));
    return t * t * (R(3) - R(2) * t);
  }

  void G2P() {  // g2p.cpp:12-135
    std::fill(pic.begin(), pic.end(), V3<R>());
    std::fill(flip.begin(), flip.end(), V3<R>());
    std::fill(Bmat.begin(), Bmat.end(), M3<R>());
#pragma omp parallel for num_threads(n_threads)
    for (long p = 0; p < (long)Np; ++p) {
      if (!active[p]) continue;
      const unsigned* b = nb_base[p].data();
      const V3<R> xp = x[p];
      V3<R> vp, fp;
      M3<R> Bp, L;
      std::array<R, 7> gl{};
      R gs = 0;
      int cnt = 0;
      for (unsigned i = b[0]; i < b[0] + 4; ++i)
        for (unsigned j = b[1]; j < b[1] + 4; ++j)
          for (unsigned k = b[2]; k < b[2] + 4; ++k) {
            R w = nb_w[size_t(p) * 64 + cnt];
            const V3<R>& g = nb_g[size_t(p) * 64 + cnt];
            ++cnt;
            if (!inGrid(i, j, k)) continue;
            unsigned id = ind(i, j, k);
            const V3<R>& gv = g_v[id];
            vp += gv * w;
            if (flip_ratio < 0) {
              V3<R> pd(gx[i] - xp[0], gy[j] - xp[1], gz[k] - xp[2]);
              for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) Bp.m[r][c] += gv[r] * pd[c] * w;
            }
            if (flip_ratio >= -1) fp += g_flip[id] * w;
            for (int r = 0; r < 3; ++r)
              for (int c = 0; c < 3; ++c) L.m[r][c] += gv[r] * g[c];
            for (int c = 0; c < 7; ++c) gl[c] += g_lat[id][c] * w;
            gs += g_shear[id] * w;
          }
      pic[p] = vp;
      if (flip_ratio < 0) Bmat[p] = Bp;
      if (flip_ratio >= -1) flip[p] = fp;
      M3<R> S = (L + L.T()) * R(0.5);
      diffusion[p] = S.frob();
      R mixf = smoothStep(D_edge0, D_edge1, gs);
      R ct = time;
      R tf = 1;
      if (ct > start_boost && end_boost > start_boost) {
        R tt = (ct - start_boost) / (end_boost - start_boost);
        tt = std::min(R(1), std::max(R(0), tt));
        tf = R(1) + tt * (boost_factor - R(1));
      }
      R dyn = D_max * tf;
      R smix = std::min(R(1), std::max(R(0), dyn * mixf * dt));
      for (int c = 0; c < 7; ++c) lat[p][c] = (R(1) - smix) * lat[p][c] + smix * gl[c];
      R s = lat[p][0] + lat[p][1] + lat[p][2] + lat[p][3];
      if (s > R(1e-6)) for (int c = 0; c < 4; ++c) lat[p][c] /= s;
    }
  }

  void velocityBlend(long p) {  // musl.cpp:13-26 / position_update.cpp:300-309
    if (flip_ratio < -1) v[p] = pic[p];
    else if (flip_ratio < 0) v[p] = (v[p] + flip[p]) * (-flip_ratio) + pic[p] * (R(1) - (-flip_ratio));
    else v[p] = (v[p] + flip[p]) * flip_ratio + pic[p] * (R(1) - flip_ratio);
  }

  void MUSL() {  // musl.cpp:6-98
#pragma omp parallel for schedule(static) num_threads(n_threads)
    for (long p = 0; p < (long)Np; ++p) {
      if (!active[p]) continue;
      velocityBlend(p);
    }
    std::fill(g_v.begin(), g_v.end(), V3<R>());
#pragma omp parallel num_threads(n_threads)
    {
      std::vector<V3<R>> lv(grid_nodes);
#pragma omp for nowait
      for (long p = 0; p < (long)Np; ++p) {
        if (!active[p]) continue;
        const V3<R> xp = x[p];
        const unsigned* b = nb_base[p].data();
        int cnt = 0;
        for (unsigned i = b[0]; i < b[0] + 4; ++i)
          for (unsigned j = b[1]; j < b[1] + 4; ++j)
            for (unsigned k = b[2]; k < b[2] + 4; ++k) {
              R w = nb_w[size_t(p) * 64 + cnt++];
              if (w > R(1e-25) && inGrid(i, j, k)) {
                unsigned id = ind(i, j, k);
                lv[id] += v[p] * w;
                if (flip_ratio < 0) {
                  V3<R> pd(gx[i] - xp[0], gy[j] - xp[1], gz[k] - xp[2]);
                  lv[id] += (Bmat[p] * pd) * (apicDinverse * w);
                }
              }
            }
      }
#pragma omp critical
      {
        for (unsigned l = 0; l < grid_nodes; ++l) g_v[l] += lv[l];
      }
    }
    for (unsigned l = 0; l < grid_nodes; ++l) {
      R mi = g_mass[l];
      if (mi > 0) g_v[l] = g_v[l] * (R(1) / (mi / particle_mass));
      else g_v[l] = V3<R>();
    }
  }

  void plasticity(long p, unsigned& pc, M3<R>& Fe) {  // plasticity.cpp:10-340
    if (plastic_model == PM_NOPLASTICITY) return;
    M3<R> U, V; V3<R> sg;
    svd3(Fe, U, sg, V);
    V3<R> h;
    for (int i = 0; i < 3; ++i) h[i] = std::log(std::max(std::abs(sg[i]), R(1e-4)));
    R htr = h[0] + h[1] + h[2];
    V3<R> hd = h - V3<R>(1, 1, 1) * (htr / R(3));
    R hdn = hd.norm();
    if (hdn > 0) hd = hd * (R(1) / hdn);
    auto rebuild = [&](const V3<R>& hh) {
      M3<R> D;
      for (int i = 0; i < 3; ++i) D.m[i][i] = std::exp(hh[i]);
      F[p] = U * D * V.T();
    };
    if (plastic_model == PM_VMVISC) {
      R q_trial = e_mu_prefac * hdn;
      R q_yield = q_min + (q_max - q_min) * std::exp(-xi * eps_pl_dev[p]);
      R p_trial = -K * htr;
      if (p_trial < p_min * std::exp(-xi * eps_pl_vol[p])) {
        R dg = q_trial / f_mu_prefac;
        F[p] = U * V.T();
        eps_pl_vol[p] += -p_trial / K;
        eps_pl_dev[p] += (R(1) / d_prefac) * dg;
        delta_gamma[p] = dg / dt;
      } else if (q_trial > q_yield) {
        ++pc;
        R dg;
        if (perzyna_exp == 1 && xi == 0) {
          dg = (q_trial - q_yield) / (f_mu_prefac + q_yield * perzyna_visc / dt);
          if (dg < 0) error_flags |= ERR_NEG_DGAMMA;
        } else {
          dg = R(0.01) * (q_trial - q_yield) / f_mu_prefac;
          const int max_iter = 60;
          for (int it = 0; it < max_iter; ++it) {
            if (it == max_iter - 1) error_flags |= ERR_NEWTON_NOCONV;
            R tm = perzyna_visc * dg + dt;
            R tmp = dt / tm;
            R tmp1 = std::pow(tmp, perzyna_exp);
            q_yield = q_min + (q_max - q_min) * std::exp(-xi * (eps_pl_dev[p] + (R(1) / d_prefac) * dg));
            R res = (q_trial - f_mu_prefac * dg) * tmp1 - q_yield;
            if (std::abs(res) < R(1e-2)) break;
            R qyd = -xi / d_prefac * (q_max - q_min) * std::exp(-xi * (eps_pl_dev[p] + (R(1) / d_prefac) * dg));
            R rd = -f_mu_prefac * tmp1 +
                   (q_trial - f_mu_prefac * dg) * perzyna_exp * std::pow(tmp, perzyna_exp - 1) * (-perzyna_visc * dt) / (tm * tm) - qyd;
            if (std::abs(rd) < R(1e-14)) error_flags |= ERR_NEWTON_FLAT;
            dg -= res / rd;
            if (dg < 0) dg = R(1e-10);
          }
        }
        h = h - hd * ((R(1) / d_prefac) * dg);
        rebuild(h);
        eps_pl_dev[p] += (R(1) / d_prefac) * dg;
        delta_gamma[p] = dg / dt;
      }
    } else if (plastic_model == PM_DPVISC) {
      R p_trial = -K * htr;
      R q_trial = e_mu_prefac * hdn;
      R p_tip = -q_cohesion / M;
      R p_shift = use_pradhana ? -K * eps_pl_vol_pradhana[p] : R(0);
      R q_yield = M * (p_trial + p_shift) + q_cohesion;
      if ((p_trial + p_shift) < p_tip) {
        R dg = d_prefac * hdn;
        R p_proj = p_tip;
        R epv = (p_proj - p_trial) / K;
        ++pc;
        V3<R> hh = V3<R>(1, 1, 1) * (-p_proj / (K * R(3)));
        rebuild(hh);
        delta_gamma[p] = dg / dt;
        eps_pl_dev[p] += (R(1) / d_prefac) * dg;
        eps_pl_vol[p] += epv;
        if (use_pradhana) eps_pl_vol_pradhana[p] += epv;
      } else {
        if (use_pradhana) eps_pl_vol_pradhana[p] = 0;
        delta_gamma[p] = 0;
      }
      if ((p_trial + p_shift) > p_tip && q_trial > q_yield) {
        ++pc;
        R dg;
        if (perzyna_exp == 1) {
          dg = (q_trial - q_yield) / (f_mu_prefac + q_yield * perzyna_visc / dt);
          if (dg < 0) error_flags |= ERR_NEG_DGAMMA;
        } else {
          dg = R(0.01) * (q_trial - q_yield) / f_mu_prefac;
          const int max_iter = 60;
          for (int it = 0; it < max_iter; ++it) {
            if (it == max_iter - 1) error_flags |= ERR_NEWTON_NOCONV;
            R tm = perzyna_visc * dg + dt;
            R tmp = dt / tm;
            R tmp1 = std::pow(tmp, perzyna_exp);
            R res = (q_trial - f_mu_prefac * dg) * tmp1 - q_yield;
            if (std::abs(res) < R(1e-2)) break;
            R rd = -f_mu_prefac * tmp1 +
                   (q_trial - f_mu_prefac * dg) * perzyna_exp * std::pow(tmp, perzyna_exp - 1) * (-perzyna_visc * dt) / (tm * tm);
            if (std::abs(rd) < R(1e-14)) error_flags |= ERR_NEWTON_FLAT;
            dg -= res / rd;
            if (dg < 0) dg = R(1e-10);
          }
        }
        h = h - hd * ((R(1) / d_prefac) * dg);
        rebuild(h);
        eps_pl_dev[p] += (R(1) / d_prefac) * dg;
        delta_gamma[p] = dg / dt;
      }
    }
  }

  void deformationUpdate() {  // deformation_update.cpp:7-52
    std::fill(delta_gamma.begin(), delta_gamma.end(), R(0));
    unsigned pc = 0;
    unsigned ef = 0;
#pragma omp parallel for reduction(+ : pc) reduction(| : ef) num_threads(n_threads)
    for (long p = 0; p < (long)Np; ++p) {
      if (!active[p]) continue;
      const unsigned* b = nb_base[p].data();
      M3<R> sum;
      int cnt = 0;
      for (unsigned i = b[0]; i < b[0] + 4; ++i)
        for (unsigned j = b[1]; j < b[1] + 4; ++j)
          for (unsigned k = b[2]; k < b[2] + 4; ++k) {
            const V3<R>& g = nb_g[size_t(p) * 64 + cnt++];
            if (!inGrid(i, j, k)) continue;
            const V3<R>& gv = g_v[ind(i, j, k)];
            for (int r = 0; r < 3; ++r)
              for (int c = 0; c < 3; ++c) sum.m[r][c] += gv[r] * g[c];
          }
      M3<R> Fe = F[p];
      Fe = Fe + (sum * Fe) * dt;
      F[p] = Fe;
      unsigned pcl = 0;
      plasticity(p, pcl, Fe);
      pc += pcl;
    }
    plastic_count = pc;
    error_flags |= ef;
  }

  void positionUpdate() {  // position_update.cpp:6-91
    unsigned ef = 0;
#pragma omp parallel for schedule(static) reduction(| : ef) num_threads(n_threads)
    for (long p = 0; p < (long)Np; ++p) {
      if (!active[p]) continue;
      x[p] = x[p] + pic[p] * dt;
      if (!use_musl) velocityBlend(p);
      bool bad = false;
      for (int d = 0; d < 3; ++d)
        if (std::isnan(x[p][d]) || std::isinf(x[p][d]) || std::isnan(v[p][d]) || std::isinf(v[p][d])) bad = true;
      if (bad) {
        active[p] = 0;
        for (int d = 0; d < 3; ++d) { v[p][d] = 0; x[p][d] = use_particle_boundaries ? particle_boundary_min[d] : R(0); }
        ef |= ERR_NAN_PARTICLE;
        continue;
      }
      if (x[p][1] < 0) { x[p][1] = 0; if (v[p][1] < 0) v[p][1] = 0; }
      if (use_particle_boundaries) {
        for (int d = 0; d < 3; ++d) {
          if (x[p][d] < particle_boundary_min[d]) { x[p][d] = particle_boundary_min[d]; active[p] = 0; v[p][d] = 0; }
          else if (x[p][d] > particle_boundary_max[d]) { x[p][d] = particle_boundary_max[d]; active[p] = 0; v[p][d] = 0; }
        }
        if (!active[p]) v[p] = V3<R>();
      }
    }
    error_flags |= ef;
  }

  void moveObjects() {  // simulation.cpp:284-291
    for (auto& pl : plates) pl.move(dt, frame_dt, time);
    if (spatula_index >= 0) objects[spatula_index].move(dt);
  }

  void advanceStep() {  // simulation.cpp:225-280 (pbc off)
    updateDt();
    if (step_count == 0) remeshInit(); else remeshCont();
    resizeGrid();
    precomputeWeights();
    P2G();
    explicitEulerUpdate();
    G2P();
    if (use_musl) MUSL();
    deformationUpdate();
    positionUpdate();
    moveObjects();
  }

  void step() {  // simulation_units.cpp:217-233
    advanceStep();
    time += dt;
    ++step_count;
  }
  bool frameFinished() {  // simulation_units.cpp:235-241
    if (frame_dt * R(frame + 1) - time < min_dt * R(1.1)) { ++frame; return true; }
    return false;
  }
  bool isFinished() const { return frame >= end_frame || time >= final_time; }
};

}  // namespace oracle

// ---------------------------------------------------------------------------------------
// C ABI (ctypes).  Names mirror the product's pm_* calls with a pmo_ prefix.
// ---------------------------------------------------------------------------------------
using namespace oracle;

struct pmo_sim {
  int prec;
  Sim<float>* f = nullptr;
  Sim<double>* d = nullptr;
};

template <class Fn> static auto dispatch(pmo_sim* h, Fn fn) {
  if (h->prec == 32) return fn(*h->f);
  return fn(*h->d);
}

template <class R> static int setParam(Sim<R>& s, const char* n, double v) {
  std::string k(n);
#define P(name, field) if (k == name) { s.field = (decltype(s.field))v; return 0; }
  P("n_threads", n_threads) P("end_frame", end_frame) P("frame", frame)
  if (k == "use_musl") { s.use_musl = s.use_musl_user = v != 0; return 0; }
  P("use_particle_boundaries", use_particle_boundaries) P("use_pradhana", use_pradhana) P("min_dt", min_dt)
  P("fps", fps) P("cfl", cfl) P("cfl_elastic", cfl_elastic) P("flip_ratio", flip_ratio) P("rho", rho) P("E", E)
  P("nu", nu) P("xi", xi) P("q_max", q_max) P("q_min", q_min) P("p_min", p_min) P("M", M)
  P("q_cohesion", q_cohesion) P("perzyna_exp", perzyna_exp) P("perzyna_visc", perzyna_visc)
  P("q_prefac", q_prefac) P("pigment_D_max", D_max) P("pigment_D_edge0", D_edge0) P("pigment_D_edge1", D_edge1)
  P("start_boost_time", start_boost) P("end_boost_time", end_boost) P("boost_factor", boost_factor)
  P("plastic_model", plastic_model) P("particle_mass", particle_mass) P("particle_volume", particle_volume)
  P("dx", dx)
#undef P
  return 1;
}
template <class R> static int getParam(Sim<R>& s, const char* n, double* out) {
  std::string k(n);
#define G(name, expr) if (k == name) { *out = (double)(expr); return 0; }
  G("time", s.time) G("dt", s.dt) G("frame", s.frame) G("step", s.step_count) G("dx", s.dx) G("Np", s.Np)
  G("particle_mass", s.particle_mass) G("particle_volume", s.particle_volume) G("plastic_count", s.plastic_count)
  G("error_flags", s.error_flags) G("mu", s.mu) G("lambda", s.lambda) G("K", s.K) G("dt_max", s.dt_max)
  G("frame_dt", s.frame_dt) G("final_time", s.final_time) G("Nx", s.Nx) G("Ny", s.Ny) G("Nz", s.Nz)
  G("flip_ratio", s.flip_ratio) G("use_musl", s.use_musl) G("end_frame", s.end_frame)
#undef G
  return 1;
}

extern "C" {

pmo_sim* pmo_create(int precision) {
  pmo_sim* h = new pmo_sim();
  h->prec = precision == 32 ? 32 : 64;
  if (h->prec == 32) h->f = new Sim<float>(); else h->d = new Sim<double>();
  return h;
}
void pmo_destroy(pmo_sim* h) {
  if (!h) return;
  delete h->f; delete h->d; delete h;
}
int pmo_set_param(pmo_sim* h, const char* name, double v) {
  return dispatch(h, [&](auto& s) { return setParam(s, name, v); });
}
int pmo_get_param(pmo_sim* h, const char* name, double* out) {
  return dispatch(h, [&](auto& s) { return getParam(s, name, out); });
}
int pmo_set_param3(pmo_sim* h, const char* name, const double* v3) {
  return dispatch(h, [&](auto& s) {
    using R = std::decay_t<decltype(s.dx)>;
    std::string k(name);
    V3<R> v((R)v3[0], (R)v3[1], (R)v3[2]);
    if (k == "gravity") s.gravity = v;
    else if (k == "particle_boundary_min") s.particle_boundary_min = v;
    else if (k == "particle_boundary_max") s.particle_boundary_max = v;
    else if (k == "grid_reference_point") s.grid_reference_point = v;
    else return 1;
    return 0;
  });
}
// x: n*3, latent: n*7, v: n*3 or null.  Positions and latents are given in float.
int pmo_set_particles(pmo_sim* h, unsigned n, const float* x, const float* latent, const float* v) {
  return dispatch(h, [&](auto& s) {
    using R = std::decay_t<decltype(s.dx)>;
    s.resizeParticles(n);
    for (unsigned p = 0; p < n; ++p) {
      for (int d = 0; d < 3; ++d) s.x[p][d] = (R)x[3 * p + d];
      if (v) for (int d = 0; d < 3; ++d) s.v[p][d] = (R)v[3 * p + d];
      if (latent) for (int c = 0; c < 7; ++c) s.lat[p][c] = (R)latent[7 * p + c];
    }
    return 0;
  });
}
int pmo_add_plate(pmo_sim* h, double pos, int type, int bc, double friction, double lower, double upper, double vx,
                  double vy, double vz, double vmin_factor, double load_factor) {
  return dispatch(h, [&](auto& s) {
    using R = std::decay_t<decltype(s.dx)>;
    Plate<R> p;
    p.pos = (R)pos; p.type = type; p.bc = bc; p.friction = (R)friction; p.lower = (R)lower; p.upper = (R)upper;
    p.vx = p.vx0 = (R)vx; p.vy = p.vy0 = (R)vy; p.vz = p.vz0 = (R)vz;
    p.vmin_factor = (R)vmin_factor; p.load_factor = (R)load_factor;
    s.plates.push_back(p);
    return 0;
  });
}
// frames: n*7 floats (pos xyz, quat xyzw) as in spatula_motion.bin
int pmo_add_spatula(pmo_sim* h, int bc, double friction, const float* frames, unsigned n) {
  return dispatch(h, [&](auto& s) {
    using R = std::decay_t<decltype(s.dx)>;
    GObject<R> o;
    o.kind = OBJ_SPATULA; o.bc = bc; o.friction = (R)friction;
    o.frames.assign(frames, frames + size_t(n) * 7);
    if (n > 0) o.setPose(V3<R>(frames[0], frames[1], frames[2]), Quat<R>{R(frames[6]), R(frames[3]), R(frames[4]), R(frames[5])});
    else o.setPose(V3<R>(), Quat<R>{1, 0, 0, 0});
    s.objects.push_back(o);
    s.spatula_index = (int)s.objects.size() - 1;
    return 0;
  });
}
// half: 3, waypoints: n*3, quat: orientation (w, x, y, z)
int pmo_add_box_knife(pmo_sim* h, int bc, double friction, const double* half, const double* waypoints, unsigned n,
                      double speed, const double* quat_wxyz) {
  return dispatch(h, [&](auto& s) {
    using R = std::decay_t<decltype(s.dx)>;
    GObject<R> o;
    o.kind = OBJ_BOXKNIFE; o.bc = bc; o.friction = (R)friction;
    o.half = V3<R>((R)half[0], (R)half[1], (R)half[2]);
    for (unsigned i = 0; i < n; ++i) o.path.push_back(V3<R>((R)waypoints[3 * i], (R)waypoints[3 * i + 1], (R)waypoints[3 * i + 2]));
    o.speed = (R)speed;
    Quat<R> q{1, 0, 0, 0};
    if (quat_wxyz) q = Quat<R>{(R)quat_wxyz[0], (R)quat_wxyz[1], (R)quat_wxyz[2], (R)quat_wxyz[3]};
    o.setPose(n > 0 ? o.path[0] : V3<R>(), q);
    s.objects.push_back(o);
    s.spatula_index = (int)s.objects.size() - 1;
    return 0;
  });
}
int pmo_add_ground(pmo_sim* h, int bc, double friction, double y0) {
  return dispatch(h, [&](auto& s) {
    using R = std::decay_t<decltype(s.dx)>;
    GObject<R> o; o.kind = OBJ_GROUND; o.bc = bc; o.friction = (R)friction; o.y0 = (R)y0;
    o.setPose(V3<R>(), Quat<R>{1, 0, 0, 0});
    s.objects.push_back(o);
    return 0;
  });
}
int pmo_add_curve(pmo_sim* h, int bc, double friction) {
  return dispatch(h, [&](auto& s) {
    using R = std::decay_t<decltype(s.dx)>;
    GObject<R> o; o.kind = OBJ_CURVE; o.bc = bc; o.friction = (R)friction;
    o.setPose(V3<R>(), Quat<R>{1, 0, 0, 0});
    s.objects.push_back(o);
    return 0;
  });
}
int pmo_prepare(pmo_sim* h) { return dispatch(h, [&](auto& s) { s.prepare(); return 0; }); }
int pmo_step(pmo_sim* h, unsigned nsteps) {
  return dispatch(h, [&](auto& s) { for (unsigned i = 0; i < nsteps; ++i) s.step(); return 0; });
}
// nsteps of (step; frameFinished) -- the render-loop idiom; returns frames finished
int pmo_advance(pmo_sim* h, unsigned nsteps, unsigned* frames_done) {
  return dispatch(h, [&](auto& s) {
    unsigned fd = 0;
    for (unsigned i = 0; i < nsteps; ++i) { s.step(); if (s.frameFinished()) ++fd; }
    if (frames_done) *frames_done = fd;
    return 0;
  });
}
// The reference's offline driver: simulation.cpp:339-474 (simulate) after prepare-style setup,
// run until end_frame, USL unless use_musl was set.
int pmo_simulate(pmo_sim* h) {
  return dispatch(h, [&](auto& s) {
    using R = std::decay_t<decltype(s.dx)>;
    s.prepare();
    s.use_musl = s.use_musl_user;
    while (s.frame < s.end_frame) {
      s.advanceStep();
      s.time += s.dt;
      ++s.step_count;
      if (s.frame_dt * R(s.frame + 1) - s.time < s.min_dt * R(1.1)) ++s.frame;
      if (std::abs(s.final_time - s.time) < s.min_dt * R(1.1) || s.final_time < s.time) break;
    }
    return 0;
  });
}
int pmo_frame_finished(pmo_sim* h, int* out) { return dispatch(h, [&](auto& s) { *out = s.frameFinished(); return 0; }); }
int pmo_is_finished(pmo_sim* h, int* out) { return dispatch(h, [&](auto& s) { *out = s.isFinished(); return 0; }); }
int pmo_get_grid_boundaries(pmo_sim* h, double* lo, double* hi) {
  return dispatch(h, [&](auto& s) { for (int d = 0; d < 3; ++d) { lo[d] = s.low[d]; hi[d] = s.high[d]; } return 0; });
}
// Any output pointer may be null.  F and B are row-major 3x3 per particle.
int pmo_get_particles(pmo_sim* h, float* x, float* v, float* latent, float* diffusion, unsigned char* active,
                      float* F, float* B, float* plastic4) {
  return dispatch(h, [&](auto& s) {
    for (unsigned p = 0; p < s.Np; ++p) {
      if (x) for (int d = 0; d < 3; ++d) x[3 * p + d] = (float)s.x[p][d];
      if (v) for (int d = 0; d < 3; ++d) v[3 * p + d] = (float)s.v[p][d];
      if (latent) for (int c = 0; c < 7; ++c) latent[7 * p + c] = (float)s.lat[p][c];
      if (diffusion) diffusion[p] = (float)s.diffusion[p];
      if (active) active[p] = s.active[p] ? 1 : 0;
      if (F) for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) F[9 * p + 3 * r + c] = (float)s.F[p].m[r][c];
      if (B) for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) B[9 * p + 3 * r + c] = (float)s.Bmat[p].m[r][c];
      if (plastic4) {
        plastic4[4 * p + 0] = (float)s.eps_pl_dev[p];
        plastic4[4 * p + 1] = (float)s.eps_pl_vol[p];
        plastic4[4 * p + 2] = (float)s.eps_pl_vol_pradhana[p];
        plastic4[4 * p + 3] = (float)s.delta_gamma[p];
      }
    }
    return 0;
  });
}
// Double-precision readback of positions, velocities and latents.
int pmo_get_particles_f64(pmo_sim* h, double* x, double* v, double* latent) {
  return dispatch(h, [&](auto& s) {
    for (unsigned p = 0; p < s.Np; ++p) {
      if (x) for (int d = 0; d < 3; ++d) x[3 * p + d] = (double)s.x[p][d];
      if (v) for (int d = 0; d < 3; ++d) v[3 * p + d] = (double)s.v[p][d];
      if (latent) for (int c = 0; c < 7; ++c) latent[7 * p + c] = (double)s.lat[p][c];
    }
    return 0;
  });
}
// Grid after the last step: node coordinates of (0,0,0), dims, and per node mass, the
// velocity after the grid update (before MUSL), the final grid velocity (after MUSL when on),
// flip, latent (7) and shear intensity.
int pmo_get_grid(pmo_sim* h, double* origin3, unsigned* dims3, float* mass, float* v_update, float* v_final,
                 float* flip, float* latent, float* shear) {
  return dispatch(h, [&](auto& s) {
    origin3[0] = s.low[0]; origin3[1] = s.low[1]; origin3[2] = s.low[2];
    dims3[0] = s.Nx; dims3[1] = s.Ny; dims3[2] = s.Nz;
    for (unsigned l = 0; l < s.grid_nodes; ++l) {
      if (mass) mass[l] = (float)s.g_mass[l];
      if (v_update) for (int d = 0; d < 3; ++d) v_update[3 * l + d] = l < s.g_v_update.size() ? (float)s.g_v_update[l][d] : 0.f;
      if (v_final) for (int d = 0; d < 3; ++d) v_final[3 * l + d] = (float)s.g_v[l][d];
      if (flip) for (int d = 0; d < 3; ++d) flip[3 * l + d] = (float)s.g_flip[l][d];
      if (latent) for (int c = 0; c < 7; ++c) latent[7 * l + c] = (float)s.g_lat[l][c];
      if (shear) shear[l] = (float)s.g_shear[l];
    }
    return 0;
  });
}
// Knife pose: world->local affine (row-major 4x4), linear and angular velocity.
int pmo_get_knife(pmo_sim* h, double* inv4x4, double* vlin, double* omega) {
  return dispatch(h, [&](auto& s) {
    if (s.spatula_index < 0) return 1;
    auto& o = s.objects[s.spatula_index];
    auto tl = o.Rinv * o.t;
    for (int r = 0; r < 3; ++r) {
      for (int c = 0; c < 3; ++c) inv4x4[4 * r + c] = o.Rinv.m[r][c];
      inv4x4[4 * r + 3] = -tl[r];
    }
    inv4x4[12] = inv4x4[13] = inv4x4[14] = 0; inv4x4[15] = 1;
    for (int d = 0; d < 3; ++d) { vlin[d] = o.vlin[d]; omega[d] = o.omega[d]; }
    return 0;
  });
}
// Direct access to the restated pieces for unit tests.
void pmo_svd3(const double* A, double* U, double* s, double* V) {
  M3<double> a, u, vv; V3<double> sv;
  for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) a.m[r][c] = A[3 * r + c];
  svd3(a, u, sv, vv);
  for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) { U[3 * r + c] = u.m[r][c]; V[3 * r + c] = vv.m[r][c]; }
  for (int i = 0; i < 3; ++i) s[i] = sv[i];
}
double pmo_sd_spatula(const double* p) {
  GObject<double> o; V3<double> q(p[0], p[1], p[2]);
  return o.sdSpatula(q);
}
void pmo_slerp(const double* q0_wxyz, const double* q1_wxyz, double t, double* out_wxyz) {
  Quat<double> a{q0_wxyz[0], q0_wxyz[1], q0_wxyz[2], q0_wxyz[3]}, b{q1_wxyz[0], q1_wxyz[1], q1_wxyz[2], q1_wxyz[3]};
  Quat<double> r = slerp(a, b, t);
  out_wxyz[0] = r.w; out_wxyz[1] = r.x; out_wxyz[2] = r.y; out_wxyz[3] = r.z;
}

}  // extern "C"
