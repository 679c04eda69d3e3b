// Device element math for the implicit step, templated on the real type (float for the
// FP32 path, double where the mixed-precision path asks for FP64). Each function restates
// the reference function named beside it in the same operation order; the translation
// unit that includes this header is compiled without FMA contraction so FP32 results
// round like the reference's scalar f32 code.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace mg {

template <class R>
struct V3 {
  R x, y, z;
  __host__ __device__ V3() : x(0), y(0), z(0) {}
  __host__ __device__ V3(R a, R b, R c) : x(a), y(b), z(c) {}
  __host__ __device__ R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  __host__ __device__ R& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  __host__ __device__ V3 operator+(const V3& o) const { return V3(x + o.x, y + o.y, z + o.z); }
  __host__ __device__ V3 operator-(const V3& o) const { return V3(x - o.x, y - o.y, z - o.z); }
  __host__ __device__ V3 operator-() const { return V3(-x, -y, -z); }
  __host__ __device__ V3 operator*(R s) const { return V3(x * s, y * s, z * s); }
  __host__ __device__ V3 operator/(R s) const { return V3(x / s, y / s, z / s); }
  __host__ __device__ V3& operator+=(const V3& o) { x += o.x; y += o.y; z += o.z; return *this; }
  __host__ __device__ R dot(const V3& o) const { return x * o.x + y * o.y + z * o.z; }
  __host__ __device__ V3 cross(const V3& o) const { return V3(y * o.z - o.y * z, z * o.x - o.z * x, x * o.y - o.x * y); }
  __host__ __device__ R length_squared() const { return dot(*this); }
  __host__ __device__ R length() const { return sqrt(dot(*this)); }
  __host__ __device__ V3 normalize() const { return (*this) * (R(1) / length()); }
  __host__ __device__ V3 normalize_or(const V3& fb) const {
    R rcp = R(1) / length();
    if (isfinite(rcp) && rcp > R(0)) return (*this) * rcp;
    return fb;
  }
  __host__ __device__ V3 normalize_or_zero() const { return normalize_or(V3()); }
  template <class S>
  __host__ __device__ V3<S> cast() const { return V3<S>(S(x), S(y), S(z)); }
};

template <class R> __host__ __device__ inline R rmax(R a, R b) { return fmax(a, b); }
template <class R> __host__ __device__ inline R rmin(R a, R b) { return fmin(a, b); }
template <> __host__ __device__ inline float rmax<float>(float a, float b) { return fmaxf(a, b); }
template <> __host__ __device__ inline float rmin<float>(float a, float b) { return fminf(a, b); }
template <class R> __host__ __device__ inline R rclamp(R v, R lo, R hi) { return v < lo ? lo : (v > hi ? hi : v); }

template <class R>
__device__ inline V3<R> ld3(const float* p, uint32_t i) {
  return V3<R>((R)p[3 * i], (R)p[3 * i + 1], (R)p[3 * i + 2]);
}

// ---------------------------------------------------------------------------------------
// contact.rs
// ---------------------------------------------------------------------------------------
// closest_point_on_triangle_bary (contact.rs:84-124)
template <class R>
__device__ inline V3<R> closest_point_bary(const V3<R>& p, const V3<R>& a, const V3<R>& b, const V3<R>& c, R w[3]) {
  V3<R> ab = b - a, ac = c - a, ap = p - a;
  R d1 = ab.dot(ap), d2 = ac.dot(ap);
  if (d1 <= 0 && d2 <= 0) { w[0] = 1; w[1] = 0; w[2] = 0; return a; }
  V3<R> bp = p - b;
  R d3 = ab.dot(bp), d4 = ac.dot(bp);
  if (d3 >= 0 && d4 <= d3) { w[0] = 0; w[1] = 1; w[2] = 0; return b; }
  R vc = d1 * d4 - d3 * d2;
  if (vc <= 0 && d1 >= 0 && d3 <= 0) {
    R den = d1 - d3;
    R v = den != 0 ? d1 / den : R(0);
    w[0] = R(1) - v; w[1] = v; w[2] = 0;
    return a + ab * v;
  }
  V3<R> cp = p - c;
  R d5 = ab.dot(cp), d6 = ac.dot(cp);
  if (d6 >= 0 && d5 <= d6) { w[0] = 0; w[1] = 0; w[2] = 1; return c; }
  R vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) {
    R den = d2 - d6;
    R ww = den != 0 ? d2 / den : R(0);
    w[0] = R(1) - ww; w[1] = 0; w[2] = ww;
    return a + ac * ww;
  }
  R va = d3 * d6 - d5 * d4;
  if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
    R den = (d4 - d3) + (d5 - d6);
    R ww = den != 0 ? (d4 - d3) / den : R(0);
    w[0] = 0; w[1] = R(1) - ww; w[2] = ww;
    return b + (c - b) * ww;
  }
  R den = va + vb + vc;
  if (den == 0) { w[0] = 1; w[1] = 0; w[2] = 0; return a; }
  R denom = R(1) / den;
  R v = vb * denom, ww = vc * denom;
  w[0] = R(1) - v - ww; w[1] = v; w[2] = ww;
  return a + ab * v + ac * ww;
}

template <class R>
__device__ inline R point_triangle_distance(const V3<R>& p, const V3<R>& a, const V3<R>& b, const V3<R>& c) {
  R w[3];
  return (p - closest_point_bary(p, a, b, c, w)).length();
}

// point_tri_distance_grad (contact.rs:836-857); `inside` negates (contact.rs:889-915)
template <class R>
__device__ inline R point_tri_distance_grad(const V3<R>& p, const V3<R>& a, const V3<R>& b, const V3<R>& c, bool inside,
                                            V3<R> g[4]) {
  R w[3];
  V3<R> q = closest_point_bary(p, a, b, c, w);
  V3<R> e = p - q;
  R d = e.length();
  if (d < R(1.0e-12)) {
    for (int k = 0; k < 4; ++k) g[k] = V3<R>();
    return inside ? -d : d;
  }
  V3<R> n = e / d;
  g[0] = n;
  g[1] = n * (-w[0]);
  g[2] = n * (-w[1]);
  g[3] = n * (-w[2]);
  if (inside) {
    for (int k = 0; k < 4; ++k) g[k] = -g[k];
    return -d;
  }
  return d;
}

template <class R>
__device__ inline void point_edge_coeff(const V3<R>& p, const V3<R>& e0, const V3<R>& e1, R out[2]) {
  V3<R> r = e1 - e0;
  R d = r.dot(r);
  if (d > 0) {
    R t = r.dot(p - e0) / d;
    out[0] = R(1) - t;
    out[1] = t;
  } else {
    out[0] = R(0.5);
    out[1] = R(0.5);
  }
}

// edge_edge_witness (contact.rs:238-311)
template <class R>
__device__ inline void edge_edge_witness(const V3<R>& ea0, const V3<R>& ea1, const V3<R>& eb0, const V3<R>& eb1, R out[4]) {
  V3<R> cog = (ea0 + ea1 + eb0 + eb1) * R(0.25);
  V3<R> a0 = ea0 - cog, a1 = ea1 - cog, b0v = eb0 - cog, b1v = eb1 - cog;
  auto dist2 = [&](const R c[4]) {
    V3<R> x0 = a0 * c[0] + a1 * c[1];
    V3<R> x1 = b0v * c[2] + b1v * c[3];
    return (x1 - x0).length_squared();
  };
  R pe[2];
  point_edge_coeff(ea0, eb0, eb1, pe);
  R cls[4] = {1, 0, pe[0], pe[1]};
  V3<R> r0 = ea1 - ea0, r1 = eb1 - eb0;
  R a00 = r0.dot(r0), a01 = -r0.dot(r1), a11 = r1.dot(r1);
  V3<R> rhs = eb0 - ea0;
  R b0 = r0.dot(rhs), b1 = -r1.dot(rhs);
  R det = a00 * a11 - a01 * a01;
  if (det != 0) {
    R sp = (a11 * b0 - a01 * b1) / det;
    R tp = (a00 * b1 - a01 * b0) / det;
    R direct[4] = {R(1) - sp, sp, R(1) - tp, tp};
    if (dist2(direct) < dist2(cls))
      for (int k = 0; k < 4; ++k) cls[k] = direct[k];
  }
  bool in01 = true;
  for (int k = 0; k < 4; ++k)
    if (!(cls[k] >= 0 && cls[k] <= 1)) in01 = false;
  if (in01) {
    for (int k = 0; k < 4; ++k) out[k] = cls[k];
    return;
  }
  auto snap = [](R c[2]) {
    if (c[0] < 0) { c[0] = 0; c[1] = 1; }
    else if (c[0] > 1) { c[0] = 1; c[1] = 0; }
  };
  R c1[2], c2[2], c3[2], c4[2];
  point_edge_coeff(ea0, eb0, eb1, c1); snap(c1);
  point_edge_coeff(ea1, eb0, eb1, c2); snap(c2);
  point_edge_coeff(eb0, ea0, ea1, c3); snap(c3);
  point_edge_coeff(eb1, ea0, ea1, c4); snap(c4);
  R types[4][4] = {{1, 0, c1[0], c1[1]}, {0, 1, c2[0], c2[1]}, {c3[0], c3[1], 1, 0}, {c4[0], c4[1], 0, 1}};
  int best = 0;
  R best_d = R(INFINITY);
  for (int k = 0; k < 4; ++k) {
    R d = dist2(types[k]);
    if (d < best_d) { best_d = d; best = k; }
  }
  for (int k = 0; k < 4; ++k) out[k] = types[best][k];
}

// segment_segment_distance (contact.rs:439-487)
template <class R>
__device__ inline R segment_segment_distance(const V3<R>& p1, const V3<R>& q1, const V3<R>& p2, const V3<R>& q2) {
  V3<R> d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
  R a = d1.dot(d1), e = d2.dot(d2), f = d2.dot(r);
  const R EPS = R(1.0e-12);
  R s, t;
  if (a <= EPS && e <= EPS) return (p1 - p2).length();
  if (a <= EPS) {
    s = 0;
    t = rclamp(f / e, R(0), R(1));
  } else {
    R c = d1.dot(r);
    if (e <= EPS) {
      t = 0;
      s = rclamp(-c / a, R(0), R(1));
    } else {
      R b = d1.dot(d2);
      R denom = a * e - b * b;
      R s0 = denom > EPS ? rclamp((b * f - c * e) / denom, R(0), R(1)) : R(0);
      R t0 = (b * s0 + f) / e;
      if (t0 < 0) {
        t = 0;
        s = rclamp(-c / a, R(0), R(1));
      } else if (t0 > 1) {
        t = 1;
        s = rclamp((b - c) / a, R(0), R(1));
      } else {
        s = s0;
        t = t0;
      }
    }
  }
  V3<R> c1 = p1 + d1 * s, c2 = p2 + d2 * t;
  return (c1 - c2).length();
}

// segment_segment_distance_grad (contact.rs:489-518)
template <class R>
__device__ inline R segment_segment_distance_grad(const V3<R>& p1, const V3<R>& q1, const V3<R>& p2, const V3<R>& q2,
                                                  V3<R> g[4]) {
  R w[4];
  edge_edge_witness(p1, q1, p2, q2, w);
  V3<R> ca = p1 * w[0] + q1 * w[1];
  V3<R> cb = p2 * w[2] + q2 * w[3];
  V3<R> e = ca - cb;
  R d = e.length();
  if (d < R(1.0e-12)) {
    for (int k = 0; k < 4; ++k) g[k] = V3<R>();
    return d;
  }
  V3<R> n = e / d;
  g[0] = n * w[0];
  g[1] = n * w[1];
  g[2] = n * (-w[2]);
  g[3] = n * (-w[3]);
  return d;
}

// accd_toi (contact.rs:378-437); kind 0 = point-triangle, 1 = edge-edge squared distance.
template <class R>
__device__ inline R accd_toi(const V3<R> x0[4], const V3<R> dx[4], R offset, R max_t, R reduction, uint32_t max_iter,
                             int kind, bool* hit_cap) {
  *hit_cap = false;
  auto sq = [&](const V3<R> p[4]) {
    R d = kind == 0 ? point_triangle_distance(p[0], p[1], p[2], p[3]) : segment_segment_distance(p[0], p[1], p[2], p[3]);
    return d * d;
  };
  R u_max = 0;
  for (int i = 0; i < 4; ++i)
    for (int j = i + 1; j < 4; ++j) u_max = rmax(u_max, (dx[i] - dx[j]).length());
  if (u_max < R(1.0e-12)) return max_t;
  R inv_u_max = R(1) / u_max;
  R d0 = sqrt(rmax(sq(x0), R(0)));
  R eps = reduction * (d0 - offset);
  if (eps <= 0) return max_t;
  R target = eps + offset;
  R eps_sqr = eps * eps;
  R toi = 0;
  V3<R> moved[4];
  uint32_t it = 0;
  for (; it < max_iter; ++it) {
    for (int k = 0; k < 4; ++k) moved[k] = x0[k] + dx[k] * toi;
    R d2 = rmax(sq(moved), R(0));
    R dmt = (d2 - target * target) / (sqrt(d2) + target);
    if ((max_t - toi) * u_max < dmt - eps) return max_t;
    if (toi > 0 && dmt * dmt < eps_sqr) break;
    R toi_next = toi + dmt * inv_u_max;
    if (toi_next != toi)
      toi = toi_next;
    else
      break;
    if (toi > max_t) return max_t;
  }
  if (it == max_iter) *hit_cap = true;
  return rmax(toi, R(0));
}

// barrier (contact.rs:1014-1027) / cubic_barrier (:580-592) via barrier_of (:723-730)
template <class R>
__device__ inline bool barrier_of(int kind, R d, R dhat, R kappa, R& g, R& h) {
  if (kind == 0) {
    if (d >= dhat) return false;
    d = rmax(d, R(1.0e-6));
    R t = d - dhat;
    R ld = log(d / dhat);
    g = -kappa * (R(2) * t * ld + t * t / d);
    h = -kappa * (R(2) * ld + R(4) * t / d - (t * t) / (d * d));
    return true;
  }
  R y = d - dhat;
  if (y >= 0) return false;
  g = kappa * (R(-2) * y * y / dhat);
  h = kappa * (R(4) * (R(1) - d / dhat));
  return true;
}

// rayleigh_stiffness (contact.rs:750-834) for n <= 4 participants.
template <class R>
__device__ inline R rayleigh_stiffness(const R (*elastic)[9], const R* mass, const R* weights, int n, const V3<R>& e) {
  R g = e.length();
  if (g <= 0 || n == 0) return 0;
  R sqr_x = g * g;
  R m_max = 0;
  for (int i = 0; i < n; ++i) m_max = rmax(m_max, mass[i]);
  R w[12];
  for (int ii = 0; ii < n; ++ii) {
    V3<R> v = e * weights[ii];
    w[3 * ii] = v.x;
    w[3 * ii + 1] = v.y;
    w[3 * ii + 2] = v.z;
  }
  R ss = 0;
  for (int k = 0; k < 3 * n; ++k) ss += w[k] * w[k];
  R norm = sqrt(ss);
  if (norm <= 0) return 0;
  for (int k = 0; k < 3 * n; ++k) w[k] /= norm;
  R acc = 0;
  for (int ii = 0; ii < n; ++ii) {
    R m_ii = mass[ii] > 0 ? mass[ii] : m_max;
    for (int jj = 0; jj < n; ++jj) {
      const R* blk = elastic[ii * n + jj];
      for (int r = 0; r < 3; ++r) {
        R row = 0;
        for (int c = 0; c < 3; ++c) {
          R v = blk[3 * r + c];
          if (ii == jj && r == c) v += m_ii / sqr_x;
          row += v * w[3 * jj + c];
        }
        acc += w[3 * ii + r] * row;
      }
    }
  }
  return acc;
}

// friction (contact.rs:613-644)
template <class R>
__device__ inline bool friction(const V3<R>& force_contact, const V3<R>& dx, const V3<R>& normal, R mu, R min_dx,
                                V3<R>& grad, R hess[9]) {
  if (mu <= 0) return false;
  R contact = -normal.dot(force_contact);
  V3<R> pdx = dx - normal * normal.dot(dx);
  R eps = rmax(min_dx, R(1.0e-12));
  R denom = rmax(pdx.length(), eps);
  R lambda = mu * contact / denom;
  if (lambda <= 0) return false;
  grad = pdx * lambda;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) hess[3 * r + c] = lambda * ((r == c ? R(1) : R(0)) - normal[r] * normal[c]);
  return true;
}

// surface_normal_at (contact.rs:935-942)
template <class R>
__device__ inline V3<R> surface_normal_at(const R bary[3], const V3<R>& face, const V3<R> pn[3]) {
  if (bary[0] > R(1.0e-4) && bary[1] > R(1.0e-4) && bary[2] > R(1.0e-4)) return face;
  return (pn[0] * bary[0] + pn[1] * bary[1] + pn[2] * bary[2]).normalize_or_zero();
}

// ---------------------------------------------------------------------------------------
// shell_model.rs (StVK)
// ---------------------------------------------------------------------------------------
template <class R>
struct M2 {  // glam column-major: x_axis = (xx, xy), y_axis = (yx, yy)
  R xx, xy, yx, yy;
  __device__ M2 transpose() const { return M2{xx, yx, xy, yy}; }
  __device__ R at(int r, int c) const { return c == 0 ? (r == 0 ? xx : xy) : (r == 0 ? yx : yy); }
};

template <class R>
struct M32 {
  V3<R> c0, c1;
  __device__ M32 mul(const M2<R>& m) const { return M32{c0 * m.xx + c1 * m.xy, c0 * m.yx + c1 * m.yy}; }
};

// sym_eig2 (shell_model.rs:60-78)
template <class R>
__device__ inline void sym_eig2(R p, R q, R r, R lam[2], M2<R>& v) {
  R tr = p + r;
  R diff = sqrt(rmax((p - r) * (p - r) + R(4) * q * q, R(0)));
  R l0 = R(0.5) * (tr + diff), l1 = R(0.5) * (tr - diff);
  R v0x, v0y;
  if (fabs(q) > R(1.0e-20)) {
    R x = q, y = l0 - p;
    R rcp = R(1) / sqrt(x * x + y * y);
    if (isfinite(rcp) && rcp > 0) {
      v0x = x * rcp;
      v0y = y * rcp;
    } else {
      v0x = 1;
      v0y = 0;
    }
  } else if (p >= r) {
    v0x = 1; v0y = 0;
  } else {
    v0x = 0; v0y = 1;
  }
  lam[0] = l0;
  lam[1] = l1;
  v = M2<R>{v0x, v0y, -v0y, v0x};
}

// svd3x2 (shell_model.rs:84-106)
template <class R>
__device__ inline void svd3x2(const M32<R>& f, M32<R>& u, R s[2], M2<R>& v) {
  R lam[2];
  sym_eig2(f.c0.dot(f.c0), f.c0.dot(f.c1), f.c1.dot(f.c1), lam, v);
  s[0] = sqrt(rmax(lam[0], R(0)));
  s[1] = sqrt(rmax(lam[1], R(0)));
  R eps = R(1.0e-9) * rmax(s[0], R(1));
  V3<R> X(1, 0, 0), Y(0, 1, 0);
  V3<R> u0 = (s[0] > eps ? (f.c0 * v.xx + f.c1 * v.xy) / s[0] : X).normalize_or(X);
  V3<R> u1_raw;
  if (s[1] > eps) {
    u1_raw = (f.c0 * v.yx + f.c1 * v.yy) / s[1];
  } else {
    V3<R> t = fabs(u0.x) < R(0.9) ? X : Y;
    u1_raw = t - u0 * t.dot(u0);
  }
  u.c0 = u0;
  u.c1 = (u1_raw - u0 * u1_raw.dot(u0)).normalize_or(Y);
}

// StVK shell element gradient alone (shell_model.rs:366-380), as in shell_grad_hess.
template <class R>
__device__ inline void shell_grad(const V3<R> p[3], const M2<R>& dm, R area, R mu, R lambda, V3<R> grad[3]) {
  M32<R> f = M32<R>{p[1] - p[0], p[2] - p[0]}.mul(dm);
  M32<R> u;
  R s[2];
  M2<R> v;
  svd3x2(f, u, s, v);
  R j = s[0] * s[1];
  R s0m = s[0] - R(1), s1m = s[1] - R(1);
  R deda[2] = {mu * (s0m * (s0m * s0m)) + lambda * s[1] * (j - R(1)),
               mu * (s1m * (s1m * s1m)) + lambda * s[0] * (j - R(1))};
  M32<R> pk1 = M32<R>{u.c0 * deda[0], u.c1 * deda[1]}.mul(v.transpose());
  M32<R> hh = pk1.mul(dm.transpose());
  V3<R> g1 = hh.c0 * area, g2 = hh.c1 * area;
  grad[0] = -(g1 + g2);
  grad[1] = g1;
  grad[2] = g2;
}

// scale * dF/dx^T d2Psi/dF2 dF/dx over a triangle from the principal-stretch derivatives
// (shell_d2psi_df2_from_derivs, shell_model.rs:242-290 with the eigenpairs of :188-240;
// dF/dx of :384-400). deda = dPsi/dsigma, d2 = d2Psi/dsigma2 (2x2, row-major). project = false
// keeps the negative eigenvalues: the exact Hessian (the six eigenpairs span the 3x2
// deformation gradients).
template <class R>
__device__ inline void shell_hess_from_derivs(const M32<R>& u, const R s[2], const M2<R>& v, const R deda[2],
                                              const R d2[4], R eps, const M2<R>& dm, R scale, R* h /*81*/,
                                              bool project) {
  R ev[2];
  M2<R> evec;
  sym_eig2(d2[0], d2[1], d2[3], ev, evec);
  const R Rr = R(0.70710678118654752440);
  V3<R> qc0[6] = {V3<R>(0, -Rr, 0), V3<R>(0, Rr, 0), V3<R>(0, 0, 1), V3<R>(0, 0, 0), V3<R>(evec.xx, 0, 0),
                  V3<R>(evec.yx, 0, 0)};
  V3<R> qc1[6] = {V3<R>(Rr, 0, 0), V3<R>(Rr, 0, 0), V3<R>(0, 0, 0), V3<R>(0, 0, 1), V3<R>(0, evec.xy, 0),
                  V3<R>(0, evec.yy, 0)};
  R a = s[0], b = s[1];
  R denom = a - b;
  R fallback = R(0.5) * (d2[0] + d2[3]) - R(0.5) * (d2[1] + d2[2]);
  R lam[6] = {(deda[0] + deda[1]) / (a + b), fabs(denom) > eps ? (deda[0] - deda[1]) / denom : fallback,
              deda[0] / a, deda[1] / b, ev[0], ev[1]};
  V3<R> u2 = u.c0.cross(u.c1);
  R a6[36];
  for (int k = 0; k < 36; ++k) a6[k] = 0;
  M2<R> vt = v.transpose();
  for (int k = 0; k < 6; ++k) {
    R l = project ? rmax(lam[k], R(0)) : lam[k];
    if (l == 0) continue;
    M32<R> uq{u.c0 * qc0[k].x + u.c1 * qc0[k].y + u2 * qc0[k].z, u.c0 * qc1[k].x + u.c1 * qc1[k].y + u2 * qc1[k].z};
    M32<R> m = uq.mul(vt);
    R qv[6] = {m.c0.x, m.c1.x, m.c0.y, m.c1.y, m.c0.z, m.c1.z};
    for (int r = 0; r < 6; ++r)
      for (int c = 0; c < 6; ++c) a6[r * 6 + c] += l * qv[r] * qv[c];
  }
  // dF/dx (shell_model.rs:384-400): row 2i+jj, column 3k+i
  R bm[54];
  for (int k = 0; k < 54; ++k) bm[k] = 0;
  for (int i = 0; i < 3; ++i)
    for (int jj = 0; jj < 2; ++jj) {
      int row = 2 * i + jj;
      R sum = 0;
      for (int k = 0; k < 2; ++k) {
        R d = dm.at(k, jj);
        bm[row * 9 + 3 * (k + 1) + i] = d;
        sum += d;
      }
      bm[row * 9 + i] = -sum;
    }
  R ab[54];
  for (int r = 0; r < 6; ++r)
    for (int c = 0; c < 9; ++c) {
      R acc = 0;
      for (int k = 0; k < 6; ++k) acc += a6[r * 6 + k] * bm[k * 9 + c];
      ab[r * 9 + c] = acc;
    }
  for (int r = 0; r < 9; ++r)
    for (int c = 0; c < 9; ++c) {
      R acc = 0;
      for (int k = 0; k < 6; ++k) acc += bm[k * 9 + r] * ab[k * 9 + c];
      h[r * 9 + c] = scale * acc;
    }
}

// StVK shell element: gradient (shell_model.rs:366-380) and eigen-projected Hessian
// (shell_model.rs:178-290 + :403-438). dm = inverse rest shape (column-major 2x2).
// project = false keeps the negative eigenvalues: the exact Hessian.
template <class R>
__device__ inline void shell_grad_hess(const V3<R> p[3], const M2<R>& dm, R area, R mu, R lambda, R eps, V3<R> grad[3],
                                       R* h /*81*/, bool project = true) {
  M32<R> f = M32<R>{p[1] - p[0], p[2] - p[0]}.mul(dm);
  M32<R> u;
  R s[2];
  M2<R> v;
  svd3x2(f, u, s, v);
  R j = s[0] * s[1];
  R s0m = s[0] - R(1), s1m = s[1] - R(1);
  R deda[2] = {mu * (s0m * (s0m * s0m)) + lambda * s[1] * (j - R(1)),
               mu * (s1m * (s1m * s1m)) + lambda * s[0] * (j - R(1))};
  // gradient
  M32<R> pk1 = M32<R>{u.c0 * deda[0], u.c1 * deda[1]}.mul(v.transpose());
  M32<R> hh = pk1.mul(dm.transpose());
  V3<R> g1 = hh.c0 * area, g2 = hh.c1 * area;
  grad[0] = -(g1 + g2);
  grad[1] = g1;
  grad[2] = g2;
  // eigen-projected d2Psi/dF2
  R cross = lambda * (R(2) * s[0] * s[1] - R(1));
  R d2[4] = {R(3) * mu * s0m * s0m + lambda * s[1] * s[1], cross, cross, R(3) * mu * s1m * s1m + lambda * s[0] * s[0]};
  shell_hess_from_derivs(u, s, v, deda, d2, eps, dm, area, h, project);
}

// ---- face strain limit (shell_model.rs:438-640) -------------------------------------------
// The barrier argument never drops below this fraction of the limit (SL_GAP_FLOOR,
// shell_model.rs:444).
#define MG_SL_GAP_FLOOR 1.0e-3

// strain_limit_derivs (shell_model.rs:456-484): energy derivatives over the two principal
// stretch excesses a = sigma - 1 (deda, diagonal d2); false when neither exceeds rest.
template <class R>
__device__ inline bool sl_derivs(const R s[2], R limit, int kind, R deda[2], R d2[4]) {
  if (!(limit > 0)) return false;
  deda[0] = deda[1] = R(0);
  d2[0] = d2[1] = d2[2] = d2[3] = R(0);
  bool active = false;
  for (int i = 0; i < 2; ++i) {
    const R a = s[i] - R(1);
    if (a <= 0) continue;
    const R y = rmax(limit - a, R(MG_SL_GAP_FLOOR) * limit);
    R g, h;
    if (barrier_of<R>(kind, y, limit, R(1), g, h)) {
      deda[i] = -g;
      d2[3 * i] = h;
      active = true;
    }
  }
  return active;
}

// The largest principal-stretch excess max(sigma - 1) of a face (what the strain-limit line
// search bisects on, implicit.rs:1719-1729).
template <class R>
__device__ inline R max_stretch_excess(const V3<R> p[3], const M2<R>& dm) {
  M32<R> f = M32<R>{p[1] - p[0], p[2] - p[0]}.mul(dm);
  R lam[2];
  M2<R> v;
  sym_eig2(f.c0.dot(f.c0), f.c0.dot(f.c1), f.c1.dot(f.c1), lam, v);
  const R s0 = sqrt(rmax(lam[0], R(0))), s1 = sqrt(rmax(lam[1], R(0)));
  return rmax(s0 - R(1), s1 - R(1));
}

// strain_limit_assembly (shell_model.rs:582-640): the face barrier's gradient and 9x9
// Hessian at the dynamic stiffness max(elastic_k, 0) + face_mass / d^2, d the headroom
// limit - max(sigma - 1) floored at the gap floor. False when inactive.
template <class R>
__device__ inline bool sl_face_grad_hess(const V3<R> p[3], const M2<R>& dm, R limit, R face_mass, R elastic_k,
                                         int kind, R eps, V3<R> grad[3], R* h /*81*/) {
  M32<R> f = M32<R>{p[1] - p[0], p[2] - p[0]}.mul(dm);
  M32<R> u;
  R s[2];
  M2<R> v;
  svd3x2(f, u, s, v);
  R deda[2], d2[4];
  if (!sl_derivs(s, limit, kind, deda, d2)) return false;
  const R max_a = rmax(s[0] - R(1), s[1] - R(1));
  const R d = rmax(limit - max_a, R(MG_SL_GAP_FLOOR) * limit);
  const R stiffness = rmax(elastic_k, R(0)) + face_mass / (d * d);
  if (!(stiffness > 0)) return false;
  M32<R> pk1 = M32<R>{u.c0 * deda[0], u.c1 * deda[1]}.mul(v.transpose());
  M32<R> hg = pk1.mul(dm.transpose());
  const V3<R> g1 = hg.c0 * stiffness, g2 = hg.c1 * stiffness;
  grad[0] = -(g1 + g2);
  grad[1] = g1;
  grad[2] = g2;
  shell_hess_from_derivs(u, s, v, deda, d2, eps, dm, stiffness, h, true);
  return true;
}

// ---------------------------------------------------------------------------------------
// bending.rs
// ---------------------------------------------------------------------------------------
template <class R>
__device__ inline R dihedral_angle(const V3<R> p[4]) {
  V3<R> n1 = (p[1] - p[0]).cross(p[2] - p[0]);
  V3<R> n2 = (p[1] - p[2]).cross(p[3] - p[2]);
  V3<R> e = (p[2] - p[1]).normalize_or_zero();
  V3<R> n1n = n1.normalize_or_zero(), n2n = n2.normalize_or_zero();
  R s = n1n.cross(n2n).dot(e);
  R c = rclamp(n1n.dot(n2n), R(-1), R(1));
  return atan2(s, c);
}

template <class R>
__device__ inline void dihedral_grad(const V3<R> p[4], V3<R> g[4]) {
  V3<R> m1 = (p[1] - p[0]).cross(p[2] - p[0]);
  V3<R> m2 = (p[1] - p[2]).cross(p[3] - p[2]);
  V3<R> e = p[2] - p[1];
  R a1 = m1.length(), a2 = m2.length(), l2 = e.length_squared();
  if (a1 < R(1.0e-12) || a2 < R(1.0e-12) || l2 < R(1.0e-24)) {
    // degenerate flap: central differences of the angle (bending.rs:51-68)
    R scale = rmax(p[0].length() + p[1].length() + p[2].length() + p[3].length(), R(1));
    R h = R(1.0e-4) * scale;
    R inv = R(1) / (R(2) * h);
    for (int vi = 0; vi < 4; ++vi)
      for (int c = 0; c < 3; ++c) {
        V3<R> pp[4] = {p[0], p[1], p[2], p[3]}, pm[4] = {p[0], p[1], p[2], p[3]};
        pp[vi][c] += h;
        pm[vi][c] -= h;
        g[vi][c] = (dihedral_angle(pp) - dihedral_angle(pm)) * inv;
      }
    return;
  }
  R l = sqrt(l2);
  V3<R> n1 = m1 / a1, n2 = m2 / a2;
  V3<R> g0 = n1 * (-l / a1);
  V3<R> g3 = n2 * (-l / a2);
  R ta = (p[0] - p[1]).dot(e) / l2;
  R tb = (p[3] - p[1]).dot(e) / l2;
  g[0] = g0;
  g[1] = g0 * (ta - R(1)) + g3 * (tb - R(1));
  g[2] = g0 * (-ta) + g3 * (-tb);
  g[3] = g3;
}

// ---------------------------------------------------------------------------------------
// Baraff-Witkin membrane (engine-core/src/membrane.rs): warp, weft and shear conditions of
// the deformation's columns wu, wv (F = Ds Dm^-1, Dm^-1 row-major dm[4]): Cu = |wu| - 1,
// Cv = |wv| - 1, Csh = wu.wv; energy area (kw Cu^2 + kf Cv^2 + ks Csh^2) / 2; the stretch
// blocks use n n^T + max(0, 1 - 1/|w|)(I - n n^T) and the shear block its eigen-projected
// 6x6 form (membrane.rs:100-205). Gradient per vertex (g[a]) and 3x3 blocks h[3 a + b].
template <class R>
__device__ void bw_add_outer(R m[3][3], const V3<R>& u, const V3<R>& v, R s) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) m[r][c] += s * u[r] * v[c];
}

template <class R>
__device__ void bw_proj_perp(const V3<R>& w, R q[3][3]) {
  const V3<R> n = w.normalize_or_zero();
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) q[r][c] = (r == c ? R(1) : R(0)) - n[r] * n[c];
}

template <class R>
__device__ void bw_stretch_material(const V3<R>& w, R m[3][3]) {
  const R s = w.length();
  const V3<R> n = w.normalize_or_zero();
  const R perp = s > R(1.0e-6) ? rmax(R(1) - R(1) / s, R(0)) : R(0);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      const R nnt = n[r] * n[c];
      m[r][c] = nnt + perp * ((r == c ? R(1) : R(0)) - nnt);
    }
}

template <class R>
__device__ void bw_shear_material(const V3<R>& wu, const V3<R>& wv, R m[4][3][3]) {
  const R f = wu.dot(wv);
  const R a = wu.length_squared() + wv.length_squared();
  const R disc = sqrt(rmax(a * a + R(12) * f * f, R(0)));
  const R mu[2] = {R(0.5) * (a + disc), R(0.5) * (a - disc)};
  for (int b = 0; b < 4; ++b)
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) m[b][r][c] = 0;
  for (int k = 0; k < 2; ++k) {
    const V3<R> top = wv * mu[k] + wu * f, bot = wu * mu[k] + wv * f;
    const R n = top.length_squared() + bot.length_squared();
    if (n > R(1e-20)) {
      const R sc = rmax(mu[k], R(0)) / n;
      bw_add_outer(m[0], top, top, sc);
      bw_add_outer(m[1], top, bot, sc);
      bw_add_outer(m[2], bot, top, sc);
      bw_add_outer(m[3], bot, bot, sc);
    }
  }
  const R fp = R(0.5) * rmax(f, R(0));
  if (fp != 0) {
    R qp[3][3];
    bw_proj_perp(wu + wv, qp);
    for (int b = 0; b < 4; ++b)
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) m[b][r][c] += fp * qp[r][c];
  }
  const R fm = R(0.5) * rmax(-f, R(0));
  if (fm != 0) {
    R qm[3][3];
    bw_proj_perp(wv - wu, qm);
    const R sgn[4] = {R(1), R(-1), R(-1), R(1)};
    for (int b = 0; b < 4; ++b)
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) m[b][r][c] += (sgn[b] * fm) * qm[r][c];
  }
}

template <class R>
__device__ void membrane_grad_hess(const V3<R> p[3], const R dm[4], R area, R kw, R kf, R ks, V3<R> g[3],
                                   R h[9][9]) {
  const V3<R> ds0 = p[1] - p[0], ds1 = p[2] - p[0];
  const V3<R> wu = ds0 * dm[0] + ds1 * dm[2];
  const V3<R> wv = ds0 * dm[1] + ds1 * dm[3];
  const R cnd[3] = {wu.length() - R(1), wv.length() - R(1), wu.dot(wv)};
  const R cu[3] = {-(dm[0] + dm[2]), dm[0], dm[2]};
  const R cv[3] = {-(dm[1] + dm[3]), dm[1], dm[3]};
  const V3<R> nu = wu.normalize_or_zero(), nv = wv.normalize_or_zero();
  R mu_[3][3], mv_[3][3], sm[4][3][3];
  bw_stretch_material(wu, mu_);
  bw_stretch_material(wv, mv_);
  bw_shear_material(wu, wv, sm);
  for (int a = 0; a < 3; ++a) g[a] = V3<R>();
  for (int i = 0; i < 9; ++i)
    for (int j = 0; j < 9; ++j) h[i][j] = 0;
  const R kc[3] = {kw, kf, ks};
  for (int ci = 0; ci < 3; ++ci) {
    const R ka = kc[ci] * area;
    if (!(ka > 0)) continue;
    for (int a = 0; a < 3; ++a) {
      const V3<R> ga = ci == 0 ? nu * cu[a] : (ci == 1 ? nv * cv[a] : wv * cu[a] + wu * cv[a]);
      g[a] += ga * (ka * cnd[ci]);
      for (int b = 0; b < 3; ++b)
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) {
            R v;
            if (ci == 0)
              v = ka * cu[a] * cu[b] * mu_[r][c];
            else if (ci == 1)
              v = ka * cv[a] * cv[b] * mv_[r][c];
            else
              v = ka * (cu[a] * cu[b] * sm[0][r][c] + cu[a] * cv[b] * sm[1][r][c] + cv[a] * cu[b] * sm[2][r][c] +
                        cv[a] * cv[b] * sm[3][r][c]);
            h[3 * a + r][3 * b + c] += v;
          }
    }
  }
}

}  // namespace mg
