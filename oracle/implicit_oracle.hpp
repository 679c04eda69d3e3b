// CPU oracle (TEST INFRASTRUCTURE ONLY): a restatement of the reference's implicit
// backward-Euler IPC step, templated on the real type (float = the reference's f32 path,
// double = the FP64 oracle of the whole step).
//
// Follows, function by function:
//   engine-core/src/contact.rs   (colliders, closest point, distances + gradients, ACCD,
//                                 barriers, Rayleigh stiffness, friction, pseudonormals)
//   engine-core/src/shell_model.rs (svd3x2, StVK derivatives, eigen-projected Hessian)
//   engine-core/src/bending.rs   (hinges, dihedral angle, analytic gradient)
//   engine-core/src/stitch.rs    (six-participant seam spring)
//   engine-core/src/strain_limit.rs (one-sided edge strain limit)
//   engine-core/src/membrane.rs  (Baraff-Witkin warp / weft / shear membrane)
//   engine-core/src/broadphase.rs (uniform hash grid V-T / E-E, 1-ring exclusion)
//   engine-core/src/implicit.rs  (new, stencils, Rayleigh gather, assemble + Asm push order,
//                                 ccd_max_step with the strain-limit and static-pin clamps,
//                                 pins, pulls, step)
// Restated element kinds: inertia, stretch springs (+ the one-sided edge strain limit), the
// Baraff-Witkin membrane, StVK shells, hinges, stitches, the per-face strain-limit barrier,
// pins and pulls, analytic colliders, static-mesh colliders with a signed gap, and
// vertex-triangle / edge-edge self contact (+ friction when mu > 0).
// Added to both this oracle and the CUDA path: a Newton termination on the step actually
// taken, max_i |t dx_i| < newton_tol (0 disables it).
#pragma once
#include <functional>
#include <map>
#include <unordered_map>

#include "mguso_oracle.hpp"

namespace mo {

template <class R>
using Vt = V3<R>;

// powi expansions as LLVM emits them for constant exponents: x^3 = x * (x*x),
// x^4 = (x*x) * (x*x).
template <class R> inline R pow3(R x) { return x * (x * x); }
template <class R> inline R pow4(R x) { R x2 = x * x; return x2 * x2; }

// ---------------------------------------------------------------------------------------
// contact.rs
// ---------------------------------------------------------------------------------------
enum class BarrierKind : int { Log = 0, Cubic = 1 };

template <class R>
struct Collider {
  int kind = 1;  // 0 = half-space (point a, unit normal n), 1 = sphere (center a, radius)
  Vt<R> a, n;
  R radius = 0;
  // Collider::distance (contact.rs:33-51)
  void distance(const Vt<R>& x, R& d, Vt<R>& nrm) const {
    if (kind == 0) {
      d = (x - a).dot(n);
      nrm = n;
      return;
    }
    Vt<R> v = x - a;
    R l = v.length();
    if (l < R(1.0e-9)) {
      d = -radius;
      nrm = Vt<R>(0, 1, 0);
    } else {
      d = l - radius;
      nrm = v / l;
    }
  }
};

// closest_point_on_triangle_bary (contact.rs:84-124)
template <class R>
inline Vt<R> closest_point_bary(const Vt<R>& p, const Vt<R>& a, const Vt<R>& b, const Vt<R>& c, R w[3]) {
  Vt<R> ab = b - a, ac = c - a, ap = p - a;
  R d1 = ab.dot(ap), d2 = ac.dot(ap);
  if (d1 <= 0 && d2 <= 0) { w[0] = 1; w[1] = 0; w[2] = 0; return a; }
  Vt<R> bp = p - b;
  R d3 = ab.dot(bp), d4 = ac.dot(bp);
  if (d3 >= 0 && d4 <= d3) { w[0] = 0; w[1] = 1; w[2] = 0; return b; }
  R vc = d1 * d4 - d3 * d2;
  if (vc <= 0 && d1 >= 0 && d3 <= 0) {
    R den = d1 - d3;
    R v = den != 0 ? d1 / den : R(0);
    w[0] = R(1) - v; w[1] = v; w[2] = 0;
    return a + ab * v;
  }
  Vt<R> cp = p - c;
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
inline R point_triangle_distance(const Vt<R>& p, const Vt<R>& a, const Vt<R>& b, const Vt<R>& c) {
  R w[3];
  return (p - closest_point_bary(p, a, b, c, w)).length();
}

// point_tri_distance_grad (contact.rs:836-857)
template <class R>
inline R point_tri_distance_grad(const Vt<R>& p, const Vt<R>& a, const Vt<R>& b, const Vt<R>& c, Vt<R> g[4]) {
  R w[3];
  Vt<R> q = closest_point_bary(p, a, b, c, w);
  Vt<R> e = p - q;
  R d = e.length();
  if (d < R(1.0e-12)) {
    for (int k = 0; k < 4; ++k) g[k] = Vt<R>();
    return d;
  }
  Vt<R> n = e / d;
  g[0] = n;
  g[1] = n * (-w[0]);
  g[2] = n * (-w[1]);
  g[3] = n * (-w[2]);
  return d;
}

// signed_point_tri_distance_grad (contact.rs:889-915)
template <class R>
inline R signed_point_tri_distance_grad(const Vt<R>& p, const Vt<R>& a, const Vt<R>& b, const Vt<R>& c, bool inside,
                                        Vt<R> g[4]) {
  R d = point_tri_distance_grad(p, a, b, c, g);
  if (inside) {
    for (int k = 0; k < 4; ++k) g[k] = -g[k];
    return -d;
  }
  return d;
}

// point_edge_coeff (contact.rs:193-202)
template <class R>
inline void point_edge_coeff(const Vt<R>& p, const Vt<R>& e0, const Vt<R>& e1, R out[2]) {
  Vt<R> r = e1 - e0;
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
inline void edge_edge_witness(const Vt<R>& ea0, const Vt<R>& ea1, const Vt<R>& eb0, const Vt<R>& eb1, R out[4]) {
  Vt<R> cog = (ea0 + ea1 + eb0 + eb1) * R(0.25);
  Vt<R> a0 = ea0 - cog, a1 = ea1 - cog, b0v = eb0 - cog, b1v = eb1 - cog;
  auto dist2 = [&](const R c[4]) {
    Vt<R> x0 = a0 * c[0] + a1 * c[1];
    Vt<R> x1 = b0v * c[2] + b1v * c[3];
    return (x1 - x0).length_squared();
  };
  R pe[2];
  point_edge_coeff(ea0, eb0, eb1, pe);
  R cls[4] = {1, 0, pe[0], pe[1]};
  Vt<R> r0 = ea1 - ea0, r1 = eb1 - eb0;
  R a00 = r0.dot(r0), a01 = -r0.dot(r1), a11 = r1.dot(r1);
  Vt<R> rhs = eb0 - ea0;
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
  R best_d = std::numeric_limits<R>::infinity();
  for (int k = 0; k < 4; ++k) {
    R d = dist2(types[k]);
    if (d < best_d) { best_d = d; best = k; }
  }
  for (int k = 0; k < 4; ++k) out[k] = types[best][k];
}

// segment_segment_distance (contact.rs:439-487)
template <class R>
inline R segment_segment_distance(const Vt<R>& p1, const Vt<R>& q1, const Vt<R>& p2, const Vt<R>& q2) {
  Vt<R> d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
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
  Vt<R> c1 = p1 + d1 * s, c2 = p2 + d2 * t;
  return (c1 - c2).length();
}

// segment_segment_distance_grad (contact.rs:489-518)
template <class R>
inline R segment_segment_distance_grad(const Vt<R>& p1, const Vt<R>& q1, const Vt<R>& p2, const Vt<R>& q2,
                                       Vt<R> g[4]) {
  R w[4];
  edge_edge_witness(p1, q1, p2, q2, w);
  Vt<R> ca = p1 * w[0] + q1 * w[1];
  Vt<R> cb = p2 * w[2] + q2 * w[3];
  Vt<R> e = ca - cb;
  R d = e.length();
  if (d < R(1.0e-12)) {
    for (int k = 0; k < 4; ++k) g[k] = Vt<R>();
    return d;
  }
  Vt<R> n = e / d;
  g[0] = n * w[0];
  g[1] = n * w[1];
  g[2] = n * (-w[2]);
  g[3] = n * (-w[3]);
  return d;
}

// edge_triangle_intersect (contact.rs:324-352)
template <class R>
inline bool edge_triangle_intersect(const Vt<R>& e0, const Vt<R>& e1, const Vt<R>& v0, const Vt<R>& v1,
                                    const Vt<R>& v2) {
  Vt<R> d1 = v1 - v0, d2 = v2 - v0, a0 = e0 - v0, a1 = e1 - v0;
  Vt<R> n = d1.cross(d2);
  R s1 = a0.dot(n), s2 = a1.dot(n);
  if (s1 * s2 < 0) {
    R t = s1 / (s1 - s2);
    Vt<R> r = a0 * (R(1) - t) + a1 * t;
    R a = d1.dot(d1), b = d1.dot(d2), c = d2.dot(d2);
    R det = a * c - b * b;
    if (det == 0) return false;
    R p = d1.dot(r), q = d2.dot(r);
    R u = (c * p - b * q) / det, v = (a * q - b * p) / det;
    return u >= 0 && v >= 0 && u + v <= 1;
  }
  return false;
}

// accd_toi (contact.rs:378-437). `hit_cap` reports whether max_iter ran out.
template <class R, class SqDist>
inline R accd_toi(const Vt<R> x0[4], const Vt<R> dx[4], R offset, R max_t, R reduction, uint32_t max_iter,
                  SqDist square_dist, bool* hit_cap = nullptr) {
  if (hit_cap) *hit_cap = false;
  R u_max = 0;
  for (int i = 0; i < 4; ++i)
    for (int j = i + 1; j < 4; ++j) u_max = rmax(u_max, (dx[i] - dx[j]).length());
  if (u_max < R(1.0e-12)) return max_t;
  R inv_u_max = R(1) / u_max;
  R d0 = std::sqrt(rmax(square_dist(x0), R(0)));
  R eps = reduction * (d0 - offset);
  if (eps <= 0) return max_t;
  R target = eps + offset;
  R eps_sqr = eps * eps;
  R toi = 0;
  Vt<R> moved[4];
  uint32_t it = 0;
  for (; it < max_iter; ++it) {
    for (int k = 0; k < 4; ++k) moved[k] = x0[k] + dx[k] * toi;
    R d2 = rmax(square_dist(moved), R(0));
    R dmt = (d2 - target * target) / (std::sqrt(d2) + target);
    if ((max_t - toi) * u_max < dmt - eps) return max_t;
    if (toi > 0 && dmt * dmt < eps_sqr) break;
    R toi_next = toi + dmt * inv_u_max;
    if (toi_next != toi)
      toi = toi_next;
    else
      break;
    if (toi > max_t) return max_t;
  }
  if (it == max_iter && hit_cap) *hit_cap = true;
  return rmax(toi, R(0));
}

// barrier (contact.rs:1014-1027): IPC log barrier (e, dE/dd, d2E/dd2).
template <class R>
inline bool barrier_log(R d, R dhat, R kappa, R& e, R& g, R& h) {
  if (d >= dhat) return false;
  d = rmax(d, R(1.0e-6));
  R t = d - dhat;
  R ld = std::log(d / dhat);
  e = -kappa * t * t * ld;
  g = -kappa * (R(2) * t * ld + t * t / d);
  h = -kappa * (R(2) * ld + R(4) * t / d - (t * t) / (d * d));
  return true;
}

// cubic_barrier (contact.rs:580-592)
template <class R>
inline bool cubic_barrier(R g, R ghat, R offset, R& e, R& de, R& d2e) {
  g = g - offset;
  R y = g - ghat;
  if (y >= 0) return false;
  e = R(-2) * (y * y * y) / (R(3) * ghat);
  de = R(-2) * y * y / ghat;
  d2e = R(4) * (R(1) - g / ghat);
  return true;
}

// barrier_of (contact.rs:723-730)
template <class R>
inline bool barrier_of(BarrierKind kind, R d, R dhat, R kappa, R& e, R& g, R& h) {
  if (kind == BarrierKind::Log) return barrier_log(d, dhat, kappa, e, g, h);
  R ce, cg, ch;
  if (!cubic_barrier(d, dhat, R(0), ce, cg, ch)) return false;
  e = kappa * ce;
  g = kappa * cg;
  h = kappa * ch;
  return true;
}

// rayleigh_stiffness (contact.rs:750-834); elastic is n*n row-major 3x3 blocks.
template <class R>
inline R rayleigh_stiffness(const R (*elastic)[9], const R* mass, const R* weights, int n, const Vt<R>& e, R offset) {
  R g = e.length() - offset;
  if (g <= 0 || n == 0) return 0;
  R sqr_x = g * g;
  R m_max = 0;
  for (int i = 0; i < n; ++i) m_max = rmax(m_max, mass[i]);
  R w[12];
  for (int ii = 0; ii < n; ++ii) {
    Vt<R> v = e * weights[ii];
    w[3 * ii] = v.x;
    w[3 * ii + 1] = v.y;
    w[3 * ii + 2] = v.z;
  }
  R ss = 0;
  for (int k = 0; k < 3 * n; ++k) ss += w[k] * w[k];
  R norm = std::sqrt(ss);
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

// dynamic_stiffness (contact.rs:984-996)
template <class R>
inline R dynamic_stiffness(R kappa_base, R coupling, R mass_eff, R gap, R dhat) {
  if (coupling <= 0 || mass_eff <= 0) return kappa_base;
  R d = rmax(rmax(gap, R(0.1) * dhat), R(1.0e-6));
  return kappa_base * (R(1) + coupling * mass_eff / (d * d));
}

// friction (contact.rs:613-644)
template <class R>
inline bool friction(const Vt<R>& force_contact, const Vt<R>& dx, const Vt<R>& normal, R mu, R min_dx, Vt<R>& grad,
                     R hess[3][3]) {
  if (mu <= 0) return false;
  R contact = -normal.dot(force_contact);
  Vt<R> pdx = dx - normal * normal.dot(dx);
  R eps = rmax(min_dx, R(1.0e-12));
  R denom = rmax(pdx.length(), eps);
  R lambda = mu * contact / denom;
  if (lambda <= 0) return false;
  grad = pdx * lambda;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) hess[r][c] = lambda * ((r == c ? R(1) : R(0)) - normal[r] * normal[c]);
  return true;
}

// stencil_friction (contact.rs:659-705)
template <class R>
inline bool stencil_friction(const Vt<R> g[4], const Vt<R> dx[4], R barrier_grad, R mu, R min_dx, Vt<R> grad[4],
                             R hess[144]) {
  if (mu <= 0) return false;
  R nlen = g[0].length();
  if (nlen < R(1.0e-12)) return false;
  Vt<R> n = g[0] / nlen;
  R w[4];
  Vt<R> slip;
  for (int a = 0; a < 4; ++a) {
    w[a] = g[a].dot(n);
    slip += dx[a] * w[a];
  }
  Vt<R> f_c = n * barrier_grad;
  Vt<R> fg;
  R fh[3][3];
  if (!friction(f_c, slip, n, mu, min_dx, fg, fh)) return false;
  if (fg == Vt<R>()) return false;
  for (int a = 0; a < 4; ++a) grad[a] = fg * w[a];
  for (int k = 0; k < 144; ++k) hess[k] = 0;
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      R wab = w[a] * w[b];
      if (wab == 0) continue;
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) hess[(3 * a + r) * 12 + (3 * b + c)] = wab * fh[r][c];
    }
  return true;
}

// vertex_contact_full (contact.rs:1082-1125)
template <class R>
inline void vertex_contact_full(const Vt<R>& x, const std::vector<Collider<R>>& colliders, R dhat, R kappa,
                                R coupling, R mass_eff, BarrierKind kind, const R* elastic, bool has_slip,
                                const Vt<R>& slip_dx, R mu, R eps, Vt<R>& grad, R hess[3][3]) {
  grad = Vt<R>();
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) hess[r][c] = 0;
  for (const auto& col : colliders) {
    R d;
    Vt<R> n;
    col.distance(x, d, n);
    R k;
    if (elastic) {
      R el[1][9];
      for (int q = 0; q < 9; ++q) el[0][q] = elastic[q];
      R one = 1;
      k = rayleigh_stiffness<R>(el, &mass_eff, &one, 1, n * d, R(0));
    } else {
      k = dynamic_stiffness(kappa, coupling, mass_eff, d, dhat);
    }
    R e, g, h;
    if (!barrier_of(kind, d, dhat, k, e, g, h)) continue;
    Vt<R> f_c = n * g;
    grad += f_c;
    R hp = rmax(h, R(0));
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) hess[r][c] += hp * n[r] * n[c];
    if (has_slip) {
      Vt<R> fg;
      R fh[3][3];
      if (friction(f_c, slip_dx, n, mu, eps, fg, fh)) {
        grad += fg;
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) hess[r][c] += fh[r][c];
      }
    }
  }
}

// surface_normal_at (contact.rs:935-942)
template <class R>
inline Vt<R> surface_normal_at(const R bary[3], const Vt<R>& face, const Vt<R> pn[3]) {
  if (bary[0] > R(1.0e-4) && bary[1] > R(1.0e-4) && bary[2] > R(1.0e-4)) return face;
  return (pn[0] * bary[0] + pn[1] * bary[1] + pn[2] * bary[2]).normalize_or_zero();
}

// pseudonormals (contact.rs:963-1001): angle-weighted, welded on exact position bits.
template <class R>
inline std::vector<Vt<R>> pseudonormals(const std::vector<Vt<R>>& pos, const std::vector<std::array<uint32_t, 3>>& tris) {
  auto bits = [](R c) -> uint64_t {
    if (c == 0) c = 0;
    uint64_t b = 0;
    std::memcpy(&b, &c, sizeof(R));
    return b;
  };
  struct Key {
    uint64_t a, b, c;
    bool operator==(const Key& o) const { return a == o.a && b == o.b && c == o.c; }
  };
  struct H {
    size_t operator()(const Key& k) const { return k.a * 1000003u ^ k.b * 9176u ^ k.c; }
  };
  std::unordered_map<Key, uint32_t, H> weld;
  std::vector<uint32_t> of(pos.size());
  for (size_t i = 0; i < pos.size(); ++i) {
    Key k{bits(pos[i].x), bits(pos[i].y), bits(pos[i].z)};
    auto it = weld.find(k);
    if (it == weld.end()) {
      uint32_t nx = (uint32_t)weld.size();
      weld.emplace(k, nx);
      of[i] = nx;
    } else {
      of[i] = it->second;
    }
  }
  std::vector<Vt<R>> acc(weld.size());
  for (const auto& t : tris) {
    Vt<R> p[3] = {pos[t[0]], pos[t[1]], pos[t[2]]};
    Vt<R> face = (p[1] - p[0]).cross(p[2] - p[0]).normalize_or_zero();
    if (face == Vt<R>()) continue;
    for (int k = 0; k < 3; ++k) {
      Vt<R> u = (p[(k + 1) % 3] - p[k]).normalize_or_zero();
      Vt<R> v = (p[(k + 2) % 3] - p[k]).normalize_or_zero();
      acc[of[t[k]]] += face * std::acos(rclamp(u.dot(v), R(-1), R(1)));
    }
  }
  std::vector<Vt<R>> out(pos.size());
  for (size_t i = 0; i < pos.size(); ++i) out[i] = acc[of[i]].normalize_or_zero();
  return out;
}

// ---------------------------------------------------------------------------------------
// shell_model.rs (isotropic StVK shells on a 3x2 SVD)
// ---------------------------------------------------------------------------------------
template <class R>
struct Mat2 {  // column-major like glam: x = column 0, y = column 1
  R xx, xy, yx, yy;  // x_axis = (xx, xy), y_axis = (yx, yy)
  R det() const { return xx * yy - yx * xy; }
  Mat2 inverse() const {
    R inv = R(1) / det();
    return Mat2{yy * inv, xy * -inv, yx * -inv, xx * inv};
  }
  Mat2 transpose() const { return Mat2{xx, yx, xy, yy}; }
  R at(int r, int c) const { return c == 0 ? (r == 0 ? xx : xy) : (r == 0 ? yx : yy); }
};

template <class R>
struct Mat3x2 {
  Vt<R> c0, c1;
  Mat3x2 mul_mat2(const Mat2<R>& m) const { return Mat3x2{c0 * m.xx + c1 * m.xy, c0 * m.yx + c1 * m.yy}; }
  Mat2<R> ata() const { return Mat2<R>{c0.dot(c0), c1.dot(c0), c0.dot(c1), c1.dot(c1)}; }
  void vec6(R o[6]) const { o[0] = c0.x; o[1] = c1.x; o[2] = c0.y; o[3] = c1.y; o[4] = c0.z; o[5] = c1.z; }
};

// sym_eig2 (shell_model.rs:60-78); eigenvalues descending, eigenvectors as columns.
template <class R>
inline void sym_eig2(const Mat2<R>& a, R lam[2], Mat2<R>& v) {
  R p = a.xx, q = a.yx, r = a.yy;
  R tr = p + r;
  R diff = std::sqrt(rmax((p - r) * (p - r) + R(4) * q * q, R(0)));
  R l0 = R(0.5) * (tr + diff), l1 = R(0.5) * (tr - diff);
  R v0x, v0y;
  if (std::fabs(q) > R(1.0e-20)) {
    R x = q, y = l0 - p;
    R len = std::sqrt(x * x + y * y);
    R rcp = R(1) / len;
    if (std::isfinite(rcp) && rcp > 0) {
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
  v = Mat2<R>{v0x, v0y, -v0y, v0x};
}

// svd3x2 (shell_model.rs:84-106)
template <class R>
inline void svd3x2(const Mat3x2<R>& f, Mat3x2<R>& u, R sigma[2], Mat2<R>& v) {
  R lam[2];
  sym_eig2(f.ata(), lam, v);
  sigma[0] = std::sqrt(rmax(lam[0], R(0)));
  sigma[1] = std::sqrt(rmax(lam[1], R(0)));
  R eps = R(1.0e-9) * rmax(sigma[0], R(1));
  auto fv = [&](R vx, R vy) { return f.c0 * vx + f.c1 * vy; };
  Vt<R> X(1, 0, 0), Y(0, 1, 0);
  Vt<R> u0 = (sigma[0] > eps ? fv(v.xx, v.xy) / sigma[0] : X).normalize_or(X);
  Vt<R> u1_raw;
  if (sigma[1] > eps) {
    u1_raw = fv(v.yx, v.yy) / sigma[1];
  } else {
    Vt<R> t = std::fabs(u0.x) < R(0.9) ? X : Y;
    u1_raw = t - u0 * t.dot(u0);
  }
  Vt<R> u1 = (u1_raw - u0 * u1_raw.dot(u0)).normalize_or(Y);
  u = Mat3x2<R>{u0, u1};
}

// StVK derivative tables (shell_model.rs:131-176).
template <class R>
inline void stvk_dpsi(const R s[2], R mu, R lambda, R out[2]) {
  R j = s[0] * s[1];
  out[0] = mu * pow3(s[0] - R(1)) + lambda * s[1] * (j - R(1));
  out[1] = mu * pow3(s[1] - R(1)) + lambda * s[0] * (j - R(1));
}
template <class R>
inline void stvk_d2psi(const R s[2], R mu, R lambda, R out[4]) {
  R a = s[0], b = s[1];
  R cross = lambda * (R(2) * a * b - R(1));
  out[0] = R(3) * mu * (a - R(1)) * (a - R(1)) + lambda * b * b;
  out[1] = cross;
  out[2] = cross;
  out[3] = R(3) * mu * (b - R(1)) * (b - R(1)) + lambda * a * a;
}
template <class R>
inline R stvk_density(const R s[2], R mu, R lambda) {
  R j = s[0] * s[1];
  return mu * (pow4(s[0] - R(1)) + pow4(s[1] - R(1))) / R(4) + R(0.5) * lambda * (j - R(1)) * (j - R(1));
}

// shell_d2psi_df2_from_derivs (shell_model.rs:242-290 + eigenpairs :188-240)
template <class R>
inline void shell_d2psi_df2(const Mat3x2<R>& u, const R sigma[2], const Mat2<R>& v, const R deda[2], const R d2[4],
                            R eps, R out[36]) {
  R eigval[2];
  Mat2<R> ev;
  sym_eig2(Mat2<R>{d2[0], d2[2], d2[1], d2[3]}, eigval, ev);
  const R Rr = R(0.70710678118654752440);
  Vt<R> qc0[6], qc1[6];
  qc0[0] = Vt<R>(0, -Rr, 0); qc1[0] = Vt<R>(Rr, 0, 0);
  qc0[1] = Vt<R>(0, Rr, 0);  qc1[1] = Vt<R>(Rr, 0, 0);
  qc0[2] = Vt<R>(0, 0, 1);   qc1[2] = Vt<R>(0, 0, 0);
  qc0[3] = Vt<R>(0, 0, 0);   qc1[3] = Vt<R>(0, 0, 1);
  qc0[4] = Vt<R>(ev.xx, 0, 0); qc1[4] = Vt<R>(0, ev.xy, 0);
  qc0[5] = Vt<R>(ev.yx, 0, 0); qc1[5] = Vt<R>(0, ev.yy, 0);
  R a = sigma[0], b = sigma[1];
  R denom = a - b;
  R fallback = R(0.5) * (d2[0] + d2[3]) - R(0.5) * (d2[1] + d2[2]);
  R lam[6] = {(deda[0] + deda[1]) / (a + b), std::fabs(denom) > eps ? (deda[0] - deda[1]) / denom : fallback,
              deda[0] / a, deda[1] / b, eigval[0], eigval[1]};
  Vt<R> u2 = u.c0.cross(u.c1);
  for (int k = 0; k < 36; ++k) out[k] = 0;
  Mat2<R> vt = v.transpose();
  for (int k = 0; k < 6; ++k) {
    R l = rmax(lam[k], R(0));
    if (l == 0) continue;
    auto col = [&](const Vt<R>& c) { return u.c0 * c.x + u.c1 * c.y + u2 * c.z; };
    Mat3x2<R> uq{col(qc0[k]), col(qc1[k])};
    R qv[6];
    uq.mul_mat2(vt).vec6(qv);
    for (int r = 0; r < 6; ++r)
      for (int c = 0; c < 6; ++c) out[r * 6 + c] += l * qv[r] * qv[c];
  }
}

template <class R>
struct ShellEl {
  uint32_t v[3];
  Mat2<R> dm_inv;
  R area;
};

// build_shells (shell_model.rs:310-348)
template <class R>
inline bool build_shell(const Vt<R>& p0, const Vt<R>& p1, const Vt<R>& p2, R min_area, ShellEl<R>& el) {
  Vt<R> e1 = p1 - p0, e2 = p2 - p0;
  Vt<R> n = e1.cross(e2);
  R area = R(0.5) * n.length();
  if (area <= min_area) return false;
  Vt<R> ax = e1.normalize();
  Vt<R> ay = (e2 - ax * e2.dot(ax)).normalize();
  Mat2<R> dm{e1.dot(ax), e1.dot(ay), e2.dot(ax), e2.dot(ay)};
  if (std::fabs(dm.det()) < R(1.0e-20)) return false;
  el.dm_inv = dm.inverse();
  el.area = area;
  return true;
}

template <class R>
inline Mat3x2<R> shell_F(const Vt<R> p[3], const Mat2<R>& dm_inv) {
  return Mat3x2<R>{p[1] - p[0], p[2] - p[0]}.mul_mat2(dm_inv);
}

// shell_gradient_analytic (shell_model.rs:366-380)
template <class R>
inline void shell_gradient(const Vt<R> p[3], const ShellEl<R>& el, R mu, R lambda, Vt<R> out[3]) {
  Mat3x2<R> f = shell_F(p, el.dm_inv);
  Mat3x2<R> u;
  R sigma[2];
  Mat2<R> v;
  svd3x2(f, u, sigma, v);
  R d[2];
  stvk_dpsi(sigma, mu, lambda, d);
  Mat3x2<R> pk1 = Mat3x2<R>{u.c0 * d[0], u.c1 * d[1]}.mul_mat2(v.transpose());
  Mat3x2<R> h = pk1.mul_mat2(el.dm_inv.transpose());
  Vt<R> g1 = h.c0 * el.area, g2 = h.c1 * el.area;
  out[0] = -(g1 + g2);
  out[1] = g1;
  out[2] = g2;
}

template <class R>
inline R shell_energy(const Vt<R> p[3], const ShellEl<R>& el, R mu, R lambda) {
  Mat3x2<R> f = shell_F(p, el.dm_inv);
  Mat3x2<R> u;
  R sigma[2];
  Mat2<R> v;
  svd3x2(f, u, sigma, v);
  return el.area * stvk_density(sigma, mu, lambda);
}

// shell_dfdx (shell_model.rs:384-400): dvec(F)/dx as a 6 x 9 row-major matrix.
template <class R>
inline void shell_dfdx(const Mat2<R>& dm_inv, R b[54]) {
  for (int k = 0; k < 54; ++k) b[k] = 0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 2; ++j) {
      int row = 2 * i + j;
      R sum = 0;
      for (int k = 0; k < 2; ++k) {
        R d = dm_inv.at(k, j);
        b[row * 9 + 3 * (k + 1) + i] = d;
        sum += d;
      }
      b[row * 9 + i] = -sum;
    }
}

// shell_hessian_analytic (shell_model.rs:403-438)
template <class R>
inline void shell_hessian(const Vt<R> p[3], const ShellEl<R>& el, R mu, R lambda, R eps, R h[81]) {
  Mat3x2<R> f = shell_F(p, el.dm_inv);
  Mat3x2<R> u;
  R sigma[2];
  Mat2<R> v;
  svd3x2(f, u, sigma, v);
  R deda[2], d2[4];
  stvk_dpsi(sigma, mu, lambda, deda);
  stvk_d2psi(sigma, mu, lambda, d2);
  R a6[36];
  shell_d2psi_df2(u, sigma, v, deda, d2, eps, a6);
  R b[54];
  shell_dfdx(el.dm_inv, b);
  R ab[54];
  for (int r = 0; r < 6; ++r)
    for (int c = 0; c < 9; ++c) {
      R acc = 0;
      for (int k = 0; k < 6; ++k) acc += a6[r * 6 + k] * b[k * 9 + c];
      ab[r * 9 + c] = acc;
    }
  for (int r = 0; r < 9; ++r)
    for (int c = 0; c < 9; ++c) {
      R acc = 0;
      for (int k = 0; k < 6; ++k) acc += b[k * 9 + r] * ab[k * 9 + c];
      h[r * 9 + c] = el.area * acc;
    }
}

// ---------------------------------------------------------------------------------------
// Strain limiting: the per-face barrier on the principal-stretch excess
// (shell_model.rs:438-640) and the one-sided per-edge spring (strain_limit.rs:24-63).
// ---------------------------------------------------------------------------------------
// SL_GAP_FLOOR (shell_model.rs:444): the barrier argument never drops below this fraction
// of the limit.
template <class R>
inline R sl_gap_floor() { return R(1.0e-3); }

// strain_limit_derivs (shell_model.rs:456-484): (E, dE/da, d2E/da2) over the two principal
// stretch excesses a = sigma - 1; false when neither exceeds rest.
template <class R>
inline bool strain_limit_derivs(const R sigma[2], R limit, BarrierKind kind, R& energy, R deda[2], R d2[4]) {
  if (limit <= 0) return false;
  energy = 0;
  deda[0] = deda[1] = 0;
  d2[0] = d2[1] = d2[2] = d2[3] = 0;
  bool active = false;
  for (int i = 0; i < 2; ++i) {
    R a = sigma[i] - R(1);
    if (a <= 0) continue;
    R y = rmax(limit - a, sl_gap_floor<R>() * limit);
    R e, g, h;
    if (barrier_of(kind, y, limit, R(1), e, g, h)) {
      energy += e;
      deda[i] = -g;
      d2[i * 2 + i] = h;
      active = true;
    }
  }
  return active;
}

// strain_limit_energy (shell_model.rs:493-502), no area factor.
template <class R>
inline R strain_limit_energy(const Vt<R> p[3], const ShellEl<R>& el, R limit, BarrierKind kind) {
  Mat3x2<R> f = shell_F(p, el.dm_inv);
  Mat3x2<R> u;
  R sigma[2];
  Mat2<R> v;
  svd3x2(f, u, sigma, v);
  R e, deda[2], d2[4];
  return strain_limit_derivs(sigma, limit, kind, e, deda, d2) ? e : R(0);
}

// The barrier's 9-vector gradient and 9x9 Hessian at unit stiffness (shell_model.rs:508-561)
// when `stiffness` is 1 and `elastic_k`/`face_mass` are unused; strain_limit_assembly
// (:582-640) otherwise: stiffness = max(elastic_k, 0) + face_mass / d^2 with d the headroom
// limit - max(sigma - 1), floored. Returns false when the term is inactive.
template <class R>
inline bool strain_limit_eval(const Vt<R> p[3], const ShellEl<R>& el, R limit, R face_mass, R elastic_k,
                              BarrierKind kind, R eps, bool dynamic_stiffness, Vt<R> grad[3], R hess[81]) {
  Mat3x2<R> f = shell_F(p, el.dm_inv);
  Mat3x2<R> u;
  R sigma[2];
  Mat2<R> v;
  svd3x2(f, u, sigma, v);
  R energy, deda[2], d2[4];
  if (!strain_limit_derivs(sigma, limit, kind, energy, deda, d2)) return false;
  R stiffness = R(1);
  if (dynamic_stiffness) {
    R max_a = rmax(sigma[0] - R(1), sigma[1] - R(1));
    R d = rmax(limit - max_a, sl_gap_floor<R>() * limit);
    stiffness = rmax(elastic_k, R(0)) + face_mass / (d * d);
    if (stiffness <= 0) return false;
  }
  Mat3x2<R> pk1 = Mat3x2<R>{u.c0 * deda[0], u.c1 * deda[1]}.mul_mat2(v.transpose());
  Mat3x2<R> hg = pk1.mul_mat2(el.dm_inv.transpose());
  Vt<R> g1 = dynamic_stiffness ? hg.c0 * stiffness : hg.c0;
  Vt<R> g2 = dynamic_stiffness ? hg.c1 * stiffness : hg.c1;
  grad[0] = -(g1 + g2);
  grad[1] = g1;
  grad[2] = g2;
  R a6[36];
  shell_d2psi_df2(u, sigma, v, deda, d2, eps, a6);
  R b[54];
  shell_dfdx(el.dm_inv, b);
  R ab[54];
  for (int r = 0; r < 6; ++r)
    for (int c = 0; c < 9; ++c) {
      R acc = 0;
      for (int k = 0; k < 6; ++k) acc += a6[r * 6 + k] * b[k * 9 + c];
      ab[r * 9 + c] = acc;
    }
  for (int r = 0; r < 9; ++r)
    for (int c = 0; c < 9; ++c) {
      R acc = 0;
      for (int k = 0; k < 6; ++k) acc += b[k * 9 + r] * ab[k * 9 + c];
      hess[r * 9 + c] = dynamic_stiffness ? stiffness * acc : acc;
    }
  return true;
}

// The largest principal-stretch excess max(sigma - 1) of a face at positions p
// (the quantity the strain-limit line search bisects on, implicit.rs:1719-1729).
template <class R>
inline R max_stretch_excess(const Vt<R> p[3], const Mat2<R>& dm_inv) {
  Mat3x2<R> f = shell_F(p, dm_inv);
  Mat3x2<R> u;
  R sigma[2];
  Mat2<R> v;
  svd3x2(f, u, sigma, v);
  return rmax(sigma[0] - R(1), sigma[1] - R(1));
}

// ---------------------------------------------------------------------------------------
// bending.rs
// ---------------------------------------------------------------------------------------
template <class R>
struct Hinge {
  uint32_t v[4];
  R rest, w;
};

template <class R>
inline R dihedral_angle(const Vt<R> p[4]) {
  Vt<R> n1 = (p[1] - p[0]).cross(p[2] - p[0]);
  Vt<R> n2 = (p[1] - p[2]).cross(p[3] - p[2]);
  Vt<R> e = (p[2] - p[1]).normalize_or_zero();
  Vt<R> n1n = n1.normalize_or_zero(), n2n = n2.normalize_or_zero();
  R s = n1n.cross(n2n).dot(e);
  R c = rclamp(n1n.dot(n2n), R(-1), R(1));
  return std::atan2(s, c);
}

template <class R>
inline void dihedral_grad_fd(const Vt<R> p[4], Vt<R> g[4]) {
  R scale = rmax(p[0].length() + p[1].length() + p[2].length() + p[3].length(), R(1));
  R h = R(1.0e-4) * scale;
  R inv = R(1) / (R(2) * h);
  for (int vi = 0; vi < 4; ++vi)
    for (int c = 0; c < 3; ++c) {
      Vt<R> pp[4] = {p[0], p[1], p[2], p[3]}, pm[4] = {p[0], p[1], p[2], p[3]};
      pp[vi][c] += h;
      pm[vi][c] -= h;
      g[vi][c] = (dihedral_angle(pp) - dihedral_angle(pm)) * inv;
    }
}

// dihedral_grad_analytic (bending.rs:77-103)
template <class R>
inline void dihedral_grad(const Vt<R> p[4], Vt<R> g[4]) {
  Vt<R> m1 = (p[1] - p[0]).cross(p[2] - p[0]);
  Vt<R> m2 = (p[1] - p[2]).cross(p[3] - p[2]);
  Vt<R> e = p[2] - p[1];
  R a1 = m1.length(), a2 = m2.length(), l2 = e.length_squared();
  if (a1 < R(1.0e-12) || a2 < R(1.0e-12) || l2 < R(1.0e-24)) {
    dihedral_grad_fd(p, g);
    return;
  }
  R l = std::sqrt(l2);
  Vt<R> n1 = m1 / a1, n2 = m2 / a2;
  Vt<R> g0 = n1 * (-l / a1);
  Vt<R> g3 = n2 * (-l / a2);
  R ta = (p[0] - p[1]).dot(e) / l2;
  R tb = (p[3] - p[1]).dot(e) / l2;
  g[0] = g0;
  g[1] = g0 * (ta - R(1)) + g3 * (tb - R(1));
  g[2] = g0 * (-ta) + g3 * (-tb);
  g[3] = g3;
}

// build_hinges (bending.rs:126-158): edge key sorted; hinge = [opp0, a, b, opp1].
template <class R>
inline std::vector<Hinge<R>> build_hinges(const std::vector<std::array<uint32_t, 3>>& tris,
                                          const std::vector<Vt<R>>& pos) {
  std::map<std::pair<uint32_t, uint32_t>, std::vector<uint32_t>> m;
  for (const auto& t : tris) {
    uint32_t e[3][3] = {{t[1], t[2], t[0]}, {t[0], t[2], t[1]}, {t[0], t[1], t[2]}};
    for (auto& x : e) {
      auto key = x[0] < x[1] ? std::make_pair(x[0], x[1]) : std::make_pair(x[1], x[0]);
      m[key].push_back(x[2]);
    }
  }
  std::vector<Hinge<R>> out;
  for (auto& kv : m) {
    if (kv.second.size() != 2) continue;
    Hinge<R> h;
    h.v[0] = kv.second[0];
    h.v[1] = kv.first.first;
    h.v[2] = kv.first.second;
    h.v[3] = kv.second[1];
    Vt<R> p[4] = {pos[h.v[0]], pos[h.v[1]], pos[h.v[2]], pos[h.v[3]]};
    h.rest = dihedral_angle(p);
    h.w = 1;
    out.push_back(h);
  }
  return out;
}

// ---------------------------------------------------------------------------------------
// stitch.rs
// ---------------------------------------------------------------------------------------
template <class R>
struct Stitch {
  uint32_t index[6];
  R weight[6];
  R stiffness, l0, l_cap;
};

// force_hessian (stitch.rs:57-107) at unit stiffness; hess is 18 x 18 row-major.
template <class R>
inline void stitch_force_hessian(const Vt<R> x[6], const R w[6], R l0, R l_cap, Vt<R> grad[6], R* hess) {
  R sw[6];
  for (int k = 0; k < 6; ++k) sw[k] = k < 3 ? w[k] : -w[k];
  Vt<R> t;
  for (int k = 0; k < 6; ++k) t += x[k] * sw[k];
  R tn = t.length();
  for (int k = 0; k < 324; ++k) hess[k] = 0;
  if (tn < R(1.0e-12) || l0 <= 0) {
    for (int k = 0; k < 6; ++k) grad[k] = Vt<R>();
    return;
  }
  R l = rmin(tn, l_cap);
  Vt<R> n = t / l;
  Vt<R> dedt = n * (l / l0 - R(1));
  for (int k = 0; k < 6; ++k) grad[k] = dedt * sw[k];
  R r = (l - l0) / l;
  R c0 = rmax(R(1) - r, R(0)) / l0;
  R c1 = rmax(r / l0, R(0));
  Vt<R> gv[6];
  for (int k = 0; k < 6; ++k) gv[k] = n * sw[k];
  for (int a = 0; a < 6; ++a)
    for (int b = 0; b < 6; ++b) {
      R iden = c1 * sw[a] * sw[b];
      for (int rr = 0; rr < 3; ++rr)
        for (int cc = 0; cc < 3; ++cc) {
          R v = c0 * gv[a][rr] * gv[b][cc];
          if (rr == cc) v += iden;
          hess[(3 * a + rr) * 18 + 3 * b + cc] = v;
        }
    }
}

// spring_block (implicit.rs:3240-3263)
template <class R>
inline void spring_block(const Vt<R>& d, R rest, R k, R h[3][3], Vt<R>& g) {
  R l = d.length();
  if (l < R(1.0e-9)) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) h[i][j] = i == j ? k : R(0);
    g = Vt<R>();
    return;
  }
  Vt<R> nrm = d / l;
  R coeff_t = rmax(R(1) - rest / l, R(0));
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      R nnt = nrm[i] * nrm[j];
      R iden = i == j ? R(1) : R(0);
      h[i][j] = k * (nnt + coeff_t * (iden - nnt));
    }
  g = nrm * (k * (l - rest));
}

// strain_energy / strain_block (strain_limit.rs:31-63): a spring of rest length
// max_ratio * rest acting only while the edge is longer than that. Returns grad_i and h_ii
// (grad_j = -grad_i, h_jj = h_ii, h_ij = h_ji = -h_ii).
template <class R>
inline R edge_strain_energy(const Vt<R>& xi, const Vt<R>& xj, R rest, R max_ratio, R k) {
  R l = (xi - xj).length();
  R r = rest * max_ratio;
  return l > r ? R(0.5) * k * (l - r) * (l - r) : R(0);
}
template <class R>
inline void edge_strain_block(const Vt<R>& xi, const Vt<R>& xj, R rest, R max_ratio, R k, Vt<R>& g, R h[3][3]) {
  Vt<R> d = xi - xj;
  R r = rest * max_ratio;
  if (d.length() <= r) {
    g = Vt<R>();
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) h[i][j] = 0;
    return;
  }
  spring_block(d, r, k, h, g);
}

// ---------------------------------------------------------------------------------------
// membrane.rs: Baraff-Witkin membrane (warp / weft stretch and shear conditions)
// ---------------------------------------------------------------------------------------
template <class R>
struct MembraneEl {
  uint32_t tri[3];
  R dm_inv[2][2];  // row-major
  R area;
};

// deformation (membrane.rs:43-51): the columns wu, wv of F = Ds Dm^-1.
template <class R>
inline void bw_deformation(const Vt<R> p[3], const R dm[2][2], Vt<R>& wu, Vt<R>& wv) {
  Vt<R> ds0 = p[1] - p[0], ds1 = p[2] - p[0];
  wu = ds0 * dm[0][0] + ds1 * dm[1][0];
  wv = ds0 * dm[0][1] + ds1 * dm[1][1];
}

// conditions (membrane.rs:53-57): Cu = |wu| - 1, Cv = |wv| - 1, Csh = wu.wv.
template <class R>
inline void bw_conditions(const Vt<R> p[3], const R dm[2][2], R c[3]) {
  Vt<R> wu, wv;
  bw_deformation(p, dm, wu, wv);
  c[0] = wu.length() - R(1);
  c[1] = wv.length() - R(1);
  c[2] = wu.dot(wv);
}

// stretch_coeffs (membrane.rs:86-91): wu = sum cu_j x_j, wv = sum cv_j x_j.
template <class R>
inline void bw_coeffs(const R dm[2][2], R cu[3], R cv[3]) {
  R a0 = dm[0][0], a1 = dm[1][0], b0 = dm[0][1], b1 = dm[1][1];
  cu[0] = -(a0 + a1); cu[1] = a0; cu[2] = a1;
  cv[0] = -(b0 + b1); cv[1] = b0; cv[2] = b1;
}

// condition_grads (membrane.rs:65-84): g[condition][vertex].
template <class R>
inline void bw_condition_grads(const Vt<R> p[3], const R dm[2][2], Vt<R> g[3][3]) {
  Vt<R> wu, wv;
  bw_deformation(p, dm, wu, wv);
  R cu[3], cv[3];
  bw_coeffs(dm, cu, cv);
  Vt<R> nu = wu.normalize_or_zero(), nv = wv.normalize_or_zero();
  for (int j = 0; j < 3; ++j) {
    g[0][j] = nu * cu[j];
    g[1][j] = nv * cv[j];
    g[2][j] = wv * cu[j] + wu * cv[j];
  }
}

// stretch_eigen_material (membrane.rs:100-120): n n^T + max(0, 1 - 1/|w|) (I - n n^T).
template <class R>
inline void bw_stretch_material(const Vt<R>& w, R m[3][3]) {
  R s = w.length();
  Vt<R> n = w.normalize_or_zero();
  R perp = s > R(1.0e-6) ? rmax(R(1) - R(1) / s, R(0)) : R(0);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      R nnt = n[r] * n[c];
      R iden = r == c ? R(1) : R(0);
      m[r][c] = nnt + perp * (iden - nnt);
    }
}

template <class R>
inline void bw_add_outer(R m[3][3], const Vt<R>& u, const Vt<R>& v, R s) {
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) m[r][c] += s * u[r] * v[c];
}

template <class R>
inline void bw_proj_perp(const Vt<R>& w, R q[3][3]) {
  Vt<R> n = w.normalize_or_zero();
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) q[r][c] = (r == c ? R(1) : R(0)) - n[r] * n[c];
}

// shear_material (membrane.rs:164-205): the blocks [uu, uv, vu, vv] of the eigen-projected
// (clamp) or exact (no clamp) 6x6 shear Hessian in (wu; wv).
template <class R>
inline void bw_shear_material(const Vt<R>& wu, const Vt<R>& wv, bool clamp, R m[4][3][3]) {
  R f = wu.dot(wv);
  R a = wu.length_squared() + wv.length_squared();
  R disc = std::sqrt(rmax(a * a + R(12) * f * f, R(0)));
  R mu[2] = {R(0.5) * (a + disc), R(0.5) * (a - disc)};
  auto ev = [&](R x) { return clamp ? rmax(x, R(0)) : x; };
  for (int b = 0; b < 4; ++b)
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) m[b][r][c] = 0;
  for (R mui : mu) {
    Vt<R> top = wv * mui + wu * f, bot = wu * mui + wv * f;
    R n = top.length_squared() + bot.length_squared();
    if (n > R(1e-20)) {
      R sc = ev(mui) / n;
      bw_add_outer(m[0], top, top, sc);
      bw_add_outer(m[1], top, bot, sc);
      bw_add_outer(m[2], bot, top, sc);
      bw_add_outer(m[3], bot, bot, sc);
    }
  }
  R fp = R(0.5) * ev(f);
  if (fp != 0) {
    R qp[3][3];
    bw_proj_perp(wu + wv, qp);
    for (int b = 0; b < 4; ++b)
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) m[b][r][c] += fp * qp[r][c];
  }
  R fm = R(0.5) * ev(-f);
  if (fm != 0) {
    R qm[3][3];
    bw_proj_perp(wv - wu, qm);
    const R sgn[4] = {R(1), R(-1), R(-1), R(1)};
    for (int b = 0; b < 4; ++b)
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) m[b][r][c] += (sgn[b] * fm) * qm[r][c];
  }
}

// build_membrane (membrane.rs:272-312) for one triangle; false when degenerate.
template <class R>
inline bool build_membrane_el(const Vt<R>& x0, const Vt<R>& x1, const Vt<R>& x2, MembraneEl<R>& el) {
  Vt<R> e1 = x1 - x0, e2 = x2 - x0;
  R a = e1.length();
  Vt<R> n = e1.cross(e2);
  R area = R(0.5) * n.length();
  if (a < R(1.0e-9) || area < R(1.0e-12)) return false;
  Vt<R> t1 = e1 / a;
  Vt<R> t2 = n.cross(e1).normalize_or_zero();
  R b = e2.dot(t1), d = e2.dot(t2);
  R det = a * d;
  if (std::fabs(det) < R(1.0e-12)) return false;
  el.dm_inv[0][0] = R(1) / a;
  el.dm_inv[0][1] = -b / (a * d);
  el.dm_inv[1][0] = 0;
  el.dm_inv[1][1] = R(1) / d;
  el.area = area;
  return true;
}

// element_assembly (membrane.rs:225-270): gradient (vertex-major) and 9x9 Hessian of one
// element for stiffnesses (kw, kf, ks).
template <class R>
inline void bw_element(const Vt<R> p[3], const MembraneEl<R>& el, R kw, R kf, R ks, R grad[9], R hess[81]) {
  R c[3];
  bw_conditions(p, el.dm_inv, c);
  Vt<R> g[3][3];
  bw_condition_grads(p, el.dm_inv, g);
  R cu[3], cv[3];
  bw_coeffs(el.dm_inv, cu, cv);
  Vt<R> wu, wv;
  bw_deformation(p, el.dm_inv, wu, wv);
  R mu_[3][3], mv_[3][3], sm[4][3][3];
  bw_stretch_material(wu, mu_);
  bw_stretch_material(wv, mv_);
  bw_shear_material(wu, wv, true, sm);
  for (int k = 0; k < 9; ++k) grad[k] = 0;
  for (int k = 0; k < 81; ++k) hess[k] = 0;
  const R kc[3] = {kw, kf, ks};
  for (int ci = 0; ci < 3; ++ci) {
    R ka = kc[ci] * el.area;
    if (ka <= 0) continue;
    for (int a = 0; a < 3; ++a) {
      for (int cc = 0; cc < 3; ++cc) grad[3 * a + cc] += ka * c[ci] * g[ci][a][cc];
      for (int b = 0; b < 3; ++b)
        for (int r = 0; r < 3; ++r)
          for (int cc = 0; cc < 3; ++cc) {
            R v;
            if (ci < 2) {
              const R* co = ci == 0 ? cu : cv;
              R(*m)[3] = ci == 0 ? mu_ : mv_;
              v = ka * co[a] * co[b] * m[r][cc];
            } else {
              v = ka * (cu[a] * cu[b] * sm[0][r][cc] + cu[a] * cv[b] * sm[1][r][cc] + cv[a] * cu[b] * sm[2][r][cc] +
                        cv[a] * cv[b] * sm[3][r][cc]);
            }
            hess[(3 * a + r) * 9 + (3 * b + cc)] += v;
          }
    }
  }
}

// ---------------------------------------------------------------------------------------
// broadphase.rs: uniform hash grid
// ---------------------------------------------------------------------------------------
struct CellKey {
  int32_t x, y, z;
  bool operator==(const CellKey& o) const { return x == o.x && y == o.y && z == o.z; }
};
struct CellHash {
  size_t operator()(const CellKey& k) const {
    return (size_t)((uint64_t)(uint32_t)k.x * 73856093ull ^ (uint64_t)(uint32_t)k.y * 19349663ull ^
                    (uint64_t)(uint32_t)k.z * 83492791ull);
  }
};

// CellGrid (broadphase.rs:65-100): items of a cell in insertion order.
struct CellGrid {
  std::unordered_map<CellKey, std::pair<uint32_t, uint32_t>, CellHash> at;
  std::vector<uint32_t> items;
  void build(const std::vector<std::pair<CellKey, uint32_t>>& ins) {
    at.clear();
    for (auto& e : ins) at[e.first].second += 1;
    uint32_t acc = 0;
    for (auto& kv : at) {
      kv.second.first = acc;
      acc += kv.second.second;
      kv.second.second = 0;
    }
    items.assign(ins.size(), 0);
    for (auto& e : ins) {
      auto& c = at[e.first];
      items[c.first + c.second] = e.second;
      c.second += 1;
    }
  }
  template <class F>
  void each(const CellKey& c, F f) const {
    auto it = at.find(c);
    if (it == at.end()) return;
    for (uint32_t k = 0; k < it->second.second; ++k) f(items[it->second.first + k]);
  }
};

inline int32_t floor_i32(double v) {
  double f = std::floor(v);
  if (!(f == f)) return 0;
  if (f >= 2147483647.0) return 2147483647;
  if (f <= -2147483648.0) return (int32_t)-2147483648LL;
  return (int32_t)f;
}

template <class R>
inline R grid_cell(R search, R extent) { return rmax(rmax(search, extent), R(1.0e-6)); }

template <class R>
inline R mean_edge_len(const std::vector<Vt<R>>& pos, const std::vector<std::array<uint32_t, 2>>& edges) {
  if (edges.empty()) return 0;
  R sum = 0;
  for (auto& e : edges) sum += (pos[e[0]] - pos[e[1]]).length();
  return sum / (R)edges.size();
}

template <class R>
inline R mean_tri_extent(const std::vector<Vt<R>>& pos, const std::vector<std::array<uint32_t, 3>>& tris) {
  if (tris.empty()) return 0;
  R sum = 0;
  for (auto& t : tris) {
    Vt<R> a = pos[t[0]], b = pos[t[1]], c = pos[t[2]];
    Vt<R> d = a.vmax(b).vmax(c) - a.vmin(b).vmin(c);
    sum += rmax(rmax(d.x, d.y), d.z);
  }
  return sum / (R)tris.size();
}

// for_each_vertex_triangle_pair (broadphase.rs:263-330)
template <class R, class F>
inline void for_each_vertex_triangle_pair(const std::vector<Vt<R>>& pos, const std::vector<std::array<uint32_t, 3>>& tris,
                                          R dhat, const std::vector<std::vector<uint32_t>>& excluded,
                                          const std::vector<uint8_t>& movable, F visit) {
  if (pos.empty() || tris.empty()) return;
  R cell = grid_cell(dhat, mean_tri_extent(pos, tris));
  R inv = R(1) / cell;
  auto key = [&](const Vt<R>& p) {
    return CellKey{floor_i32((double)(p.x * inv)), floor_i32((double)(p.y * inv)), floor_i32((double)(p.z * inv))};
  };
  std::vector<std::pair<CellKey, uint32_t>> ins;
  ins.reserve(pos.size());
  for (size_t i = 0; i < pos.size(); ++i) ins.push_back({key(pos[i]), (uint32_t)i});
  CellGrid grid;
  grid.build(ins);
  Vt<R> sd(dhat, dhat, dhat);
  for (size_t ti = 0; ti < tris.size(); ++ti) {
    const auto& t = tris[ti];
    Vt<R> pa = pos[t[0]], pb = pos[t[1]], pc = pos[t[2]];
    Vt<R> lo = pa.vmin(pb).vmin(pc) - sd, hi = pa.vmax(pb).vmax(pc) + sd;
    bool tri_mov = movable.empty() || movable[t[0]] || movable[t[1]] || movable[t[2]];
    CellKey kl = key(lo), kh = key(hi);
    for (int32_t cx = kl.x; cx <= kh.x; ++cx)
      for (int32_t cy = kl.y; cy <= kh.y; ++cy)
        for (int32_t cz = kl.z; cz <= kh.z; ++cz)
          grid.each(CellKey{cx, cy, cz}, [&](uint32_t v) {
            if (!tri_mov && !movable[v]) return;
            for (uint32_t e : excluded[v])
              if (e == t[0] || e == t[1] || e == t[2]) return;
            visit(v, (uint32_t)ti);
          });
  }
}

// for_each_edge_edge_pair (broadphase.rs:395-526)
template <class R, class F>
inline void for_each_edge_edge_pair(const std::vector<Vt<R>>& pos, const std::vector<std::array<uint32_t, 2>>& edges,
                                    R search, const std::vector<uint8_t>& movable, F visit) {
  if (edges.size() < 2) return;
  std::vector<uint8_t> em;
  if (!movable.empty()) {
    em.resize(edges.size());
    for (size_t i = 0; i < edges.size(); ++i) em[i] = movable[edges[i][0]] || movable[edges[i][1]];
  }
  auto e_mov = [&](uint32_t i) { return em.empty() || em[i]; };
  R cell = grid_cell(search, mean_edge_len(pos, edges));
  R inv = R(1) / cell;
  auto key = [&](R v) { return floor_i32((double)(v * inv)); };
  auto cells = [&](const std::array<uint32_t, 2>& e, R pad, int32_t lo[3], int32_t hi[3]) {
    Vt<R> p = pos[e[0]], q = pos[e[1]];
    Vt<R> l = p.vmin(q) - Vt<R>(pad, pad, pad), h = p.vmax(q) + Vt<R>(pad, pad, pad);
    lo[0] = key(l.x); lo[1] = key(l.y); lo[2] = key(l.z);
    hi[0] = key(h.x); hi[1] = key(h.y); hi[2] = key(h.z);
  };
  std::vector<std::pair<CellKey, uint32_t>> ins;
  for (size_t ei = 0; ei < edges.size(); ++ei) {
    if (!e_mov((uint32_t)ei)) continue;
    int32_t lo[3], hi[3];
    cells(edges[ei], R(0), lo, hi);
    for (int32_t cx = lo[0]; cx <= hi[0]; ++cx)
      for (int32_t cy = lo[1]; cy <= hi[1]; ++cy)
        for (int32_t cz = lo[2]; cz <= hi[2]; ++cz) ins.push_back({CellKey{cx, cy, cz}, (uint32_t)ei});
  }
  if (ins.empty()) return;
  CellGrid grid;
  grid.build(ins);
  for (size_t j = 0; j < edges.size(); ++j) {
    uint32_t ej = (uint32_t)j;
    const auto& eb = edges[j];
    int32_t lo[3], hi[3];
    cells(eb, search, lo, hi);
    for (int32_t cx = lo[0]; cx <= hi[0]; ++cx)
      for (int32_t cy = lo[1]; cy <= hi[1]; ++cy)
        for (int32_t cz = lo[2]; cz <= hi[2]; ++cz)
          grid.each(CellKey{cx, cy, cz}, [&](uint32_t ei) {
            if (ei == ej || (ei > ej && e_mov(ej))) return;
            const auto& ea = edges[ei];
            if (ea[0] == eb[0] || ea[0] == eb[1] || ea[1] == eb[0] || ea[1] == eb[1]) return;
            visit(std::min(ei, ej), std::max(ei, ej));
          });
  }
}

// The cells of an edge's or a triangle's box padded by `search` (the edge/triangle grids of
// broadphase.rs:523-751 key a coordinate as floor(v / cell) in the scalar type).
template <class R>
struct EtCells {
  const std::vector<Vt<R>>& pos;
  R search, inv;
  CellKey key(const Vt<R>& p) const {
    return CellKey{floor_i32((double)(p.x * inv)), floor_i32((double)(p.y * inv)), floor_i32((double)(p.z * inv))};
  }
  void edge(const std::array<uint32_t, 2>& e, CellKey& lo, CellKey& hi) const {
    const Vt<R> p = pos[e[0]], q = pos[e[1]], pad(search, search, search);
    lo = key(p.vmin(q) - pad);
    hi = key(p.vmax(q) + pad);
  }
  void tri(const std::array<uint32_t, 3>& t, CellKey& lo, CellKey& hi) const {
    const Vt<R> a = pos[t[0]], b = pos[t[1]], c = pos[t[2]], pad(search, search, search);
    lo = key(a.vmin(b).vmin(c) - pad);
    hi = key(a.vmax(b).vmax(c) + pad);
  }
};

inline bool et_adjacent(const std::array<uint32_t, 2>& e, const std::array<uint32_t, 3>& t) {
  return e[0] == t[0] || e[0] == t[1] || e[0] == t[2] || e[1] == t[0] || e[1] == t[1] || e[1] == t[2];
}

// edge_triangle_pairs (broadphase.rs:523-585): every edge hashed into the cells of its box
// padded by search, every triangle's padded cells scanned; pairs sharing a vertex skipped;
// the (edge, triangle) pairs sorted and deduplicated. Cell size: grid_cell(search,
// max(mean edge length, mean triangle extent)).
template <class R>
inline std::vector<std::pair<uint32_t, uint32_t>> edge_triangle_pairs(const std::vector<Vt<R>>& pos,
                                                                      const std::vector<std::array<uint32_t, 2>>& edges,
                                                                      const std::vector<std::array<uint32_t, 3>>& tris,
                                                                      R search) {
  std::vector<std::pair<uint32_t, uint32_t>> pairs;
  if (edges.empty() || tris.empty()) return pairs;
  const R cell = grid_cell(search, rmax(mean_edge_len(pos, edges), mean_tri_extent(pos, tris)));
  const EtCells<R> cells{pos, search, R(1) / cell};
  std::vector<std::pair<CellKey, uint32_t>> ins;
  for (size_t ei = 0; ei < edges.size(); ++ei) {
    CellKey lo, hi;
    cells.edge(edges[ei], lo, hi);
    for (int32_t cx = lo.x; cx <= hi.x; ++cx)
      for (int32_t cy = lo.y; cy <= hi.y; ++cy)
        for (int32_t cz = lo.z; cz <= hi.z; ++cz) ins.push_back({CellKey{cx, cy, cz}, (uint32_t)ei});
  }
  CellGrid grid;
  grid.build(ins);
  for (size_t ti = 0; ti < tris.size(); ++ti) {
    CellKey lo, hi;
    cells.tri(tris[ti], lo, hi);
    for (int32_t cx = lo.x; cx <= hi.x; ++cx)
      for (int32_t cy = lo.y; cy <= hi.y; ++cy)
        for (int32_t cz = lo.z; cz <= hi.z; ++cz)
          grid.each(CellKey{cx, cy, cz}, [&](uint32_t ei) {
            if (!et_adjacent(edges[ei], tris[ti])) pairs.push_back({ei, (uint32_t)ti});
          });
  }
  std::sort(pairs.begin(), pairs.end());
  pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
  return pairs;
}

// any_edge_triangle_pair (broadphase.rs:587-751): the candidates of edge_triangle_pairs
// streamed to hit(edge, triangle) until it returns true (the return value). With a movable
// mask (u8 per vertex; empty = unfiltered) it runs two passes, each indexing only the
// movable primitives of one kind: pass A hashes the edges with a movable vertex and scans
// every triangle, pass B hashes the triangles with a movable vertex and scans the edges
// with none, so pairs whose every vertex is immovable are never offered. A pair may be
// offered more than once (an edge and a triangle sharing several cells).
template <class R, class F>
inline bool any_edge_triangle_pair(const std::vector<Vt<R>>& pos, const std::vector<std::array<uint32_t, 2>>& edges,
                                   const std::vector<std::array<uint32_t, 3>>& tris, R search,
                                   const std::vector<uint8_t>& movable, F hit) {
  if (edges.empty() || tris.empty()) return false;
  const R cell = grid_cell(search, rmax(mean_edge_len(pos, edges), mean_tri_extent(pos, tris)));
  const EtCells<R> cells{pos, search, R(1) / cell};
  auto e_mov = [&](const std::array<uint32_t, 2>& e) { return movable.empty() || movable[e[0]] || movable[e[1]]; };
  auto t_mov = [&](const std::array<uint32_t, 3>& t) {
    return movable.empty() || movable[t[0]] || movable[t[1]] || movable[t[2]];
  };
  // pass A: movable edges indexed, every triangle scanned
  std::vector<std::pair<CellKey, uint32_t>> ins;
  for (size_t ei = 0; ei < edges.size(); ++ei) {
    if (!e_mov(edges[ei])) continue;
    CellKey lo, hi;
    cells.edge(edges[ei], lo, hi);
    for (int32_t cx = lo.x; cx <= hi.x; ++cx)
      for (int32_t cy = lo.y; cy <= hi.y; ++cy)
        for (int32_t cz = lo.z; cz <= hi.z; ++cz) ins.push_back({CellKey{cx, cy, cz}, (uint32_t)ei});
  }
  bool found = false;
  {
    CellGrid grid;
    grid.build(ins);
    for (size_t ti = 0; ti < tris.size() && !found; ++ti) {
      CellKey lo, hi;
      cells.tri(tris[ti], lo, hi);
      for (int32_t cx = lo.x; cx <= hi.x && !found; ++cx)
        for (int32_t cy = lo.y; cy <= hi.y && !found; ++cy)
          for (int32_t cz = lo.z; cz <= hi.z && !found; ++cz)
            grid.each(CellKey{cx, cy, cz}, [&](uint32_t ei) {
              if (!found && !et_adjacent(edges[ei], tris[ti]) && hit(ei, (uint32_t)ti)) found = true;
            });
    }
  }
  if (found || movable.empty()) return found;
  // pass B: movable triangles indexed, the edges with no movable vertex scanned
  ins.clear();
  for (size_t ti = 0; ti < tris.size(); ++ti) {
    if (!t_mov(tris[ti])) continue;
    CellKey lo, hi;
    cells.tri(tris[ti], lo, hi);
    for (int32_t cx = lo.x; cx <= hi.x; ++cx)
      for (int32_t cy = lo.y; cy <= hi.y; ++cy)
        for (int32_t cz = lo.z; cz <= hi.z; ++cz) ins.push_back({CellKey{cx, cy, cz}, (uint32_t)ti});
  }
  CellGrid tgrid;
  tgrid.build(ins);
  for (size_t ei = 0; ei < edges.size() && !found; ++ei) {
    if (e_mov(edges[ei])) continue;  // pass A offered it against every triangle
    CellKey lo, hi;
    cells.edge(edges[ei], lo, hi);
    for (int32_t cx = lo.x; cx <= hi.x && !found; ++cx)
      for (int32_t cy = lo.y; cy <= hi.y && !found; ++cy)
        for (int32_t cz = lo.z; cz <= hi.z && !found; ++cz)
          tgrid.each(CellKey{cx, cy, cz}, [&](uint32_t ti) {
            if (!found && !et_adjacent(edges[ei], tris[ti]) && hit((uint32_t)ei, ti)) found = true;
          });
  }
  return found;
}

inline std::vector<std::vector<uint32_t>> one_ring_exclusion(size_t nv, const std::vector<std::array<uint32_t, 3>>& tris) {
  std::vector<std::vector<uint32_t>> ex(nv);
  for (size_t i = 0; i < nv; ++i) ex[i].push_back((uint32_t)i);
  for (auto& t : tris)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        if (a != b) ex[t[a]].push_back(t[b]);
  for (auto& e : ex) {
    std::sort(e.begin(), e.end());
    e.erase(std::unique(e.begin(), e.end()), e.end());
  }
  return ex;
}

inline std::vector<std::array<uint32_t, 2>> unique_edges(const std::vector<std::array<uint32_t, 3>>& tris) {
  std::vector<std::array<uint32_t, 2>> e;
  for (auto& t : tris) {
    uint32_t p[3][2] = {{t[0], t[1]}, {t[1], t[2]}, {t[2], t[0]}};
    for (auto& q : p) e.push_back({std::min(q[0], q[1]), std::max(q[0], q[1])});
  }
  std::sort(e.begin(), e.end());
  e.erase(std::unique(e.begin(), e.end()), e.end());
  return e;
}

// ---------------------------------------------------------------------------------------
// implicit.rs: parameters, solver, assembly, CCD, step
// ---------------------------------------------------------------------------------------
template <class R>
struct Params {
  R dt = R(1.0 / 60.0);
  Vt<R> gravity = Vt<R>(0, R(-9.8), 0);
  uint32_t newton_iters = 4;
  R stiffness = R(1.0e3);
  R bend_stiffness = 0;
  R max_dx = std::numeric_limits<R>::infinity();
  R target_toi = 0;
  uint32_t min_newton_steps = 0;
  uint32_t ccd_max_iter = 256;
  R eiganalysis_eps = R(1.0e-6);
  R contact_dhat = R(1.0e-2);
  R contact_kappa = R(1.0e2);
  R contact_dynamic = 0;
  R shell_mu = 0, shell_lambda = 0;
  R friction = 0, friction_eps = R(1.0e-3);
  R collider_friction = std::numeric_limits<R>::infinity();
  int friction_mode = 0;  // how two coefficients combine: 0 min, 1 max, 2 mean (contact.rs:141-205)
  BarrierKind barrier_kind = BarrierKind::Log;
  bool contact_rayleigh = false;
  bool self_collision = false;
  R cg_tol = R(1.0e-4);
  uint32_t cg_max_iter = 2000;
  R floor_y = -std::numeric_limits<R>::infinity();
  R constraint_tol = R(1.0e-2);  // pin gap floor as a fraction of ghat
  R membrane_warp = 0, membrane_weft = 0, membrane_shear = 0;  // Baraff-Witkin stiffnesses
  R strain_limit_ratio = 0, strain_limit_k = 0, strain_limit_ratio_weft = 0;
  R newton_tol = 0;          // added termination (0 disables)
  int precond = 2;           // 1 block Jacobi (CgCpu), 2 Schwarz
  uint32_t schwarz_domain = 32;
};

// Pin (implicit.rs:230-262, the reference's FixPair): the vertex is confined to a ball of
// radius ghat around target and pulled by k |x - target|^2 / 2 with a dynamic k.
template <class R>
struct Pin {
  uint32_t index;
  Vt<R> target;
  R ghat;
  bool kinematic;
  R stiffness;
};

// Pull (implicit.rs:264-282, the reference's PullPair): w |x - target|^2 / 2.
template <class R>
struct Pull {
  uint32_t index;
  Vt<R> target;
  R weight;
};

// A face under the strain-limit barrier: its element, allowed stretch fraction and mass.
template <class R>
struct SlFace {
  ShellEl<R> el;
  R limit, mass;
};

struct StepStats {
  uint32_t newton_iters = 0, max_cg_iters = 0, num_contacts = 0, stencils = 0, ccd_cap_hits = 0;
  double max_reresid = 0.0;
  double t_min = 1.0;
  int penetration_free = 1, all_finite = 1;
};

template <class R>
struct Stencil {
  uint32_t idx[4];
  R d;
  Vt<R> g[4];
  R ghat;
};

template <class R>
struct ImplicitSolver {
  using V = Vt<R>;
  using Tri = std::array<uint32_t, 3>;
  using Edge = std::array<uint32_t, 2>;
  // state
  std::vector<V> positions, prev_positions, velocities;
  std::vector<R> inv_mass;
  std::vector<Tri> tris;
  std::vector<Edge> stretch_edges;
  std::vector<R> stretch_rest;
  double time = 0.0;
  Params<R> params;
  // elements
  std::vector<Hinge<R>> hinges;
  std::vector<ShellEl<R>> shells;
  std::vector<std::array<R, 2>> shell_k;
  std::vector<Stitch<R>> stitches;
  std::vector<Collider<R>> colliders;
  std::vector<Tri> collision_tris;
  std::vector<uint8_t> static_collider_vert;
  std::vector<Tri> collider_tris;
  std::vector<V> collider_pn;
  std::vector<std::vector<uint32_t>> exclusion;
  std::vector<Edge> edges;
  R char_len = 1;
  std::vector<R> vertex_area;
  std::vector<Pin<R>> pins;
  std::vector<Pull<R>> pulls;
  std::vector<SlFace<R>> sl_faces;
  std::vector<std::array<R, 2>> uvs;
  std::vector<V> kinematic_dx;  // the static collider's move since the last step
  std::vector<MembraneEl<R>> membrane;               // built from every triangle at init
  std::vector<std::array<R, 3>> membrane_k;          // per-element (kw, kf, ks), or empty
  LinearSolver linear;
  std::vector<StepStats> history;

  // ImplicitSolver::new (implicit.rs:530-601) + SimState::from_mesh stretch edges
  void init(const std::vector<V>& pos, const std::vector<V>& vel, const std::vector<R>& im, const std::vector<Tri>& t,
            const Params<R>& p) {
    positions = pos;
    prev_positions = pos;
    velocities = vel;
    inv_mass = im;
    tris = t;
    params = p;
    stretch_edges = unique_edges(tris);
    stretch_rest.resize(stretch_edges.size());
    for (size_t i = 0; i < stretch_edges.size(); ++i)
      stretch_rest[i] = (pos[stretch_edges[i][0]] - pos[stretch_edges[i][1]]).length();
    hinges = build_hinges<R>(tris, positions);
    membrane.clear();
    for (auto& f : tris) {
      MembraneEl<R> el;
      el.tri[0] = f[0]; el.tri[1] = f[1]; el.tri[2] = f[2];
      if (build_membrane_el(positions[f[0]], positions[f[1]], positions[f[2]], el)) membrane.push_back(el);
    }
    exclusion = one_ring_exclusion(positions.size(), tris);
    edges = unique_edges(tris);
    if (edges.empty()) {
      char_len = 1;
    } else {
      R sum = 0;
      for (auto& e : edges) sum += (positions[e[0]] - positions[e[1]]).length();
      char_len = rmax(sum / (R)edges.size(), R(1.0e-6));
    }
    collision_tris = tris;
    vertex_area.assign(positions.size(), 0);
    for (auto& f : tris) {
      V a = positions[f[0]], b = positions[f[1]], c = positions[f[2]];
      R third = R(0.5) * (b - a).cross(c - a).length() / R(3);
      for (uint32_t v : f) vertex_area[v] += third;
    }
    linear.kind = (Precond)p.precond;
    linear.domain = p.schwarz_domain;
  }

  void set_shell_faces(const std::vector<Tri>& faces) {
    shells.clear();
    shell_k.clear();
    for (auto& f : faces) {
      ShellEl<R> el;
      el.v[0] = f[0]; el.v[1] = f[1]; el.v[2] = f[2];
      if (build_shell(positions[f[0]], positions[f[1]], positions[f[2]], R(1.0e-12), el)) shells.push_back(el);
    }
  }

  // set_static_collider_verts (implicit.rs:1258-1320)
  void set_static_collider_verts(const std::vector<uint8_t>& mask) {
    static_collider_vert.clear();
    collider_tris.clear();
    collider_pn.clear();
    if (mask.size() != positions.size()) return;
    V lo(INFINITY, INFINITY, INFINITY), hi(-INFINITY, -INFINITY, -INFINITY);
    std::vector<Tri> marked;
    for (auto& t : collision_tris) {
      if (!(mask[t[0]] && mask[t[1]] && mask[t[2]])) continue;
      for (uint32_t i : t) {
        lo = lo.vmin(positions[i]);
        hi = hi.vmax(positions[i]);
      }
      marked.push_back(t);
    }
    if (marked.empty()) return;
    V e = hi - lo;
    double box_vol = (double)(e.x * e.y * e.z);
    V mid = (lo + hi) * R(0.5);
    double vol = 0.0;
    for (auto& t : marked) {
      V a = positions[t[0]] - mid, b = positions[t[1]] - mid, c = positions[t[2]] - mid;
      vol += (double)a.cross(b).dot(c) / 6.0;
    }
    if (vol < -0.05 * box_vol) return;  // inward wound: unsigned distance stays
    static_collider_vert = mask;
    collider_tris = marked;
    collider_pn = pseudonormals(positions, collider_tris);
  }

  // set_kinematic_collider_positions (implicit.rs:1368-1398): move the static collider's
  // vertices to x (its rows only), give them the velocity of that move over one step,
  // accumulate the move into kinematic_dx (the friction slip of the next step) and recompute
  // the pseudonormals. False, with nothing written, when there is no static collider, x has
  // the wrong length or a collider row of x is not finite.
  bool set_kinematic_collider_positions(const std::vector<V>& x) {
    if (static_collider_vert.empty() || x.size() != positions.size()) return false;
    for (size_t i = 0; i < x.size(); ++i)
      if (static_collider_vert[i] && !(std::isfinite(x[i].x) && std::isfinite(x[i].y) && std::isfinite(x[i].z)))
        return false;
    if (kinematic_dx.empty()) kinematic_dx.assign(x.size(), V());
    const R inv_h = R(1) / params.dt;
    for (size_t i = 0; i < x.size(); ++i) {
      if (!static_collider_vert[i]) continue;
      V d = x[i] - positions[i];
      kinematic_dx[i] += d;
      positions[i] = x[i];
      velocities[i] = d * inv_h;
    }
    collider_pn = pseudonormals(positions, collider_tris);
    return true;
  }

  // set_pins (implicit.rs:826-838): all or nothing; false for a vertex out of range or a
  // ghat that is not positive.
  bool set_pins(const std::vector<Pin<R>>& p) {
    for (auto& q : p)
      if (q.index >= positions.size() || std::isnan(q.ghat) || q.ghat <= 0) return false;
    pins = p;
    return true;
  }

  // set_pulls (implicit.rs:852-864): false for a vertex out of range or a weight that is not
  // positive.
  bool set_pulls(const std::vector<Pull<R>>& p) {
    for (auto& q : p)
      if (q.index >= positions.size() || std::isnan(q.weight) || q.weight <= 0) return false;
    pulls = p;
    return true;
  }

  // set_strain_limit_faces (implicit.rs:1088-1121): faces with a positive limit (allowed
  // stretch fraction) and mass, rest shape from the current positions, degenerate faces
  // skipped. False when the arrays' lengths disagree.
  bool set_strain_limit_faces(const std::vector<Tri>& faces, const std::vector<R>& limits,
                              const std::vector<R>& masses) {
    if (limits.size() != faces.size() || masses.size() != faces.size()) return false;
    std::vector<SlFace<R>> out;
    for (size_t i = 0; i < faces.size(); ++i) {
      if (limits[i] <= 0 || masses[i] <= 0) continue;
      const Tri& f = faces[i];
      SlFace<R> sf;
      sf.el.v[0] = f[0]; sf.el.v[1] = f[1]; sf.el.v[2] = f[2];
      if (!build_shell(positions[f[0]], positions[f[1]], positions[f[2]], R(1.0e-12), sf.el)) continue;
      sf.limit = limits[i];
      sf.mass = masses[i];
      out.push_back(sf);
    }
    sl_faces = out;
    return true;
  }

  // edge_strain_ratio (implicit.rs:798-817): the warp ratio, or with a weft ratio set and
  // per-vertex UVs present, warp for an edge more U-aligned in UV space, else weft.
  R edge_strain_ratio(uint32_t a, uint32_t b) const {
    R warp = params.strain_limit_ratio, weft = params.strain_limit_ratio_weft;
    if (weft <= 0 || uvs.size() != positions.size()) return warp;
    R du = std::fabs(uvs[a][0] - uvs[b][0]), dv = std::fabs(uvs[a][1] - uvs[b][1]);
    return du >= dv ? warp : weft;
  }

  std::vector<uint8_t> movable_mask() const {
    std::vector<uint8_t> m(inv_mass.size());
    for (size_t i = 0; i < m.size(); ++i) m[i] = inv_mass[i] > 0;
    return m;
  }

  bool is_collider_tri(const uint32_t idx[4]) const {
    return !static_collider_vert.empty() && static_collider_vert[idx[1]] && static_collider_vert[idx[2]] &&
           static_collider_vert[idx[3]];
  }

  // collider_sides (implicit.rs:1431-1475)
  std::vector<R> collider_sides(const std::vector<V>& x) const {
    if (collider_tris.empty()) return {};
    R dhat = params.contact_dhat;
    std::vector<R> best(x.size(), std::numeric_limits<R>::infinity());
    std::vector<R> side(x.size(), R(1));
    auto mov = movable_mask();
    for_each_vertex_triangle_pair<R>(x, collider_tris, dhat, exclusion, mov, [&](uint32_t v, uint32_t ti) {
      if (static_collider_vert[v]) return;
      const Tri& t = collider_tris[ti];
      V a = x[t[0]], b = x[t[1]], c = x[t[2]];
      R l[3];
      V q = closest_point_bary(x[v], a, b, c, l);
      V e = x[v] - q;
      R d2 = e.length_squared();
      if (d2 >= best[v]) return;
      best[v] = d2;
      V pn[3] = {collider_pn[t[0]], collider_pn[t[1]], collider_pn[t[2]]};
      V n = surface_normal_at(l, (b - a).cross(c - a).normalize_or_zero(), pn);
      side[v] = e.dot(n) < 0 ? R(-1) : R(1);
    });
    for (size_t i = 0; i < side.size(); ++i)
      if (best[i] >= dhat * dhat) side[i] = 1;
    return side;
  }

  // self_collision_stencils (implicit.rs:678-753)
  // kinds (optional, one per stencil, test infrastructure for the adjoint): 0 vertex-triangle,
  // 1 vertex against a static collider triangle (signed, outside), 3 the same inside, 2 edge-edge
  std::vector<Stencil<R>> self_collision_stencils(const std::vector<V>& x, std::vector<uint8_t>* kinds = nullptr) const {
    R dhat = params.contact_dhat;
    std::vector<Stencil<R>> out;
    auto mov = movable_mask();
    auto side = collider_sides(x);
    std::vector<std::pair<uint32_t, uint32_t>> vt;
    for_each_vertex_triangle_pair<R>(x, collision_tris, dhat, exclusion, mov,
                                     [&](uint32_t v, uint32_t t) { vt.push_back({v, t}); });
    std::sort(vt.begin(), vt.end());
    vt.erase(std::unique(vt.begin(), vt.end()), vt.end());
    for (auto& pr : vt) {
      const Tri& t = collision_tris[pr.second];
      Stencil<R> s;
      s.idx[0] = pr.first; s.idx[1] = t[0]; s.idx[2] = t[1]; s.idx[3] = t[2];
      const bool col = is_collider_tri(s.idx);
      if (col)
        s.d = signed_point_tri_distance_grad(x[s.idx[0]], x[s.idx[1]], x[s.idx[2]], x[s.idx[3]], side[s.idx[0]] < 0, s.g);
      else
        s.d = point_tri_distance_grad(x[s.idx[0]], x[s.idx[1]], x[s.idx[2]], x[s.idx[3]], s.g);
      if (s.d >= dhat) continue;
      s.ghat = dhat;
      out.push_back(s);
      if (kinds) kinds->push_back(col ? (side[s.idx[0]] < 0 ? 3 : 1) : 0);
    }
    R ee_search = dhat;  // max_edge_gap() + 2 * max_edge_offset() with face edges only
    std::vector<std::pair<uint32_t, uint32_t>> ee;
    for_each_edge_edge_pair<R>(x, edges, ee_search, mov, [&](uint32_t a, uint32_t b) { ee.push_back({a, b}); });
    std::sort(ee.begin(), ee.end());
    ee.erase(std::unique(ee.begin(), ee.end()), ee.end());
    for (auto& pr : ee) {
      const Edge& ea = edges[pr.first];
      const Edge& eb = edges[pr.second];
      Stencil<R> s;
      s.idx[0] = ea[0]; s.idx[1] = ea[1]; s.idx[2] = eb[0]; s.idx[3] = eb[1];
      s.d = segment_segment_distance_grad(x[s.idx[0]], x[s.idx[1]], x[s.idx[2]], x[s.idx[3]], s.g);
      R pair_ghat = R(0.5) * (dhat + dhat);
      if (s.d >= pair_ghat) continue;
      s.ghat = pair_ghat;
      out.push_back(s);
      if (kinds) kinds->push_back(2);
    }
    return out;
  }

  // The assembly push target (implicit.rs:3175-3233).
  struct Asm {
    TripletSinkT<R>* sink;
    const std::unordered_map<uint64_t, size_t>* slots;
    std::vector<std::array<R, 9>> blocks;
    std::vector<std::array<R, 9>> diag;
    const std::vector<uint8_t>* pinned;
    bool grad_only = false;
    void push(uint32_t r, uint32_t c, R v) {
      if (grad_only) return;
      if (!diag.empty() && r / 3 == c / 3) diag[r / 3][3 * (r % 3) + (c % 3)] += v;
      if (!slots->empty()) {
        auto it = slots->find(((uint64_t)(r / 3) << 32) | (c / 3));
        if (it != slots->end()) blocks[it->second][3 * (r % 3) + (c % 3)] += v;
      }
      if (!(*pinned)[r / 3] && !(*pinned)[c / 3]) sink->push({r, c, v});
    }
  };

  // self_contact_rayleigh (implicit.rs:755-795)
  R self_contact_rayleigh(const std::vector<std::array<R, 9>>& blocks, const std::unordered_map<uint64_t, size_t>& slots,
                          const Stencil<R>& s) const {
    R nlen = s.g[0].length();
    if (nlen < R(1.0e-12)) return params.contact_kappa;
    V nrm = s.g[0] / nlen;
    R weights[4], mass[4];
    for (int a = 0; a < 4; ++a) {
      weights[a] = s.g[a].dot(nrm);
      R im = inv_mass[s.idx[a]];
      mass[a] = im > 0 ? R(1) / im : R(0);
    }
    R elastic[16][9];
    for (int a = 0; a < 16; ++a)
      for (int q = 0; q < 9; ++q) elastic[a][q] = 0;
    for (int ia = 0; ia < 4; ++ia)
      for (int ib = 0; ib < 4; ++ib) {
        auto it = slots.find(((uint64_t)s.idx[ia] << 32) | s.idx[ib]);
        if (it != slots.end())
          for (int q = 0; q < 9; ++q) elastic[ia * 4 + ib][q] = blocks[it->second][q];
      }
    R k = rayleigh_stiffness<R>(elastic, mass, weights, 4, nrm * s.d, R(0));
    return k > 0 ? k : params.contact_kappa;
  }

  // Test infrastructure for the FP64 adjoint: the mass part of a stencil's Rayleigh
  // stiffness, sum_a m_a w_a^2 / (sum_a w_a^2 d^2) (0 when the stiffness fell back to kappa).
  R rayleigh_mass_part(const Stencil<R>& s, R k_used) const {
    R nlen = s.g[0].length();
    if (nlen < R(1.0e-12) || k_used == params.contact_kappa) return 0;
    V nrm = s.g[0] / nlen;
    R m_max = 0, ws = 0, acc = 0, mass[4], w[4];
    for (int a = 0; a < 4; ++a) {
      w[a] = s.g[a].dot(nrm);
      R im = inv_mass[s.idx[a]];
      mass[a] = im > 0 ? R(1) / im : R(0);
      m_max = rmax(m_max, mass[a]);
    }
    for (int a = 0; a < 4; ++a) {
      ws += w[a] * w[a];
      acc += (mass[a] > 0 ? mass[a] : m_max) * w[a] * w[a];
    }
    return ws > 0 ? acc / ws / (s.d * s.d) : R(0);
  }

  // Adjoint support (test infrastructure): a frozen contact set, each stencil with its kind
  // (as self_collision_stencils reports it) and its stiffness split into an elastic part held
  // fixed and a mass part that goes as 1/d^2 from its value km at gap d0; when set, the
  // assembly recomputes these stencils' gaps and gradients at its x instead of collecting
  // stencils. grad_only skips the Hessian. record_contacts keeps (stiffness, mass part) of
  // every stencil the assembly used.
  struct FrozenContact {
    uint32_t idx[4];
    uint8_t kind;
    R ghat, k_el, km, d0;
  };
  const std::vector<FrozenContact>* frozen = nullptr;
  bool grad_only = false;
  bool record_contacts = false;
  std::vector<std::array<R, 2>> contact_rec;

  std::vector<Stencil<R>> frozen_stencils(const std::vector<V>& x) const {
    std::vector<Stencil<R>> out(frozen->size());
    for (size_t i = 0; i < frozen->size(); ++i) {
      const FrozenContact& f = (*frozen)[i];
      Stencil<R>& s = out[i];
      for (int a = 0; a < 4; ++a) s.idx[a] = f.idx[a];
      const V &p0 = x[f.idx[0]], &p1 = x[f.idx[1]], &p2 = x[f.idx[2]], &p3 = x[f.idx[3]];
      if (f.kind == 2)
        s.d = segment_segment_distance_grad(p0, p1, p2, p3, s.g);
      else if (f.kind == 0)
        s.d = point_tri_distance_grad(p0, p1, p2, p3, s.g);
      else
        s.d = signed_point_tri_distance_grad(p0, p1, p2, p3, f.kind == 3, s.g);
      s.ghat = f.ghat;
    }
    return out;
  }

  // assemble (implicit.rs:2280-3155), restricted to the element kinds listed in the header
  CsrT<R> assemble(const std::vector<V>& x, const std::vector<V>& x_tilde, R inv_h2, std::vector<R>& rhs,
                   uint32_t* nstencils) {
    size_t n = positions.size(), ndof = 3 * n;
    R k = params.stiffness;
    TripletSinkT<R> sink;
    sink.begin(ndof);
    std::vector<R> grad(ndof, R(0));
    std::vector<uint8_t> pinned(n);
    for (size_t i = 0; i < n; ++i) pinned[i] = inv_mass[i] <= 0;
    std::vector<Stencil<R>> sc = frozen ? frozen_stencils(x)
                                        : (params.self_collision ? self_collision_stencils(x) : std::vector<Stencil<R>>());
    if (nstencils) *nstencils = (uint32_t)sc.size();
    if (record_contacts) contact_rec.clear();
    bool want_diag = !pins.empty() || !pulls.empty() || (!colliders.empty() && params.contact_rayleigh);
    std::unordered_map<uint64_t, size_t> slots;
    for (auto& f : sl_faces)
      for (uint32_t a : f.el.v)
        for (uint32_t b : f.el.v) {
          uint64_t key = ((uint64_t)a << 32) | b;
          if (!slots.count(key)) {
            size_t kk = slots.size();
            slots[key] = kk;
          }
        }
    for (auto& s : sc)
      for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) {
          uint64_t key = ((uint64_t)s.idx[a] << 32) | s.idx[b];
          if (!slots.count(key)) {
            size_t kk = slots.size();
            slots[key] = kk;
          }
        }
    Asm trips;
    trips.sink = &sink;
    trips.grad_only = grad_only;
    trips.slots = &slots;
    trips.blocks.assign(slots.size(), std::array<R, 9>{});
    if (want_diag) trips.diag.assign(n, std::array<R, 9>{});
    trips.pinned = &pinned;

    // inertia
    for (size_t i = 0; i < n; ++i) {
      R im = inv_mass[i];
      if (im <= 0) continue;
      R m_over_h2 = (R(1) / im) * inv_h2;
      V diff = x[i] - x_tilde[i];
      for (int c = 0; c < 3; ++c) {
        trips.push((uint32_t)(3 * i + c), (uint32_t)(3 * i + c), m_over_h2);
        grad[3 * i + c] += m_over_h2 * diff[c];
      }
    }
    // stitches
    for (auto& st : stitches) {
      if (st.stiffness <= 0) continue;
      V xs[6];
      for (int q = 0; q < 6; ++q) xs[q] = x[st.index[q]];
      V g[6];
      static thread_local std::vector<R> hh(324);
      stitch_force_hessian(xs, st.weight, st.l0, st.l_cap, g, hh.data());
      for (int q = 0; q < 6; ++q)
        for (int c = 0; c < 3; ++c) grad[3 * st.index[q] + c] += st.stiffness * g[q][c];
      for (int a = 0; a < 6; ++a)
        for (int b = 0; b < 6; ++b)
          for (int rr = 0; rr < 3; ++rr)
            for (int cc = 0; cc < 3; ++cc) {
              R v = st.stiffness * hh[(3 * a + rr) * 18 + 3 * b + cc];
              if (v != 0) trips.push(3 * st.index[a] + rr, 3 * st.index[b] + cc, v);
            }
    }
    // stretch springs (pushed even at zero stiffness, as the reference does)
    for (size_t e = 0; e < stretch_edges.size(); ++e) {
      uint32_t a = stretch_edges[e][0], b = stretch_edges[e][1];
      R hk[3][3];
      V ga;
      spring_block(x[a] - x[b], stretch_rest[e], k, hk, ga);
      for (int c = 0; c < 3; ++c) {
        grad[3 * a + c] += ga[c];
        grad[3 * b + c] -= ga[c];
      }
      for (int r = 0; r < 3; ++r)
        for (int cc = 0; cc < 3; ++cc) {
          R v = hk[r][cc];
          trips.push(3 * a + r, 3 * a + cc, v);
          trips.push(3 * b + r, 3 * b + cc, v);
          trips.push(3 * a + r, 3 * b + cc, -v);
          trips.push(3 * b + r, 3 * a + cc, -v);
        }
      // one-sided strain limit on the same edge (implicit.rs:2508-2530)
      R slk = params.strain_limit_k, slr = edge_strain_ratio(a, b);
      if (slr > 0 && slk > 0) {
        V sg;
        R sh[3][3];
        edge_strain_block(x[a], x[b], stretch_rest[e], slr, slk, sg, sh);
        for (int c = 0; c < 3; ++c) {
          grad[3 * a + c] += sg[c];
          grad[3 * b + c] -= sg[c];
        }
        for (int r = 0; r < 3; ++r)
          for (int cc = 0; cc < 3; ++cc) {
            R v = sh[r][cc];
            trips.push(3 * a + r, 3 * a + cc, v);
            trips.push(3 * b + r, 3 * b + cc, v);
            trips.push(3 * a + r, 3 * b + cc, -v);
            trips.push(3 * b + r, 3 * a + cc, -v);
          }
      }
    }
    // Baraff-Witkin membrane (implicit.rs:2532-2596)
    if (params.membrane_warp > 0 || params.membrane_weft > 0 || params.membrane_shear > 0 || !membrane_k.empty()) {
      for (size_t ei = 0; ei < membrane.size(); ++ei) {
        const auto& el = membrane[ei];
        R kw = membrane_k.empty() ? params.membrane_warp : membrane_k[ei][0];
        R kf = membrane_k.empty() ? params.membrane_weft : membrane_k[ei][1];
        R ks = membrane_k.empty() ? params.membrane_shear : membrane_k[ei][2];
        V p[3] = {x[el.tri[0]], x[el.tri[1]], x[el.tri[2]]};
        R cnd[3];
        bw_conditions(p, el.dm_inv, cnd);
        V g[3][3];
        bw_condition_grads(p, el.dm_inv, g);
        R cu[3], cv[3];
        bw_coeffs(el.dm_inv, cu, cv);
        V wu, wv;
        bw_deformation(p, el.dm_inv, wu, wv);
        R mu_[3][3], mv_[3][3], sm[4][3][3];
        bw_stretch_material(wu, mu_);
        bw_stretch_material(wv, mv_);
        bw_shear_material(wu, wv, true, sm);
        const R kc[3] = {kw, kf, ks};
        // pushed per condition, vertex pair and entry, in the reference's order
        for (int ci = 0; ci < 3; ++ci) {
          R ka = kc[ci] * el.area;
          if (ka <= 0) continue;
          for (int a = 0; a < 3; ++a) {
            uint32_t va = el.tri[a];
            for (int c = 0; c < 3; ++c) grad[3 * va + c] += ka * cnd[ci] * g[ci][a][c];
            for (int b = 0; b < 3; ++b) {
              uint32_t vb = el.tri[b];
              for (int r = 0; r < 3; ++r)
                for (int cc = 0; cc < 3; ++cc) {
                  R v;
                  if (ci < 2) {
                    const R* co = ci == 0 ? cu : cv;
                    R(*m)[3] = ci == 0 ? mu_ : mv_;
                    v = ka * co[a] * co[b] * m[r][cc];
                  } else {
                    v = ka * (cu[a] * cu[b] * sm[0][r][cc] + cu[a] * cv[b] * sm[1][r][cc] +
                              cv[a] * cu[b] * sm[2][r][cc] + cv[a] * cv[b] * sm[3][r][cc]);
                  }
                  if (v != 0) trips.push(3 * va + r, 3 * vb + cc, v);
                }
            }
          }
        }
      }
    }
    // shells
    if (!shells.empty() && (params.shell_mu > 0 || params.shell_lambda > 0 || !shell_k.empty())) {
      for (size_t ei = 0; ei < shells.size(); ++ei) {
        const auto& el = shells[ei];
        R smu = shell_k.empty() ? params.shell_mu : shell_k[ei][0];
        R slam = shell_k.empty() ? params.shell_lambda : shell_k[ei][1];
        V p[3] = {x[el.v[0]], x[el.v[1]], x[el.v[2]]};
        V eg[3];
        shell_gradient(p, el, smu, slam, eg);
        R eh[81];
        shell_hessian(p, el, smu, slam, params.eiganalysis_eps, eh);
        for (int a = 0; a < 3; ++a) {
          uint32_t va = el.v[a];
          for (int c = 0; c < 3; ++c) grad[3 * va + c] += eg[a][c];
          for (int b = 0; b < 3; ++b) {
            uint32_t vb = el.v[b];
            for (int r = 0; r < 3; ++r)
              for (int cc = 0; cc < 3; ++cc) {
                R v = eh[(3 * a + r) * 9 + 3 * b + cc];
                if (v != 0) trips.push(3 * va + r, 3 * vb + cc, v);
              }
          }
        }
      }
    }
    // hinges
    R kb = params.bend_stiffness;
    if (kb > 0) {
      for (auto& h : hinges) {
        V p[4] = {x[h.v[0]], x[h.v[1]], x[h.v[2]], x[h.v[3]]};
        R theta = dihedral_angle(p);
        V g[4];
        dihedral_grad(p, g);
        R kwt = kb * h.w;
        if (kwt <= 0) continue;
        R gval = theta - h.rest;
        for (int a = 0; a < 4; ++a) {
          uint32_t va = h.v[a];
          for (int c = 0; c < 3; ++c) grad[3 * va + c] += kwt * gval * g[a][c];
          for (int b = 0; b < 4; ++b) {
            uint32_t vb = h.v[b];
            for (int r = 0; r < 3; ++r)
              for (int cc = 0; cc < 3; ++cc) {
                R v = kwt * g[a][r] * g[b][cc];
                if (v != 0) trips.push(3 * va + r, 3 * vb + cc, v);
              }
          }
        }
      }
    }
    // strain-limit barrier (implicit.rs:2743-2807): every elastic term is in, so the
    // gathered blocks give each face the elastic half of its stiffness, w.(H_elastic w) with
    // w the face's positions about their centroid, unnormalised.
    if (!sl_faces.empty()) {
      auto blocks = trips.blocks;
      for (auto& f : sl_faces) {
        const uint32_t* vs = f.el.v;
        V p[3] = {x[vs[0]], x[vs[1]], x[vs[2]]};
        V centroid = (p[0] + p[1] + p[2]) / R(3);
        V w[3] = {p[0] - centroid, p[1] - centroid, p[2] - centroid};
        R elastic_k = 0;
        for (int ia = 0; ia < 3; ++ia)
          for (int ib = 0; ib < 3; ++ib) {
            auto it = slots.find(((uint64_t)vs[ia] << 32) | vs[ib]);
            if (it == slots.end()) continue;
            const auto& blk = blocks[it->second];
            for (int r = 0; r < 3; ++r)
              for (int c = 0; c < 3; ++c) elastic_k += w[ia][r] * blk[3 * r + c] * w[ib][c];
          }
        V eg[3];
        R eh[81];
        if (!strain_limit_eval(p, f.el, f.limit, f.mass, elastic_k, params.barrier_kind, params.eiganalysis_eps, true,
                               eg, eh))
          continue;
        for (int a = 0; a < 3; ++a) {
          uint32_t va = vs[a];
          for (int c = 0; c < 3; ++c) grad[3 * va + c] += eg[a][c];
          for (int b = 0; b < 3; ++b) {
            uint32_t vb = vs[b];
            for (int r = 0; r < 3; ++r)
              for (int cc = 0; cc < 3; ++cc) {
                R v = eh[(3 * a + r) * 9 + (3 * b + cc)];
                if (v != 0) trips.push(3 * va + r, 3 * vb + cc, v);
              }
          }
        }
      }
    }
    // pins (implicit.rs:2809-2856): k = (H w).w / |w|^2 + m / gap^2 from the vertex's own
    // elastic diagonal block, gap = max(ghat - |w|, constraint_tol ghat); kinematic pins
    // scale k by their stiffness.
    if (!pins.empty()) {
      auto diag = trips.diag;
      for (auto& pin : pins) {
        size_t i = pin.index;
        if (inv_mass[i] <= 0) continue;
        R m = R(1) / inv_mass[i];
        V w = x[i] - pin.target;
        R d = w.length();
        R floor = params.constraint_tol * pin.ghat;
        R gap = rmax(pin.ghat - d, floor);
        R d2 = w.length_squared();
        R tmp = 0;
        if (d2 > 0) {
          const auto& hb = diag[i];
          V hw(hb[0] * w.x + hb[1] * w.y + hb[2] * w.z, hb[3] * w.x + hb[4] * w.y + hb[5] * w.z,
               hb[6] * w.x + hb[7] * w.y + hb[8] * w.z);
          tmp = hw.dot(w) / d2;
        }
        R kp = tmp + m / (gap * gap);
        if (pin.kinematic) kp *= pin.stiffness;
        V gp = w * kp;
        for (int c = 0; c < 3; ++c) {
          grad[3 * i + c] += gp[c];
          trips.push((uint32_t)(3 * i + c), (uint32_t)(3 * i + c), kp);
        }
      }
    }
    // pulls (implicit.rs:2858-2872)
    for (auto& pl : pulls) {
      size_t i = pl.index;
      if (inv_mass[i] <= 0) continue;
      V d = (x[i] - pl.target) * pl.weight;
      for (int c = 0; c < 3; ++c) {
        grad[3 * i + c] += d[c];
        trips.push((uint32_t)(3 * i + c), (uint32_t)(3 * i + c), pl.weight);
      }
    }
    // analytic colliders (implicit.rs:2954-3021)
    if (!colliders.empty()) {
      R dhat = params.contact_dhat, kappa = params.contact_kappa;
      std::vector<std::array<R, 9>> ediag;
      if (params.contact_rayleigh) ediag = trips.diag;
      for (size_t i = 0; i < n; ++i) {
        if (inv_mass[i] <= 0) continue;
        R m = R(1) / inv_mass[i];
        R mu_i = params.friction;
        // combined with the collider's own coefficient only when it is set (implicit.rs:2975-2990)
        if (std::isfinite(params.collider_friction)) {
          R cf = params.collider_friction;
          mu_i = params.friction_mode == 1 ? rmax(mu_i, cf) : params.friction_mode == 2 ? R(0.5) * (mu_i + cf) : rmin(mu_i, cf);
        }
        bool has_slip = mu_i > 0;
        V cg;
        R ch[3][3];
        vertex_contact_full<R>(x[i], colliders, dhat, kappa, params.contact_dynamic, m, params.barrier_kind,
                               params.contact_rayleigh ? ediag[i].data() : nullptr, has_slip, x[i] - positions[i],
                               mu_i, params.friction_eps, cg, ch);
        for (int c = 0; c < 3; ++c) grad[3 * i + c] += cg[c];
        for (int r = 0; r < 3; ++r)
          for (int cc = 0; cc < 3; ++cc)
            if (ch[r][cc] != 0) trips.push((uint32_t)(3 * i + r), (uint32_t)(3 * i + cc), ch[r][cc]);
      }
    }
    // self contact (implicit.rs:3026-3103)
    if (!sc.empty()) {
      auto blocks = trips.blocks;
      for (size_t si = 0; si < sc.size(); ++si) {
        const Stencil<R>& s = sc[si];
        R kk;
        if (frozen) {
          const FrozenContact& f = (*frozen)[si];
          kk = f.k_el + (f.km > 0 ? f.km * (f.d0 * f.d0) / (s.d * s.d) : R(0));
        } else {
          kk = self_contact_rayleigh(blocks, slots, s);
        }
        if (record_contacts) contact_rec.push_back({kk, rayleigh_mass_part(s, kk)});
        BarrierKind kind = s.d < 0 ? BarrierKind::Cubic : params.barrier_kind;
        R e, bg, bh;
        if (!barrier_of(kind, s.d, s.ghat, kk, e, bg, bh)) continue;
        R hp = rmax(bh, R(0));
        for (int a = 0; a < 4; ++a) {
          for (int c = 0; c < 3; ++c) grad[3 * s.idx[a] + c] += bg * s.g[a][c];
          for (int b = 0; b < 4; ++b)
            for (int r = 0; r < 3; ++r)
              for (int cc = 0; cc < 3; ++cc) {
                R vh = hp * s.g[a][r] * s.g[b][cc];
                if (vh != 0) trips.push(3 * s.idx[a] + r, 3 * s.idx[b] + cc, vh);
              }
        }
        R mu_s = params.friction;
        if (mu_s > 0) {
          V dxs[4];
          // the slip is relative (fdx_override, implicit.rs:3068-3078): a re-posed collider
          // vertex contributes the displacement it was moved by before this step
          for (int a = 0; a < 4; ++a) {
            uint32_t i = s.idx[a];
            dxs[a] = x[i] - positions[i] + (kinematic_dx.empty() ? V() : kinematic_dx[i]);
          }
          V fg[4];
          R fh[144];
          if (stencil_friction(s.g, dxs, bg, mu_s, params.friction_eps, fg, fh)) {
            for (int a = 0; a < 4; ++a) {
              for (int c = 0; c < 3; ++c) grad[3 * s.idx[a] + c] += fg[a][c];
              for (int b = 0; b < 4; ++b)
                for (int r = 0; r < 3; ++r)
                  for (int cc = 0; cc < 3; ++cc) {
                    R vh = fh[(3 * a + r) * 12 + 3 * b + cc];
                    if (vh != 0) trips.push(3 * s.idx[a] + r, 3 * s.idx[b] + cc, vh);
                  }
            }
          }
        }
      }
    }
    rhs.assign(ndof, R(0));
    for (size_t i = 0; i < ndof; ++i) rhs[i] = -grad[i];
    for (size_t i = 0; i < n; ++i)
      if (pinned[i])
        for (int c = 0; c < 3; ++c) rhs[3 * i + c] = 0;
    if (grad_only) return CsrT<R>();
    return sink.finish(pinned);
  }

  // ccd_max_step (implicit.rs:1690-1947)
  R ccd_max_step(const std::vector<V>& x, const std::vector<V>& dx, uint32_t* cap_hits) const {
    bool has_self = params.self_collision;
    bool has_static_pins = false;
    for (auto& p : pins)
      if (!p.kinematic) has_static_pins = true;
    if (colliders.empty() && !has_self && !has_static_pins && sl_faces.empty()) return 1;
    const R GAP = R(0.2), T_MIN = 0;
    size_t n = x.size();
    R t = 1;
    // strain-limit line search (implicit.rs:1709-1753): per face, bisect the step fraction
    // on max(sigma(x + t dx) - 1) < limit over [0, 1.25] until the window stops shrinking.
    if (!sl_faces.empty()) {
      const R LS_MAX_T = R(1.25);
      for (auto& f : sl_faces) {
        const uint32_t* vs = f.el.v;
        auto at = [&](R frac) {
          V p[3] = {x[vs[0]] + dx[vs[0]] * frac, x[vs[1]] + dx[vs[1]] * frac, x[vs[2]] + dx[vs[2]] * frac};
          return max_stretch_excess(p, f.el.dm_inv);
        };
        if (at(LS_MAX_T) < f.limit) continue;
        R lo = 0, hi = LS_MAX_T;
        R window = hi - lo;
        for (int it = 0; it < 64; ++it) {
          R mid = R(0.5) * (lo + hi);
          if (at(mid) - f.limit < 0)
            lo = mid;
          else
            hi = mid;
          R w = hi - lo;
          if (w == window) break;
          window = w;
        }
        t = rmin(t, lo);
      }
    }
    // static-pin confinement (implicit.rs:1755-1789): radius interpolated linearly over the
    // extended horizon 1.25 dx, clamped to land on the ghat sphere.
    if (has_static_pins) {
      const R LS_MAX_T = R(1.25);
      for (auto& pin : pins) {
        if (pin.kinematic) continue;
        size_t i = pin.index;
        if (inv_mass[i] <= 0) continue;
        R r0 = (x[i] - pin.target).length();
        if (r0 >= pin.ghat) continue;
        R r1 = (x[i] + dx[i] * LS_MAX_T - pin.target).length();
        if (r1 > pin.ghat) {
          R denom = r1 - r0;
          if (denom != 0) t = rmin(t, LS_MAX_T * (pin.ghat - r0) / denom);
        }
      }
    }
    for (size_t i = 0; i < n; ++i) {
      if (inv_mass[i] <= 0) continue;
      for (auto& c : colliders) {
        R d0;
        V nrm;
        c.distance(x[i], d0, nrm);
        if (d0 <= 0) continue;
        if (c.kind == 0) {
          R rate = dx[i].dot(nrm);
          if (rate < 0) t = rmin(t, (GAP - R(1)) * d0 / rate);
        } else {
          R l = dx[i].length();
          if (l > R(1.0e-12)) t = rmin(t, (R(1) - GAP) * d0 / l);
        }
      }
    }
    if (has_self) {
      const R MAX_T = R(1.25), REDUCTION = R(0.01);
      uint32_t ccd_iters = std::max<uint32_t>(params.ccd_max_iter, 1);
      R max_disp = 0;
      for (auto& d : dx) max_disp = rmax(max_disp, d.length());
      R fixed = params.contact_dhat;
      R allowed = rmax(rmin(R(0.5) * char_len, max_disp), R(1.0e-9));
      auto mov = movable_mask();
      auto side = collider_sides(x);
      for (;;) {
        bool full = allowed >= max_disp;
        R search = fixed + R(2) * allowed;
        R t_self = 1;
        for_each_vertex_triangle_pair<R>(x, collision_tris, search, exclusion, mov, [&](uint32_t v, uint32_t ti) {
          const Tri& tri = collision_tris[ti];
          uint32_t idx[4] = {v, tri[0], tri[1], tri[2]};
          if (is_collider_tri(idx) && side[idx[0]] < 0) return;
          V x0[4] = {x[idx[0]], x[idx[1]], x[idx[2]], x[idx[3]]};
          V dd[4] = {dx[idx[0]], dx[idx[1]], dx[idx[2]], dx[idx[3]]};
          bool cap = false;
          R toi = accd_toi<R>(x0, dd, R(0), MAX_T, REDUCTION, ccd_iters,
                              [](const V* p) {
                                R d = point_triangle_distance(p[0], p[1], p[2], p[3]);
                                return d * d;
                              },
                              &cap);
          if (cap && cap_hits) ++*cap_hits;
          t_self = rmin(t_self, toi / MAX_T);
        });
        for_each_edge_edge_pair<R>(x, edges, search, mov, [&](uint32_t ei, uint32_t ej) {
          const Edge& ea = edges[ei];
          const Edge& eb = edges[ej];
          uint32_t idx[4] = {ea[0], ea[1], eb[0], eb[1]};
          V x0[4] = {x[idx[0]], x[idx[1]], x[idx[2]], x[idx[3]]};
          V dd[4] = {dx[idx[0]], dx[idx[1]], dx[idx[2]], dx[idx[3]]};
          bool cap = false;
          R toi = accd_toi<R>(x0, dd, R(0), MAX_T, REDUCTION, ccd_iters,
                              [](const V* p) {
                                R d = segment_segment_distance(p[0], p[1], p[2], p[3]);
                                return d * d;
                              },
                              &cap);
          if (cap && cap_hits) ++*cap_hits;
          t_self = rmin(t_self, toi / MAX_T);
        });
        if (full || t_self * max_disp <= allowed) {
          t = rmin(t, t_self);
          break;
        }
        allowed = rmin(allowed * R(4), max_disp);
      }
    }
    return rclamp(t, T_MIN, R(1));
  }

  // has_self_intersection (implicit.rs:618-650): positions_self_intersect (implicit.rs:618-643)
  // streams the candidates of any_edge_triangle_pair (broadphase.rs:587-751) at search =
  // char_len over the movable mask and stops at the first pair that edge_triangle_intersect
  // reports piercing.
  bool positions_self_intersect(const std::vector<V>& x) const {
    if (edges.empty() || collision_tris.empty()) return false;
    return any_edge_triangle_pair<R>(x, edges, collision_tris, char_len, movable_mask(),
                                     [&](uint32_t ei, uint32_t ti) {
                                       const Edge& e = edges[ei];
                                       const Tri& t = collision_tris[ti];
                                       return edge_triangle_intersect(x[e[0]], x[e[1]], x[t[0]], x[t[1]], x[t[2]]);
                                     });
  }

  // step (implicit.rs:1951-2191)
  StepStats step(bool check_intersection) {
    StepStats st;
    size_t n = positions.size();
    R h = params.dt;
    R inv_h2 = R(1) / (h * h);
    V g = params.gravity;
    std::vector<V> x0 = positions;
    std::vector<V> x_tilde(n);
    for (size_t i = 0; i < n; ++i)
      x_tilde[i] = inv_mass[i] > 0 ? x0[i] + velocities[i] * h + g * (h * h) : x0[i];
    std::vector<V> x = x0;
    uint32_t cap = std::max<uint32_t>(params.newton_iters, 1);
    bool final_step = false;
    uint32_t taken = 0;
    std::vector<R> rhs, dxflat(3 * n);
    std::vector<V> dx(n);
    for (uint32_t it = 0; it < cap; ++it) {
      ++taken;
      uint32_t nst = 0;
      CsrT<R> a = assemble(x, x_tilde, inv_h2, rhs, &nst);
      st.stencils = std::max(st.stencils, nst);
      linear.solve(a, rhs.data(), params.cg_tol, params.cg_max_iter, dxflat.data());
      st.max_reresid = std::max(st.max_reresid, linear.last.residual);
      st.max_cg_iters = std::max(st.max_cg_iters, linear.last.iters);
      for (size_t i = 0; i < n; ++i) dx[i] = V(dxflat[3 * i], dxflat[3 * i + 1], dxflat[3 * i + 2]);
      R max_norm = 0;
      for (auto& d : dx) max_norm = rmax(max_norm, d.length());
      if (max_norm > 0) {
        R rescale = rmin(params.max_dx / max_norm, R(1));
        if (rescale < 1)
          for (auto& d : dx) d *= rescale;
      }
      R t = ccd_max_step(x, dx, &st.ccd_cap_hits);
      st.t_min = std::min(st.t_min, (double)t);
      R max_step = 0;
      for (size_t i = 0; i < n; ++i) {
        V d = dx[i] * t;
        x[i] += d;
        max_step = rmax(max_step, d.length());
      }
      if (max_step < R(1.0e-7)) break;
      if (params.newton_tol > 0 && max_step < params.newton_tol) break;
      if (final_step) break;
      if (params.target_toi > 0 && t >= params.target_toi && taken > params.min_newton_steps) final_step = true;
    }
    R floor = params.floor_y;
    for (size_t i = 0; i < n; ++i)
      if (inv_mass[i] > 0 && std::isfinite(floor) && x[i].y < floor) x[i].y = floor;
    bool finite = true;
    for (auto& p : x)
      if (!p.finite()) finite = false;
    R inv_h = R(1) / h;
    for (size_t i = 0; i < n; ++i) {
      if (finite) {
        velocities[i] = inv_mass[i] > 0 ? (x[i] - x0[i]) * inv_h : V();
        prev_positions[i] = x0[i];
        positions[i] = x[i];
      } else {
        velocities[i] = V();
        prev_positions[i] = x0[i];
        positions[i] = x0[i];
      }
    }
    time += (double)h;
    // the collider move described this step only (implicit.rs:2065-2070)
    for (auto& d : kinematic_dx) d = V();
    st.newton_iters = taken;
    st.all_finite = finite ? 1 : 0;
    // count_active_contacts (implicit.rs:2213-2232)
    if (!colliders.empty()) {
      for (size_t i = 0; i < n; ++i) {
        if (inv_mass[i] <= 0) continue;
        for (auto& c : colliders) {
          R d;
          V nn;
          c.distance(positions[i], d, nn);
          if (d < params.contact_dhat) {
            ++st.num_contacts;
            break;
          }
        }
      }
    }
    // penetration_free (implicit.rs:2235-2268)
    bool pf = finite;
    R tol = R(-1.0e-3) * rmax(params.contact_dhat, R(1.0e-6));
    for (size_t i = 0; i < n && pf; ++i) {
      if (inv_mass[i] <= 0) continue;
      for (auto& c : colliders) {
        R d;
        V nn;
        c.distance(positions[i], d, nn);
        if (d < tol) pf = false;
      }
    }
    if (pf && params.self_collision && check_intersection) pf = !positions_self_intersect(positions);
    st.penetration_free = pf ? 1 : 0;
    history.push_back(st);
    return st;
  }
};

}  // namespace mo
