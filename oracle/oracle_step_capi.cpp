// C entry points over the implicit-step oracle (TEST INFRASTRUCTURE ONLY): whole steps in
// float (the reference's f32 path) or double (the FP64 oracle), and the element-level
// functions the reference's unit tests pin (distances, ACCD, barriers, shells, hinges,
// stitches, Rayleigh stiffness).
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#include "implicit_oracle.hpp"

using namespace mo;

extern "C" {

// Scene description shared with the CUDA library's mguso_scene_desc (same field meaning).
struct OracleParams {
  float dt, gravity[3];
  uint32_t newton_iters;
  float stiffness, bend_stiffness, max_dx, target_toi;
  uint32_t min_newton_steps, ccd_max_iter;
  float eiganalysis_eps, contact_dhat, contact_kappa, contact_dynamic;
  float shell_mu, shell_lambda, friction, friction_eps;
  int barrier_kind, contact_rayleigh, self_collision;
  float cg_tol;
  uint32_t cg_max_iter;
  float floor_y, newton_tol;
  int precond;
  uint32_t schwarz_domain;
};

struct OracleStats {
  uint32_t newton_iters, max_cg_iters, num_contacts, stencils, ccd_cap_hits;
  double max_reresid, t_min;
  int penetration_free, all_finite;
};

}  // extern "C"

namespace {

struct AnySolver {
  int prec;  // 0 float, 1 double
  std::unique_ptr<ImplicitSolver<float>> f;
  std::unique_ptr<ImplicitSolver<double>> d;
};

template <class R>
std::unique_ptr<ImplicitSolver<R>> make_solver(uint32_t nv, const float* pos, const float* vel, const float* inv_mass,
                                               uint32_t nt, const uint32_t* tris, const uint8_t* static_mask,
                                               uint32_t nshell, const uint32_t* shell_faces, uint32_t nstitch,
                                               const uint32_t* st_idx, const float* st_w, const float* st_kl,
                                               uint32_t ncol, const float* cols, const OracleParams* p) {
  auto s = std::make_unique<ImplicitSolver<R>>();
  std::vector<Vt<R>> P(nv), Vv(nv);
  std::vector<R> im(nv);
  for (uint32_t i = 0; i < nv; ++i) {
    P[i] = Vt<R>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
    Vv[i] = vel ? Vt<R>(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]) : Vt<R>();
    im[i] = inv_mass[i];
  }
  std::vector<std::array<uint32_t, 3>> T(nt);
  for (uint32_t t = 0; t < nt; ++t) T[t] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
  Params<R> q;
  q.dt = p->dt;
  q.gravity = Vt<R>(p->gravity[0], p->gravity[1], p->gravity[2]);
  q.newton_iters = p->newton_iters;
  q.stiffness = p->stiffness;
  q.bend_stiffness = p->bend_stiffness;
  q.max_dx = p->max_dx;
  q.target_toi = p->target_toi;
  q.min_newton_steps = p->min_newton_steps;
  q.ccd_max_iter = p->ccd_max_iter;
  q.eiganalysis_eps = p->eiganalysis_eps;
  q.contact_dhat = p->contact_dhat;
  q.contact_kappa = p->contact_kappa;
  q.contact_dynamic = p->contact_dynamic;
  q.shell_mu = p->shell_mu;
  q.shell_lambda = p->shell_lambda;
  q.friction = p->friction;
  q.friction_eps = p->friction_eps;
  q.barrier_kind = (BarrierKind)p->barrier_kind;
  q.contact_rayleigh = p->contact_rayleigh != 0;
  q.self_collision = p->self_collision != 0;
  q.cg_tol = p->cg_tol;
  q.cg_max_iter = p->cg_max_iter;
  q.floor_y = p->floor_y;
  q.newton_tol = p->newton_tol;
  q.precond = p->precond;
  q.schwarz_domain = p->schwarz_domain;
  s->init(P, Vv, im, T, q);
  std::vector<std::array<uint32_t, 3>> SF(nshell);
  for (uint32_t i = 0; i < nshell; ++i) SF[i] = {shell_faces[3 * i], shell_faces[3 * i + 1], shell_faces[3 * i + 2]};
  s->set_shell_faces(SF);
  for (uint32_t i = 0; i < nstitch; ++i) {
    Stitch<R> st;
    for (int k = 0; k < 6; ++k) {
      st.index[k] = st_idx[6 * i + k];
      st.weight[k] = st_w[6 * i + k];
    }
    st.stiffness = st_kl[3 * i];
    st.l0 = st_kl[3 * i + 1];
    st.l_cap = st_kl[3 * i + 2];
    s->stitches.push_back(st);
  }
  for (uint32_t i = 0; i < ncol; ++i) {
    const float* c = cols + 8 * i;
    Collider<R> col;
    col.kind = (int)c[0];
    col.a = Vt<R>(c[1], c[2], c[3]);
    col.n = Vt<R>(c[4], c[5], c[6]);
    col.radius = c[7];
    s->colliders.push_back(col);
  }
  if (static_mask) s->set_static_collider_verts(std::vector<uint8_t>(static_mask, static_mask + nv));
  return s;
}

template <class R>
void fill_stats(const StepStats& s, OracleStats* o) {
  o->newton_iters = s.newton_iters;
  o->max_cg_iters = s.max_cg_iters;
  o->num_contacts = s.num_contacts;
  o->stencils = s.stencils;
  o->ccd_cap_hits = s.ccd_cap_hits;
  o->max_reresid = s.max_reresid;
  o->t_min = s.t_min;
  o->penetration_free = s.penetration_free;
  o->all_finite = s.all_finite;
}

// StVK shell element built from rest positions; returns 0 if the rest triangle is degenerate.
template <class R>
int shell_eval(const double* rest9, const double* p9, double mu, double lambda, double eps, double* energy,
                      double* grad9, double* hess81) {
  ShellEl<R> el;
  Vt<R> r[3], p[3];
  for (int k = 0; k < 3; ++k) {
    r[k] = Vt<R>((R)rest9[3 * k], (R)rest9[3 * k + 1], (R)rest9[3 * k + 2]);
    p[k] = Vt<R>((R)p9[3 * k], (R)p9[3 * k + 1], (R)p9[3 * k + 2]);
  }
  if (!build_shell(r[0], r[1], r[2], R(1.0e-12), el)) return 0;
  Vt<R> g[3];
  shell_gradient(p, el, (R)mu, (R)lambda, g);
  R h[81];
  shell_hessian(p, el, (R)mu, (R)lambda, (R)eps, h);
  *energy = shell_energy(p, el, (R)mu, (R)lambda);
  for (int k = 0; k < 3; ++k)
    for (int c = 0; c < 3; ++c) grad9[3 * k + c] = g[k][c];
  for (int k = 0; k < 81; ++k) hess81[k] = h[k];
  return 1;
}

}  // namespace

namespace {
// Replaces the shell elements with explicit rest data: per face its vertices, the inverse
// rest shape (column-major 2x2) and area (5 values), and its (mu, lambda).
template <class R>
static void set_shells(ImplicitSolver<R>& s, uint32_t n, const uint32_t* faces, const double* rest, const double* mu,
                       const double* lam) {
  s.shells.clear();
  s.shell_k.clear();
  for (uint32_t f = 0; f < n; ++f) {
    ShellEl<R> el;
    for (int k = 0; k < 3; ++k) el.v[k] = faces[3 * f + k];
    el.dm_inv = Mat2<R>{(R)rest[5 * f], (R)rest[5 * f + 1], (R)rest[5 * f + 2], (R)rest[5 * f + 3]};
    el.area = (R)rest[5 * f + 4];
    s.shells.push_back(el);
    s.shell_k.push_back({(R)mu[f], (R)lam[f]});
  }
}

template <class R>
static int set_pins_t(ImplicitSolver<R>& s, uint32_t n, const uint32_t* idx, const double* target, const double* ghat,
                      const int* kinematic, const double* stiffness) {
  std::vector<Pin<R>> p(n);
  for (uint32_t i = 0; i < n; ++i) {
    p[i].index = idx[i];
    p[i].target = Vt<R>((R)target[3 * i], (R)target[3 * i + 1], (R)target[3 * i + 2]);
    p[i].ghat = (R)ghat[i];
    p[i].kinematic = kinematic[i] != 0;
    p[i].stiffness = (R)stiffness[i];
  }
  return s.set_pins(p);
}

template <class R>
static int set_pulls_t(ImplicitSolver<R>& s, uint32_t n, const uint32_t* idx, const double* target,
                       const double* weight) {
  std::vector<Pull<R>> p(n);
  for (uint32_t i = 0; i < n; ++i) {
    p[i].index = idx[i];
    p[i].target = Vt<R>((R)target[3 * i], (R)target[3 * i + 1], (R)target[3 * i + 2]);
    p[i].weight = (R)weight[i];
  }
  return s.set_pulls(p);
}

template <class R>
static int set_sl_faces_t(ImplicitSolver<R>& s, uint32_t n, const uint32_t* faces, const double* limits,
                          const double* masses, uint32_t nl, uint32_t nm) {
  std::vector<std::array<uint32_t, 3>> f(n);
  for (uint32_t i = 0; i < n; ++i) f[i] = {faces[3 * i], faces[3 * i + 1], faces[3 * i + 2]};
  std::vector<R> l(limits, limits + nl), m(masses, masses + nm);
  if (!s.set_strain_limit_faces(f, l, m)) return -1;
  return (int)s.sl_faces.size();
}

template <class R>
static void set_limits_t(ImplicitSolver<R>& s, double constraint_tol, double ratio, double k, double ratio_weft,
                         uint32_t nuv, const double* uv) {
  s.params.constraint_tol = (R)constraint_tol;
  s.params.strain_limit_ratio = (R)ratio;
  s.params.strain_limit_k = (R)k;
  s.params.strain_limit_ratio_weft = (R)ratio_weft;
  s.uvs.assign(nuv, {});
  for (uint32_t i = 0; i < nuv; ++i) s.uvs[i] = {(R)uv[2 * i], (R)uv[2 * i + 1]};
}

template <class R>
static void set_stretch_edges_t(ImplicitSolver<R>& s, uint32_t n, const uint32_t* edges) {
  s.stretch_edges.assign(n, {});
  s.stretch_rest.assign(n, R(0));
  for (uint32_t i = 0; i < n; ++i) {
    s.stretch_edges[i] = {edges[2 * i], edges[2 * i + 1]};
    s.stretch_rest[i] = (s.positions[edges[2 * i]] - s.positions[edges[2 * i + 1]]).length();
  }
}

template <class R>
static int strain_limit_face_t(int kind, const double* rest9, const double* p9, double limit, double mass,
                               double elastic_k, double eps, int dynamic, double* energy, double* grad9,
                               double* hess81) {
  ShellEl<R> el;
  Vt<R> r[3], p[3];
  for (int k = 0; k < 3; ++k) {
    r[k] = Vt<R>((R)rest9[3 * k], (R)rest9[3 * k + 1], (R)rest9[3 * k + 2]);
    p[k] = Vt<R>((R)p9[3 * k], (R)p9[3 * k + 1], (R)p9[3 * k + 2]);
  }
  if (!build_shell(r[0], r[1], r[2], R(1.0e-12), el)) return -1;
  *energy = strain_limit_energy(p, el, (R)limit, (BarrierKind)kind);
  Vt<R> g[3];
  R h[81];
  bool on = strain_limit_eval(p, el, (R)limit, (R)mass, (R)elastic_k, (BarrierKind)kind, (R)eps, dynamic != 0, g, h);
  for (int k = 0; k < 3; ++k)
    for (int c = 0; c < 3; ++c) grad9[3 * k + c] = on ? (double)g[k][c] : 0.0;
  for (int k = 0; k < 81; ++k) hess81[k] = on ? (double)h[k] : 0.0;
  return on ? 1 : 0;
}

}  // namespace

extern "C" {

void* oracle_solver_new(int precision, uint32_t nv, const float* pos, const float* vel, const float* inv_mass,
                        uint32_t nt, const uint32_t* tris, const uint8_t* static_mask, uint32_t nshell,
                        const uint32_t* shell_faces, uint32_t nstitch, const uint32_t* st_idx, const float* st_w,
                        const float* st_kl, uint32_t ncol, const float* cols, const OracleParams* p) {
  auto* a = new AnySolver();
  a->prec = precision;
  if (precision == 0)
    a->f = make_solver<float>(nv, pos, vel, inv_mass, nt, tris, static_mask, nshell, shell_faces, nstitch, st_idx,
                              st_w, st_kl, ncol, cols, p);
  else
    a->d = make_solver<double>(nv, pos, vel, inv_mass, nt, tris, static_mask, nshell, shell_faces, nstitch, st_idx,
                               st_w, st_kl, ncol, cols, p);
  return a;
}

void oracle_solver_free(void* h) { delete (AnySolver*)h; }

int oracle_solver_step(void* h, int nsteps, int check_intersection, OracleStats* out) {
  auto* a = (AnySolver*)h;
  for (int k = 0; k < nsteps; ++k) {
    if (a->prec == 0) {
      StepStats s = a->f->step(check_intersection != 0);
      if (out) fill_stats<float>(s, out + k);
    } else {
      StepStats s = a->d->step(check_intersection != 0);
      if (out) fill_stats<double>(s, out + k);
    }
  }
  return 0;
}

// positions / velocities as f64 (whichever precision the solver runs in)
void oracle_solver_state(void* h, double* pos, double* vel) {
  auto* a = (AnySolver*)h;
  size_t n = a->prec == 0 ? a->f->positions.size() : a->d->positions.size();
  for (size_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      if (a->prec == 0) {
        if (pos) pos[3 * i + c] = a->f->positions[i][c];
        if (vel) vel[3 * i + c] = a->f->velocities[i][c];
      } else {
        if (pos) pos[3 * i + c] = a->d->positions[i][c];
        if (vel) vel[3 * i + c] = a->d->velocities[i][c];
      }
    }
}

// Multiplies every stitch's stiffness by factor[i] (in the solver's precision).
void oracle_solver_scale_stitches(void* h, const double* factor) {
  auto* a = (AnySolver*)h;
  if (a->prec == 0) {
    for (size_t i = 0; i < a->f->stitches.size(); ++i) a->f->stitches[i].stiffness *= (float)factor[i];
  } else {
    for (size_t i = 0; i < a->d->stitches.size(); ++i) a->d->stitches[i].stiffness *= factor[i];
  }
}

void oracle_solver_set_shells(void* h, uint32_t n, const uint32_t* faces, const double* rest, const double* mu,
                              const double* lam) {
  auto* a = (AnySolver*)h;
  if (a->prec == 0)
    set_shells(*a->f, n, faces, rest, mu, lam);
  else
    set_shells(*a->d, n, faces, rest, mu, lam);
}

int oracle_solver_set_kinematic(void* h, const double* pos) {
  auto* a = (AnySolver*)h;
  if (a->prec == 0) {
    std::vector<Vt<float>> x(a->f->positions.size());
    for (size_t i = 0; i < x.size(); ++i) x[i] = Vt<float>((float)pos[3 * i], (float)pos[3 * i + 1], (float)pos[3 * i + 2]);
    return a->f->set_kinematic_collider_positions(x);
  }
  std::vector<Vt<double>> x(a->d->positions.size());
  for (size_t i = 0; i < x.size(); ++i) x[i] = Vt<double>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
  return a->d->set_kinematic_collider_positions(x);
}

// Baraff-Witkin membrane stiffnesses (warp, weft, shear) and optional per-element values
// (n = 0 clears them; otherwise n must be the element count): 1 accepted, 0 not.
int oracle_solver_set_membrane(void* h, double kw, double kf, double ks, uint32_t n, const double* k3) {
  auto* a = (AnySolver*)h;
  auto apply = [&](auto& s) {
    using R = typename std::decay_t<decltype(s.membrane_k)>::value_type::value_type;
    if (n && n != s.membrane.size()) return 0;
    s.params.membrane_warp = (R)kw;
    s.params.membrane_weft = (R)kf;
    s.params.membrane_shear = (R)ks;
    s.membrane_k.assign(n, {});
    for (uint32_t i = 0; i < n; ++i) s.membrane_k[i] = {(R)k3[3 * i], (R)k3[3 * i + 1], (R)k3[3 * i + 2]};
    return 1;
  };
  return a->prec == 0 ? apply(*a->f) : apply(*a->d);
}

// set_shell_stiffness (per-face (mu, lambda) for the current shells, in their order):
// 1 when accepted, 0 when n is not the shell count (nothing changed).
int oracle_solver_set_shell_stiffness(void* h, uint32_t n, const double* mu_lam) {
  auto* a = (AnySolver*)h;
  auto apply = [&](auto& s) {
    using R = typename std::decay_t<decltype(s.shell_k)>::value_type::value_type;
    if (n != s.shells.size()) return 0;
    s.shell_k.assign(n, {});
    for (uint32_t i = 0; i < n; ++i) s.shell_k[i] = {(R)mu_lam[2 * i], (R)mu_lam[2 * i + 1]};
    return 1;
  };
  return a->prec == 0 ? apply(*a->f) : apply(*a->d);
}

// The hinges (build_hinges, bending.rs:126-158): vertices u32[4 n] and rest angles f64[n],
// up to cap; returns the count.
uint32_t oracle_solver_hinges(void* h, uint32_t* idx, double* rest, uint32_t cap) {
  auto* a = (AnySolver*)h;
  auto copy = [&](auto& s) {
    for (size_t i = 0; i < s.hinges.size() && i < cap; ++i) {
      for (int k = 0; k < 4; ++k) idx[4 * i + k] = s.hinges[i].v[k];
      rest[i] = (double)s.hinges[i].rest;
    }
    return (uint32_t)s.hinges.size();
  };
  return a->prec == 0 ? copy(*a->f) : copy(*a->d);
}

// positions_self_intersect (implicit.rs:618-650) at positions pos (f32[3 nv]).
int oracle_solver_self_intersect(void* h, const float* pos) {
  auto* a = (AnySolver*)h;
  if (a->prec != 0) return -1;
  std::vector<Vt<float>> x(a->f->positions.size());
  for (size_t i = 0; i < x.size(); ++i) x[i] = Vt<float>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
  return a->f->positions_self_intersect(x) ? 1 : 0;
}

// collider_sides (implicit.rs:1431-1475) at the current positions: +1 outside, -1 inside,
// per vertex (f32[nv]); returns 0 when there is no static collider (nothing written).
int oracle_solver_collider_sides(void* h, float* out) {
  auto* a = (AnySolver*)h;
  if (a->prec != 0) return 0;
  auto side = a->f->collider_sides(a->f->positions);
  for (size_t i = 0; i < side.size(); ++i) out[i] = side[i];
  return side.empty() ? 0 : 1;
}

// Pins (FixPair): 1 when accepted, 0 when rejected (nothing changed).
int oracle_solver_set_pins(void* h, uint32_t n, const uint32_t* idx, const double* target, const double* ghat,
                           const int* kinematic, const double* stiffness) {
  auto* a = (AnySolver*)h;
  return a->prec == 0 ? set_pins_t(*a->f, n, idx, target, ghat, kinematic, stiffness)
                      : set_pins_t(*a->d, n, idx, target, ghat, kinematic, stiffness);
}

// Pulls (PullPair): 1 when accepted, 0 when rejected.
int oracle_solver_set_pulls(void* h, uint32_t n, const uint32_t* idx, const double* target, const double* weight) {
  auto* a = (AnySolver*)h;
  return a->prec == 0 ? set_pulls_t(*a->f, n, idx, target, weight) : set_pulls_t(*a->d, n, idx, target, weight);
}

// Strain-limit barrier faces: the number of faces kept, or -1 when the lengths disagree.
int oracle_solver_set_strain_limit_faces(void* h, uint32_t n, const uint32_t* faces, const double* limits,
                                         const double* masses, uint32_t nl, uint32_t nm) {
  auto* a = (AnySolver*)h;
  return a->prec == 0 ? set_sl_faces_t(*a->f, n, faces, limits, masses, nl, nm)
                      : set_sl_faces_t(*a->d, n, faces, limits, masses, nl, nm);
}

// Pin gap floor, per-edge strain limit (warp ratio, stiffness, weft ratio) and per-vertex
// UVs (nuv pairs; 0 clears them).
void oracle_solver_set_limits(void* h, double constraint_tol, double ratio, double k, double ratio_weft, uint32_t nuv,
                              const double* uv) {
  auto* a = (AnySolver*)h;
  if (a->prec == 0)
    set_limits_t(*a->f, constraint_tol, ratio, k, ratio_weft, nuv, uv);
  else
    set_limits_t(*a->d, constraint_tol, ratio, k, ratio_weft, nuv, uv);
}

// The collider's friction coefficient (infinity: unset) and the friction mode (0 min, 1 max,
// 2 mean) it combines with the cloth's under.
void oracle_solver_set_friction(void* h, double collider_friction, int mode) {
  auto* a = (AnySolver*)h;
  if (a->prec == 0) {
    a->f->params.collider_friction = (float)collider_friction;
    a->f->params.friction_mode = mode;
  } else {
    a->d->params.collider_friction = collider_friction;
    a->d->params.friction_mode = mode;
  }
}

// Replaces the stretch edges (a mesh with explicit edges, as the reference's Mesh carries);
// rest lengths from the current positions.
void oracle_solver_set_stretch_edges(void* h, uint32_t n, const uint32_t* edges) {
  auto* a = (AnySolver*)h;
  if (a->prec == 0)
    set_stretch_edges_t(*a->f, n, edges);
  else
    set_stretch_edges_t(*a->d, n, edges);
}

void oracle_solver_set_state(void* h, const double* pos, const double* vel) {
  auto* a = (AnySolver*)h;
  size_t n = a->prec == 0 ? a->f->positions.size() : a->d->positions.size();
  for (size_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      if (a->prec == 0) {
        if (pos) a->f->positions[i][c] = (float)pos[3 * i + c];
        if (vel) a->f->velocities[i][c] = (float)vel[3 * i + c];
      } else {
        if (pos) a->d->positions[i][c] = pos[3 * i + c];
        if (vel) a->d->velocities[i][c] = vel[3 * i + c];
      }
    }
}

// Element counts: hinges, shells, edges, exclusion entries.
void oracle_solver_counts(void* h, uint32_t* out4) {
  auto* a = (AnySolver*)h;
  if (a->prec == 0) {
    out4[0] = (uint32_t)a->f->hinges.size();
    out4[1] = (uint32_t)a->f->shells.size();
    out4[2] = (uint32_t)a->f->edges.size();
    out4[3] = (uint32_t)a->f->collider_tris.size();
  } else {
    out4[0] = (uint32_t)a->d->hinges.size();
    out4[1] = (uint32_t)a->d->shells.size();
    out4[2] = (uint32_t)a->d->edges.size();
    out4[3] = (uint32_t)a->d->collider_tris.size();
  }
}

// Active self-contact stencils at the current positions: idx u32[4*cap], d f32[cap].
uint32_t oracle_solver_stencils(void* h, uint32_t* idx, float* d, uint32_t cap) {
  auto* a = (AnySolver*)h;
  if (a->prec != 0) return 0;
  auto st = a->f->self_collision_stencils(a->f->positions);
  for (size_t i = 0; i < st.size() && i < cap; ++i) {
    for (int k = 0; k < 4; ++k) idx[4 * i + k] = st[i].idx[k];
    d[i] = st[i].d;
  }
  return (uint32_t)st.size();
}

// One assembly at the current positions (x = x_tilde = positions unless given):
// returns the scalar CSR through the oracle_csr_* handle API and rhs f32[3n].
void* oracle_solver_assemble(void* h, const float* x_in, const float* xt_in, float* rhs_out) {
  auto* a = (AnySolver*)h;
  auto& s = *a->f;
  size_t n = s.positions.size();
  std::vector<Vt<float>> x = s.positions, xt = s.positions;
  for (size_t i = 0; i < n; ++i) {
    if (x_in) x[i] = Vt<float>(x_in[3 * i], x_in[3 * i + 1], x_in[3 * i + 2]);
    if (xt_in) xt[i] = Vt<float>(xt_in[3 * i], xt_in[3 * i + 1], xt_in[3 * i + 2]);
  }
  float h2 = s.params.dt * s.params.dt;
  std::vector<float> rhs;
  auto* m = new Csr(s.assemble(x, xt, 1.0f / h2, rhs, nullptr));
  std::memcpy(rhs_out, rhs.data(), 4 * rhs.size());
  return m;
}

// CCD step fraction for the current positions and a search direction dx f32[3n].
float oracle_solver_ccd(void* h, const float* dx_in) {
  auto* a = (AnySolver*)h;
  auto& s = *a->f;
  size_t n = s.positions.size();
  std::vector<Vt<float>> dx(n);
  for (size_t i = 0; i < n; ++i) dx[i] = Vt<float>(dx_in[3 * i], dx_in[3 * i + 1], dx_in[3 * i + 2]);
  uint32_t caps = 0;
  return s.ccd_max_step(s.positions, dx, &caps);
}

// ---- element-level functions (float) --------------------------------------------------
float oracle_point_tri(const float* p12, float* g12, float* bary3) {
  Vt<float> p[4];
  for (int k = 0; k < 4; ++k) p[k] = Vt<float>(p12[3 * k], p12[3 * k + 1], p12[3 * k + 2]);
  Vt<float> g[4];
  float d = point_tri_distance_grad(p[0], p[1], p[2], p[3], g);
  for (int k = 0; k < 4; ++k)
    for (int c = 0; c < 3; ++c) g12[3 * k + c] = g[k][c];
  float w[3];
  closest_point_bary(p[0], p[1], p[2], p[3], w);
  for (int k = 0; k < 3; ++k) bary3[k] = w[k];
  return d;
}

float oracle_seg_seg(const float* p12, float* g12, float* plain) {
  Vt<float> p[4];
  for (int k = 0; k < 4; ++k) p[k] = Vt<float>(p12[3 * k], p12[3 * k + 1], p12[3 * k + 2]);
  Vt<float> g[4];
  float d = segment_segment_distance_grad(p[0], p[1], p[2], p[3], g);
  for (int k = 0; k < 4; ++k)
    for (int c = 0; c < 3; ++c) g12[3 * k + c] = g[k][c];
  *plain = segment_segment_distance(p[0], p[1], p[2], p[3]);
  return d;
}

// kind 0 = point-triangle, 1 = edge-edge
float oracle_accd(const float* x12, const float* dx12, float offset, float max_t, float reduction, uint32_t max_iter,
                  int kind) {
  Vt<float> x0[4], dx[4];
  for (int k = 0; k < 4; ++k) {
    x0[k] = Vt<float>(x12[3 * k], x12[3 * k + 1], x12[3 * k + 2]);
    dx[k] = Vt<float>(dx12[3 * k], dx12[3 * k + 1], dx12[3 * k + 2]);
  }
  if (kind == 0)
    return accd_toi<float>(x0, dx, offset, max_t, reduction, max_iter, [](const Vt<float>* p) {
      float d = point_triangle_distance(p[0], p[1], p[2], p[3]);
      return d * d;
    });
  return accd_toi<float>(x0, dx, offset, max_t, reduction, max_iter, [](const Vt<float>* p) {
    float d = segment_segment_distance(p[0], p[1], p[2], p[3]);
    return d * d;
  });
}

int oracle_barrier(int kind, double d, double dhat, double kappa, int f64, double* egh) {
  if (f64) {
    double e = 0, g = 0, h = 0;
    bool on = barrier_of<double>((BarrierKind)kind, d, dhat, kappa, e, g, h);
    egh[0] = e; egh[1] = g; egh[2] = h;
    return on;
  }
  float e = 0, g = 0, h = 0;
  bool on = barrier_of<float>((BarrierKind)kind, (float)d, (float)dhat, (float)kappa, e, g, h);
  egh[0] = e; egh[1] = g; egh[2] = h;
  return on;
}

// friction (contact.rs:613-644) in f32: gradient g3 and Hessian h9 (row-major); 0 when
// nothing applies (mu <= 0 or a separating contact), with g3/h9 zeroed.
int oracle_friction(const float* fc3, const float* dx3, const float* n3, float mu, float eps, float* g3, float* h9) {
  Vt<float> g;
  float h[3][3] = {};
  bool on = friction<float>(Vt<float>(fc3[0], fc3[1], fc3[2]), Vt<float>(dx3[0], dx3[1], dx3[2]),
                            Vt<float>(n3[0], n3[1], n3[2]), mu, eps, g, h);
  for (int c = 0; c < 3; ++c) g3[c] = on ? g[c] : 0.f;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) h9[3 * r + c] = on ? h[r][c] : 0.f;
  return on;
}

// Strain-limit barrier of one face (rest shape rest9): energy, and the gradient and Hessian
// at unit stiffness (dynamic = 0) or as assembled (dynamic = 1: elastic_k + mass / d^2).
// Returns 1 active, 0 inactive, -1 degenerate rest face.
int oracle_strain_limit_face(int f64, int kind, const double* rest9, const double* p9, double limit, double mass,
                             double elastic_k, double eps, int dynamic, double* energy, double* grad9,
                             double* hess81) {
  return f64 ? strain_limit_face_t<double>(kind, rest9, p9, limit, mass, elastic_k, eps, dynamic, energy, grad9, hess81)
             : strain_limit_face_t<float>(kind, rest9, p9, limit, mass, elastic_k, eps, dynamic, energy, grad9, hess81);
}

// Baraff-Witkin element (f32) from a rest triangle rest9 at positions p9: conditions c3,
// element gradient g9 and Hessian h81 (element_assembly); returns 0 for a degenerate rest
// triangle. wuv6, when given, receives the deformation columns wu, wv.
int oracle_membrane_element(const float* rest9, const float* p9, float kw, float kf, float ks, float* c3, float* g9,
                            float* h81, float* wuv6) {
  Vt<float> r[3], p[3];
  for (int k = 0; k < 3; ++k) {
    r[k] = Vt<float>(rest9[3 * k], rest9[3 * k + 1], rest9[3 * k + 2]);
    p[k] = Vt<float>(p9[3 * k], p9[3 * k + 1], p9[3 * k + 2]);
  }
  MembraneEl<float> el;
  if (!build_membrane_el(r[0], r[1], r[2], el)) return 0;
  bw_conditions(p, el.dm_inv, c3);
  bw_element(p, el, kw, kf, ks, g9, h81);
  if (wuv6) {
    Vt<float> wu, wv;
    bw_deformation(p, el.dm_inv, wu, wv);
    for (int c = 0; c < 3; ++c) {
      wuv6[c] = wu[c];
      wuv6[3 + c] = wv[c];
    }
  }
  return 1;
}

// Baraff-Witkin materials (f32): stretch material of w3 into m9, shear blocks of (wu, wv)
// into m36 ([uu, uv, vu, vv], each row-major), clamped or exact.
void oracle_membrane_materials(const float* w3, const float* wu3, const float* wv3, int clamp, float* m9,
                               float* m36) {
  float m[3][3], sm[4][3][3];
  bw_stretch_material(Vt<float>(w3[0], w3[1], w3[2]), m);
  bw_shear_material(Vt<float>(wu3[0], wu3[1], wu3[2]), Vt<float>(wv3[0], wv3[1], wv3[2]), clamp != 0, sm);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) m9[3 * r + c] = m[r][c];
  for (int b = 0; b < 4; ++b)
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) m36[9 * b + 3 * r + c] = sm[b][r][c];
}

// One-sided edge strain limit in f32: energy, grad_i g3 and h_ii h9 (row-major).
float oracle_edge_strain(const float* xi3, const float* xj3, float rest, float ratio, float k, float* g3, float* h9) {
  Vt<float> xi(xi3[0], xi3[1], xi3[2]), xj(xj3[0], xj3[1], xj3[2]), g;
  float h[3][3];
  edge_strain_block(xi, xj, rest, ratio, k, g, h);
  for (int c = 0; c < 3; ++c) g3[c] = g[c];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) h9[3 * r + c] = h[r][c];
  return edge_strain_energy(xi, xj, rest, ratio, k);
}

// vertex_triangle_pairs / edge_edge_pairs (broadphase.rs:250-264, 356-367) in f32: the
// candidate pairs sorted and deduplicated into out (2 u32 each, up to cap); returns the count.
// exclude_one_ring applies one_ring_exclusion over tris; movable (u8 per vertex) may be null.
uint64_t oracle_vt_pairs(uint32_t nv, const float* pos, uint32_t nt, const uint32_t* tris, float search,
                         int exclude_one_ring, const uint8_t* movable, uint32_t* out, uint64_t cap) {
  std::vector<Vt<float>> P(nv);
  for (uint32_t i = 0; i < nv; ++i) P[i] = Vt<float>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
  std::vector<std::array<uint32_t, 3>> T(nt);
  for (uint32_t t = 0; t < nt; ++t) T[t] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
  std::vector<std::vector<uint32_t>> ex = exclude_one_ring ? one_ring_exclusion(nv, T)
                                                           : std::vector<std::vector<uint32_t>>(nv);
  std::vector<uint8_t> mov = movable ? std::vector<uint8_t>(movable, movable + nv) : std::vector<uint8_t>();
  std::vector<std::pair<uint32_t, uint32_t>> pr;
  for_each_vertex_triangle_pair<float>(P, T, search, ex, mov, [&](uint32_t v, uint32_t t) { pr.push_back({v, t}); });
  std::sort(pr.begin(), pr.end());
  pr.erase(std::unique(pr.begin(), pr.end()), pr.end());
  for (size_t i = 0; i < pr.size() && i < cap; ++i) {
    out[2 * i] = pr[i].first;
    out[2 * i + 1] = pr[i].second;
  }
  return pr.size();
}

uint64_t oracle_ee_pairs(uint32_t nv, const float* pos, uint32_t ne, const uint32_t* edges, float search,
                         const uint8_t* movable, uint32_t* out, uint64_t cap) {
  std::vector<Vt<float>> P(nv);
  for (uint32_t i = 0; i < nv; ++i) P[i] = Vt<float>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
  std::vector<std::array<uint32_t, 2>> E(ne);
  for (uint32_t e = 0; e < ne; ++e) E[e] = {edges[2 * e], edges[2 * e + 1]};
  std::vector<uint8_t> mov = movable ? std::vector<uint8_t>(movable, movable + nv) : std::vector<uint8_t>();
  std::vector<std::pair<uint32_t, uint32_t>> pr;
  for_each_edge_edge_pair<float>(P, E, search, mov, [&](uint32_t a, uint32_t b) { pr.push_back({a, b}); });
  std::sort(pr.begin(), pr.end());
  pr.erase(std::unique(pr.begin(), pr.end()), pr.end());
  for (size_t i = 0; i < pr.size() && i < cap; ++i) {
    out[2 * i] = pr[i].first;
    out[2 * i + 1] = pr[i].second;
  }
  return pr.size();
}

// The assembler's elastic-block gather (Asm::push into its requested blocks, implicit.rs
// Asm; the blocks the Rayleigh stiffnesses read): the n_trips triplets (row trip_rc[2k],
// column trip_rc[2k + 1], value trip_v[k], scalar indices) pushed in order over nv vertices
// with the vertex pairs (slot_keys[2s], slot_keys[2s + 1]) requested as slots s; each slot's
// row-major 3x3 block into out (9 floats per slot).
void oracle_asm_blocks(uint32_t nv, uint32_t n_slots, const uint32_t* slot_keys, uint32_t n_trips,
                       const uint32_t* trip_rc, const float* trip_v, float* out) {
  std::unordered_map<uint64_t, size_t> slots;
  for (uint32_t k = 0; k < n_slots; ++k) slots[((uint64_t)slot_keys[2 * k] << 32) | slot_keys[2 * k + 1]] = k;
  TripletSinkT<float> sink;
  sink.begin(3 * (size_t)nv);
  std::vector<uint8_t> pinned(nv, 0);
  ImplicitSolver<float>::Asm a;
  a.sink = &sink;
  a.slots = &slots;
  a.blocks.assign(n_slots, std::array<float, 9>{});
  a.pinned = &pinned;
  for (uint32_t k = 0; k < n_trips; ++k) a.push(trip_rc[2 * k], trip_rc[2 * k + 1], trip_v[k]);
  for (uint32_t k = 0; k < n_slots; ++k)
    for (int q = 0; q < 9; ++q) out[9 * k + q] = a.blocks[k][q];
}

// sym_eig2 (shell_model.rs:60-78) in f32 of the symmetric [[p, q], [q, r]] (a3 = p, q, r):
// eigenvalues descending into l2, eigenvectors as the columns of v4 (column-major).
void oracle_sym_eig2(const float* a3, float* l2, float* v4) {
  Mat2<float> a{a3[0], a3[1], a3[1], a3[2]}, v{};
  sym_eig2(a, l2, v);
  v4[0] = v.xx;
  v4[1] = v.xy;
  v4[2] = v.yx;
  v4[3] = v.yy;
}

// svd3x2 (shell_model.rs:84-106) in f32 of F (f6: column 0 xyz, then column 1 xyz): U's two
// columns into u6 the same way, sigma descending into s2, V column-major into v4.
void oracle_svd3x2(const float* f6, float* u6, float* s2, float* v4) {
  Mat3x2<float> f{Vt<float>(f6[0], f6[1], f6[2]), Vt<float>(f6[3], f6[4], f6[5])}, u{};
  Mat2<float> v{};
  svd3x2(f, u, s2, v);
  const float uu[6] = {u.c0.x, u.c0.y, u.c0.z, u.c1.x, u.c1.y, u.c1.z};
  for (int k = 0; k < 6; ++k) u6[k] = uu[k];
  v4[0] = v.xx;
  v4[1] = v.xy;
  v4[2] = v.yx;
  v4[3] = v.yy;
}

// The StVK shell density over principal stretches (shell_model.rs:131-176) in f32: returns
// psi(s2), its gradient into g2 and its Hessian (row-major 2x2) into h4.
float oracle_stvk_density(const float* s2, float mu, float lambda, float* g2, float* h4) {
  stvk_dpsi(s2, mu, lambda, g2);
  stvk_d2psi(s2, mu, lambda, h4);
  return stvk_density(s2, mu, lambda);
}

// edge_triangle_pairs (broadphase.rs:523-585) in f32: the sorted unique (edge, triangle)
// candidate pairs into out (2 u32 each, up to cap); returns the count.
uint64_t oracle_et_pairs(uint32_t nv, const float* pos, uint32_t ne, const uint32_t* edges, uint32_t nt,
                         const uint32_t* tris, float search, uint32_t* out, uint64_t cap) {
  std::vector<Vt<float>> P(nv);
  for (uint32_t i = 0; i < nv; ++i) P[i] = Vt<float>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
  std::vector<std::array<uint32_t, 2>> E(ne);
  for (uint32_t e = 0; e < ne; ++e) E[e] = {edges[2 * e], edges[2 * e + 1]};
  std::vector<std::array<uint32_t, 3>> T(nt);
  for (uint32_t t = 0; t < nt; ++t) T[t] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
  const auto pr = edge_triangle_pairs<float>(P, E, T, search);
  for (size_t i = 0; i < pr.size() && i < cap; ++i) {
    out[2 * i] = pr[i].first;
    out[2 * i + 1] = pr[i].second;
  }
  return pr.size();
}

// any_edge_triangle_pair (broadphase.rs:587-751) in f32 with one of three predicates: mode 0
// never matches (every candidate offered is written to out, repeats included, up to cap),
// mode 1 matches the first candidate offered, mode 2 is edge_triangle_intersect. movable
// (u8 per vertex) may be null. *offered = the number of candidates the predicate saw; returns
// 1 when it matched.
int oracle_et_any(uint32_t nv, const float* pos, uint32_t ne, const uint32_t* edges, uint32_t nt,
                  const uint32_t* tris, float search, const uint8_t* movable, int mode, uint32_t* out, uint64_t cap,
                  uint64_t* offered) {
  std::vector<Vt<float>> P(nv);
  for (uint32_t i = 0; i < nv; ++i) P[i] = Vt<float>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
  std::vector<std::array<uint32_t, 2>> E(ne);
  for (uint32_t e = 0; e < ne; ++e) E[e] = {edges[2 * e], edges[2 * e + 1]};
  std::vector<std::array<uint32_t, 3>> T(nt);
  for (uint32_t t = 0; t < nt; ++t) T[t] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
  std::vector<uint8_t> mov = movable ? std::vector<uint8_t>(movable, movable + nv) : std::vector<uint8_t>();
  uint64_t n = 0;
  const bool found = any_edge_triangle_pair<float>(P, E, T, search, mov, [&](uint32_t ei, uint32_t ti) {
    if (mode == 0 && out && n < cap) {
      out[2 * n] = ei;
      out[2 * n + 1] = ti;
    }
    ++n;
    if (mode == 1) return true;
    if (mode == 2) {
      const auto& e = E[ei];
      const auto& t = T[ti];
      return edge_triangle_intersect(P[e[0]], P[e[1]], P[t[0]], P[t[1]], P[t[2]]);
    }
    return false;
  });
  if (offered) *offered = n;
  return found ? 1 : 0;
}

// unique_edges (broadphase.rs:332-343) into out (2 u32 each, room for 3 nt); returns the count.
uint32_t oracle_unique_edges(uint32_t nt, const uint32_t* tris, uint32_t* out) {
  std::vector<std::array<uint32_t, 3>> T(nt);
  for (uint32_t t = 0; t < nt; ++t) T[t] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
  auto e = unique_edges(T);
  for (size_t i = 0; i < e.size(); ++i) {
    out[2 * i] = e[i][0];
    out[2 * i + 1] = e[i][1];
  }
  return (uint32_t)e.size();
}

float oracle_grid_cell(float search, float extent) { return grid_cell(search, extent); }

// edge_triangle_intersect (contact.rs:324-352) for the segment p0p1 against triangle abc.
int oracle_edge_triangle_intersect(const float* p15) {
  Vt<float> v[5];
  for (int k = 0; k < 5; ++k) v[k] = Vt<float>(p15[3 * k], p15[3 * k + 1], p15[3 * k + 2]);
  return edge_triangle_intersect(v[0], v[1], v[2], v[3], v[4]) ? 1 : 0;
}

// closest_point_on_triangle_bary (contact.rs:84-124): q3 and weights w3 for p12 = p, a, b, c.
void oracle_closest_point(const float* p12, float* q3, float* w3) {
  Vt<float> v[4];
  for (int k = 0; k < 4; ++k) v[k] = Vt<float>(p12[3 * k], p12[3 * k + 1], p12[3 * k + 2]);
  Vt<float> q = closest_point_bary(v[0], v[1], v[2], v[3], w3);
  for (int c = 0; c < 3; ++c) q3[c] = q[c];
}

// edge_edge_witness (contact.rs:238-311): the four witness weights for p12 = ea0, ea1, eb0, eb1.
void oracle_ee_witness(const float* p12, float* w4) {
  Vt<float> v[4];
  for (int k = 0; k < 4; ++k) v[k] = Vt<float>(p12[3 * k], p12[3 * k + 1], p12[3 * k + 2]);
  edge_edge_witness(v[0], v[1], v[2], v[3], w4);
}

// signed_point_tri_distance_grad (contact.rs:889-915) with the side taken the way the
// stencil collection takes it for a one-triangle mesh: pseudonormals of that triangle,
// surface_normal_at the closest point, inside when (p - q).n < 0. Returns the signed gap,
// gradient in g12 and the side in *inside.
float oracle_signed_point_tri(const float* p12, float* g12, int* inside) {
  Vt<float> v[4];
  for (int k = 0; k < 4; ++k) v[k] = Vt<float>(p12[3 * k], p12[3 * k + 1], p12[3 * k + 2]);
  auto pn = pseudonormals<float>({v[1], v[2], v[3]}, {{0u, 1u, 2u}});
  float w[3];
  Vt<float> q = closest_point_bary(v[0], v[1], v[2], v[3], w);
  Vt<float> pnv[3] = {pn[0], pn[1], pn[2]};
  Vt<float> n = surface_normal_at(w, (v[2] - v[1]).cross(v[3] - v[1]).normalize_or_zero(), pnv);
  bool in = (v[0] - q).dot(n) < 0;
  Vt<float> g[4];
  float d = signed_point_tri_distance_grad(v[0], v[1], v[2], v[3], in, g);
  for (int k = 0; k < 4; ++k)
    for (int c = 0; c < 3; ++c) g12[3 * k + c] = g[k][c];
  *inside = in ? 1 : 0;
  return d;
}

// Collider::distance (contact.rs:33-51) of col8 = (kind, a xyz, n xyz, radius) at x3.
float oracle_collider_distance(const float* col8, const float* x3, float* n3) {
  Collider<float> c;
  c.kind = (int)col8[0];
  c.a = Vt<float>(col8[1], col8[2], col8[3]);
  c.n = Vt<float>(col8[4], col8[5], col8[6]);
  c.radius = col8[7];
  float d;
  Vt<float> n;
  c.distance(Vt<float>(x3[0], x3[1], x3[2]), d, n);
  for (int k = 0; k < 3; ++k) n3[k] = n[k];
  return d;
}

// vertex_contact (contact.rs:1029-1050): log barrier, dynamic stiffness, no friction.
void oracle_vertex_contact(const float* x3, uint32_t ncol, const float* cols, float dhat, float kappa, float coupling,
                           float mass, float* g3, float* h9) {
  std::vector<Collider<float>> cs(ncol);
  for (uint32_t i = 0; i < ncol; ++i) {
    const float* c = cols + 8 * i;
    cs[i].kind = (int)c[0];
    cs[i].a = Vt<float>(c[1], c[2], c[3]);
    cs[i].n = Vt<float>(c[4], c[5], c[6]);
    cs[i].radius = c[7];
  }
  Vt<float> g;
  float h[3][3];
  vertex_contact_full<float>(Vt<float>(x3[0], x3[1], x3[2]), cs, dhat, kappa, coupling, mass, BarrierKind::Log,
                             nullptr, false, Vt<float>(), 0.f, 0.f, g, h);
  for (int c = 0; c < 3; ++c) g3[c] = g[c];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) h9[3 * r + c] = h[r][c];
}

float oracle_dynamic_stiffness(float base, float coupling, float mass, float gap, float dhat) {
  return dynamic_stiffness(base, coupling, mass, gap, dhat);
}

// stencil_friction (contact.rs:659-705): gradient fg12 and Hessian fh144 (row-major);
// 0 with both zeroed when nothing applies.
int oracle_stencil_friction(const float* g12, const float* dx12, float barrier_grad, float mu, float eps, float* fg12,
                            float* fh144) {
  Vt<float> g[4], dx[4], fg[4];
  for (int k = 0; k < 4; ++k) {
    g[k] = Vt<float>(g12[3 * k], g12[3 * k + 1], g12[3 * k + 2]);
    dx[k] = Vt<float>(dx12[3 * k], dx12[3 * k + 1], dx12[3 * k + 2]);
  }
  bool on = stencil_friction(g, dx, barrier_grad, mu, eps, fg, fh144);
  for (int k = 0; k < 4; ++k)
    for (int c = 0; c < 3; ++c) fg12[3 * k + c] = on ? fg[k][c] : 0.f;
  if (!on)
    for (int k = 0; k < 144; ++k) fh144[k] = 0.f;
  return on ? 1 : 0;
}

float oracle_rayleigh(int n, const float* elastic, const float* mass, const float* weights, const float* e3,
                      float offset) {
  float el[16][9];
  for (int i = 0; i < n * n; ++i)
    for (int q = 0; q < 9; ++q) el[i][q] = elastic[9 * i + q];
  return rayleigh_stiffness<float>(el, mass, weights, n, Vt<float>(e3[0], e3[1], e3[2]), offset);
}

int oracle_shell(int f64, const double* rest9, const double* p9, double mu, double lambda, double eps, double* energy,
                 double* grad9, double* hess81) {
  return f64 ? shell_eval<double>(rest9, p9, mu, lambda, eps, energy, grad9, hess81)
             : shell_eval<float>(rest9, p9, mu, lambda, eps, energy, grad9, hess81);
}

double oracle_hinge(int f64, const double* p12, double* grad12, double* grad_fd12) {
  if (f64) {
    Vt<double> p[4], g[4], gf[4];
    for (int k = 0; k < 4; ++k) p[k] = Vt<double>(p12[3 * k], p12[3 * k + 1], p12[3 * k + 2]);
    dihedral_grad(p, g);
    dihedral_grad_fd(p, gf);
    for (int k = 0; k < 4; ++k)
      for (int c = 0; c < 3; ++c) {
        grad12[3 * k + c] = g[k][c];
        grad_fd12[3 * k + c] = gf[k][c];
      }
    return dihedral_angle(p);
  }
  Vt<float> p[4], g[4], gf[4];
  for (int k = 0; k < 4; ++k) p[k] = Vt<float>((float)p12[3 * k], (float)p12[3 * k + 1], (float)p12[3 * k + 2]);
  dihedral_grad(p, g);
  dihedral_grad_fd(p, gf);
  for (int k = 0; k < 4; ++k)
    for (int c = 0; c < 3; ++c) {
      grad12[3 * k + c] = g[k][c];
      grad_fd12[3 * k + c] = gf[k][c];
    }
  return dihedral_angle(p);
}

void oracle_stitch(const double* x18, const double* w6, double l0, double lcap, double* grad18, double* hess324) {
  Vt<double> x[6], g[6];
  double w[6];
  for (int k = 0; k < 6; ++k) {
    x[k] = Vt<double>(x18[3 * k], x18[3 * k + 1], x18[3 * k + 2]);
    w[k] = w6[k];
  }
  stitch_force_hessian(x, w, l0, lcap, g, hess324);
  for (int k = 0; k < 6; ++k)
    for (int c = 0; c < 3; ++c) grad18[3 * k + c] = g[k][c];
}


// ---- FP64 reference adjoint (test infrastructure) ---------------------------------------
// One step's adjoint system, in FP64 on the oracle's assembly, at the converged state x_{n+1}
// of step n (x_n, v_n its start): the Jacobian H = dG/dx and dG/dtheta of the step's
// equilibrium residual G(x) = M/h^2 (x - x~) + grad Phi(x; theta) (implicit.rs:2280-3155
// restated in FP64), x~ = x_n + h v_n + h^2 g on free vertices. The contact set is the one
// collected at x_{n+1}, held fixed; each stencil's stiffness is split into its elastic part,
// held fixed, and its mass part, which goes as 1/d^2 from its value at x_{n+1} (the
// definition of the GPU adjoint's exact Hessian). Both derivatives are central differences
// of G: H column by column, many columns at once by a distance-2 colouring of the vertices'
// element graph (shells, hinges, stitches, stretch edges, stencils), step eps; dG/dtheta
// parameter by parameter, step 1e-6 theta_j. theta = [stiff_p (P), warp_p, weft_p (2P),
// seam_q (S)]: shell (mu, lambda) = base * stiff_p, rest shape = pattern triangle scaled by
// (weft, warp) along (u, v), stitch stiffness = base * seam_q.
// H is n3 x n3 row-major (pinned rows and columns 0), dG is (3P + S) x n3. Returns the
// number of stencils, or -1 for a float solver.
// Diagnostics of the reference adjoint: 0 freezes each contact stiffness whole (no 1/d^2 mass
// part), to measure how much that part of the exact Hessian moves a gradient.
static int g_adjoint_km = 1;
void oracle_adjoint_set_km(int on) { g_adjoint_km = on; }

int oracle_adjoint_system(void* h, uint32_t npanel, uint32_t nseam, const float* uv, const uint8_t* panel,
                          const uint8_t* seam, const double* stitch_k0, const double* theta, const double* xn,
                          const double* vn, const double* xn1, double eps, double* H, double* dG) {
  auto* any = (AnySolver*)h;
  if (any->prec != 1) return -1;
  ImplicitSolver<double>& s = *any->d;
  using V = Vt<double>;
  const size_t nv = s.positions.size(), n3 = 3 * nv;
  const uint32_t P = npanel, S = nseam, np = 3 * P + S;
  const double mu0 = s.params.shell_mu, lam0 = s.params.shell_lambda;
  std::vector<double> th(theta, theta + np);
  auto apply_theta = [&](const std::vector<double>& t) {
    s.shell_k.resize(s.shells.size());
    for (size_t f = 0; f < s.shells.size(); ++f) {
      const uint32_t p = panel[f];
      const double su = t[P + 2 * p + 1], sv = t[P + 2 * p];
      const float* q = uv + 6 * f;
      const double xx = su * ((double)q[2] - (double)q[0]), xy = sv * ((double)q[3] - (double)q[1]);
      const double yx = su * ((double)q[4] - (double)q[0]), yy = sv * ((double)q[5] - (double)q[1]);
      const double det = xx * yy - yx * xy;
      s.shells[f].dm_inv = Mat2<double>{yy / det, -xy / det, -yx / det, xx / det};
      s.shells[f].area = 0.5 * std::fabs(det);
      s.shell_k[f] = {mu0 * t[p], lam0 * t[p]};
    }
    for (size_t i = 0; i < s.stitches.size(); ++i) s.stitches[i].stiffness = stitch_k0[i] * t[3 * P + seam[i]];
  };
  apply_theta(th);
  const double dt = s.params.dt, inv_h2 = 1.0 / (dt * dt);
  std::vector<V> x0(nv), x1(nv), xt(nv);
  for (size_t i = 0; i < nv; ++i) {
    x0[i] = V(xn[3 * i], xn[3 * i + 1], xn[3 * i + 2]);
    x1[i] = V(xn1[3 * i], xn1[3 * i + 1], xn1[3 * i + 2]);
    const V v(vn[3 * i], vn[3 * i + 1], vn[3 * i + 2]);
    xt[i] = s.inv_mass[i] > 0 ? x0[i] + v * dt + s.params.gravity * (dt * dt) : x0[i];
  }
  // stencils at x_{n+1}, their kinds and the stiffnesses the step's assembly gives them
  std::vector<uint8_t> kinds;
  std::vector<Stencil<double>> sts =
      s.params.self_collision ? s.self_collision_stencils(x1, &kinds) : std::vector<Stencil<double>>();
  std::vector<double> rhs;
  s.frozen = nullptr;
  s.grad_only = false;
  s.record_contacts = true;
  s.assemble(x1, xt, inv_h2, rhs, nullptr);
  s.record_contacts = false;
  using FC = typename ImplicitSolver<double>::FrozenContact;
  std::vector<FC> fr(sts.size());
  for (size_t i = 0; i < sts.size(); ++i) {
    FC& f = fr[i];
    for (int a = 0; a < 4; ++a) f.idx[a] = sts[i].idx[a];
    f.kind = kinds[i];
    f.ghat = sts[i].ghat;
    f.km = g_adjoint_km ? s.contact_rec[i][1] : 0.0;
    f.k_el = s.contact_rec[i][0] - f.km;
    f.d0 = sts[i].d;
  }
  s.frozen = &fr;
  s.grad_only = true;
  std::vector<double> gp(n3), gm(n3);
  auto G = [&](const std::vector<V>& x, std::vector<double>& out) {
    s.assemble(x, xt, inv_h2, rhs, nullptr);
    for (size_t i = 0; i < n3; ++i) out[i] = -rhs[i];
  };
  // vertex coupling graph
  std::vector<std::vector<uint32_t>> nb(nv);
  auto couple = [&](const uint32_t* v, int k) {
    for (int a = 0; a < k; ++a)
      for (int b = 0; b < k; ++b) nb[v[a]].push_back(v[b]);
  };
  for (auto& sh : s.shells) couple(sh.v, 3);
  for (auto& hg : s.hinges) couple(hg.v, 4);
  for (auto& st : s.stitches) couple(st.index, 6);
  for (auto& e : s.stretch_edges) couple(e.data(), 2);
  for (auto& f : fr) couple(f.idx, 4);
  for (size_t i = 0; i < nv; ++i) {
    nb[i].push_back((uint32_t)i);
    std::sort(nb[i].begin(), nb[i].end());
    nb[i].erase(std::unique(nb[i].begin(), nb[i].end()), nb[i].end());
  }
  // greedy distance-2 colouring of the free vertices
  std::vector<int> color(nv, -1);
  int ncolor = 0;
  std::vector<int> mark;
  for (size_t j = 0; j < nv; ++j) {
    if (!(s.inv_mass[j] > 0)) continue;
    mark.assign(ncolor + 1, 0);
    for (uint32_t a : nb[j])
      for (uint32_t b : nb[a])
        if (color[b] >= 0) mark[color[b]] = 1;
    int c = 0;
    while (mark[c]) ++c;
    color[j] = c;
    ncolor = std::max(ncolor, c + 1);
  }
  std::fill(H, H + n3 * n3, 0.0);
  std::vector<V> xp(x1), xm(x1);
  for (int c = 0; c < ncolor; ++c)
    for (int k = 0; k < 3; ++k) {
      xp = x1;
      xm = x1;
      for (size_t j = 0; j < nv; ++j)
        if (color[j] == c) {
          xp[j][k] += eps;
          xm[j][k] -= eps;
        }
      G(xp, gp);
      G(xm, gm);
      for (size_t j = 0; j < nv; ++j) {
        if (color[j] != c) continue;
        for (uint32_t i : nb[j]) {
          if (!(s.inv_mass[i] > 0)) continue;
          for (int r = 0; r < 3; ++r) H[(3 * i + r) * n3 + 3 * j + k] = (gp[3 * i + r] - gm[3 * i + r]) / (2 * eps);
        }
      }
    }
  // parameter partials
  for (uint32_t j = 0; j < np; ++j) {
    const double d = 1e-6 * th[j];
    std::vector<double> t = th;
    t[j] = th[j] + d;
    apply_theta(t);
    G(x1, gp);
    t[j] = th[j] - d;
    apply_theta(t);
    G(x1, gm);
    for (size_t i = 0; i < n3; ++i) dG[(size_t)j * n3 + i] = (gp[i] - gm[i]) / (2 * d);
  }
  apply_theta(th);
  s.frozen = nullptr;
  s.grad_only = false;
  return (int)fr.size();
}

}  // extern "C"
