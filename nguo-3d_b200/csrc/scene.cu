// Scene construction (host): topology, rest state, block patterns and push-order gather
// lists for the implicit step, plus the scene half of the C ABI.
//
// Rest quantities are computed in f32 in the reference's operation order:
//   ImplicitSolver::new (implicit.rs:530-601): hinges, 1-ring exclusion, unique edges,
//     characteristic edge length;
//   SimState::from_mesh (state.rs:37-61): stretch springs on the unique edges;
//   build_shells (shell_model.rs:310-348): in-plane frame, Dm^-1, rest area;
//   set_static_collider_verts (implicit.rs:1258-1320): winding check and angle-weighted
//     pseudonormals (contact.rs:963-1001).
#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <map>
#include <unordered_map>

#include "elements.cuh"
#include "scene.cuh"

namespace mg {

namespace {

using HV = V3<float>;

HV hp(const float* p, uint32_t i) { return HV(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }

// Angle-weighted pseudonormals of the static collider's triangles `ctris` at positions P
// (contact.rs:963-1001), welded on exact position bits within an instance (-0 folded to
// +0); pn gets 3 per vertex (zero off the collider).
static void collider_pseudonormals(const float* P, uint32_t nv, const std::vector<std::array<uint32_t, 3>>& ctris,
                                   const std::vector<uint8_t>& vinst, std::vector<float>& pn) {
  std::vector<HV> acc;
  std::vector<uint32_t> of(nv);
  auto bits = [](float c) { if (c == 0.f) c = 0.f; uint32_t b; std::memcpy(&b, &c, 4); return (uint64_t)b; };
  std::map<std::array<uint64_t, 3>, uint32_t> wmap;
  for (uint32_t i = 0; i < nv; ++i) {
    std::array<uint64_t, 3> kk = {bits(P[3 * i]) | ((uint64_t)vinst[i] << 32), bits(P[3 * i + 1]),
                                  bits(P[3 * i + 2])};
    auto it = wmap.find(kk);
    if (it == wmap.end()) {
      uint32_t id = (uint32_t)wmap.size();
      wmap.emplace(kk, id);
      of[i] = id;
    } else {
      of[i] = it->second;
    }
  }
  acc.assign(wmap.size(), HV());
  for (const auto& tv : ctris) {
    HV q[3] = {hp(P, tv[0]), hp(P, tv[1]), hp(P, tv[2])};
    HV face = (q[1] - q[0]).cross(q[2] - q[0]).normalize_or_zero();
    if (face.x == 0.f && face.y == 0.f && face.z == 0.f) continue;
    for (int k = 0; k < 3; ++k) {
      HV u = (q[(k + 1) % 3] - q[k]).normalize_or_zero();
      HV w = (q[(k + 2) % 3] - q[k]).normalize_or_zero();
      float dt = u.dot(w);
      dt = dt < -1.f ? -1.f : (dt > 1.f ? 1.f : dt);
      acc[of[tv[k]]] += face * std::acos(dt);
    }
  }
  pn.assign(3 * (size_t)nv, 0.f);
  for (uint32_t i = 0; i < nv; ++i) {
    HV n = acc[of[i]].normalize_or_zero();
    pn[3 * i] = n.x;
    pn[3 * i + 1] = n.y;
    pn[3 * i + 2] = n.z;
  }
}

float host_dihedral(const HV p[4]) {
  HV n1 = (p[1] - p[0]).cross(p[2] - p[0]);
  HV n2 = (p[1] - p[2]).cross(p[3] - p[2]);
  HV e = (p[2] - p[1]).normalize_or_zero();
  HV n1n = n1.normalize_or_zero(), n2n = n2.normalize_or_zero();
  float s = n1n.cross(n2n).dot(e);
  float c = n1n.dot(n2n);
  c = c < -1.f ? -1.f : (c > 1.f ? 1.f : c);
  return std::atan2(s, c);
}

// build_shells (shell_model.rs:310-348) for one triangle: the inverse rest shape dm
// (column-major 2x2) in the triangle's own in-plane frame and the rest area; false for a
// degenerate triangle.
bool shell_rest_shape(const HV& p0, const HV& p1, const HV& p2, float dm[4], float& area) {
  HV e1 = p1 - p0, e2 = p2 - p0;
  area = 0.5f * e1.cross(e2).length();
  if (area <= 1e-12f) return false;
  HV ax = e1.normalize();
  HV ay = (e2 - ax * e2.dot(ax)).normalize();
  float xx = e1.dot(ax), xy = e1.dot(ay), yx = e2.dot(ax), yy = e2.dot(ay);
  float det = xx * yy - yx * xy;
  if (std::fabs(det) < 1e-20f) return false;
  float inv = 1.f / det;
  dm[0] = yy * inv;
  dm[1] = xy * -inv;
  dm[2] = yx * -inv;
  dm[3] = xx * inv;
  return true;
}

struct Contribution {
  uint32_t row, col;
};
constexpr uint32_t PAD_ENTRY = 0xffffffffu;  // alignment padding in the contribution lists

}  // namespace

// The checks a description must pass before anything is built: index ranges, the stitch
// rules of ImplicitSolver::set_stitches (implicit.rs:939-966) and the parameters. Host only.
static int validate_desc(const mguso_scene_desc* d) {
  MG_CHECK_ARG(d && d->positions && d->inv_mass && (d->nt == 0 || d->tris), "scene: null arrays");
  MG_CHECK_ARG(d->nv > 0 && d->nv < (1u << 30), "scene: vertex count out of range");
  MG_CHECK_ARG(d->nshell == 0 || d->shell_faces, "scene: null arrays");
  MG_CHECK_ARG(d->nstitch == 0 || (d->stitch_idx && d->stitch_w && d->stitch_kl), "scene: null arrays");
  const uint32_t nv = d->nv, nt = d->nt;
  for (uint32_t t = 0; t < 3 * nt; ++t) MG_CHECK_ARG(d->tris[t] < nv, "scene: triangle index out of range");
  for (uint32_t t = 0; t < 3 * d->nshell; ++t) MG_CHECK_ARG(d->shell_faces[t] < nv, "scene: shell face index out of range");
  for (uint32_t i = 0; i < d->nstitch; ++i) {
    for (int k = 0; k < 6; ++k) MG_CHECK_ARG(d->stitch_idx[6 * i + k] < nv, "scene: stitch references a missing vertex");
    const float* kl = d->stitch_kl + 3 * i;
    MG_CHECK_ARG(std::isfinite(kl[0]) && kl[0] >= 0, "scene: stitch stiffness must be finite and >= 0");
    MG_CHECK_ARG(std::isfinite(kl[1]) && kl[1] > 0, "scene: stitch rest length must be > 0");
    MG_CHECK_ARG(std::isfinite(kl[2]) && kl[2] >= kl[1], "scene: stitch cap below its rest length");
    float ws = d->stitch_w[6 * i] + d->stitch_w[6 * i + 1] + d->stitch_w[6 * i + 2];
    float wt = d->stitch_w[6 * i + 3] + d->stitch_w[6 * i + 4] + d->stitch_w[6 * i + 5];
    MG_CHECK_ARG(std::fabs(ws - 1.f) <= 1e-3f && std::fabs(wt - 1.f) <= 1e-3f, "scene: stitch weights must sum to 1 per side");
  }
  MG_CHECK_ARG(d->params.dt > 0, "scene: dt must be > 0");
  MG_CHECK_ARG(d->params.precond == MGUSO_PRECOND_BLOCK_JACOBI || d->params.precond == MGUSO_PRECOND_SCHWARZ,
               "scene: unknown preconditioner");
  MG_CHECK_ARG(d->params.pcg_mode >= 0 && d->params.pcg_mode <= 2, "scene: pcg_mode must be 0, 1 or 2");
  MG_CHECK_ARG(d->params.factor_storage >= 0 && d->params.factor_storage <= 2, "scene: factor_storage must be 0, 1 or 2");
  MG_CHECK_ARG(d->params.schwarz_levels <= 2, "scene: schwarz_levels must be 1 or 2");
  MG_CHECK_ARG(std::isfinite(d->params.membrane_warp) && std::isfinite(d->params.membrane_weft) &&
                   std::isfinite(d->params.membrane_shear) && d->params.membrane_warp >= 0 &&
                   d->params.membrane_weft >= 0 && d->params.membrane_shear >= 0,
               "scene: membrane stiffnesses must be finite and >= 0");
  MG_CHECK_ARG(d->params.pcg_variant >= 0 && d->params.pcg_variant <= 24, "scene: pcg_variant must be in [0, 24]");
  MG_CHECK_ARG(std::isfinite(d->params.schwarz_weight) && d->params.schwarz_weight >= 0.f,
               "scene: schwarz_weight must be finite and >= 0");
  MG_CHECK_ARG(std::isfinite(d->params.strain_limit_ratio) && std::isfinite(d->params.strain_limit_k) &&
                   std::isfinite(d->params.strain_limit_ratio_weft) && d->params.strain_limit_ratio >= 0 &&
                   d->params.strain_limit_k >= 0 && d->params.strain_limit_ratio_weft >= 0,
               "scene: strain limit ratios and stiffness must be finite and >= 0");
  MG_CHECK_ARG(d->nstretch == 0 || d->stretch_edges, "scene: null arrays");
  for (uint32_t e = 0; e < 2 * d->nstretch; ++e)
    MG_CHECK_ARG(d->stretch_edges[e] < nv, "scene: stretch edge index out of range");
  return MGUSO_OK;
}

int scene_build(Scene& s, const mguso_scene_desc* d, const std::vector<uint32_t>& inst_vert) {
  MG_TRY(validate_desc(d));
  const uint32_t nv = d->nv, nt = d->nt;
  s.p = d->params;
  s.nv = nv;
  s.nt = nt;
  s.mixed = d->params.precision == MGUSO_PRECISION_MIXED;
  // Schwarz factor storage: FP32 tiles for plain FP32 (and whenever asked), FP16 tiles
  // scaled per domain for mixed precision unless the caller (or the adjoint) chose FP32
  if (d->params.factor_storage == 1 || (d->params.factor_storage == 0 && !s.mixed)) s.fp16_factor = false;
  if (d->params.factor_storage == 2) s.fp16_factor = true;
  s.st = s.ctx->stream;
  cudaStream_t st = s.st;
  const float* P = d->positions;
  MG_CHECK_ARG(inst_vert.size() >= 2 && inst_vert.size() <= PCG_MAX_INST + 1 && inst_vert.front() == 0 &&
                   inst_vert.back() == nv,
               "scene: instance vertex ranges");
  s.ninst = (uint32_t)inst_vert.size() - 1;
  s.inst_vert = inst_vert;
  std::vector<uint8_t> vinst(nv);
  for (uint32_t k = 0; k < s.ninst; ++k) {
    MG_CHECK_ARG(inst_vert[k] < inst_vert[k + 1], "scene: empty instance");
    for (uint32_t v = inst_vert[k]; v < inst_vert[k + 1]; ++v) vinst[v] = (uint8_t)k;
  }
  MG_TRY(s.vinst.upload(vinst.data(), nv, st));
  // every triangle, stitch and shell face lies in one instance, triangles in instance order
  s.inst_tri.assign(s.ninst + 1, nt);
  s.inst_tri[0] = 0;
  {
    uint32_t k = 0;
    for (uint32_t t = 0; t < nt; ++t) {
      const uint32_t a = vinst[d->tris[3 * t]];
      MG_CHECK_ARG(a == vinst[d->tris[3 * t + 1]] && a == vinst[d->tris[3 * t + 2]] && a >= k,
                   "scene: triangles must be grouped by instance");
      while (k < a) s.inst_tri[++k] = t;
    }
    while (k < s.ninst) s.inst_tri[++k] = nt;
  }
  for (uint32_t f = 0; f < d->nshell; ++f)
    MG_CHECK_ARG(vinst[d->shell_faces[3 * f]] == vinst[d->shell_faces[3 * f + 1]] &&
                     vinst[d->shell_faces[3 * f]] == vinst[d->shell_faces[3 * f + 2]],
                 "scene: a shell face spans two instances");
  for (uint32_t i = 0; i < d->nstitch; ++i)
    for (int k = 1; k < 6; ++k)
      MG_CHECK_ARG(vinst[d->stitch_idx[6 * i + k]] == vinst[d->stitch_idx[6 * i]], "scene: a stitch spans two instances");

  // ---- state -------------------------------------------------------------------------
  s.h_inv_mass.assign(d->inv_mass, d->inv_mass + nv);
  s.h_pinned.resize(nv);
  std::vector<uint32_t> free_verts;
  for (uint32_t i = 0; i < nv; ++i) {
    s.h_pinned[i] = s.h_inv_mass[i] <= 0.f;
    if (!s.h_pinned[i]) free_verts.push_back(i);
  }
  s.n_free = (uint32_t)free_verts.size();
  MG_TRY(s.x.upload(P, 3 * (size_t)nv, st));
  std::vector<float> vel(3 * (size_t)nv, 0.f);
  if (d->velocities) std::memcpy(vel.data(), d->velocities, 4 * vel.size());
  MG_TRY(s.v.upload(vel.data(), vel.size(), st));
  MG_TRY(s.x0.reserve(3 * (size_t)nv));
  MG_TRY(s.xt.reserve(3 * (size_t)nv));
  MG_TRY(s.xstep.reserve(3 * (size_t)nv));
  MG_TRY(s.dx.reserve(3 * (size_t)nv));
  MG_TRY(s.inv_mass.upload(s.h_inv_mass.data(), nv, st));
  MG_TRY(s.pinned.upload(s.h_pinned.data(), nv, st));
  if (free_verts.empty())
    MG_TRY(s.free_verts.reserve(1));
  else
    MG_TRY(s.free_verts.upload(free_verts.data(), free_verts.size(), st));
  auto vfree = [&](uint32_t v) { return !s.h_pinned[v]; };

  // ---- topology ------------------------------------------------------------------------
  std::vector<std::array<uint32_t, 3>> tris(nt);
  for (uint32_t t = 0; t < nt; ++t) tris[t] = {d->tris[3 * t], d->tris[3 * t + 1], d->tris[3 * t + 2]};
  // unique edges (geometry.rs:38-47 / broadphase.rs:334-346): sorted (min, max)
  std::vector<std::array<uint32_t, 2>> edges;
  edges.reserve(3 * nt);
  for (auto& t : tris)
    for (int k = 0; k < 3; ++k) {
      uint32_t a = t[k], b = t[(k + 1) % 3];
      edges.push_back({std::min(a, b), std::max(a, b)});
    }
  std::sort(edges.begin(), edges.end());
  edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
  s.n_edge = (uint32_t)edges.size();
  // sorted (min, max) edges are grouped by instance
  s.inst_edge.assign(s.ninst + 1, s.n_edge);
  s.inst_edge[0] = 0;
  {
    uint32_t k = 0;
    for (uint32_t e = 0; e < s.n_edge; ++e)
      while (k < vinst[edges[e][0]]) s.inst_edge[++k] = e;
  }
  // characteristic length per instance: mean unique-edge length, summed in order
  // (implicit.rs:533-542)
  s.char_len.assign(s.ninst, 1.f);
  for (uint32_t k = 0; k < s.ninst; ++k) {
    if (s.inst_edge[k + 1] == s.inst_edge[k]) continue;
    float sum = 0.f;
    for (uint32_t e = s.inst_edge[k]; e < s.inst_edge[k + 1]; ++e)
      sum += (hp(P, edges[e][0]) - hp(P, edges[e][1])).length();
    s.char_len[k] = std::max(sum / (float)(s.inst_edge[k + 1] - s.inst_edge[k]), 1e-6f);
  }
  // hinges (bending.rs:126-158): sorted edge key -> opposite vertices in triangle order
  std::map<std::pair<uint32_t, uint32_t>, std::vector<uint32_t>> em;
  for (auto& t : tris) {
    uint32_t e3[3][3] = {{t[1], t[2], t[0]}, {t[0], t[2], t[1]}, {t[0], t[1], t[2]}};
    for (auto& x : e3) em[{std::min(x[0], x[1]), std::max(x[0], x[1])}].push_back(x[2]);
  }
  std::vector<uint32_t> hinge_v;
  std::vector<float> hinge_rest;
  if (s.p.bend_stiffness > 0) {
    for (auto& kv : em) {
      if (kv.second.size() != 2) continue;
      uint32_t hv[4] = {kv.second[0], kv.first.first, kv.first.second, kv.second[1]};
      HV pp[4] = {hp(P, hv[0]), hp(P, hv[1]), hp(P, hv[2]), hp(P, hv[3])};
      for (uint32_t q : hv) hinge_v.push_back(q);
      hinge_rest.push_back(host_dihedral(pp));
    }
  }
  s.n_hinge = (uint32_t)hinge_rest.size();
  // Baraff-Witkin membrane elements (membrane.rs:272-312) on every triangle, rest frame from
  // the initial positions; degenerate triangles are skipped
  std::vector<uint32_t> mem_v;
  std::vector<float> mem_dm, mem_area;
  if (s.p.membrane_warp > 0 || s.p.membrane_weft > 0 || s.p.membrane_shear > 0) {
    for (auto& t : tris) {
      HV x0 = hp(P, t[0]), x1 = hp(P, t[1]), x2 = hp(P, t[2]);
      HV e1 = x1 - x0, e2 = x2 - x0;
      const float a = e1.length();
      HV n = e1.cross(e2);
      const float area = 0.5f * n.length();
      if (a < 1.0e-9f || area < 1.0e-12f) continue;
      HV t1 = e1 / a;
      HV t2 = n.cross(e1).normalize_or_zero();
      const float b = e2.dot(t1), dd = e2.dot(t2);
      const float det = a * dd;
      if (std::fabs(det) < 1.0e-12f) continue;
      mem_v.insert(mem_v.end(), {t[0], t[1], t[2]});
      mem_dm.insert(mem_dm.end(), {1.0f / a, -b / (a * dd), 0.0f, 1.0f / dd});
      mem_area.push_back(area);
    }
  }
  s.n_mem = (uint32_t)mem_area.size();
  // shells (shell_model.rs:310-348), StVK, per-scene (mu, lambda)
  std::vector<uint32_t> shell_v;
  std::vector<float> shell_dm, shell_area, shell_mu, shell_lam;
  if (s.p.shell_mu > 0 || s.p.shell_lambda > 0) {
    for (uint32_t f = 0; f < d->nshell; ++f) {
      const uint32_t* fv = d->shell_faces + 3 * f;
      const float k = d->shell_stiff ? d->shell_stiff[f] : 1.f;
      if (d->shell_rest) {
        const float* r = d->shell_rest + 5 * f;
        shell_v.insert(shell_v.end(), {fv[0], fv[1], fv[2]});
        shell_dm.insert(shell_dm.end(), {r[0], r[1], r[2], r[3]});
        shell_area.push_back(r[4]);
        shell_mu.push_back(s.p.shell_mu * k);
        shell_lam.push_back(s.p.shell_lambda * k);
        continue;
      }
      float dm[4], area;
      if (!shell_rest_shape(hp(P, fv[0]), hp(P, fv[1]), hp(P, fv[2]), dm, area)) continue;
      shell_v.insert(shell_v.end(), {fv[0], fv[1], fv[2]});
      shell_dm.insert(shell_dm.end(), {dm[0], dm[1], dm[2], dm[3]});
      shell_area.push_back(area);
      shell_mu.push_back(s.p.shell_mu * k);
      shell_lam.push_back(s.p.shell_lambda * k);
    }
  }
  s.n_shell = (uint32_t)shell_area.size();
  // stretch springs on the unique edges (state.rs:37-61), or on the description's stretch
  // edges, rest = initial length. At zero stiffness, with the edge strain limit off, every
  // spring block and gradient entry is exactly 0, so they are left out. Each spring carries
  // its strain-limit ratio (edge_strain_ratio, implicit.rs:798-817): warp, or with a weft
  // ratio and uvs, weft for an edge less U- than V-aligned in UV space.
  std::vector<std::array<uint32_t, 2>> stretch = edges;
  if (d->nstretch) {
    stretch.resize(d->nstretch);
    for (uint32_t e = 0; e < d->nstretch; ++e) stretch[e] = {d->stretch_edges[2 * e], d->stretch_edges[2 * e + 1]};
    for (auto& e : stretch)
      MG_CHECK_ARG(vinst[e[0]] == vinst[e[1]], "scene: a stretch edge spans two instances");
  }
  const bool edge_limit = s.p.strain_limit_ratio > 0.f && s.p.strain_limit_k > 0.f;
  std::vector<uint32_t> spring_v;
  std::vector<float> spring_rest, spring_slr;
  if (s.p.stiffness != 0.f || edge_limit)
    for (auto& e : stretch) {
      spring_v.insert(spring_v.end(), {e[0], e[1]});
      spring_rest.push_back((hp(P, e[0]) - hp(P, e[1])).length());
      float ratio = s.p.strain_limit_ratio;
      if (s.p.strain_limit_ratio_weft > 0.f && d->uvs) {
        const float du = std::fabs(d->uvs[2 * e[0]] - d->uvs[2 * e[1]]);
        const float dv = std::fabs(d->uvs[2 * e[0] + 1] - d->uvs[2 * e[1] + 1]);
        if (!(du >= dv)) ratio = s.p.strain_limit_ratio_weft;
      }
      spring_slr.push_back(ratio);
    }
  s.n_spring = (uint32_t)spring_rest.size();
  s.edge_limit = edge_limit;
  // stitches with stiffness > 0 (implicit.rs:2456-2485 skips the rest)
  std::vector<uint32_t> stitch_idx;
  std::vector<float> stitch_w, stitch_kl;
  for (uint32_t i = 0; i < d->nstitch; ++i) {
    if (!(d->stitch_kl[3 * i] > 0)) continue;
    stitch_idx.insert(stitch_idx.end(), d->stitch_idx + 6 * i, d->stitch_idx + 6 * i + 6);
    stitch_w.insert(stitch_w.end(), d->stitch_w + 6 * i, d->stitch_w + 6 * i + 6);
    stitch_kl.insert(stitch_kl.end(), d->stitch_kl + 3 * i, d->stitch_kl + 3 * i + 3);
  }
  s.n_stitch = (uint32_t)(stitch_kl.size() / 3);

  auto up = [&](auto& buf, const auto& vec) -> int {
    if (vec.empty()) return buf.reserve(1);
    return buf.upload(vec.data(), vec.size(), st);
  };
  MG_TRY(up(s.mem_v, mem_v));
  MG_TRY(up(s.mem_dm, mem_dm));
  MG_TRY(up(s.mem_area, mem_area));
  MG_TRY(up(s.shell_v, shell_v));
  MG_TRY(up(s.shell_dm, shell_dm));
  MG_TRY(up(s.shell_area, shell_area));
  MG_TRY(up(s.shell_mu, shell_mu));
  MG_TRY(up(s.shell_lam, shell_lam));
  MG_TRY(up(s.hinge_v, hinge_v));
  MG_TRY(up(s.hinge_rest, hinge_rest));
  MG_TRY(up(s.spring_v, spring_v));
  MG_TRY(up(s.spring_rest, spring_rest));
  MG_TRY(up(s.spring_slr, spring_slr));
  MG_TRY(up(s.stitch_idx, stitch_idx));
  MG_TRY(up(s.stitch_w, stitch_w));
  MG_TRY(up(s.stitch_kl, stitch_kl));

  // active (>= 1 free vertex) element lists
  auto active = [&](const std::vector<uint32_t>& vv, uint32_t k, uint32_t n, std::vector<uint32_t>& out) {
    out.clear();
    for (uint32_t e = 0; e < n; ++e) {
      bool a = false;
      for (uint32_t q = 0; q < k; ++q) a = a || vfree(vv[k * e + q]);
      if (a) out.push_back(e);
    }
  };
  std::vector<uint32_t> act;
  active(mem_v, 3, s.n_mem, act);
  s.n_act_mem = (uint32_t)act.size();
  MG_TRY(up(s.act_mem, act));
  active(shell_v, 3, s.n_shell, act);
  s.n_act_shell = (uint32_t)act.size();
  MG_TRY(up(s.act_shell, act));
  active(hinge_v, 4, s.n_hinge, act);
  s.n_act_hinge = (uint32_t)act.size();
  MG_TRY(up(s.act_hinge, act));
  active(spring_v, 2, s.n_spring, act);
  s.n_act_spring = (uint32_t)act.size();
  MG_TRY(up(s.act_spring, act));
  active(stitch_idx, 6, s.n_stitch, act);
  s.n_act_stitch = (uint32_t)act.size();
  MG_TRY(up(s.act_stitch, act));

  // ---- contributions in push order (implicit.rs:2394-2740) ----------------------------
  std::vector<Contribution> cb;   // block contributions
  std::vector<uint32_t> gvert;    // gradient entry -> vertex
  s.cb_inertia = cb.size();
  s.gb_inertia = gvert.size();
  for (uint32_t v : free_verts) {
    cb.push_back({v, v});
    gvert.push_back(v);
  }
  s.cb_stitch = cb.size();
  s.gb_stitch = gvert.size();
  for (uint32_t e = 0; e < s.n_stitch; ++e) {
    const uint32_t* ix = stitch_idx.data() + 6 * e;
    for (int a = 0; a < 6; ++a) gvert.push_back(ix[a]);
    for (int a = 0; a < 6; ++a)
      for (int b = 0; b < 6; ++b) cb.push_back({ix[a], ix[b]});
  }
  s.cb_spring = cb.size();
  s.gb_spring = gvert.size();
  for (uint32_t e = 0; e < s.n_spring; ++e) {
    uint32_t a = spring_v[2 * e], b = spring_v[2 * e + 1];
    gvert.push_back(a);
    gvert.push_back(b);
    cb.push_back({a, a});
    cb.push_back({b, b});
    cb.push_back({a, b});
    cb.push_back({b, a});
  }
  s.cb_mem = cb.size();
  s.gb_mem = gvert.size();
  for (uint32_t e = 0; e < s.n_mem; ++e) {
    const uint32_t* mv = mem_v.data() + 3 * e;
    for (int a = 0; a < 3; ++a) gvert.push_back(mv[a]);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) cb.push_back({mv[a], mv[b]});
  }
  s.cb_shell = cb.size();
  s.gb_shell = gvert.size();
  for (uint32_t e = 0; e < s.n_shell; ++e) {
    const uint32_t* sv = shell_v.data() + 3 * e;
    for (int a = 0; a < 3; ++a) gvert.push_back(sv[a]);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) cb.push_back({sv[a], sv[b]});
  }
  // the hinges' blocks and gradient entries start 16-byte aligned (k_hinge stores them as
  // float4): padding entries before them, which no slot and no vertex gathers
  while (cb.size() % 4) cb.push_back({PAD_ENTRY, PAD_ENTRY});
  while (gvert.size() % 4) gvert.push_back(PAD_ENTRY);
  s.cb_hinge = cb.size();
  s.gb_hinge = gvert.size();
  for (uint32_t e = 0; e < s.n_hinge; ++e) {
    const uint32_t* hv = hinge_v.data() + 4 * e;
    for (int a = 0; a < 4; ++a) gvert.push_back(hv[a]);
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) cb.push_back({hv[a], hv[b]});
  }
  s.n_cblocks = cb.size();
  s.n_gentries = gvert.size();

  // ---- patterns -------------------------------------------------------------------------
  auto key = [](uint32_t r, uint32_t c) { return ((uint64_t)r << 32) | c; };
  std::vector<uint64_t> ks, kp;
  ks.reserve(cb.size() + nv);
  for (auto& c : cb) {
    if (c.row == PAD_ENTRY) continue;
    if (vfree(c.row) && vfree(c.col))
      ks.push_back(key(c.row, c.col));
    else
      kp.push_back(key(c.row, c.col));
  }
  for (uint32_t v = 0; v < nv; ++v) ks.push_back(key(v, v));  // every vertex owns a diagonal block
  std::sort(ks.begin(), ks.end());
  ks.erase(std::unique(ks.begin(), ks.end()), ks.end());
  std::sort(kp.begin(), kp.end());
  kp.erase(std::unique(kp.begin(), kp.end()), kp.end());
  auto to_pattern = [&](const std::vector<uint64_t>& k, BlockPattern& pat) {
    pat.nnz = (uint32_t)k.size();
    pat.h_row_ptr.assign(nv + 1, 0);
    pat.h_col.resize(k.size());
    for (size_t i = 0; i < k.size(); ++i) {
      pat.h_row_ptr[(k[i] >> 32) + 1]++;
      pat.h_col[i] = (uint32_t)k[i];
    }
    for (uint32_t v = 0; v < nv; ++v) pat.h_row_ptr[v + 1] += pat.h_row_ptr[v];
  };
  to_pattern(ks, s.Ps);
  to_pattern(kp, s.Pp);
  MG_TRY(s.Ps.row_ptr.upload(s.Ps.h_row_ptr.data(), nv + 1, st));
  MG_TRY(up(s.Ps.col, s.Ps.h_col));
  MG_TRY(s.Pp.row_ptr.upload(s.Pp.h_row_ptr.data(), nv + 1, st));
  MG_TRY(up(s.Pp.col, s.Pp.h_col));
  auto slot_of = [&](uint32_t r, uint32_t c) -> uint32_t {
    bool sys = vfree(r) && vfree(c);
    const BlockPattern& pat = sys ? s.Ps : s.Pp;
    auto b = pat.h_col.begin() + pat.h_row_ptr[r], e = pat.h_col.begin() + pat.h_row_ptr[r + 1];
    auto it = std::lower_bound(b, e, c);
    uint32_t local = (uint32_t)(it - pat.h_col.begin());
    return sys ? local : s.Ps.nnz + local;
  };
  // per-slot contribution lists in push order (counting sort on the slot)
  uint32_t nslots = s.Ps.nnz + s.Pp.nnz;
  std::vector<uint32_t> slot_ptr(nslots + 1, 0), slot_of_c(cb.size());
  for (size_t i = 0; i < cb.size(); ++i) {
    if (cb[i].row == PAD_ENTRY) {
      slot_of_c[i] = PAD_ENTRY;
      continue;
    }
    slot_of_c[i] = slot_of(cb[i].row, cb[i].col);
    slot_ptr[slot_of_c[i] + 1]++;
  }
  for (uint32_t k = 0; k < nslots; ++k) slot_ptr[k + 1] += slot_ptr[k];
  std::vector<uint32_t> cursor(slot_ptr.begin(), slot_ptr.end() - 1),
      slot_list(std::max<uint32_t>(slot_ptr[nslots], 1));
  for (size_t i = 0; i < cb.size(); ++i)
    if (slot_of_c[i] != PAD_ENTRY) slot_list[cursor[slot_of_c[i]]++] = (uint32_t)i;
  MG_TRY(up(s.slot_ptr, slot_ptr));
  MG_TRY(up(s.slot_list, slot_list));
  std::vector<uint32_t> gv_ptr(nv + 1, 0);
  for (uint32_t v : gvert)
    if (v != PAD_ENTRY) gv_ptr[v + 1]++;
  for (uint32_t k = 0; k < nv; ++k) gv_ptr[k + 1] += gv_ptr[k];
  std::vector<uint32_t> gcur(gv_ptr.begin(), gv_ptr.end() - 1), gv_list(std::max<uint32_t>(gv_ptr[nv], 1));
  for (size_t i = 0; i < gvert.size(); ++i)
    if (gvert[i] != PAD_ENTRY) gv_list[gcur[gvert[i]]++] = (uint32_t)i;
  MG_TRY(up(s.gv_ptr, gv_ptr));
  MG_TRY(up(s.gv_list, gv_list));
  std::vector<uint32_t> diag(nv);
  for (uint32_t v = 0; v < nv; ++v) {
    if (vfree(v)) {
      diag[v] = slot_of(v, v);
    } else {
      auto b = s.Pp.h_col.begin() + s.Pp.h_row_ptr[v], e = s.Pp.h_col.begin() + s.Pp.h_row_ptr[v + 1];
      auto it = std::lower_bound(b, e, v);
      diag[v] = (it != e && *it == v) ? s.Ps.nnz + (uint32_t)(it - s.Pp.h_col.begin()) : 0xffffffffu;
    }
  }
  MG_TRY(up(s.diag_slot, diag));
  // each slot's instance (its row's), for gathers that skip the instances a batch no longer
  // iterates
  std::vector<uint8_t> slot_inst(std::max<uint32_t>(nslots, 1), 0);
  for (uint32_t r = 0; r < nv; ++r) {
    for (uint32_t k = s.Ps.h_row_ptr[r]; k < s.Ps.h_row_ptr[r + 1]; ++k) slot_inst[k] = vinst[r];
    for (uint32_t k = s.Pp.h_row_ptr[r]; k < s.Pp.h_row_ptr[r + 1]; ++k) slot_inst[s.Ps.nnz + k] = vinst[r];
  }
  MG_TRY(s.slot_inst.upload(slot_inst.data(), slot_inst.size(), st));
  MG_TRY(s.cblocks.reserve(9 * std::max<uint64_t>(s.n_cblocks, 1)));
  MG_TRY(s.gentries.reserve(3 * std::max<uint64_t>(s.n_gentries, 1)));
  MG_CUDA(cudaMemsetAsync(s.cblocks.p, 0, 36 * std::max<uint64_t>(s.n_cblocks, 1), st));
  MG_CUDA(cudaMemsetAsync(s.gentries.p, 0, 12 * std::max<uint64_t>(s.n_gentries, 1), st));
  MG_TRY(s.valp.reserve(9 * (size_t)std::max<uint32_t>(s.Pp.nnz, 1)));
  MG_TRY(s.grad.reserve(3 * (size_t)nv));
  MG_TRY(s.rhs.reserve(3 * (size_t)nv));
  // the system operator over Ps
  s.A = std::make_unique<mguso_bsr>();
  s.A->ctx = s.ctx;
  std::vector<float> zeros(9 * (size_t)s.Ps.nnz, 0.f);
  MG_TRY(bsr_upload(s.A.get(), nv, s.Ps.h_row_ptr, s.Ps.h_col, zeros.data()));
  s.A->variant = SPMV_DIRECT;

  // ---- colliders -------------------------------------------------------------------------
  s.n_col = d->ncollider;
  s.h_colliders.assign(d->colliders, d->colliders + 8 * (size_t)d->ncollider);
  MG_TRY(up(s.colliders, s.h_colliders));

  // ---- collision topology -------------------------------------------------------------------
  if (nt)
    MG_TRY(s.tris.upload(d->tris, 3 * (size_t)nt, st));
  else
    MG_TRY(s.tris.reserve(3));
  std::vector<uint32_t> ev, etris;
  for (auto& e : edges) {
    ev.insert(ev.end(), {e[0], e[1]});
    etris.insert(etris.end(), {e[0], e[1], e[1]});
  }
  MG_TRY(up(s.edges, ev));
  MG_TRY(up(s.edge_tris, etris));
  {
    std::vector<uint32_t> tail(PCG_MAX_INST, 0);
    for (uint32_t k = 0; k < s.ninst; ++k) {
      uint32_t t = s.inst_edge[k + 1];
      while (t > s.inst_edge[k] && s.h_pinned[edges[t - 1][0]] && s.h_pinned[edges[t - 1][1]]) --t;
      tail[k] = t;
    }
    MG_TRY(up(s.ee_tail, tail));
  }
  // 1-ring exclusion: the vertex and its triangle neighbours, sorted
  std::vector<std::vector<uint32_t>> ex(nv);
  for (uint32_t i = 0; i < nv; ++i) ex[i].push_back(i);
  for (auto& t : tris)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        if (a != b) ex[t[a]].push_back(t[b]);
  std::vector<uint32_t> ex_ptr(nv + 1, 0), ex_list;
  for (uint32_t i = 0; i < nv; ++i) {
    std::sort(ex[i].begin(), ex[i].end());
    ex[i].erase(std::unique(ex[i].begin(), ex[i].end()), ex[i].end());
    ex_list.insert(ex_list.end(), ex[i].begin(), ex[i].end());
    ex_ptr[i + 1] = (uint32_t)ex_list.size();
  }
  MG_TRY(up(s.ex_ptr, ex_ptr));
  MG_TRY(up(s.ex_list, ex_list));
  // static mesh collider: winding check + pseudonormals (implicit.rs:1258-1320)
  std::vector<uint8_t> svert(nv, 0), ctri(std::max<uint32_t>(nt, 1), 0);
  std::vector<float> pn(3 * (size_t)nv, 0.f);
  s.has_static = false;
  if (d->static_mask) {
    HV lo(INFINITY, INFINITY, INFINITY), hi(-INFINITY, -INFINITY, -INFINITY);
    std::vector<uint32_t> marked;
    for (uint32_t t = 0; t < nt; ++t) {
      auto& tv = tris[t];
      if (!(d->static_mask[tv[0]] && d->static_mask[tv[1]] && d->static_mask[tv[2]])) continue;
      for (uint32_t i : tv) {
        HV q = hp(P, i);
        lo = HV(std::min(lo.x, q.x), std::min(lo.y, q.y), std::min(lo.z, q.z));
        hi = HV(std::max(hi.x, q.x), std::max(hi.y, q.y), std::max(hi.z, q.z));
      }
      marked.push_back(t);
    }
    if (!marked.empty()) {
      HV e = hi - lo;
      double box_vol = (double)(e.x * e.y * e.z);
      HV mid = (lo + hi) * 0.5f;
      double vol = 0.0;
      for (uint32_t t : marked) {
        HV a = hp(P, tris[t][0]) - mid, b = hp(P, tris[t][1]) - mid, c = hp(P, tris[t][2]) - mid;
        vol += (double)a.cross(b).dot(c) / 6.0;
      }
      if (!(vol < -0.05 * box_vol)) {
        s.has_static = true;
        for (uint32_t i = 0; i < nv; ++i) svert[i] = d->static_mask[i] ? 1 : 0;
        for (uint32_t t : marked) ctri[t] = 1;
        std::vector<std::array<uint32_t, 3>> ctris;
        for (uint32_t t : marked) ctris.push_back(tris[t]);
        collider_pseudonormals(P, nv, ctris, vinst, pn);
        s.h_static = svert;
        s.h_ctris = ctris;
        s.h_vinst = vinst;
      }
    }
  }
  MG_TRY(up(s.static_vert, svert));
  MG_TRY(up(s.collider_tri, ctri));
  MG_TRY(up(s.collider_pn, pn));
  s.sorter.ctx = s.ctx;
  for (uint32_t k = 0; k < s.ninst; ++k) {
    s.tri_bvh.push_back(std::make_unique<Lbvh>());
    s.edge_bvh.push_back(std::make_unique<Lbvh>());
    s.tri_bvh.back()->ctx = s.ctx;
    s.edge_bvh.back()->ctx = s.ctx;
  }

  // ---- working set -------------------------------------------------------------------------
  s.cap_pairs = std::max<uint32_t>(1u << 16, 8 * nv);
  s.cap_stencils = std::max<uint32_t>(1u << 14, 2 * nv);
  MG_TRY(s.pairs.reserve(2 * (size_t)s.cap_pairs));
  MG_TRY(s.counters.reserve(8));
  MG_TRY(s.side_best.reserve(nv));
  MG_TRY(s.red.reserve(RED_STRIDE * s.ninst));
  MG_TRY(s.status.reserve(4));
  MG_CUDA(cudaMemsetAsync(s.status.p, 0, 16, st));
  // the sorts and BVH builds of the step report a look-back timeout in the step's status
  s.sorter.err_sink = s.status.p;
  for (uint32_t k = 0; k < s.ninst; ++k) s.tri_bvh[k]->err_sink = s.edge_bvh[k]->err_sink = s.status.p;
  s.cap_c = std::max<uint32_t>(1u << 14, 4 * nv);
  MG_TRY(s.c_row_ptr.reserve(nv + 1));
  MG_TRY(s.c_count.reserve(4));
  MG_CUDA(cudaMemsetAsync(s.c_row_ptr.p, 0, 4 * ((size_t)nv + 1), st));

  // ---- linear solver ---------------------------------------------------------------------
  if (s.p.precond == MGUSO_PRECOND_SCHWARZ) {
    MG_CHECK_ARG(s.p.schwarz_domain >= 1 && s.p.schwarz_domain <= 32, "Schwarz domain size must be in [1, 32]");
    s.schwarz = std::make_unique<mguso_schwarz>();
    s.schwarz->a = s.A.get();
    s.schwarz->domain = s.p.schwarz_domain;
    s.schwarz->half = s.fp16_factor;  // FP16 factor tiles: the apply moves half the bytes
    s.schwarz->inst_vert = s.inst_vert;
    if (s.p.schwarz_levels == 2) {
      // two-level Schwarz: single scenes, stepped with the per-kernel PCG
      MG_CHECK_ARG(s.ninst == 1, "scene: two-level Schwarz is for single scenes, not batches");
      s.schwarz->levels = 2;
      s.schwarz->weight = s.p.schwarz_weight > 0.f ? s.p.schwarz_weight : 0.7f;
    }
    MG_TRY(schwarz_build(s.schwarz.get()));
  } else {
    MG_TRY(s.bjinv.reserve(9 * (size_t)nv));
  }
  MG_TRY(s.work.reserve(3 * nv));
  MG_CUDA(cudaStreamSynchronize(st));
  return MGUSO_OK;
}

// Pins and pulls grouped by vertex, each vertex's in their order of setting (the order the
// reference pushes them), onto the device.
int upload_pins(Scene& s) {
  std::vector<uint32_t> verts;
  for (auto& p : s.h_pins) verts.push_back(p.index);
  for (auto& p : s.h_pulls) verts.push_back(p.index);
  std::sort(verts.begin(), verts.end());
  verts.erase(std::unique(verts.begin(), verts.end()), verts.end());
  const uint32_t nvp = (uint32_t)verts.size();
  std::vector<uint32_t> pin_ptr(nvp + 1, 0), pull_ptr(nvp + 1, 0);
  auto slot = [&](uint32_t v) { return (uint32_t)(std::lower_bound(verts.begin(), verts.end(), v) - verts.begin()); };
  for (auto& p : s.h_pins) pin_ptr[slot(p.index) + 1]++;
  for (auto& p : s.h_pulls) pull_ptr[slot(p.index) + 1]++;
  for (uint32_t i = 0; i < nvp; ++i) {
    pin_ptr[i + 1] += pin_ptr[i];
    pull_ptr[i + 1] += pull_ptr[i];
  }
  std::vector<uint32_t> pc(pin_ptr.begin(), pin_ptr.end() - 1), qc(pull_ptr.begin(), pull_ptr.end() - 1);
  const size_t np = s.h_pins.size(), nq = s.h_pulls.size();
  std::vector<float> pt(3 * np + 1), pg(np + 1), pst(np + 1), qt(3 * nq + 1), qw(nq + 1);
  std::vector<uint8_t> pk(np + 1);
  std::vector<uint32_t> pvert(np + 1);
  s.n_static_pin = 0;
  for (auto& p : s.h_pins) {
    const uint32_t j = pc[slot(p.index)]++;
    for (int c = 0; c < 3; ++c) pt[3 * j + c] = p.target[c];
    pg[j] = p.ghat;
    pst[j] = p.stiffness;
    pk[j] = p.kinematic;
    pvert[j] = p.index;
    if (!p.kinematic) s.n_static_pin++;
  }
  for (auto& p : s.h_pulls) {
    const uint32_t j = qc[slot(p.index)]++;
    for (int c = 0; c < 3; ++c) qt[3 * j + c] = p.target[c];
    qw[j] = p.weight;
  }
  verts.push_back(0);
  cudaStream_t st = s.st;
  MG_TRY(s.pv.upload(verts.data(), verts.size(), st));
  MG_TRY(s.pv_pin.upload(pin_ptr.data(), pin_ptr.size(), st));
  MG_TRY(s.pv_pull.upload(pull_ptr.data(), pull_ptr.size(), st));
  MG_TRY(s.pin_vert.upload(pvert.data(), pvert.size(), st));
  MG_TRY(s.pin_target.upload(pt.data(), pt.size(), st));
  MG_TRY(s.pin_ghat.upload(pg.data(), pg.size(), st));
  MG_TRY(s.pin_stiff.upload(pst.data(), pst.size(), st));
  MG_TRY(s.pin_kin.upload(pk.data(), pk.size(), st));
  MG_TRY(s.pull_target.upload(qt.data(), qt.size(), st));
  MG_TRY(s.pull_weight.upload(qw.data(), qw.size(), st));
  MG_CUDA(cudaStreamSynchronize(st));
  s.n_pv = nvp;
  s.n_pin = (uint32_t)np;
  s.n_pull = (uint32_t)nq;
  return MGUSO_OK;
}

// The gather slot of block (r, c): Ps when both vertices are free, else Pp (numbered after
// Ps); -1 when the pattern has no such block.
int slot_of_pair(const Scene& s, uint32_t r, uint32_t c) {
  const bool sys = !s.h_pinned[r] && !s.h_pinned[c];
  const BlockPattern& pat = sys ? s.Ps : s.Pp;
  auto b = pat.h_col.begin() + pat.h_row_ptr[r], e = pat.h_col.begin() + pat.h_row_ptr[r + 1];
  auto it = std::lower_bound(b, e, c);
  if (it == e || *it != c) return -1;
  const uint32_t local = (uint32_t)(it - pat.h_col.begin());
  return (int)(sys ? local : s.Ps.nnz + local);
}

}  // namespace mg

using namespace mg;

extern "C" {

int mguso_scene_validate(const mguso_scene_desc* desc) { return validate_desc(desc); }

int mguso_scene_create(mguso_ctx* ctx, const mguso_scene_desc* desc, mguso_scene** out) {
  MG_CHECK_ARG(ctx && desc && out, "null argument");
  MG_CUDA(cudaSetDevice(ctx->device));
  auto sc = std::make_unique<mguso_scene>();
  sc->s.ctx = ctx;
  MG_TRY(scene_build(sc->s, desc, {0, desc->nv}));
  *out = sc.release();
  return MGUSO_OK;
}

int mguso_scene_destroy(mguso_scene* s) {
  if (s) cudaStreamSynchronize(s->s.st);
  delete s;
  return MGUSO_OK;
}

// Several independent drapes as one scene: the descriptions are concatenated (vertex,
// triangle, shell-face and stitch indices offset), every instance keeps its own Newton
// loop, and the launches of a step are shared. All instances share one mguso_params and one
// set of analytic colliders.
int mguso_batch_create(mguso_ctx* ctx, const mguso_scene_desc* descs, uint32_t n, mguso_scene** out) {
  MG_CHECK_ARG(ctx && descs && out && n >= 1, "null argument");
  MG_CHECK_ARG(n <= PCG_MAX_INST, "batch: at most 8 instances");
  const mguso_scene_desc& d0 = descs[0];
  uint64_t nv = 0, nt = 0, nsh = 0, nst = 0;
  bool any_mask = false;
  for (uint32_t k = 0; k < n; ++k) {
    const mguso_scene_desc& d = descs[k];
    MG_CHECK_ARG(d.positions && d.inv_mass && d.nv > 0 && (d.nt == 0 || d.tris), "batch: null arrays");
    MG_CHECK_ARG(std::memcmp(&d.params, &d0.params, sizeof(mguso_params)) == 0, "batch: instances must share params");
    MG_CHECK_ARG(d.ncollider == d0.ncollider &&
                     (d.ncollider == 0 || std::memcmp(d.colliders, d0.colliders, 32 * (size_t)d.ncollider) == 0),
                 "batch: instances must share their analytic colliders");
    nv += d.nv;
    nt += d.nt;
    nsh += d.nshell;
    nst += d.nstitch;
    any_mask = any_mask || d.static_mask;
    MG_CHECK_ARG(!d.shell_rest && !d.shell_stiff, "batch: per-shell overrides are not supported");
  }
  MG_CHECK_ARG(nv < (1u << 30), "batch: too many vertices");
  std::vector<float> pos, vel, im, skl, sw, uvs;
  std::vector<uint32_t> tri, shf, sidx, sedge, inst{0};
  std::vector<uint8_t> mask;
  bool any_uv = false, any_stretch = false;
  for (uint32_t k = 0; k < n; ++k) {
    any_uv = any_uv || descs[k].uvs;
    any_stretch = any_stretch || descs[k].nstretch;
  }
  MG_CHECK_ARG(!any_stretch || std::all_of(descs, descs + n, [](const mguso_scene_desc& d) { return d.nstretch > 0; }),
               "batch: give stretch edges for every instance or for none");
  pos.reserve(3 * nv);
  for (uint32_t k = 0; k < n; ++k) {
    const mguso_scene_desc& d = descs[k];
    const uint32_t o = (uint32_t)(pos.size() / 3);
    pos.insert(pos.end(), d.positions, d.positions + 3 * (size_t)d.nv);
    if (d.velocities)
      vel.insert(vel.end(), d.velocities, d.velocities + 3 * (size_t)d.nv);
    else
      vel.insert(vel.end(), 3 * (size_t)d.nv, 0.f);
    im.insert(im.end(), d.inv_mass, d.inv_mass + d.nv);
    if (any_mask) {
      if (d.static_mask)
        mask.insert(mask.end(), d.static_mask, d.static_mask + d.nv);
      else
        mask.insert(mask.end(), d.nv, 0);
    }
    for (uint64_t i = 0; i < 3ull * d.nt; ++i) {
      MG_CHECK_ARG(d.tris[i] < d.nv, "batch: triangle index out of range");
      tri.push_back(d.tris[i] + o);
    }
    for (uint64_t i = 0; i < 3ull * d.nshell; ++i) {
      MG_CHECK_ARG(d.shell_faces[i] < d.nv, "batch: shell face index out of range");
      shf.push_back(d.shell_faces[i] + o);
    }
    for (uint64_t i = 0; i < 6ull * d.nstitch; ++i) {
      MG_CHECK_ARG(d.stitch_idx[i] < d.nv, "batch: stitch index out of range");
      sidx.push_back(d.stitch_idx[i] + o);
    }
    if (d.nstitch) {
      sw.insert(sw.end(), d.stitch_w, d.stitch_w + 6 * (size_t)d.nstitch);
      skl.insert(skl.end(), d.stitch_kl, d.stitch_kl + 3 * (size_t)d.nstitch);
    }
    // an instance without uvs reads zeros, which give every edge the warp ratio, as no uvs do
    if (any_uv) {
      if (d.uvs)
        uvs.insert(uvs.end(), d.uvs, d.uvs + 2 * (size_t)d.nv);
      else
        uvs.insert(uvs.end(), 2 * (size_t)d.nv, 0.f);
    }
    MG_CHECK_ARG(d.nstretch == 0 || d.stretch_edges, "batch: null arrays");
    for (uint64_t i = 0; i < 2ull * d.nstretch; ++i) {
      MG_CHECK_ARG(d.stretch_edges[i] < d.nv, "batch: stretch edge index out of range");
      sedge.push_back(d.stretch_edges[i] + o);
    }
    inst.push_back(o + d.nv);
  }
  mguso_scene_desc u = d0;
  u.nv = (uint32_t)nv;
  u.positions = pos.data();
  u.velocities = vel.data();
  u.inv_mass = im.data();
  u.nt = (uint32_t)nt;
  u.tris = tri.empty() ? nullptr : tri.data();
  u.static_mask = any_mask ? mask.data() : nullptr;
  u.nshell = (uint32_t)nsh;
  u.shell_faces = shf.empty() ? nullptr : shf.data();
  u.nstitch = (uint32_t)nst;
  u.stitch_idx = sidx.empty() ? nullptr : sidx.data();
  u.stitch_w = sw.empty() ? nullptr : sw.data();
  u.stitch_kl = skl.empty() ? nullptr : skl.data();
  u.uvs = any_uv ? uvs.data() : nullptr;
  u.nstretch = (uint32_t)(sedge.size() / 2);
  u.stretch_edges = sedge.empty() ? nullptr : sedge.data();
  MG_CUDA(cudaSetDevice(ctx->device));
  auto sc = std::make_unique<mguso_scene>();
  sc->s.ctx = ctx;
  MG_TRY(scene_build(sc->s, &u, inst));
  *out = sc.release();
  return MGUSO_OK;
}

int mguso_scene_instances(mguso_scene* sc, uint32_t* n, uint32_t* vert_offsets) {
  MG_CHECK_ARG(sc && n, "bad argument");
  *n = sc->s.ninst;
  if (vert_offsets) std::memcpy(vert_offsets, sc->s.inst_vert.data(), 4 * sc->s.inst_vert.size());
  return MGUSO_OK;
}

int mguso_step(mguso_scene* sc, int nsteps, mguso_step_stats* stats) {
  MG_CHECK_ARG(sc && nsteps >= 0, "bad argument");
  MG_CUDA(cudaSetDevice(sc->s.ctx->device));
  const uint32_t K = sc->s.ninst;
  for (int k = 0; k < nsteps; ++k) {
    mguso_step_stats st[PCG_MAX_INST];
    MG_TRY(scene_step(sc->s, st));
    if (stats)
      for (uint32_t i = 0; i < K; ++i) stats[(size_t)k * K + i] = st[i];
  }
  return MGUSO_OK;
}

static int copy_state(mguso_scene* sc, DevBuf<float>& buf, float* out, const float* in) {
  MG_CHECK_ARG(sc && (out || in), "null argument");
  size_t bytes = 12 * (size_t)sc->s.nv;
  if (out) MG_CUDA(cudaMemcpyAsync(out, buf.p, bytes, cudaMemcpyDeviceToHost, sc->s.st));
  if (in) MG_CUDA(cudaMemcpyAsync(buf.p, in, bytes, cudaMemcpyHostToDevice, sc->s.st));
  MG_CUDA(cudaStreamSynchronize(sc->s.st));
  return MGUSO_OK;
}

// set_kinematic_collider_positions (implicit.rs:1368-1398).
int mguso_set_kinematic_collider_positions(mguso_scene* sc, const float* x) {
  MG_CHECK_ARG(sc && x, "null argument");
  Scene& s = sc->s;
  MG_CHECK_ARG(s.has_static && !s.h_static.empty(), "kinematic collider: the scene has no static collider");
  const uint32_t nv = s.nv;
  for (uint32_t i = 0; i < nv; ++i)
    if (s.h_static[i])
      MG_CHECK_ARG(std::isfinite(x[3 * i]) && std::isfinite(x[3 * i + 1]) && std::isfinite(x[3 * i + 2]),
                   "kinematic collider: a collider position is not finite");
  MG_CUDA(cudaSetDevice(s.ctx->device));
  std::vector<float> pos(3 * (size_t)nv), vel(3 * (size_t)nv);
  MG_CUDA(cudaMemcpyAsync(pos.data(), s.x.p, 12 * (size_t)nv, cudaMemcpyDeviceToHost, s.st));
  MG_CUDA(cudaMemcpyAsync(vel.data(), s.v.p, 12 * (size_t)nv, cudaMemcpyDeviceToHost, s.st));
  MG_CUDA(cudaStreamSynchronize(s.st));
  const float inv_h = 1.0f / s.p.dt;
  if (!s.kin_dx_set) s.h_kin_dx.assign(3 * (size_t)nv, 0.f);
  for (uint32_t i = 0; i < nv; ++i) {
    if (!s.h_static[i]) continue;
    for (int c = 0; c < 3; ++c) {
      const float dd = x[3 * i + c] - pos[3 * i + c];
      pos[3 * i + c] = x[3 * i + c];
      vel[3 * i + c] = dd * inv_h;
      s.h_kin_dx[3 * i + c] += dd;  // accumulated until the next step consumes it
    }
  }
  MG_TRY(s.kin_dx.upload(s.h_kin_dx.data(), s.h_kin_dx.size(), s.st));
  s.kin_dx_set = true;
  std::vector<float> pn;
  collider_pseudonormals(pos.data(), nv, s.h_ctris, s.h_vinst, pn);
  MG_CUDA(cudaMemcpyAsync(s.x.p, pos.data(), 12 * (size_t)nv, cudaMemcpyHostToDevice, s.st));
  MG_CUDA(cudaMemcpyAsync(s.v.p, vel.data(), 12 * (size_t)nv, cudaMemcpyHostToDevice, s.st));
  MG_CUDA(cudaMemcpyAsync(s.collider_pn.p, pn.data(), 4 * pn.size(), cudaMemcpyHostToDevice, s.st));
  MG_CUDA(cudaStreamSynchronize(s.st));
  s.static_done = false;  // contributions of all-pinned elements move with the collider
  return MGUSO_OK;
}

// set_pins / set_pulls (implicit.rs:826-864): all or nothing.
int mguso_set_pins(mguso_scene* sc, uint32_t n, const uint32_t* index, const float* target, const float* ghat,
                   const uint8_t* kinematic, const float* stiffness) {
  MG_CHECK_ARG(sc && (n == 0 || (index && target && ghat)), "null argument");
  Scene& s = sc->s;
  std::vector<Scene::HostPin> pins(n);
  for (uint32_t i = 0; i < n; ++i) {
    MG_CHECK_ARG(index[i] < s.nv, "set_pins: a pin's vertex is out of range");
    MG_CHECK_ARG(std::isfinite(ghat[i]) && ghat[i] > 0.f, "set_pins: a pin's ghat must be positive");
    MG_CHECK_ARG(std::isfinite(target[3 * i]) && std::isfinite(target[3 * i + 1]) && std::isfinite(target[3 * i + 2]),
                 "set_pins: a pin's target is not finite");
    pins[i].index = index[i];
    for (int c = 0; c < 3; ++c) pins[i].target[c] = target[3 * i + c];
    pins[i].ghat = ghat[i];
    pins[i].kinematic = kinematic ? (kinematic[i] ? 1 : 0) : 0;
    pins[i].stiffness = stiffness ? stiffness[i] : 1.f;
  }
  MG_CUDA(cudaSetDevice(s.ctx->device));
  s.h_pins = std::move(pins);
  return upload_pins(s);
}

int mguso_set_pulls(mguso_scene* sc, uint32_t n, const uint32_t* index, const float* target, const float* weight) {
  MG_CHECK_ARG(sc && (n == 0 || (index && target && weight)), "null argument");
  Scene& s = sc->s;
  std::vector<Scene::HostPull> pulls(n);
  for (uint32_t i = 0; i < n; ++i) {
    MG_CHECK_ARG(index[i] < s.nv, "set_pulls: a pull's vertex is out of range");
    MG_CHECK_ARG(std::isfinite(weight[i]) && weight[i] > 0.f, "set_pulls: a pull's weight must be positive");
    MG_CHECK_ARG(std::isfinite(target[3 * i]) && std::isfinite(target[3 * i + 1]) && std::isfinite(target[3 * i + 2]),
                 "set_pulls: a pull's target is not finite");
    pulls[i].index = index[i];
    for (int c = 0; c < 3; ++c) pulls[i].target[c] = target[3 * i + c];
    pulls[i].weight = weight[i];
  }
  MG_CUDA(cudaSetDevice(s.ctx->device));
  s.h_pulls = std::move(pulls);
  return upload_pins(s);
}

// set_strain_limit_faces (implicit.rs:1088-1121): all or nothing.
int mguso_set_strain_limit_faces(mguso_scene* sc, uint32_t n, const uint32_t* faces, const float* limits,
                                 const float* masses, uint32_t* kept) {
  MG_CHECK_ARG(sc && (n == 0 || (faces && limits && masses)), "null argument");
  Scene& s = sc->s;
  std::vector<uint8_t> vinst(s.nv);
  for (uint32_t k = 0; k < s.ninst; ++k)
    for (uint32_t v = s.inst_vert[k]; v < s.inst_vert[k + 1]; ++v) vinst[v] = (uint8_t)k;
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t* f = faces + 3 * i;
    MG_CHECK_ARG(f[0] < s.nv && f[1] < s.nv && f[2] < s.nv, "set_strain_limit_faces: a face index is out of range");
    MG_CHECK_ARG(vinst[f[0]] == vinst[f[1]] && vinst[f[0]] == vinst[f[2]],
                 "set_strain_limit_faces: a face spans two instances");
    MG_CHECK_ARG(std::isfinite(limits[i]) && std::isfinite(masses[i]),
                 "set_strain_limit_faces: a limit or mass is not finite");
  }
  MG_CUDA(cudaSetDevice(s.ctx->device));
  std::vector<float> pos(3 * (size_t)s.nv);
  MG_CUDA(cudaMemcpyAsync(pos.data(), s.x.p, 12 * (size_t)s.nv, cudaMemcpyDeviceToHost, s.st));
  MG_CUDA(cudaStreamSynchronize(s.st));
  std::vector<uint32_t> fv, fslot;
  std::vector<float> fdm, flim, fmass;
  for (uint32_t i = 0; i < n; ++i) {
    if (limits[i] <= 0.f || masses[i] <= 0.f) continue;
    const uint32_t* f = faces + 3 * i;
    float dm[4], area;
    if (!shell_rest_shape(hp(pos.data(), f[0]), hp(pos.data(), f[1]), hp(pos.data(), f[2]), dm, area)) continue;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        const int sl = slot_of_pair(s, f[a], f[b]);
        if (sl < 0 && (!s.h_pinned[f[a]] || !s.h_pinned[f[b]])) {
          set_error("set_strain_limit_faces: a face's vertex pair shares no element, so its block lies "
                    "outside the scene's Hessian pattern");
          return MGUSO_ERR_UNSUPPORTED;
        }
        fslot.push_back(sl < 0 ? ~0u : (uint32_t)sl);
      }
    fv.insert(fv.end(), {f[0], f[1], f[2]});
    fdm.insert(fdm.end(), {dm[0], dm[1], dm[2], dm[3]});
    flim.push_back(limits[i]);
    fmass.push_back(masses[i]);
  }
  const uint32_t m = (uint32_t)flim.size();
  // contributions per touched slot and per touched vertex, in face order
  std::vector<uint32_t> slots, verts;
  for (uint32_t x : fslot)
    if (x != ~0u) slots.push_back(x);
  std::sort(slots.begin(), slots.end());
  slots.erase(std::unique(slots.begin(), slots.end()), slots.end());
  verts = fv;
  std::sort(verts.begin(), verts.end());
  verts.erase(std::unique(verts.begin(), verts.end()), verts.end());
  std::vector<uint32_t> sptr(slots.size() + 1, 0), vptr(verts.size() + 1, 0);
  auto rank = [](const std::vector<uint32_t>& v, uint32_t x) {
    return (uint32_t)(std::lower_bound(v.begin(), v.end(), x) - v.begin());
  };
  for (uint32_t x : fslot)
    if (x != ~0u) sptr[rank(slots, x) + 1]++;
  for (uint32_t x : fv) vptr[rank(verts, x) + 1]++;
  for (size_t k = 0; k < slots.size(); ++k) sptr[k + 1] += sptr[k];
  for (size_t k = 0; k < verts.size(); ++k) vptr[k + 1] += vptr[k];
  std::vector<uint32_t> slist(sptr.back()), vlist(vptr.back());
  {
    std::vector<uint32_t> sc2(sptr.begin(), sptr.end() - 1), vc(vptr.begin(), vptr.end() - 1);
    for (uint32_t e = 0; e < 9 * m; ++e)
      if (fslot[e] != ~0u) slist[sc2[rank(slots, fslot[e])]++] = e;
    for (uint32_t e = 0; e < 3 * m; ++e) vlist[vc[rank(verts, fv[e])]++] = e;
  }
  cudaStream_t st = s.st;
  auto up = [&](auto& buf, const auto& vec) -> int {
    if (vec.empty()) return buf.reserve(1);
    return buf.upload(vec.data(), vec.size(), st);
  };
  MG_TRY(up(s.sl_v, fv));
  MG_TRY(up(s.sl_slot, fslot));
  MG_TRY(up(s.sl_dm, fdm));
  MG_TRY(up(s.sl_limit, flim));
  MG_TRY(up(s.sl_mass, fmass));
  MG_TRY(up(s.sl_slots, slots));
  MG_TRY(up(s.sl_sptr, sptr));
  MG_TRY(up(s.sl_slist, slist));
  MG_TRY(up(s.sl_verts, verts));
  MG_TRY(up(s.sl_vptr, vptr));
  MG_TRY(up(s.sl_vlist, vlist));
  MG_TRY(s.sl_c.reserve(90 * (size_t)std::max<uint32_t>(m, 1)));
  MG_CUDA(cudaStreamSynchronize(st));
  s.n_sl = m;
  s.n_sl_slots = (uint32_t)slots.size();
  s.n_sl_verts = (uint32_t)verts.size();
  if (kept) *kept = m;
  return MGUSO_OK;
}

int mguso_read_positions(mguso_scene* s, float* out) { return copy_state(s, s->s.x, out, nullptr); }
int mguso_write_positions(mguso_scene* s, const float* in) { return copy_state(s, s->s.x, nullptr, in); }
int mguso_read_velocities(mguso_scene* s, float* out) { return copy_state(s, s->s.v, out, nullptr); }
int mguso_write_velocities(mguso_scene* s, const float* in) { return copy_state(s, s->s.v, nullptr, in); }

int mguso_scene_info(mguso_scene* sc, uint32_t* out6) {
  MG_CHECK_ARG(sc && out6, "null argument");
  Scene& s = sc->s;
  uint32_t nct = 0;
  std::vector<uint8_t> ct(std::max<uint32_t>(s.nt, 1));
  MG_CUDA(cudaMemcpy(ct.data(), s.collider_tri.p, ct.size(), cudaMemcpyDeviceToHost));
  for (uint32_t t = 0; t < s.nt; ++t) nct += ct[t];
  out6[0] = s.n_hinge;
  out6[1] = s.n_shell;
  out6[2] = s.n_edge;
  out6[3] = nct;
  out6[4] = s.Ps.nnz;
  out6[5] = s.Pp.nnz;
  return MGUSO_OK;
}

}  // extern "C"

extern "C" int mguso_scene_spmv_time(mguso_scene* sc, int reps, float* us, double* bytes) {
  MG_CHECK_ARG(sc && us && bytes && reps > 0, "bad argument");
  Scene& s = sc->s;
  cudaStream_t st = s.st;
  DevBuf<float> x, y;
  MG_TRY(x.reserve(3 * (size_t)s.nv));
  MG_TRY(y.reserve(3 * (size_t)s.nv));
  MG_CUDA(cudaMemsetAsync(x.p, 0, 12 * (size_t)s.nv, st));
  for (int i = 0; i < 3; ++i) MG_TRY(system_spmv(s, x.p, y.p, st, nullptr));
  cudaEvent_t e0, e1;
  MG_CUDA(cudaEventCreate(&e0));
  MG_CUDA(cudaEventCreate(&e1));
  cudaEventRecord(e0, st);
  for (int i = 0; i < reps; ++i) MG_TRY(system_spmv(s, x.p, y.p, st, nullptr));
  cudaEventRecord(e1, st);
  MG_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  uint32_t nc = 0;
  MG_CUDA(cudaMemcpy(&nc, s.c_count.p, 4, cudaMemcpyDeviceToHost));
  *us = 1000.f * ms / reps;
  double nnz = (double)s.Ps.nnz + nc;
  *bytes = 40.0 * nnz + 4.0 * 2 * (s.nv + 1) + 24.0 * s.nv;
  return MGUSO_OK;
}

// One Newton-system assembly at positions x (and inertia target x_tilde, x when null), as
// one Newton iteration of mguso_step does it; the scene's positions are left at x.
extern "C" int mguso_scene_ccd(mguso_scene* sc, const float* x, const float* dx, float* t_out, uint32_t* cap_hits) {
  MG_CHECK_ARG(sc && x && dx && t_out, "bad argument");
  Scene& s = sc->s;
  cudaStream_t st = s.st;
  const size_t bytes = 12 * (size_t)s.nv;
  MG_CUDA(cudaMemcpyAsync(s.x.p, x, bytes, cudaMemcpyHostToDevice, st));
  MG_CUDA(cudaMemcpyAsync(s.dx.p, dx, bytes, cudaMemcpyHostToDevice, st));
  if (s.p.self_collision) {
    uint32_t nst = 0;
    MG_TRY(build_bvhs(s, s.x.p));
    MG_TRY(collect_stencils(s, &nst));  // also decides each vertex's side of a static collider
  }
  std::vector<float> t(s.ninst, 1.f);
  std::vector<uint32_t> caps(s.ninst, 0u);
  MG_TRY(ccd_step(s, (s.ninst >= 32 ? ~0u : ((1u << s.ninst) - 1u))));
  MG_TRY(ccd_results(s, t.data(), caps.data()));
  MG_CUDA(cudaStreamSynchronize(st));
  for (uint32_t k = 0; k < s.ninst; ++k) {
    t_out[k] = t[k];
    if (cap_hits) cap_hits[k] = caps[k];
  }
  return MGUSO_OK;
}

extern "C" int mguso_scene_assemble(mguso_scene* sc, const float* x, const float* x_tilde, uint32_t* out3) {
  MG_CHECK_ARG(sc && x && out3, "bad argument");
  Scene& s = sc->s;
  cudaStream_t st = s.st;
  const size_t bytes = 12 * (size_t)s.nv;
  MG_CUDA(cudaMemcpyAsync(s.x.p, x, bytes, cudaMemcpyHostToDevice, st));
  MG_CUDA(cudaMemcpyAsync(s.xt.p, x_tilde ? x_tilde : x, bytes, cudaMemcpyHostToDevice, st));
  uint32_t nst = 0;
  if (s.p.self_collision) {
    MG_TRY(build_bvhs(s, s.x.p));
    MG_TRY(collect_stencils(s, &nst));
  }
  MG_TRY(assemble_elastic(s));
  MG_TRY(assemble_colliders(s));
  MG_TRY(assemble_contacts(s, nst));
  MG_TRY(finish_rhs(s));
  uint32_t nc = 0;
  MG_CUDA(cudaMemcpyAsync(&nc, s.c_count.p, 4, cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaStreamSynchronize(st));
  out3[0] = s.Ps.nnz;
  out3[1] = nc;
  out3[2] = nst;
  s.last_nst = nst;
  return MGUSO_OK;
}

// The adjoint's exact Hessian at x (inertia target x_tilde, x when null), as the backward
// pass of mguso_adjoint_backward assembles it: the step's projected system first, for the
// contact stiffnesses it records, then the exact one (no eigenvalue clamps, second-derivative
// terms of hinges and barriers, the contact stiffnesses' gap dependence) into the same Ps + C
// that mguso_scene_system downloads; the right-hand side is the negative gradient.
extern "C" int mguso_scene_assemble_exact(mguso_scene* sc, const float* x, const float* x_tilde, uint32_t* out3) {
  MG_CHECK_ARG(sc && x && out3, "bad argument");
  Scene& s = sc->s;
  cudaStream_t st = s.st;
  const size_t bytes = 12 * (size_t)s.nv;
  MG_CUDA(cudaMemcpyAsync(s.x.p, x, bytes, cudaMemcpyHostToDevice, st));
  MG_CUDA(cudaMemcpyAsync(s.xt.p, x_tilde ? x_tilde : x, bytes, cudaMemcpyHostToDevice, st));
  uint32_t nst = 0;
  if (s.p.self_collision) {
    MG_TRY(build_bvhs(s, s.x.p));
    MG_TRY(collect_stencils(s, &nst));
  }
  s.hess_mode = 0;
  MG_TRY(assemble_elastic(s));
  MG_TRY(assemble_colliders(s));
  MG_TRY(contact_stiffness(s, nst));
  s.hess_mode = 2;
  int rc = assemble_elastic(s);
  if (rc == MGUSO_OK) rc = assemble_colliders(s);
  if (rc == MGUSO_OK) rc = assemble_contacts(s, nst);
  s.hess_mode = 0;
  MG_TRY(rc);
  MG_TRY(finish_rhs(s));
  uint32_t nc = 0;
  MG_CUDA(cudaMemcpyAsync(&nc, s.c_count.p, 4, cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaStreamSynchronize(st));
  out3[0] = s.Ps.nnz;
  out3[1] = nc;
  out3[2] = nst;
  s.last_nst = nst;
  return MGUSO_OK;
}

// The contact stencils of the last mguso_scene_assemble, in assembly order: participants
// u32[4 n], kind u32[n] (0 vertex-triangle, 1 edge-edge), gap f64[n]. Writes min(n, cap).
extern "C" int mguso_scene_stencils(mguso_scene* sc, uint32_t cap, uint32_t* idx4, uint32_t* kind, double* d,
                                    uint32_t* n_out) {
  MG_CHECK_ARG(sc && n_out && (cap == 0 || (idx4 && kind && d)), "bad argument");
  Scene& s = sc->s;
  const uint32_t n = std::min(cap, s.last_nst);
  *n_out = s.last_nst;
  if (n == 0) return MGUSO_OK;
  std::vector<Stencil> h(n);
  MG_CUDA(cudaMemcpyAsync(h.data(), s.stencils_sorted.p, sizeof(Stencil) * n, cudaMemcpyDeviceToHost, s.st));
  MG_CUDA(cudaStreamSynchronize(s.st));
  for (uint32_t i = 0; i < n; ++i) {
    for (int k = 0; k < 4; ++k) idx4[4 * i + k] = h[i].idx[k];
    kind[i] = h[i].kind;
    d[i] = h[i].d;
  }
  return MGUSO_OK;
}

// The last assembled system: fixed pattern Ps (row_ptr nv+1, col, 9 floats per block),
// contact-only blocks C (same layout), right-hand side f32[3 nv].
extern "C" int mguso_scene_system(mguso_scene* sc, uint32_t* ps_rp, uint32_t* ps_col, float* ps_val, uint32_t* c_rp,
                                  uint32_t* c_col, float* c_val, float* rhs) {
  MG_CHECK_ARG(sc && ps_rp && ps_col && ps_val && c_rp && rhs, "bad argument");
  Scene& s = sc->s;
  cudaStream_t st = s.st;
  uint32_t nc = 0;
  MG_CUDA(cudaMemcpyAsync(&nc, s.c_count.p, 4, cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaStreamSynchronize(st));
  MG_CHECK_ARG(nc == 0 || (c_col && c_val), "bad argument");
  const size_t nv1 = (size_t)s.nv + 1;
  MG_CUDA(cudaMemcpyAsync(ps_rp, s.Ps.row_ptr.p, 4 * nv1, cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaMemcpyAsync(ps_col, s.Ps.col.p, 4 * (size_t)s.Ps.nnz, cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaMemcpyAsync(ps_val, s.A->val.p, 36 * (size_t)s.Ps.nnz, cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaMemcpyAsync(c_rp, s.c_row_ptr.p, 4 * nv1, cudaMemcpyDeviceToHost, st));
  if (nc) {
    MG_CUDA(cudaMemcpyAsync(c_col, s.c_col.p, 4 * (size_t)nc, cudaMemcpyDeviceToHost, st));
    MG_CUDA(cudaMemcpyAsync(c_val, s.c_val.p, 36 * (size_t)nc, cudaMemcpyDeviceToHost, st));
  }
  MG_CUDA(cudaMemcpyAsync(rhs, s.work.b.p, 12 * (size_t)s.nv, cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaStreamSynchronize(st));
  return MGUSO_OK;
}

namespace mg {
int schwarz_factor_with(mguso_schwarz* s, const uint32_t* c_rp, const uint32_t* c_col, const float* c_val,
                        cudaStream_t st);
}

// Mean device time of the step's linear-solver kernels at the last assembled system, each
// timed alone over `reps` launches with CUDA events on the scene's stream:
// us4 = {system SpMV, preconditioner apply, preconditioner factorisation, PCG vector update}
// and bytes4 their algorithmic bytes per launch (the minimum each must move: every stored
// block or factor entry once, the vectors once).
extern "C" int mguso_scene_profile(mguso_scene* sc, int reps, float* us4, double* bytes4) {
  MG_CHECK_ARG(sc && us4 && bytes4 && reps > 0, "bad argument");
  Scene& s = sc->s;
  cudaStream_t st = s.st;
  const size_t n3 = 3 * (size_t)s.nv;
  DevBuf<float> x, y;
  MG_TRY(x.reserve(n3));
  MG_TRY(y.reserve(n3));
  MG_CUDA(cudaMemsetAsync(x.p, 0, 4 * n3, st));
  uint32_t nc = 0;
  MG_CUDA(cudaMemcpyAsync(&nc, s.c_count.p, 4, cudaMemcpyDeviceToHost, st));
  MG_CUDA(cudaStreamSynchronize(st));
  cudaEvent_t e0, e1;
  MG_CUDA(cudaEventCreate(&e0));
  MG_CUDA(cudaEventCreate(&e1));
  auto timed = [&](auto&& fn, float* out) -> int {
    for (int i = 0; i < 3; ++i) MG_TRY(fn());
    MG_CUDA(cudaEventRecord(e0, st));
    for (int i = 0; i < reps; ++i) MG_TRY(fn());
    MG_CUDA(cudaEventRecord(e1, st));
    MG_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    MG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    *out = 1000.f * ms / reps;
    return MGUSO_OK;
  };
  int rc = MGUSO_OK;
  const double nnz = (double)s.Ps.nnz + nc;
  bytes4[0] = 40.0 * nnz + 8.0 * (s.nv + 1) + 24.0 * s.nv;
  if (rc == MGUSO_OK) rc = timed([&]() { return system_spmv(s, x.p, y.p, st, nullptr); }, &us4[0]);
  if (s.schwarz) {
    mguso_schwarz* sw = s.schwarz.get();
    double packed = 0, vert = 0;
    for (uint32_t d = 0; d < sw->ndom; ++d) {
      double m = 3.0 * (sw->h_dom_start[d + 1] - sw->h_dom_start[d]);
      if (sw->h_dom_diag[d])
        vert += 24.0 * (sw->h_dom_start[d + 1] - sw->h_dom_start[d]);  // 6 FP32 per vertex
      else
        packed += m * (m + 1) / 2;
    }
    // factor entries at their stored width (2 bytes in FP16 plus a scale per domain)
    const double fe = sw->half ? 2.0 : 4.0, fs = sw->half ? 4.0 * sw->ndom : 0.0;
    bytes4[1] = fe * packed + vert + fs + 4.0 * s.nv + 24.0 * s.nv + 8.0 * (sw->ndom + 1);
    bytes4[2] = 36.0 * nnz + fe * packed + vert + fs;
    if (rc == MGUSO_OK) rc = timed([&]() { return schwarz_apply(sw, x.p, y.p, st, nullptr); }, &us4[1]);
    if (rc == MGUSO_OK)
      rc = timed([&]() { return schwarz_factor_with(sw, s.c_row_ptr.p, s.c_col.p, s.c_val.p, st); }, &us4[2]);
  } else {
    bytes4[1] = 36.0 * s.nv + 24.0 * s.nv;
    bytes4[2] = 36.0 * s.Ps.nnz + 36.0 * s.nv;
    if (rc == MGUSO_OK)
      rc = timed([&]() { return bj_apply(s.bjinv.p, x.p, y.p, s.nv, s.ctx->sm_count, st, nullptr); }, &us4[1]);
    if (rc == MGUSO_OK) rc = timed([&]() { return blockjacobi_factor(s.A.get(), s.bjinv.p, st); }, &us4[2]);
  }
  // the PCG update x += a p, r -= a Ap with its fused r.r: 4 vectors in, 2 out
  bytes4[3] = 24.0 * n3;
  if (rc == MGUSO_OK && cudaMemsetAsync(s.work.sc.p, 0, sizeof(PcgScalars), st) != cudaSuccess) rc = MGUSO_ERR_CUDA;
  if (rc == MGUSO_OK) rc = timed([&]() { return pcg_vector_update(s.work, s.mixed, s.ctx->sm_count, st); }, &us4[3]);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

// Device time of the two fused PCG kernels inside a solve of the last assembled system
// (pcg_fused_profile: `iters` iterations, every launch bracketed by its own events), with
// their algorithmic bytes per launch: rows = every block and column index of Ps and C once,
// both row-pointer arrays, z and the old direction read, the new direction and Ap written;
// domains = the factor's packed lower triangle at its stored width (FP16 plus a scale per
// domain, or FP32), x and r read and written, the direction and Ap read, z written, the
// domain vertex lists and offsets (block Jacobi: the 3x3 inverses instead of the factor).
extern "C" int mguso_scene_profile_pcg(mguso_scene* sc, int iters, float* us2, double* bytes2) {
  MG_CHECK_ARG(sc && us2 && bytes2 && iters > 0, "bad argument");
  Scene& s = sc->s;
  uint32_t nc = 0;
  MG_CUDA(cudaMemcpyAsync(&nc, s.c_count.p, 4, cudaMemcpyDeviceToHost, s.st));
  MG_CUDA(cudaStreamSynchronize(s.st));
  const double nv = s.nv;
  bytes2[0] = 40.0 * ((double)s.Ps.nnz + nc) + 8.0 * (nv + 1) + 48.0 * nv;
  if (s.schwarz) {
    mguso_schwarz* sw = s.schwarz.get();
    double packed = 0, vert = 0;
    for (uint32_t d = 0; d < sw->ndom; ++d) {
      const double m = 3.0 * (sw->h_dom_start[d + 1] - sw->h_dom_start[d]);
      if (sw->h_dom_diag[d])
        vert += 24.0 * (sw->h_dom_start[d + 1] - sw->h_dom_start[d]);  // 6 FP32 per vertex
      else
        packed += m * (m + 1) / 2;
    }
    const double fe = sw->half ? 2.0 : 4.0, fs = sw->half ? 4.0 * sw->ndom : 0.0;
    bytes2[1] = fe * packed + vert + fs + 88.0 * nv + 13.0 * sw->ndom;
  } else {
    bytes2[1] = 36.0 * nv + 84.0 * nv;
  }
  return pcg_fused_profile(s, (uint32_t)iters, us2);
}

// Piercing (edge, triangle) pairs of every instance at positions x (host f32[3 nv]), the
// self-intersection scan of penetration_free (has_self_intersection, implicit.rs:618-650);
// the scene's positions are left at x.
extern "C" int mguso_scene_self_intersections(mguso_scene* sc, const float* x, uint32_t* counts) {
  MG_CHECK_ARG(sc && x && counts, "null argument");
  Scene& s = sc->s;
  MG_CUDA(cudaMemcpyAsync(s.x.p, x, 12 * (size_t)s.nv, cudaMemcpyHostToDevice, s.st));
  MG_CUDA(cudaMemsetAsync(s.red.p, 0, 4 * RED_STRIDE * (size_t)s.ninst, s.st));
  MG_TRY(self_intersections(s));
  std::vector<unsigned int> h(RED_STRIDE * (size_t)s.ninst);
  uint32_t st = 0;
  MG_CUDA(cudaMemcpyAsync(h.data(), s.red.p, 4 * h.size(), cudaMemcpyDeviceToHost, s.st));
  MG_CUDA(cudaMemcpyAsync(&st, s.status.p, 4, cudaMemcpyDeviceToHost, s.st));
  MG_CUDA(cudaStreamSynchronize(s.st));
  if (st & ST_STACK_OVERFLOW) {
    set_error("self-intersection scan: BVH traversal stack overflow");
    return MGUSO_ERR_BVH_STACK;
  }
  for (uint32_t k = 0; k < s.ninst; ++k) counts[k] = h[RED_STRIDE * k + 14];
  return MGUSO_OK;
}

// The fused PCG kernels in use (after the autotuner, or pcg_variant): out2 = {rows variant
// (0: 2 lanes per block row, 1: 1, 2: 4), domain variant (0: one warp per domain, 4 per CTA;
// 1, 2, 3: three warps per domain, 1, 2 or 4 domains per CTA)}; -1 before the first solve.
extern "C" int mguso_scene_pcg_kernels(mguso_scene* sc, int* out2) {
  MG_CHECK_ARG(sc && out2, "null argument");
  out2[0] = sc->s.fr_tuned ? sc->s.fr_rows_variant : -1;
  out2[1] = sc->s.fr_tuned ? sc->s.fr_dom_variant : -1;
  return MGUSO_OK;
}

