// Device layout of one implicit-step scene.
//
// Positions, velocities and the Newton iterate are AoS f32[3*nv]. Element data is SoA per
// kind. The Hessian lives in two fixed 3x3 block patterns built once from the topology:
//   Ps: the system pattern, every block whose row and column vertices are both free, plus
//       an identity diagonal block per pinned vertex (the Dirichlet filter of
//       csr.rs:385-415, applied structurally);
//   Pp: every block that touches a pinned vertex. It is never solved with; it holds the
//       unfiltered elastic blocks the contact Rayleigh stiffness gathers
//       (implicit.rs:755-795 reads the Hessian before the Dirichlet filter).
// Each element writes its local 3x3 blocks into a contribution buffer at positions fixed
// by the reference's push order (implicit.rs:2394-2740); a gather kernel then sums every
// slot's contributions in that order, so the assembly is deterministic and needs no
// atomics. Self-contact blocks that land outside Ps form a per-iteration block matrix C.
#pragma once
#include <array>
#include "lbvh.cuh"
#include "pcg.cuh"

namespace mg {

struct Stencil {  // one active self-contact stencil (implicit.rs:678-753)
  uint32_t idx[4];
  uint32_t kind;    // 0 vertex-triangle, 1 edge-edge
  uint32_t pad;
  double d;         // gap (signed for static-collider triangles)
  double ghat;
  double g[12];     // distance gradient per participant
};

struct BlockPattern {
  uint32_t nnz = 0;
  std::vector<uint32_t> h_row_ptr, h_col;
  DevBuf<uint32_t> row_ptr, col;
};

constexpr uint32_t RED_STRIDE = 16;

enum : uint32_t {
  EXACT_SHELLS = 1,
  EXACT_STITCHES = 2,
  EXACT_HINGES = 4,
  EXACT_CONTACTS = 8,
  EXACT_SPRINGS = 16,
  EXACT_ALL = 31
};

struct Scene {
  mguso_ctx* ctx = nullptr;
  cudaStream_t st = nullptr;
  mguso_params p{};
  uint32_t nv = 0, nt = 0;
  bool mixed = true;

  // state
  std::vector<float> h_inv_mass;
  std::vector<uint8_t> h_pinned;
  DevBuf<float> x, x0, xt, v, xstep, inv_mass, dx;
  DevBuf<uint8_t> pinned;
  double time = 0.0;

  // elements (device, SoA)
  uint32_t n_free = 0, n_shell = 0, n_hinge = 0, n_spring = 0, n_stitch = 0;
  DevBuf<uint32_t> free_verts;
  DevBuf<uint32_t> shell_v;      // 3 per shell
  DevBuf<float> shell_dm;        // 4 per shell (dm_inv, glam column-major)
  DevBuf<float> shell_area, shell_mu, shell_lam;
  DevBuf<uint32_t> hinge_v;      // 4 per hinge
  DevBuf<float> hinge_rest;
  DevBuf<uint32_t> spring_v;     // 2 per spring
  DevBuf<float> spring_rest;
  DevBuf<float> spring_slr;      // per spring: its edge strain-limit ratio (used when edge_limit)
  bool edge_limit = false;       // strain_limit_ratio > 0 and strain_limit_k > 0
  DevBuf<uint32_t> mem_v;        // 3 per Baraff-Witkin membrane element
  DevBuf<float> mem_dm, mem_area; // 4 per element (Dm^-1 row-major), area
  uint32_t n_mem = 0, n_act_mem = 0;
  DevBuf<uint32_t> act_mem;
  uint64_t cb_mem = 0, gb_mem = 0;
  DevBuf<uint32_t> stitch_idx;   // 6 per stitch
  DevBuf<float> stitch_w, stitch_kl;
  // elements with at least one free vertex (recomputed every Newton iteration); the
  // contributions of all-pinned elements are constant and computed once
  uint32_t n_act_shell = 0, n_act_hinge = 0, n_act_spring = 0, n_act_stitch = 0;
  DevBuf<uint32_t> act_shell, act_hinge, act_spring, act_stitch;
  bool static_done = false;
  // the static collider on the host (for re-posing it): its vertex mask, its triangles and
  // every vertex's instance (empty without a static collider)
  std::vector<uint8_t> h_static, h_vinst;
  std::vector<std::array<uint32_t, 3>> h_ctris;
  // the collider's move since the last step (the friction slip of its vertices in the next
  // step, implicit.rs:3063-3078), kept while kin_dx_set
  std::vector<float> h_kin_dx;
  DevBuf<float> kin_dx;
  bool kin_dx_set = false;
  // Hessians the assembly writes: 0 the step's PSD-projected ones; 2 the exact ones (shells
  // without the eigenvalue clamp, stitches below rest length, hinges and barriers with their
  // second-derivative terms), the contact stiffness held at `contact_k` (2 per stencil:
  // stiffness and its mass part) recorded by contact_stiffness()
  bool fp16_factor = true;  // Schwarz factor tiles in FP16 (false: FP32, as the adjoint uses)
  int hess_mode = 0;
  uint32_t exact_terms = EXACT_ALL;  // which element kinds mode 2 writes exactly
  DevBuf<double> contact_k;

  // contribution buffers: blocks (9 floats) and gradient entries (3 floats)
  uint64_t cb_inertia = 0, cb_stitch = 0, cb_spring = 0, cb_shell = 0, cb_hinge = 0, n_cblocks = 0;
  uint64_t gb_inertia = 0, gb_stitch = 0, gb_spring = 0, gb_shell = 0, gb_hinge = 0, n_gentries = 0;
  DevBuf<float> cblocks, gentries;

  // patterns + gather lists (slot < Ps.nnz: Ps; else Pp)
  BlockPattern Ps, Pp;
  DevBuf<uint32_t> slot_ptr, slot_list;     // contributions per slot, push order
  DevBuf<uint8_t> slot_inst;                // instance of each slot (Ps, then Pp)
  DevBuf<uint32_t> gv_ptr, gv_list;         // gradient entries per vertex, push order
  DevBuf<uint32_t> diag_slot;               // per vertex: its diagonal slot (Ps if free, Pp if pinned)
  std::unique_ptr<mguso_bsr> A;             // Ps values live in A->val
  DevBuf<float> valp;                       // Pp values
  DevBuf<float> grad, rhs;

  // pins (FixPair, implicit.rs:230-262) and pulls (PullPair, implicit.rs:264-282), grouped by
  // vertex in their order of setting: pv the vertices having any, pv_pin / pv_pull the ranges
  // (n_pv + 1 each) into the pin and pull arrays
  struct HostPin {
    uint32_t index;
    float target[3], ghat, stiffness;
    uint8_t kinematic;
  };
  struct HostPull {
    uint32_t index;
    float target[3], weight;
  };
  std::vector<HostPin> h_pins;
  std::vector<HostPull> h_pulls;
  uint32_t n_pv = 0, n_pin = 0, n_pull = 0, n_static_pin = 0;
  DevBuf<uint32_t> pv, pv_pin, pv_pull, pin_vert;
  DevBuf<float> pin_target, pin_ghat, pin_stiff, pull_target, pull_weight;
  DevBuf<uint8_t> pin_kin;
  // strain-limit barrier faces (implicit.rs:1088-1121): vertices (3 per face), inverse rest
  // shape (4, column-major as shells), limit and mass; per face its 9 block slots (a, b) in
  // the slot numbering of the gather (~0u: absent, both vertices pinned) and its
  // contribution (81 Hessian entries, row-major 9x9, then 9 gradient entries). The touched
  // slots and vertices have their contributions listed in face order (entry = 9 face + 3 a
  // + b for blocks, 3 face + a for gradients).
  uint32_t n_sl = 0, n_sl_slots = 0, n_sl_verts = 0;
  DevBuf<uint32_t> sl_v, sl_slot, sl_slots, sl_sptr, sl_slist, sl_verts, sl_vptr, sl_vlist;
  DevBuf<float> sl_dm, sl_limit, sl_mass, sl_c;
  // colliders
  uint32_t n_col = 0;
  std::vector<float> h_colliders;
  DevBuf<float> colliders;

  // collision topology
  uint32_t n_edge = 0;
  DevBuf<uint32_t> tris, edge_tris;         // edges as degenerate triangles (a, b, b)
  DevBuf<uint32_t> edges;                   // 2 per edge
  DevBuf<uint32_t> ee_tail;                 // per instance: first edge of its static tail (all
                                            // later edges of the instance have both ends pinned)
  DevBuf<uint32_t> ex_ptr, ex_list;         // 1-ring exclusion (broadphase.rs:756-775)
  DevBuf<uint8_t> static_vert, collider_tri;
  bool has_static = false;
  DevBuf<float> collider_pn;                // 3 per vertex
  // instances: a batch of independent drapes in one scene (one for a single scene), as
  // contiguous vertex, triangle and edge ranges; every element and stencil lies in one
  uint32_t ninst = 1;
  std::vector<uint32_t> inst_vert, inst_tri, inst_edge;  // ninst + 1 each
  DevBuf<uint8_t> vinst;                                 // per vertex
  std::vector<float> char_len;                           // per instance
  std::vector<std::unique_ptr<Lbvh>> tri_bvh, edge_bvh;  // per instance
  Lbvh sorter;                                           // radix-sort scratch

  // self-contact working set
  uint32_t cap_pairs = 0, cap_stencils = 0;
  // the instances the current Newton iteration of a step works on (all outside a step): BVH
  // builds, stencil collection and collider sides skip the others
  uint32_t iter_active = 0xffffffffu;
  DevBuf<uint32_t> pairs;                   // 2 per candidate
  DevBuf<unsigned long long> counters;      // [0] vt pairs, [1] stencils, [2] ee candidates, [3] unique keys
  DevBuf<unsigned long long> side_best;     // per vertex (d2 bits << 32 | tri)
  DevBuf<Stencil> stencils, stencils_sorted;
  uint32_t last_nst = 0;  // stencils of the last mguso_scene_assemble
  // persistent PCG: grid (-1 until configured, 0 when it cannot be resident), barrier words,
  // per-instance results and the instance row offsets
  int pp_grid = -1;
  DevBuf<uint32_t> pp_bar, pp_inst;
  DevBuf<PcgInstResult> pp_out;
  DevBuf<uint64_t> pp_probe;
  DevBuf<double> pp_part;
  std::vector<uint32_t> pp_key;  // instance rows the uploaded layout was built for
  // fused two-kernel PCG: layout, per-instance state, partials and the cached graph
  std::vector<uint32_t> fr_key;
  std::vector<unsigned char> fr_graph_key;
  DevBuf<uint32_t> fr_lay;
  uint32_t fr_grid_rows = 0, fr_grid_dom = 0;
  DevBuf<FusedInst> fr_inst;
  DevBuf<FusedCtl> fr_ctl;
  PinnedBuf<FusedInst> fr_out;  // the last solve's per-instance results, copied back without a wait
  DevBuf<double> fr_part;
  cudaGraphExec_t fr_exec = nullptr;
  int fr_rows_variant = 0, fr_dom_variant = 0;  // the fused kernels in use (see pcg_fused.cu)
  // sliced-ELL copy of Ps for the rows kernel's SELL variant: slices of 32 consecutive rows of
  // one instance, slot base per slice (sell_base, nslices + 1), per instance the first slice
  // (sell_inst, ninst + 1), columns (sell_col, 32 per slot), values SoA (288 floats per slot:
  // entry q of the 32 rows at q * 32 + lane) and each Ps block's value offset (sell_pos)
  bool sell_built = false;
  DevBuf<uint32_t> sell_base, sell_inst, sell_col, sell_pos;
  DevBuf<float> sell_val;
  bool fr_tuned = false;
  // side streams for the instances' independent BVH builds and refits (forked from and joined
  // back into st with events), created on first use
  std::vector<cudaStream_t> aux;
  std::vector<cudaEvent_t> aux_ev;
  cudaEvent_t fork_ev = nullptr;
  ~Scene() {
    if (fr_exec) cudaGraphExecDestroy(fr_exec);
    if (ccd_exec) cudaGraphExecDestroy(ccd_exec);
    for (auto e : aux_ev) cudaEventDestroy(e);
    for (auto q : aux) cudaStreamDestroy(q);
    if (fork_ev) cudaEventDestroy(fork_ev);
  }
  DevBuf<unsigned long long> st_keys;
  DevBuf<uint32_t> st_ids;
  // contact contributions (32 blocks + 4 gradient entries per stencil)
  DevBuf<float> ccblocks, cgentries;
  DevBuf<unsigned long long> ckeys;
  DevBuf<uint32_t> cids;
  DevBuf<unsigned long long> gkeys;
  DevBuf<uint32_t> gids;
  // C: contact blocks outside Ps (rows sorted), device row pointers over all vertices
  uint32_t cap_c = 0;
  DevBuf<uint32_t> c_row_ptr, c_col, c_row;
  DevBuf<float> c_val;
  DevBuf<uint32_t> c_count;
  DevBuf<uint32_t> is_new, rank, scan_tmp;

  // reductions / CCD
  DevBuf<unsigned int> red;                 // per-iteration reductions (float bits), RED_STRIDE per instance
  DevBuf<unsigned int> ccd_acc;             // CCD per (instance, pass): step fraction bits, caps
  DevBuf<unsigned char> ccd_state;          // the device-driven CCD schedule (contact.cu)
  PinnedBuf<unsigned char> ccd_out;         // its copy for the host, read after the stream passes it
  bool ccd_half_set = false;                // half the characteristic lengths uploaded into it
  cudaGraphExec_t ccd_exec = nullptr;       // the self-contact schedule's conditional graph
  std::vector<unsigned char> ccd_key;
  DevBuf<uint32_t> status;

  // linear solve
  std::unique_ptr<mguso_schwarz> schwarz;
  DevBuf<float> bjinv;
  PcgWork work;

  std::vector<mguso_step_stats> history;
};

int scene_build(Scene& s, const mguso_scene_desc* d, const std::vector<uint32_t>& inst_vert);
int scene_step(Scene& s, mguso_step_stats* out);

// assembly (assemble.cu)
int assemble_elastic(Scene& s);
int assemble_colliders(Scene& s);  // strain-limit faces, pins and pulls first, then the analytic colliders
int upload_pins(Scene& s);          // groups h_pins / h_pulls by vertex onto the device
int slot_of_pair(const Scene& s, uint32_t r, uint32_t c);  // gather slot of block (r, c), -1 if absent
int assemble_contacts(Scene& s, uint32_t nst);
int contact_stiffness(Scene& s, uint32_t nst);  // records s.contact_k from the gathered blocks
int finish_rhs(Scene& s);
int system_spmv(Scene& s, const float* p, float* ap, cudaStream_t st, const DotSink* d);

// contact (contact.cu)
// The instances' triangle and edge LBVHs at x; refit = true keeps each tree's shape from its
// last build (the Newton iterations after a step's first) and only recomputes its boxes at x.
int build_bvhs(Scene& s, const float* x, bool refit = false);
int pcg_persistent(Scene& s, const uint32_t* h_inst_row, uint32_t ninst, uint32_t active, PcgInstResult* out);
// out == null defers the results: the caller synchronises the stream later and reads them with
// pcg_fused_results (the solve itself never waits on the host)
int pcg_fused(Scene& s, const uint32_t* h_inst_row, uint32_t ninst, uint32_t active, PcgInstResult* out);
int pcg_fused_results(Scene& s, uint32_t ninst, PcgInstResult* out);
int pcg_fused_profile(Scene& s, uint32_t iters, float* us2);
int pcg_fused_select(Scene& s);  // the fused kernels' variants: pcg_variant, or the autotuner's choice
int collect_stencils(Scene& s, uint32_t* nst);
// piercing pairs per instance at s.x into red[RED_STRIDE k + 14]; refit = true refits the
// triangle LBVHs built earlier in the step instead of rebuilding them
int self_intersections(Scene& s, bool refit = false);
// CCD step fractions of the instances in `active` along s.dx, enqueued without a host wait:
// ccd_t is the device array of fractions (0 for inactive instances), ccd_results waits for
// the stream and gives fractions and ACCD cap hits per instance
int ccd_step(Scene& s, uint32_t active);
const float* ccd_t(Scene& s);
int ccd_results(Scene& s, float* t_out, uint32_t* cap_hits);
uint32_t ccd_launches(Scene& s);  // self-contact schedule launches of the last ccd_step (after ccd_results)

}  // namespace mg

struct mguso_scene {
  mg::Scene s;
};
