// md_state.h -- host-side state of one b200_ctx and the launchers shared by
// the engine's translation units.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "md_common.cuh"

// graph pieces of a step (api.cu): initial half-step + decision, rebuild,
// forces + final half-step (with / without thermo output), and the same two
// with the next step's initial half-step and decision fused in
#define MD_NPIECES 6
// graph slots: every piece for each of the two position buffers (md_lj_step)
#define MD_NGRAPHS (2 * MD_NPIECES)
#include "../../include/b200md.h"

// timer phases of one step
enum {
  PH_INITIAL = 0,  // fix nve initial_integrate + rebuild decision
  PH_NEIGH = 1,    // wrap, cell sort, neighbor list (when taken)
  PH_PAIR1 = 2,    // LJ force, or EAM density + embedding
  PH_PAIR2 = 3,    // EAM force (empty for LJ)
  PH_FINAL = 4,    // fix nve final_integrate (+ kinetic energy, thermo row)
  MD_NPHASE = 5
};

struct EAMDev {
  int nrho = 0, nr = 0, nfrho = 0, nrhor = 0, nz2r = 0;
  double drho = 0, dr = 0, rdr = 0, rdrho = 0, rhomax = 0, cutmax = 0, cutforcesq = 0;
  // spline tables, 8 coefficients per knot (7 used): [table][knot][8];
  // embedding rows [c0..c6 -], density and pair rows [c3 c4 c5 c6 c0 c1 c2 -]
  double *frho = nullptr, *rhor = nullptr, *z2r = nullptr;
  float *frho_f = nullptr, *rhor_f = nullptr, *z2r_f = nullptr;
  float *fz_f = nullptr;  // one element: [z2 c3..c6 | rho' c0..c2 | 0] per knot
  int type2frho[MD_MAXTYPES + 1];
  int type2rhor[(MD_MAXTYPES + 1) * (MD_MAXTYPES + 1)];
  int type2z2r[(MD_MAXTYPES + 1) * (MD_MAXTYPES + 1)];
  // type2rhor[i][j] == type2rhor[j][i] for every type pair (one element, or
  // a funcfl/setfl mapping symmetric in the pair): rho'_j(r) of a pair is
  // then the same spline row as rho'_i(r) and is loaded once
  bool rhor_sym = false;
};

// blocks of tables_dev, each TABSZ doubles
enum { TAB_CUTNEIGHSQ = 0, TAB_CUTSQ, TAB_LJ1, TAB_LJ2, TAB_LJ3, TAB_LJ4, TAB_OFFSET, TAB_COUNT };
constexpr int TABSZ = (MD_MAXTYPES + 1) * (MD_MAXTYPES + 1);

struct b200_ctx {
  int device = 0;
  int prec = 0;
  cudaStream_t stream = nullptr;
  // side stream of the rebuild: a replica batch's second builder launch runs
  // beside the first (fork and join events)
  cudaStream_t s_aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  std::string err;
  long long launches = 0;

  // box and cells
  bool box_set = false;
  BoxGeom box{};
  int ncells = 0;

  // replicas (b200_set_replicas): nrep independent boxes in one context;
  // nrep == 0 is the single box `box`
  int nrep = 0;
  std::vector<int> rep_natoms, rep_atom_start, rep_cell_base, rep_tile_base;
  std::vector<double> rep_lo, rep_hi;
  std::vector<BoxGeom> rep_box;
  int ntiles = 0;  // builder tiles over all replicas
  BoxGeom *d_rep_box = nullptr;
  int *d_rep_of_atom = nullptr, *d_rep_cell_base = nullptr, *d_tile_rep = nullptr,
      *d_rep_tile_base = nullptr;
  int rep_dev_n = 0, rep_dev_tiles = 0, rep_dev_r = 0;
  Reps reps() const { return Reps{d_rep_box, d_rep_of_atom, d_rep_cell_base, d_tile_rep,
                                  d_rep_tile_base}; }

  // settings
  double skin = 0.3;
  int every = 1, delay = 10, check = 1, one_user = 0;
  int ntypes = 0;
  double mass[MD_MAXTYPES + 1] = {0};
  bool mass_set = false;
  int pstyle = 0;
  LJParamsDev lj{};
  double cutforce_max = 0.0;  // largest force cutoff
  double cutneighsq[(MD_MAXTYPES + 1) * (MD_MAXTYPES + 1)] = {0};
  double cutneighmax = 0.0;
  EAMDev eam;
  // device copy of the per-type tables, TAB_* blocks of (ntypes+1)^2 doubles
  double *tables_dev = nullptr;
  double *cutneighsq_dev = nullptr;  // = tables_dev + TAB_CUTNEIGHSQ*TABSZ

  // atoms (device, cell-sorted order)
  int n = 0, nalloc = 0, stride = 0;
  double4 *x4 = nullptr, *x4b = nullptr;
  double *v = nullptr, *vb = nullptr;  // 3 SoA planes of `stride`
  double *f = nullptr;                 // 3 SoA planes of `stride`
  int *orig = nullptr, *origb = nullptr;
  int *image = nullptr, *imageb = nullptr;
  int *cell = nullptr;        // packed cell of each sorted atom
  int *where = nullptr;       // sorted slot of each caller index (inverse of orig)
  // ghost atoms (b200_set_ghosts): per caller index, nonzero for an atom that
  // another rank owns; such atoms are neither integrated nor distance-checked
  int *ghost = nullptr;
  bool ghosts_on = false;
  int4 *xq = nullptr;         // mixed: fixed-point coordinates (md_xq)
  int4 *xqb = nullptr;        // mixed: second buffer of xq (md_lj_step)
  int pos_parity = 0;         // md_lj_step buffer swaps since allocation, mod 2
  double4 *xhold = nullptr;   // positions at the last build (check yes)
  // device staging of host transfers (upload, download, per-atom energy and
  // virial), kept between calls so a call maps no new memory
  char *xfer = nullptr;
  size_t xfer_bytes = 0;
  // overlapped transfers (b200_stage_atoms, b200_download_atoms_async): one
  // copy stream per direction, two staged input sets and two download slots
  struct XferSlot {
    char *buf = nullptr;
    size_t bytes = 0;
    int n = 0;
    bool has_v = false, used = false;
    cudaEvent_t ready = nullptr;  // input: copy done; output: caller order formed
    cudaEvent_t done = nullptr;   // output: copy to the host done
  };
  cudaStream_t s_h2d = nullptr, s_d2h = nullptr;
  XferSlot in_slot[2], out_slot[2];
  int in_head = 0, in_count = 0;  // oldest staged input set, sets waiting
  int out_next = 0;
  double *rho = nullptr, *fp = nullptr;
  float *fpf = nullptr;
  // split EAM compute (b200_eam_density, then b200_eam_force): the eflag /
  // vflag of the density call and its per-atom embedding energies
  int eam_split_eflag = -1, eam_split_vflag = -1;
  double *eam_eatom = nullptr;  // caller order, n doubles
  int eam_eatom_n = 0;
  double *mass_dev = nullptr; // per-type masses (device)
  bool have_atoms = false, sorted_once = false;

  // binning scratch
  int ncell_alloc = 0;
  int *cell_count = nullptr, *cell_start = nullptr, *scan_tmp = nullptr;
  int *slot = nullptr, *perm = nullptr, *cell_tmp = nullptr;

  // neighbor list
  int *nlist = nullptr, *numneigh = nullptr;
  int capacity = 0;     // entries per atom
  int stage_need = 0;   // staged atoms per builder tile seen by earlier builds
  long long nlist_alloc = 0;

  // run-chunk snapshot for overflow replay (x4, v, f, xhold planes + ids)
  double4 *snap_x4 = nullptr, *snap_xhold = nullptr;
  double *snap_v = nullptr, *snap_f = nullptr;
  int *snap_orig = nullptr, *snap_image = nullptr, *snap_cell = nullptr;
  int4 *snap_xq = nullptr;
  int *snap_status = nullptr;
  int snap_alloc = 0;
  int overflow_replays = 0;

  // reductions and status
  double *partial = nullptr;     // per-block partial sums
  int partial_blocks = 0;
  unsigned int *counter = nullptr;
  double *adj_gs = nullptr;    // force-matching scratch: G in the sorted order
  double *adj_gtab = nullptr;  // force-matching parameter gradients
  int adj_n = 0;
  double *ev = nullptr;          // [0] eng, [1..6] virial, [7] sum m v^2
  int *status = nullptr;         // ST_* words
  int *status_host = nullptr;    // pinned mirror
  // decision mailbox: mapped page-locked words that the device's rebuild
  // decision writes on the steps where the distance criterion decides ([0]
  // the decision, [1] the number of such decisions so far), so the host
  // reads a decision by waiting on memory instead of a copy and a stream
  // synchronize; dec_count is the device's count (kept apart from the status
  // words, which run-chunk snapshots restore) and decisions the host's count
  // of the decisions it has waited for
  int *mail_host = nullptr, *mail_dev = nullptr;
  // mapped page-locked bounce buffer of the small device-to-host reads
  // (status words, energy/virial sums), written by a one-warp kernel
  int *bounce_host = nullptr, *bounce_dev = nullptr;
  int *dec_count = nullptr;
  unsigned int decisions = 0;
  double *rows = nullptr;        // device thermo rows (9 doubles each)
  int rows_cap = 0;

  // launch shape of the pair kernels
  int tpa = 0, block = 128;
  bool tuned = false;
  // The launch-shape search made at setup ran on the caller's starting
  // state (often a perfect lattice, where the best shape can differ from
  // the thermal one); the first run repeats it once, retune_steps steps in.
  bool retune_pending = false;
  long long retune_step = -1;

  // one-launch replica step (b200_set_replica_step): each thread-block
  // cluster of rep_cs CTAs of rep_block threads owns a fixed set of whole
  // replicas (group g: atom ranges d_rep_ranges[d_rep_grp_first[g] ..
  // d_rep_grp_first[g+1]) as (start, count)), balanced by atom count
  int rep_mode = 0;       // 0 chosen on the next b200_setup, 1 graph of kernels, 2 one launch
  int rep_fix_cs = 0, rep_fix_block = 0, rep_fix_tpa = 0;  // shapes fixed by the caller (0 = tuned)
  bool rep_tuned = false;  // the form has been chosen for the current batch
  bool rep_onelaunch = false;
  int rep_cs = 0, rep_block = 0, rep_tpa = 0, rep_groups = 0;
  int *d_rep_grp_first = nullptr;
  int2 *d_rep_ranges = nullptr;
  double rep_tune_ms[2] = {0, 0};  // per-step device time of the two forms when tuned

  // CUDA graph of one MD step (captured lazily by b200_run)
  // graphs of the step pieces: [0] initial half-step + decision, [1] rebuild,
  // [2] forces + final half-step with thermo output, [3] the same without
  cudaGraphExec_t step_exec[MD_NGRAPHS] = {};
  cudaGraph_t step_graph[MD_NGRAPHS] = {};
  int step_kernels[MD_NGRAPHS] = {};                    // kernel nodes per graph
  bool graph_valid = false;
  double graph_dt = 0, graph_ftm2v = 0;
  int graph_tpa = 0;
  bool graph_timing = false;
  bool use_graphs = true;   // false: eager launches, host-side rebuild decision

  // phase timers (Timer categories of the reference, src/timer.h:19-20):
  // event-record nodes at the phase boundaries of every step graph
  bool timing = false;
  bool timing_pieces = false;  // b200_set_timing(ctx, 2): device time of whole pieces
  cudaEvent_t ph_event[MD_NPHASE + 1] = {};           // placeholders used at capture
  std::vector<cudaGraphNode_t> ev_nodes[MD_NGRAPHS];   // event-record nodes per graph
  std::vector<cudaEvent_t> ev_pool;                    // per-step events of a chunk
  double phase_ms[MD_NPHASE] = {0};
  std::vector<float> step_ms;  // device time of each timed step (first to last phase event)
  long long phase_steps = 0;
};

// The mixed form's fixed-point unit is the same in every dimension of the box
// (of every replica box, for a batch): the pair kernels then work in units.
inline bool md_q_iso(const b200_ctx *c) {
  if (!c->nrep) return c->box.qiso != 0;
  for (int r = 0; r < c->nrep; r++)
    if (!c->rep_box[r].qiso) return false;
  return true;
}

// ---- launchers (neigh.cu) -------------------------------------------------
// full rebuild: wrap, cell counting sort, permute, neighbor list
cudaError_t md_rebuild(b200_ctx *c, const int *d_flag);
int md_stage_cap(const b200_ctx *c);
bool md_stage_feedback(b200_ctx *c, int staged_max);
// LAMMPS half list derived from the full list; returns entry count via *total
cudaError_t md_half_list(b200_ctx *c, int *d_num, int *d_jowner, int *d_jimage, long long cap,
                         long long *total);
// ---- halo (halo.cu) ---------------------------------------------------------
// where[orig[k]] = k for the n sorted atoms
cudaError_t md_where(b200_ctx *c);
// buf[3i..3i+2] = x of caller atom idx[i]; idx, buf on the device
cudaError_t md_halo_pack(b200_ctx *c, int m, const int *idx, double *buf);
// x of caller atom idx[i] = buf[3i..3i+2] (and its fixed-point copy)
cudaError_t md_halo_unpack(b200_ctx *c, int m, const int *idx, const double *buf);
// x of every atom from x[3n] in caller order (device), keeping cells and list
cudaError_t md_set_positions(b200_ctx *c, const double *x);
// ---- pair kernels (pair_lj.cu, pair_eam.cu) --------------------------------
cudaError_t md_lj_compute(b200_ctx *c, bool ev, bool atom_ev, double *eatom, double *vatom);
// `mid`, when given, is recorded between the density and the force kernel;
// `stage` runs both passes or one of them (the density pass sets the global
// energy/virial sums and the per-atom embedding energies, the force pass
// adds its pair terms to them)
enum { EAM_BOTH = 0, EAM_DENSITY = 1, EAM_FORCE = 2 };
cudaError_t md_eam_compute(b200_ctx *c, bool ev, bool atom_ev, double *eatom, double *vatom,
                           cudaEvent_t mid = nullptr, int stage = EAM_BOTH);
// F'(rho) of the caller atoms idx[0..m) to buf (pack) or from it (unpack,
// ghosts only when ghosts are marked); idx and buf on the device
cudaError_t md_eam_fp_halo(b200_ctx *c, int m, const int *idx, double *buf, bool pack);
// one-launch replica step (pair_lj.cu): this step's lj/cut forces, final
// half-step and the next step's initial half-step and rebuild decision, for
// every replica, in one cluster launch (non-output steps)
cudaError_t md_rep_step(b200_ctx *c, double dtv, double dtf);
// one MD step of lj/cut in one launch (pair forces, this step's final and the
// next step's initial half-step, thermo row, rebuild decision), reading the
// current positions and writing the other position buffer; md_swap_positions
// makes that buffer current.  md_lj_step_ok: the context can use it.
bool md_lj_step_ok(const b200_ctx *c);
cudaError_t md_lj_step(b200_ctx *c, double dtv, double dtf, bool out);
void md_swap_positions(b200_ctx *c);
// the same for eam: the density pass, then the force pass with the half-steps
bool md_eam_step_ok(const b200_ctx *c);
cudaError_t md_eam_step(b200_ctx *c, double dtv, double dtf, bool out);
// the context runs a one-launch step kernel in its fused pieces
inline bool md_step_ok(const b200_ctx *c) { return md_lj_step_ok(c) || md_eam_step_ok(c); }
// group plan of the one-launch step: cluster size cs, block size, groups
int md_rep_plan(b200_ctx *c, int cs, int block, int tpa);
// ---- integration (integrate.cu) --------------------------------------------
cudaError_t md_nve_initial(b200_ctx *c, double dtv, double dtf);
cudaError_t md_decide(b200_ctx *c);
cudaError_t md_nve_final(b200_ctx *c, double dtf, bool ke);
// final half-step of this step (+ KE) and initial half-step of the next
cudaError_t md_nve_fused(b200_ctx *c, double dtv, double dtf, bool ke);
cudaError_t md_ke(b200_ctx *c);
cudaError_t md_record_row(b200_ctx *c);
cudaError_t md_zero_ev(b200_ctx *c);

// ---- force-matching adjoint (adjoint.cu) ------------------------------------
// lj1, lj2, cutsq: host (ntypes+1)^2 tables; f, g, gx: device, 3n doubles in
// the caller's order; gs: device scratch of 3n doubles; gtab: device, 2 *
// MD_ADJ_MAXTYPES^2 doubles (dL/dlj1, dL/dlj2 per type pair)
cudaError_t md_adj_forward(b200_ctx *c, const double *lj1, const double *lj2, const double *cutsq,
                           double *f);
cudaError_t md_adj_backward(b200_ctx *c, const double *lj1, const double *lj2,
                            const double *cutsq, const double *g, double *gx, double *gs,
                            double *gtab);
cudaError_t md_adj_positions(b200_ctx *c, const double *x);

// ---- replicas (replica.cu) ------------------------------------------------------
// per-replica thermo rows {natoms, sum m v^2, eng_vdwl, virial[6]} from the
// per-atom energy/virial of the last compute (eatom, vatom in caller order)
cudaError_t md_rep_rows(b200_ctx *c, const int *d_start, const double *eatom, const double *vatom,
                        double *rows);

inline int md_blocks(long long work, int block) {
  return (int)((work + block - 1) / block);
}
